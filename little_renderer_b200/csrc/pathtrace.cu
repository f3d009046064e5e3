// pathtrace.cu - the path tracer on sm_100a: the light transport of the reference's
// trace_path_sampled (engine/rt/tracer.c:364-545) and trace_image (:329-356), which its WGSL
// megakernel `main`/`trace()` restate (engine/gpu/shaders/trace/trace.wgsl:1125-1316).
//
// Per bounce: the closest hit through the world's BVH (shape ids: primitives, then triangles, as
// scene_intersect numbers them, engine/rt/accel.c:252), the hit (engine/rt/intersect.c set_hit,
// finish_*), the lamp counted by its emit mode (FULL / NONE / MIS), next event estimation of the
// lamp quad with a shadow ray to dist - RT_SHADOW_MARGIN (sample_direct_light, tracer.c:56) and
// the power heuristic, the BSDF's lobe pick and sample (bsdf.cuh), Russian roulette after 3
// bounces. Float build constants: RT_EPS 2e-3, RT_SHADOW_MARGIN 2e-2 (tracer.c:14-23).
//
// Two launch modes:
//   exact: one thread per pixel, its samples in order from the CPU's per-pixel PCG32 stream and
//          sampler (trace_image's seeding): the image is the CPU's up to transcendental rounding
//          (the parity mode);
//   fast:  one thread per (pixel, sample), each sample its own PCG32 stream (seeded from pixel,
//          sample and image seed) and the same Owen-Sobol dimensions; a pixel's samples sit in
//          neighbouring lanes and are summed by warp shuffles in a fixed order (deterministic).

#include "pt_device.cuh"
#include <algorithm>

namespace lrc {
namespace pt {

// plane 1's w after a guided call: its last sample's number (low 24 bits) + 1, as trace.wgsl keeps
// it for the temporal gradients (trace.wgsl:1306-1310)
__device__ __forceinline__ float last_sample_tag(const PtParams &P) {
    return (float)((((uint32_t)(P.spp0 + P.spp - 1)) & 0xffffffu) + 1u);
}

// exact mode: one thread per pixel of rows [y0, y0 + rows), samples [0, spp) in order from the
// CPU's per-pixel stream (trace_image, tracer.c:337-353)
template <bool MEDIA, bool GUIDED>
__global__ void __launch_bounds__(128) exact_kernel(PtScene S, PtParams P, float4 *accum, unsigned long long *ray_count,
                                                    uint32_t *err) {
    const uint32_t idx = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t x = idx % P.W, yy = idx / P.W;
    uint32_t rays = 0;
    if (yy < (uint32_t)P.rows) {
        const uint32_t y = P.y0 + yy;
        const uint64_t pixel = (uint64_t)y * P.W + x;
        Rng rng;
        rng_seed(rng, 0x853c49e6748fea9bull ^ (pixel * 0x9E3779B97F4A7C15ull) ^ (P.seed * 0xD1B54A32D192ED03ull), pixel);
        V3 sum = v3(0, 0, 0);
        float ml = 0.0f, ml2 = 0.0f, l_last = 0.0f;
        for (int k = 0; k < P.spp; k++) {
            Sampler sm{&rng, (uint32_t)k, (uint32_t)P.seed * 0x9e3779b9u, (int)x, (int)y, P.sampler_on, S.mask};
            float jx, jy;
            sampler_2d(sm, 0, jx, jy);
            float u = dvd(add((float)x, jx), (float)P.W), v = dvd(add((float)y, jy), (float)P.H);
            V3 o, d;
            camera_ray(P, u, v, o, d);
            V3 c = trace_path<MEDIA>(S, P, o, d, sm, err, rays);
            if (!is_number(c)) {
                if (GUIDED) l_last = 0.0f;           // (a dropped sample counts as black)
                continue;
            }
            c = clamp_sample(c, P.clamp);
            sum = vadd(sum, c);
            if (GUIDED) {
                const float l = sample_luma(c, P.guide[pixel]);
                ml += l;
                ml2 += l * l;
                l_last = l;
            }
        }
        float4 a = accum[pixel];
        accum[pixel] = make_float4(a.x + sum.x, a.y + sum.y, a.z + sum.z, a.w + (float)P.spp);
        if (GUIDED) {                                // (z, w: the last sample's luminance and number + 1)
            const float4 m = P.moments[pixel];
            P.moments[pixel] = make_float4(m.x + ml, m.y + ml2, l_last, last_sample_tag(P));
        }
    }
    if (ray_count) {
        unsigned long long r = rays;
        for (int o = 16; o > 0; o >>= 1) r += __shfl_xor_sync(0xffffffffu, r, o);
        if ((threadIdx.x & 31) == 0 && r) atomicAdd(ray_count, r);
    }
}

// fast mode: P.group lanes (a power of 2 dividing 32) per pixel, lane s tracing samples s, s + g,
// s + 2g, ... of [spp0, spp0 + spp), each from its own PCG32 stream; the group's sums are then added
// in a fixed order (deterministic)
template <bool MEDIA, bool GUIDED>
__global__ void __launch_bounds__(128) fast_kernel(PtScene S, PtParams P, float4 *accum, unsigned long long *ray_count,
                                                   uint32_t *err) {
    const uint32_t g = P.group;
    const uint64_t tid = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const uint64_t pix_local = tid / g;
    const uint32_t lane_s = (uint32_t)(tid % g);
    const uint64_t npix = (uint64_t)P.W * P.rows;
    uint32_t rays = 0;
    V3 c = v3(0, 0, 0);
    float cnt = 0.0f, ml = 0.0f, ml2 = 0.0f, l_last = 0.0f;
    const bool live = pix_local < npix;
    uint64_t pixel = 0;
    if (live) {
        const uint32_t x = (uint32_t)(pix_local % P.W), y = P.y0 + (uint32_t)(pix_local / P.W);
        pixel = (uint64_t)y * P.W + x;
        for (uint32_t k = lane_s; k < (uint32_t)P.spp; k += g) {
            const uint32_t kk = P.spp0 + k;
            Rng rng;
            rng_seed(rng, mix64(pixel * 0x9E3779B97F4A7C15ull ^ ((uint64_t)kk << 40) ^ P.seed), pixel);
            Sampler sm{&rng, kk, (uint32_t)P.seed * 0x9e3779b9u, (int)x, (int)y, P.sampler_on, S.mask};
            float jx, jy;
            sampler_2d(sm, 0, jx, jy);
            float u = dvd(add((float)x, jx), (float)P.W), v = dvd(add((float)y, jy), (float)P.H);
            V3 o, d;
            camera_ray(P, u, v, o, d);
            V3 s = trace_path<MEDIA>(S, P, o, d, sm, err, rays);
            s = is_number(s) ? clamp_sample(s, P.clamp) : v3(0, 0, 0);
            c = vadd(c, s);
            cnt += 1.0f;
            if (GUIDED) {
                const float l = sample_luma(s, P.guide[pixel]);
                ml += l;
                ml2 += l * l;
                l_last = l;
            }
        }
    }
    // (the pixel's last sample, spp0 + spp - 1, is lane (spp - 1) % g's last)
    if (GUIDED) l_last = __shfl_sync(0xffffffffu, l_last, (uint32_t)(P.spp - 1) % g, g);
    for (uint32_t o = 1; o < g; o <<= 1) {               // fixed-order tree sum over the group
        c.x += __shfl_down_sync(0xffffffffu, c.x, o, g);
        c.y += __shfl_down_sync(0xffffffffu, c.y, o, g);
        c.z += __shfl_down_sync(0xffffffffu, c.z, o, g);
        cnt += __shfl_down_sync(0xffffffffu, cnt, o, g);
        if (GUIDED) {
            ml += __shfl_down_sync(0xffffffffu, ml, o, g);
            ml2 += __shfl_down_sync(0xffffffffu, ml2, o, g);
        }
    }
    if (live && lane_s == 0) {
        float4 a = accum[pixel];
        accum[pixel] = make_float4(a.x + c.x, a.y + c.y, a.z + c.z, a.w + cnt);
        if (GUIDED) {                                // (z, w: the last sample's luminance and number + 1)
            const float4 m = P.moments[pixel];
            P.moments[pixel] = make_float4(m.x + ml, m.y + ml2, l_last, last_sample_tag(P));
        }
    }
    if (ray_count) {
        unsigned long long r = rays;
        for (int o = 16; o > 0; o >>= 1) r += __shfl_xor_sync(0xffffffffu, r, o);
        if ((threadIdx.x & 31) == 0 && r) atomicAdd(ray_count, r);
    }
}

// ---- the batch: one persistent kernel over the tasks of many jobs --------------------------------

// Each lane holds one task (a pixel's lane slot) and one path of it at a time. A loop pass is
// one bounce for every lane with a path; a lane whose path ends adds it to its task's sum and
// starts the task's next sample, and a lane whose task is done writes it out and takes the next
// task of the queue (one atomic per warp and pass for all such lanes). The lanes thus stay busy
// however the path lengths and the samples per task differ, within a job and across jobs, and
// the grid drains the queue with no launch per job and no tail per job.
template <int BLOCK, int MINB, bool MEDIA>
__global__ void __launch_bounds__(BLOCK, MINB) batch_kernel(const BatchJob *__restrict__ jobs, uint32_t njobs,
                                                      unsigned long long ntasks, unsigned long long *next, uint32_t *err) {
    const uint32_t lane = threadIdx.x & 31;
    const uint32_t lt_mask = (1u << lane) - 1u;
    int j = -1;                       // the job of the lane's task (-1: none)
    unsigned long long task = 0;
    uint64_t pixel = 0;               // the pixel's index in its image
    uint32_t x = 0, y = 0, slot = 0, kk = 0, kend = 0, g = 1, rays = 0;
    V3 c = v3(0, 0, 0);
    float cnt = 0.0f, ml = 0.0f, ml2 = 0.0f, l_last = 0.0f;   // the task's sum, samples, luminance moments
    bool active = false, done = false;
    PathState ps;
    Rng rng;
    rng.state = 0;
    rng.inc = 1;
    for (;;) {
        if (j >= 0 && !active && kk >= kend) {       // the task is done
            const BatchJob &J = jobs[j];
            const unsigned long long l = task - J.task0;
            J.partial[l] = make_float4(c.x, c.y, c.z, cnt);
            J.prays[l] = rays;
            if (J.pmom) J.pmom[l] = make_float4(ml, ml2, l_last, 0.0f);
            j = -1;
        }
        const bool need = !done && j < 0;
        const uint32_t m = __ballot_sync(0xffffffffu, need);
        if (m) {
            const int leader = __ffs(m) - 1;
            unsigned long long base = 0;
            if ((int)lane == leader) base = atomicAdd(next, (unsigned long long)__popc(m));
            base = __shfl_sync(0xffffffffu, base, leader);
            if (need) {
                task = base + __popc(m & lt_mask);
                if (task >= ntasks) {
                    done = true;
                } else {
                    j = (int)batch_job_of(jobs, njobs, task);
                    const BatchJob &J = jobs[j];
                    const unsigned long long l = task - J.task0;
                    g = (uint32_t)J.P.group;
                    const unsigned long long pl = l / g;
                    slot = (uint32_t)(l - pl * g);
                    x = (uint32_t)(pl % (uint32_t)J.P.W);
                    y = (uint32_t)J.P.y0 + (uint32_t)(pl / (uint32_t)J.P.W);
                    pixel = (uint64_t)y * (uint32_t)J.P.W + x;
                    kk = (uint32_t)J.P.spp0 + slot;
                    kend = (uint32_t)(J.P.spp0 + J.P.spp);
                    c = v3(0, 0, 0);
                    cnt = 0.0f;
                    ml = ml2 = l_last = 0.0f;
                    rays = 0;
                    if (J.P.exact)                    // trace_image's per-pixel stream, all samples in order
                        rng_seed(rng, 0x853c49e6748fea9bull ^ (pixel * 0x9E3779B97F4A7C15ull) ^ (J.P.seed * 0xD1B54A32D192ED03ull),
                                 pixel);
                }
            }
        }
        if (__all_sync(0xffffffffu, done)) break;
        if (j < 0) continue;                         // (only lanes that ran out of tasks)
        const BatchJob &J = jobs[j];
        Sampler sm{&rng, kk, (uint32_t)J.P.seed * 0x9e3779b9u, (int)x, (int)y, J.P.sampler_on, J.S.mask};
        if (!active) {                               // the task's next sample: its camera ray
            if (!J.P.exact)
                rng_seed(rng, mix64(pixel * 0x9E3779B97F4A7C15ull ^ ((uint64_t)kk << 40) ^ J.P.seed), pixel);
            float jx, jy;
            sampler_2d(sm, 0, jx, jy);
            float u = dvd(add((float)x, jx), (float)J.P.W), v = dvd(add((float)y, jy), (float)J.P.H);
            V3 o, d;
            camera_ray(J.P, u, v, o, d);
            path_begin(J.P.mis || (MEDIA && J.S.nvol), o, d, ps, J.P.skip_caustics, J.P.indirect_clamp);
            active = true;
        }
        if (!path_bounce<MEDIA>(J.S, J.P.max_depth, J.P.mis, ps, sm, err, rays)) {
            V3 s = is_number(ps.radiance) ? clamp_sample(ps.radiance, J.P.clamp) : v3(0, 0, 0);
            c = vadd(c, s);
            cnt += 1.0f;
            if (J.P.moments) {
                const float l = sample_luma(s, J.P.guide[pixel]);
                ml += l;
                ml2 += l * l;
                l_last = l;
            }
            active = false;
            kk += g;
        }
    }
}

// pixel i of all the batch's bands (a whole warp calls it together): the pixel's slots summed in
// the fast kernel's shuffle order (pairs, then pairs of pairs, ...) and added to its image, its rays
// to its job
__device__ __forceinline__ void resolve_pixel(const BatchJob *__restrict__ jobs, uint32_t njobs, unsigned long long npix,
                                              unsigned long long i) {
    uint32_t jj = 0xffffffffu;
    unsigned long long r = 0;
    if (i < npix) {
        uint32_t lo = 0, hi = njobs - 1;
        while (lo < hi) {
            uint32_t mid = (lo + hi + 1) >> 1;
            if (__ldg(&jobs[mid].pix0) <= i) lo = mid;
            else hi = mid - 1;
        }
        jj = lo;
        const BatchJob &J = jobs[jj];
        const unsigned long long pl = i - J.pix0;
        const uint32_t g = (uint32_t)J.P.group;
        float4 v[16];
        for (uint32_t s = 0; s < 16; s++) {
            if (s < g) {
                v[s] = J.partial[pl * g + s];
                r += J.prays[pl * g + s];
            }
        }
        for (uint32_t o = 1; o < 16; o <<= 1)
            for (uint32_t s = 0; s + o < 16; s += 2 * o)
                if (s + o < g) {
                    v[s].x += v[s + o].x;
                    v[s].y += v[s + o].y;
                    v[s].z += v[s + o].z;
                    v[s].w += v[s + o].w;
                }
        const uint32_t x = (uint32_t)(pl % (uint32_t)J.P.W), y = (uint32_t)J.P.y0 + (uint32_t)(pl / (uint32_t)J.P.W);
        const uint64_t pixel = (uint64_t)y * (uint32_t)J.P.W + x;
        float4 *a = J.accum + pixel;
        float4 av = *a;
        *a = make_float4(av.x + v[0].x, av.y + v[0].y, av.z + v[0].z, av.w + v[0].w);
        if (J.pmom) {                                // the moments, in the same order; the last sample's
            float2 mv[16];                           // (spp0 + spp - 1) from slot (spp - 1) % g
            for (uint32_t s = 0; s < 16; s++)
                if (s < g) {
                    const float4 q = J.pmom[pl * g + s];
                    mv[s] = make_float2(q.x, q.y);
                }
            for (uint32_t o = 1; o < 16; o <<= 1)
                for (uint32_t s = 0; s + o < 16; s += 2 * o)
                    if (s + o < g) {
                        mv[s].x += mv[s + o].x;
                        mv[s].y += mv[s + o].y;
                    }
            const float4 m = J.P.moments[pixel];
            const float lz = J.pmom[pl * g + (uint32_t)(J.P.spp - 1) % g].z;
            J.P.moments[pixel] = make_float4(m.x + mv[0].x, m.y + mv[0].y, lz, last_sample_tag(J.P));
        }
    }
    // the rays of the warp's pixels, one atomic per job present
    const uint32_t peers = __match_any_sync(0xffffffffu, jj);
    const uint32_t sum = __reduce_add_sync(peers, (uint32_t)r);
    if (jj != 0xffffffffu && (threadIdx.x & 31) == (uint32_t)(__ffs(peers) - 1) && sum)
        atomicAdd(jobs[jj].rays, (unsigned long long)sum);
}

// one thread per pixel
__global__ void __launch_bounds__(128) batch_resolve_kernel(const BatchJob *__restrict__ jobs, uint32_t njobs,
                                                            unsigned long long npix) {
    resolve_pixel(jobs, njobs, npix, (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x);
}

// the same over a fixed grid, the job and pixel counts read from the run block (run[1], run[3]):
// a graph captured once resolves any run
__global__ void __launch_bounds__(128) batch_resolve_run_kernel(const BatchJob *__restrict__ jobs,
                                                                const unsigned long long *__restrict__ run) {
    const uint32_t njobs = (uint32_t)run[1];
    const unsigned long long npix = run[3];
    if (!njobs) return;
    for (unsigned long long base = (unsigned long long)blockIdx.x * blockDim.x; base < npix;
         base += (unsigned long long)gridDim.x * blockDim.x)
        resolve_pixel(jobs, njobs, npix, base + threadIdx.x);
}

// closest hits over shape ids (primitives, then triangles): lrc_scene_intersect for world scenes
__global__ void __launch_bounds__(128) shapes_closest_kernel(PtScene S, const float *__restrict__ orig,
                                                             const float *__restrict__ dir, uint64_t n, float tmin, float tmax,
                                                             int32_t *__restrict__ prim, int32_t *__restrict__ inst_out,
                                                             float *__restrict__ tout, uint32_t *err) {
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    V3 o = v3(orig[3 * i], orig[3 * i + 1], orig[3 * i + 2]), d = v3(dir[3 * i], dir[3 * i + 1], dir[3 * i + 2]);
    float best = tmax;
    int32_t id = -1, inst = -1;
    if (S.nnodes) id = walk<false>(S, S.nodes, S.root, S.nnodes, S.aux, S.naux, o, d, tmin, best, err);
    if (S.ninst) {
        int ii = -1, tri = -1;
        if (walk_instances<false>(S, o, d, tmin, best, ii, tri, err)) {
            id = tri;
            inst = ii;
        }
    }
    prim[i] = id;
    if (inst_out) inst_out[i] = inst;
    tout[i] = id >= 0 ? best : -1.0f;
}

// primitive_bounds (scene.c:47-63) of each primitive (6 float4 each) into boxes (8 floats each)
__global__ void prim_boxes_kernel(const float4 *__restrict__ prims, uint32_t n, float4 *__restrict__ boxes) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float4 *pr = prims + 6 * (size_t)i;
    float4 c = __ldg(pr), q = __ldg(pr + 1), u = __ldg(pr + 2), v = __ldg(pr + 3);
    float lo[3], hi[3];
    if (q.w == 0.0f) {
        lo[0] = sub(c.x, c.w); lo[1] = sub(c.y, c.w); lo[2] = sub(c.z, c.w);
        hi[0] = add(c.x, c.w); hi[1] = add(c.y, c.w); hi[2] = add(c.z, c.w);
    } else {
        float p[4][3] = {{q.x, q.y, q.z},
                         {add(q.x, u.x), add(q.y, u.y), add(q.z, u.z)},
                         {add(q.x, v.x), add(q.y, v.y), add(q.z, v.z)},
                         {add(q.x, add(u.x, v.x)), add(q.y, add(u.y, v.y)), add(q.z, add(u.z, v.z))}};
        for (int k = 0; k < 3; k++) {
            lo[k] = p[0][k];
            hi[k] = p[0][k];
            for (int j = 1; j < 4; j++) { lo[k] = rmin(lo[k], p[j][k]); hi[k] = rmax(hi[k], p[j][k]); }
        }
    }
    boxes[2 * (size_t)i] = make_float4(sub(lo[0], 1e-3f), sub(lo[1], 1e-3f), sub(lo[2], 1e-3f), 0.0f);
    boxes[2 * (size_t)i + 1] = make_float4(add(hi[0], 1e-3f), add(hi[1], 1e-3f), add(hi[2], 1e-3f), 0.0f);
}

}  // namespace pt

cudaError_t pt_prim_boxes(const float *d_prims, uint32_t n, float *d_boxes, cudaStream_t st) {
    if (!n) return cudaSuccess;
    pt::prim_boxes_kernel<<<(n + 127) / 128, 128, 0, st>>>(reinterpret_cast<const float4 *>(d_prims), n,
                                                           reinterpret_cast<float4 *>(d_boxes));
    return cudaGetLastError();
}

cudaError_t pt_trace(const PtScene &S, const PtParams &P, float *d_accum, unsigned long long *d_rays, uint32_t *d_status,
                     cudaStream_t st) {
    if (P.rows <= 0 || P.spp <= 0 || P.W <= 0) return cudaSuccess;
    float4 *acc = reinterpret_cast<float4 *>(d_accum);
    // (kernels compiled with and without the media's tracking and the denoiser's moments: each
    // holds registers that a scene or an image without them would pay for)
    using Fn = void (*)(PtScene, PtParams, float4 *, unsigned long long *, uint32_t *);
    static const Fn exact_fns[4] = {pt::exact_kernel<false, false>, pt::exact_kernel<false, true>,
                                    pt::exact_kernel<true, false>, pt::exact_kernel<true, true>};
    static const Fn fast_fns[4] = {pt::fast_kernel<false, false>, pt::fast_kernel<false, true>,
                                   pt::fast_kernel<true, false>, pt::fast_kernel<true, true>};
    const int k = (S.nvol ? 2 : 0) + (P.moments ? 1 : 0);
    const uint64_t threads = P.exact ? (uint64_t)P.W * P.rows : (uint64_t)P.W * P.rows * P.group;
    (P.exact ? exact_fns[k] : fast_fns[k])<<<(unsigned)((threads + 127) / 128), 128, 0, st>>>(S, P, acc, d_rays, d_status);
    return cudaGetLastError();
}

namespace pt {

// a tile's gradient sample (trace.wgsl main with T.txl.w = 1): old pixel o's sample kk traced again
// in the new scene from the same random numbers (the fast kernel's stream of (o, kk, seed) and the
// sampler's dimensions of o), through the new pixel k moved by the old one's offset (dx, dy); lam[0]
// = |l - old l| / max(l, old l, 1e-3) of the two samples' luminance over their albedo, -1 where
// there is no sample or the new one is not a number
template <bool MEDIA>
__global__ void __launch_bounds__(128) grad_kernel(PtScene S, PtParams P, GradTile *tiles, uint32_t ntiles,
                                                   const float4 *__restrict__ guide, unsigned long long *ray_count,
                                                   uint32_t *err) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    uint32_t rays = 0;
    if (t < ntiles && tiles[t].o >= 0) {
        const GradTile T = tiles[t];
        const uint32_t W = (uint32_t)P.W;
        const uint32_t ox = (uint32_t)T.o % W, oy = (uint32_t)T.o / W;
        const uint32_t kx = (uint32_t)T.k % W, ky = (uint32_t)T.k / W;
        const uint64_t opix = (uint64_t)(uint32_t)T.o;
        Rng rng;
        rng_seed(rng, mix64(opix * 0x9E3779B97F4A7C15ull ^ ((uint64_t)T.kk << 40) ^ P.seed), opix);
        Sampler sm{&rng, T.kk, (uint32_t)P.seed * 0x9e3779b9u, (int)ox, (int)oy, P.sampler_on, S.mask};
        float jx, jy;
        sampler_2d(sm, 0, jx, jy);
        const float u = dvd(add(add((float)kx, T.dx), jx), (float)P.W);
        const float v = dvd(add(add((float)ky, T.dy), jy), (float)P.H);
        V3 o, d;
        camera_ray(P, u, v, o, d);
        V3 c = trace_path<MEDIA>(S, P, o, d, sm, err, rays);
        float lam = -1.0f;
        if (is_number(c) && vmax3(c) >= 0.0f) {
            c = clamp_sample(c, P.clamp);
            const float l = sample_luma(c, guide[T.k]);
            lam = fabsf(l - T.l) / fmaxf(fmaxf(l, T.l), 1e-3f);
        }
        tiles[t].lam[0] = lam;
    }
    if (ray_count) {
        unsigned long long r = rays;
        for (int o = 16; o > 0; o >>= 1) r += __shfl_xor_sync(0xffffffffu, r, o);
        if ((threadIdx.x & 31) == 0 && r) atomicAdd(ray_count, r);
    }
}

}  // namespace pt

// the batch kernel's launch shapes: threads per block and the blocks per SM its registers are
// capped for (65536 / (threads x blocks) registers a thread)
namespace {
using BatchFn = void (*)(const BatchJob *, uint32_t, unsigned long long, unsigned long long *, uint32_t *);
struct BatchVariant {
    int block, minb;
    BatchFn fn, media;   // (media: the kernel compiled with the media's tracking, for batches that have some)
};
#define LRC_BATCH_VARIANT(B, M) {B, M, pt::batch_kernel<B, M, false>, pt::batch_kernel<B, M, true>}
const BatchVariant kBatchVariants[] = {
    LRC_BATCH_VARIANT(128, 4), LRC_BATCH_VARIANT(128, 3), LRC_BATCH_VARIANT(128, 5),
    LRC_BATCH_VARIANT(256, 2), LRC_BATCH_VARIANT(64, 8),  LRC_BATCH_VARIANT(256, 3),
};
#undef LRC_BATCH_VARIANT
}  // namespace

int batch_variants() { return (int)(sizeof(kBatchVariants) / sizeof(kBatchVariants[0])); }

int batch_variant_shape(int v, int *block, int *minb) {
    if (v < 0 || v >= batch_variants()) return -1;
    *block = kBatchVariants[v].block;
    *minb = kBatchVariants[v].minb;
    int n = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, kBatchVariants[v].fn, kBatchVariants[v].block, 0)) return -1;
    return n;
}

cudaError_t batch_trace(const BatchJob *d_jobs, uint32_t njobs, unsigned long long ntasks, unsigned long long *d_next,
                        uint32_t *d_status, int variant, int grid, bool media, cudaStream_t st) {
    if (!njobs || !ntasks) return cudaSuccess;
    if (grid < 1 || variant < 0 || variant >= batch_variants()) return cudaErrorInvalidValue;
    void *args[] = {(void *)&d_jobs, (void *)&njobs, (void *)&ntasks, (void *)&d_next, (void *)&d_status};
    const BatchVariant &V = kBatchVariants[variant];
    return cudaLaunchKernel((const void *)(media ? V.media : V.fn), dim3(grid), dim3(V.block), args, 0, st);
}

cudaError_t batch_resolve(const BatchJob *d_jobs, uint32_t njobs, unsigned long long npix, cudaStream_t st) {
    if (!njobs || !npix) return cudaSuccess;
    pt::batch_resolve_kernel<<<(unsigned)((npix + 127) / 128), 128, 0, st>>>(d_jobs, njobs, npix);
    return cudaGetLastError();
}

cudaError_t batch_resolve_run(const BatchJob *d_jobs, const unsigned long long *d_run, int num_sms, cudaStream_t st) {
    pt::batch_resolve_run_kernel<<<16 * num_sms, 128, 0, st>>>(d_jobs, d_run);
    return cudaGetLastError();
}

cudaError_t pt_gradients(const PtScene &S, const PtParams &P, GradTile *d_tiles, uint32_t ntiles, const float4 *d_guide,
                         unsigned long long *d_rays, uint32_t *d_status, cudaStream_t st) {
    if (!ntiles) return cudaSuccess;
    (S.nvol ? pt::grad_kernel<true> : pt::grad_kernel<false>)<<<(ntiles + 127) / 128, 128, 0, st>>>(
        S, P, d_tiles, ntiles, d_guide, d_rays, d_status);
    return cudaGetLastError();
}

cudaError_t pt_intersect(const PtScene &S, const float *d_orig, const float *d_dir, uint64_t n, float tmin, float tmax,
                         int32_t *d_prim, int32_t *d_inst, float *d_t, uint32_t *d_status, cudaStream_t st) {
    if (!n) return cudaSuccess;
    pt::shapes_closest_kernel<<<(unsigned)((n + 127) / 128), 128, 0, st>>>(S, d_orig, d_dir, n, tmin, tmax, d_prim, d_inst,
                                                                           d_t, d_status);
    return cudaGetLastError();
}

// the instances' world boxes (records' words 24-26, 28-30) as builder boxes (8 floats each)
__global__ void inst_boxes_kernel(const float4 *__restrict__ rec, uint32_t n, float4 *__restrict__ boxes) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float4 lo = __ldg(&rec[8 * (size_t)i + 6]), hi = __ldg(&rec[8 * (size_t)i + 7]);
    boxes[2 * (size_t)i] = make_float4(lo.x, lo.y, lo.z, 0.0f);
    boxes[2 * (size_t)i + 1] = make_float4(hi.x, hi.y, hi.z, 0.0f);
}

cudaError_t pt_inst_boxes(const float *d_rec, uint32_t n, float *d_boxes, cudaStream_t st) {
    if (!n) return cudaSuccess;
    inst_boxes_kernel<<<(n + 127) / 128, 128, 0, st>>>(reinterpret_cast<const float4 *>(d_rec), n,
                                                       reinterpret_cast<float4 *>(d_boxes));
    return cudaGetLastError();
}

}  // namespace lrc
