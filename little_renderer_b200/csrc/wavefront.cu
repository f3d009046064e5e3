// wavefront.cu - the batch's wavefront path tracer: the bounce loop of trace_path_sampled
// (engine/rt/tracer.c:364-545) cut into four kernels over a pool of M path slots, looped inside
// one CUDA graph by a while node until the batch's task queue is drained.
//
//   advance    one thread per slot: adds the last bounce's shadowed contributions (lamp, then sky),
//              ends a finished sample into its task's sum, starts the task's next sample (camera
//              ray) or takes the next task from the queue (one atomic per warp), and queues the
//              slot's ray;
//   intersect  the closest hit of every queued ray (warps fetch 32 rays at a time);
//   shade      the rest of the bounce: emission, the lamp's and the sky's next event estimation
//              (their shadow rays queued, not traced), the BSDF's sample, Russian roulette;
//   shadow     the any-hit test of every queued shadow ray.
//
// Each kernel is short and holds only its own state, so traversal runs at high occupancy and is not
// held back by shading registers or divergence, and lanes whose path ended take new work at the
// next pass. The arithmetic is pt_device.cuh's, in the order the plain kernels use it (a bounce's
// shadowed contributions are added before the next bounce, lamp first), and each task's samples are
// summed in order: the images are the plain ones to the bit. The slot pool is the wavefront size
// the autotuner picks, with the closest-hit / shadow kernels' launch shape.
#include "pt_device.cuh"

namespace lrc {
namespace pt {

constexpr uint32_t F_PATH = 1u << 8, F_ENDED = 1u << 9;
constexpr unsigned long long NO_TASK = ~0ull;
constexpr int ADV_BLOCK = 256;
constexpr int SHADE_BLOCK = 128;

__device__ __forceinline__ V3 v3f(float4 a) { return v3(a.x, a.y, a.z); }

// block-aggregated append (every thread of the block calls, ADV_BLOCK of them): threads with want
// get consecutive positions from *ctr, in thread order, with one atomic per block
__device__ __forceinline__ uint32_t block_append(uint32_t *ctr, bool want, uint32_t *s_warp, uint32_t &s_base) {
    const uint32_t lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const uint32_t m = __ballot_sync(0xffffffffu, want);
    if (lane == 0) s_warp[w] = __popc(m);
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t t = 0;
        for (int k = 0; k < ADV_BLOCK / 32; k++) {
            const uint32_t c = s_warp[k];
            s_warp[k] = t;
            t += c;
        }
        s_base = t ? atomicAdd(ctr, t) : 0u;
    }
    __syncthreads();
    return s_base + s_warp[w] + __popc(m & ((1u << lane) - 1u));
}

// the slots emptied, the queues cleared, the task queue set to [0, limit)
__global__ void wf_clear_kernel(WfState W) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < 8) W.ctl[i] = 0;
    if (i == 0) {
        W.next[0] = 0;
        W.next[1] = W.run[0];
        W.next[2] = 0;                               // (the counting closest-hit kernel's box tests
        W.next[3] = 0;                               //  and triangle tests)
    }
    if (i >= W.M) return;
    W.task[i] = NO_TASK;
    W.flags[i] = 0;
}

__global__ void __launch_bounds__(ADV_BLOCK) wf_advance_kernel(const BatchJob *__restrict__ jobs, WfState W) {
    const uint32_t njobs = (uint32_t)W.run[1];
    const uint32_t i = blockIdx.x * ADV_BLOCK + threadIdx.x;   // (M is a multiple of the block: every lane has a slot)
    const uint32_t lane = threadIdx.x & 31;
    if (i == 0) {
        W.ctl[1] = 0;
        W.ctl[2] = 0;
        W.ctl[3] = 0;
    }
    const uint32_t f0 = W.flags[i];
    unsigned long long task = W.task[i];
    int j = task != NO_TASK ? (int)W.job[i] : -1;
    uint32_t kk = 0, trays = 0;
    float4 sum = make_float4(0, 0, 0, 0);
    float4 mom = make_float4(0, 0, 0, 0);
    bool path = (f0 & F_PATH) != 0, new_task = false, wrote_sum = false;
    if (j >= 0) {
        kk = W.kk[i];
        trays = W.trays[i];
        sum = W.sum[i];
        if (jobs[j].pmom) mom = W.mom[i];
    }
    if (path) {
        const BatchJob &J = jobs[j];
        const float4 r = W.rad[i];
        V3 rad = v3f(r);
        if (f0 & (NEE_L | NEE_E)) {                  // (each held to the indirect cap when it was on)
            const V3 thr = v3f(W.nthr[i]);
            const bool cap = (f0 & NEE_ROUGH) != 0;
            const float k = J.P.indirect_clamp;
            if (f0 & NEE_L)
                rad = vadd(rad, indirect_cap(vmul(thr, (f0 & NEE_RL) && W.vis[2 * i] ? v3f(W.nvl[i]) : v3(0, 0, 0)), cap, k));
            if (f0 & NEE_E)
                rad = vadd(rad, indirect_cap(vmul(thr, (f0 & NEE_RE) && W.vis[2 * i + 1] ? v3f(W.nve[i]) : v3(0, 0, 0)), cap, k));
        }
        if (f0 & F_ENDED) {                          // the sample into its task's sum
            const V3 s = is_number(rad) ? clamp_sample(rad, J.P.clamp) : v3(0, 0, 0);
            const V3 c = vadd(v3(sum.x, sum.y, sum.z), s);
            sum = make_float4(c.x, c.y, c.z, sum.w + 1.0f);
            if (J.pmom) {                            // the denoiser's moments
                const uint2 xy = W.xy[i];
                const float l = sample_luma(s, J.P.guide[(uint64_t)xy.y * (uint32_t)J.P.W + xy.x]);
                mom = make_float4(mom.x + l, mom.y + l * l, l, 0.0f);
            }
            wrote_sum = true;
            kk += (uint32_t)J.P.group;
            path = false;
        } else if (f0 & (NEE_L | NEE_E)) {
            W.rad[i] = make_float4(rad.x, rad.y, rad.z, r.w);
        }
    }
    if (!path && j >= 0) {
        const BatchJob &J = jobs[j];
        if (kk >= (uint32_t)(J.P.spp0 + J.P.spp)) {  // the task is done
            const unsigned long long l = task - J.task0;
            J.partial[l] = sum;
            J.prays[l] = trays;
            if (J.pmom) J.pmom[l] = mom;
            j = -1;
            task = NO_TASK;
            wrote_sum = false;
        }
    }
    // lanes without a task take the queue's next ones (one atomic per warp)
    const bool need = j < 0 && *reinterpret_cast<volatile unsigned long long *>(&W.next[0]) < W.next[1];
    const uint32_t m = __ballot_sync(0xffffffffu, need);
    if (m) {
        const int leader = __ffs(m) - 1;
        unsigned long long base = 0;
        if ((int)lane == leader) base = atomicAdd(&W.next[0], (unsigned long long)__popc(m));
        base = __shfl_sync(0xffffffffu, base, leader);
        if (need) {
            const unsigned long long t = base + __popc(m & ((1u << lane) - 1u));
            if (t < W.next[1]) {
                task = t;
                j = (int)batch_job_of(jobs, njobs, t);
                const BatchJob &J = jobs[j];
                const unsigned long long l = t - J.task0;
                const uint32_t g = (uint32_t)J.P.group;
                const unsigned long long pl = l / g;
                const uint32_t slot = (uint32_t)(l - pl * g);
                const uint32_t x = (uint32_t)(pl % (uint32_t)J.P.W), y = (uint32_t)J.P.y0 + (uint32_t)(pl / (uint32_t)J.P.W);
                W.xy[i] = make_uint2(x, y);
                kk = (uint32_t)J.P.spp0 + slot;
                sum = make_float4(0, 0, 0, 0);
                mom = make_float4(0, 0, 0, 0);
                trays = 0;
                new_task = true;
                wrote_sum = true;
                if (J.P.exact) {                     // trace_image's per-pixel stream, all samples in order
                    const uint64_t pixel = (uint64_t)y * (uint32_t)J.P.W + x;
                    Rng rng;
                    rng_seed(rng, 0x853c49e6748fea9bull ^ (pixel * 0x9E3779B97F4A7C15ull) ^ (J.P.seed * 0xD1B54A32D192ED03ull),
                             pixel);
                    W.rng[i] = make_ulonglong2(rng.state, rng.inc);
                }
            }
        }
    }
    if (!path && j >= 0) {                           // the task's next sample: its camera ray
        const BatchJob &J = jobs[j];
        const uint2 xy = W.xy[i];
        const uint64_t pixel = (uint64_t)xy.y * (uint32_t)J.P.W + xy.x;
        Rng rng;
        if (J.P.exact) {
            const ulonglong2 r = W.rng[i];
            rng.state = r.x;
            rng.inc = r.y;
        } else {
            rng_seed(rng, mix64(pixel * 0x9E3779B97F4A7C15ull ^ ((uint64_t)kk << 40) ^ J.P.seed), pixel);
        }
        Sampler sm{&rng, kk, (uint32_t)J.P.seed * 0x9e3779b9u, (int)xy.x, (int)xy.y, J.P.sampler_on, J.S.mask};
        float jx, jy;
        sampler_2d(sm, 0, jx, jy);
        const float u = dvd(add((float)xy.x, jx), (float)J.P.W), v = dvd(add((float)xy.y, jy), (float)J.P.H);
        V3 o, d;
        camera_ray(J.P, u, v, o, d);
        PathState ps;
        path_begin(J.P.mis || J.S.nvol, o, d, ps, J.P.skip_caustics, J.P.indirect_clamp);
        W.ro[i] = make_float4(ps.ro.x, ps.ro.y, ps.ro.z, ps.bounce_pdf);
        W.rd[i] = make_float4(ps.rd.x, ps.rd.y, ps.rd.z, __int_as_float(ps.depth | (ps.emit << 16) | (ps.caus << 24)));
        W.thr[i] = make_float4(ps.thr.x, ps.thr.y, ps.thr.z, 0.0f);
        W.rad[i] = make_float4(0, 0, 0, 0);
        W.rng[i] = make_ulonglong2(rng.state, rng.inc);
        path = true;
    }
    if (path) trays++;                               // its closest-hit ray
    __shared__ uint32_t s_warp[ADV_BLOCK / 32];
    __shared__ uint32_t s_base;
    const uint32_t q = block_append(&W.ctl[0], path, s_warp, s_base);
    if (path) W.rq[q] = i;
    W.flags[i] = path ? F_PATH : 0;
    if (new_task || task == NO_TASK) {
        W.task[i] = task;
        if (task != NO_TASK) W.job[i] = (uint32_t)j;
    }
    if (j >= 0) {
        W.kk[i] = kk;
        W.trays[i] = trays;
        if (wrote_sum) {
            W.sum[i] = sum;
            if (jobs[j].pmom) W.mom[i] = mom;
        }
    }
}

// the closest hit of every queued ray (warps fetch 32 rays at a time); sets the loop's condition
// (another pass while rays are queued)
// (COUNT: also the walks' box and triangle tests into W.next[2], W.next[3]; only the stepped runs
// that measure the engine's algorithmic bytes launch it)
template <int BLOCK, int MINB, bool INST, bool COUNT = false>
__global__ void __launch_bounds__(BLOCK, MINB) wf_intersect_kernel(const BatchJob *__restrict__ jobs, WfState W, uint32_t *err,
                                                                   cudaGraphConditionalHandle cond, int use_cond) {
    const uint32_t max_passes = (uint32_t)W.run[2];
    // (the pass counter is advanced by the shadow kernel, so every block of this one and of the
    // shade kernel reads the same value)
    uint32_t count = *reinterpret_cast<volatile uint32_t *>(&W.ctl[0]);
    if (W.ctl[4] >= max_passes) {                    // (never with sound inputs: stop, say so)
        if (blockIdx.x == 0 && threadIdx.x == 0) atomicOr(err, ST_LOOP);
        count = 0;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        if (use_cond) cudaGraphSetConditional(cond, count > 0 ? 1u : 0u);
        else W.ctl[5] = count;                       // (the stepped loop's host reads it)
    }
    const uint32_t lane = threadIdx.x & 31;
    uint32_t cnt[2] = {0, 0};
    for (;;) {
        uint32_t base = 0;
        if (lane == 0) base = atomicAdd(&W.ctl[2], 32u);
        base = __shfl_sync(0xffffffffu, base, 0);
        if (base >= count) break;
        const uint32_t k = base + lane;
        if (k < count) {
            const uint32_t s = W.rq[k];
            const BatchJob &J = jobs[W.job[s]];
            const V3 o = v3f(W.ro[s]), d = v3f(W.rd[s]);
            float t;
            int id, inst, tri;
            scene_find<INST, COUNT>(J.S, o, d, RT_EPS, 1e30f, t, id, inst, tri, err, cnt);
            W.hit[s] = make_float4(t, __int_as_float(id), __int_as_float(inst), __int_as_float(tri));
        }
    }
    if constexpr (COUNT) {
        unsigned long long a = cnt[0], b = cnt[1];
        for (int o = 16; o > 0; o >>= 1) {
            a += __shfl_xor_sync(0xffffffffu, a, o);
            b += __shfl_xor_sync(0xffffffffu, b, o);
        }
        if (lane == 0 && (a | b)) {
            atomicAdd(&W.next[2], a);
            atomicAdd(&W.next[3], b);
        }
    }
}

// the rest of every queued path's bounce; its shadow rays into the shadow queue
template <int SMINB>
__global__ void __launch_bounds__(SHADE_BLOCK, SMINB) wf_shade_kernel(const BatchJob *__restrict__ jobs, WfState W,
                                                                       uint32_t *err) {
    const uint32_t max_passes = (uint32_t)W.run[2];
    const uint32_t count = W.ctl[4] >= max_passes ? 0u : *reinterpret_cast<volatile uint32_t *>(&W.ctl[0]);
    const uint32_t lane = threadIdx.x & 31;
    const uint32_t warps = gridDim.x * (SHADE_BLOCK / 32);
    for (uint32_t base = (blockIdx.x * (SHADE_BLOCK / 32) + (threadIdx.x >> 5)) * 32; base < count; base += warps * 32) {
        const uint32_t k = base + lane;
        const bool live = k < count;
        Nee nee;
        nee.flags = 0;
        uint32_t s = 0;
        if (live) {
            s = W.rq[k];
            const BatchJob &J = jobs[W.job[s]];
            const float4 ro = W.ro[s], rd = W.rd[s], th = W.thr[s], ra = W.rad[s];
            PathState ps;
            ps.ro = v3f(ro);
            ps.bounce_pdf = ro.w;
            ps.rd = v3f(rd);
            const int de = __float_as_int(rd.w);
            ps.depth = de & 0xffff;
            ps.emit = (de >> 16) & 0xff;
            ps.caus = de >> 24;
            ps.thr = v3f(th);
            ps.radiance = v3f(ra);
            ps.icap = J.P.indirect_clamp;
            const ulonglong2 r = W.rng[s];
            Rng rng;
            rng.state = r.x;
            rng.inc = r.y;
            const uint2 xy = W.xy[s];
            Sampler sm{&rng, W.kk[s], (uint32_t)J.P.seed * 0x9e3779b9u, (int)xy.x, (int)xy.y, J.P.sampler_on, J.S.mask};
            const float4 hh = W.hit[s];
            Hit h;
            const bool found = make_hit(J.S, ps.ro, ps.rd, hh.x, __float_as_int(hh.y), __float_as_int(hh.z),
                                        __float_as_int(hh.w), h);
            uint32_t rays = 0;
            const bool cont = path_shade<true>(J.S, J.P.max_depth, J.P.mis, ps, found, h, sm, err, rays, nee);
            W.ro[s] = make_float4(ps.ro.x, ps.ro.y, ps.ro.z, ps.bounce_pdf);
            W.rd[s] = make_float4(ps.rd.x, ps.rd.y, ps.rd.z, __int_as_float(ps.depth | (ps.emit << 16) | (ps.caus << 24)));
            W.thr[s] = make_float4(ps.thr.x, ps.thr.y, ps.thr.z, 0.0f);
            W.rad[s] = make_float4(ps.radiance.x, ps.radiance.y, ps.radiance.z, 0.0f);
            W.rng[s] = make_ulonglong2(rng.state, rng.inc);
            if (rays) W.trays[s] += rays;
            W.flags[s] = F_PATH | (cont ? 0u : F_ENDED) | nee.flags;
            if (nee.flags & (NEE_L | NEE_E)) W.nthr[s] = make_float4(nee.thr.x, nee.thr.y, nee.thr.z, 0.0f);
            if (nee.flags & NEE_L) W.nvl[s] = make_float4(nee.vl.x, nee.vl.y, nee.vl.z, 0.0f);
            if (nee.flags & NEE_E) W.nve[s] = make_float4(nee.ve.x, nee.ve.y, nee.ve.z, 0.0f);
        }
        const bool rl = (nee.flags & NEE_RL) != 0, re = (nee.flags & NEE_RE) != 0;
        // (the warp's lamp rays, then its sky rays, from one atomic)
        const uint32_t ml = __ballot_sync(0xffffffffu, rl), me = __ballot_sync(0xffffffffu, re);
        uint32_t qb = 0;
        if (lane == 0 && (ml | me)) qb = atomicAdd(&W.ctl[1], (uint32_t)(__popc(ml) + __popc(me)));
        qb = __shfl_sync(0xffffffffu, qb, 0);
        const uint32_t lt = (1u << lane) - 1u;
        const uint32_t ql = qb + __popc(ml & lt), qe = qb + __popc(ml) + __popc(me & lt);
        if (rl) {
            W.sq_o[ql] = make_float4(nee.p.x, nee.p.y, nee.p.z, __uint_as_float(s << 1));
            W.sq_d[ql] = make_float4(nee.wl.x, nee.wl.y, nee.wl.z, nee.tl);
        }
        if (re) {
            W.sq_o[qe] = make_float4(nee.p.x, nee.p.y, nee.p.z, __uint_as_float(s << 1 | 1u));
            W.sq_d[qe] = make_float4(nee.we.x, nee.we.y, nee.we.z, 1e30f);
        }
    }
}

// the any-hit test of every queued shadow ray; clears the ray queue and counts the pass for the
// next one
template <int BLOCK, int MINB, bool INST>
__global__ void __launch_bounds__(BLOCK, MINB) wf_shadow_kernel(const BatchJob *__restrict__ jobs, WfState W, uint32_t *err) {
    const uint32_t count = *reinterpret_cast<volatile uint32_t *>(&W.ctl[1]);
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        W.ctl[0] = 0;
        W.ctl[4]++;
    }
    const uint32_t lane = threadIdx.x & 31;
    for (;;) {
        uint32_t base = 0;
        if (lane == 0) base = atomicAdd(&W.ctl[3], 32u);
        base = __shfl_sync(0xffffffffu, base, 0);
        if (base >= count) break;
        const uint32_t k = base + lane;
        if (k < count) {
            const float4 o = W.sq_o[k], d = W.sq_d[k];
            const uint32_t e = __float_as_uint(o.w);
            const BatchJob &J = jobs[W.job[e >> 1]];
            W.vis[e] = scene_occluded<INST>(J.S, v3f(o), v3f(d), RT_EPS, d.w, err) ? 0 : 1;
        }
    }
}

}  // namespace pt

namespace {
struct WfVariant {
    int block, minb, shade_minb;
    const void *isect, *shadow, *shade;
    const void *isect_world, *shadow_world;   // (for batches without instances)
};
#define LRC_WF_VARIANT(B, M, S)                                                                                 \
    {B, M, S, (const void *)pt::wf_intersect_kernel<B, M, true>, (const void *)pt::wf_shadow_kernel<B, M, true>,  \
     (const void *)pt::wf_shade_kernel<S>, (const void *)pt::wf_intersect_kernel<B, M, false>,                  \
     (const void *)pt::wf_shadow_kernel<B, M, false>}
const WfVariant kWfVariants[] = {
    LRC_WF_VARIANT(128, 4, 1), LRC_WF_VARIANT(128, 6, 1), LRC_WF_VARIANT(128, 8, 1), LRC_WF_VARIANT(256, 4, 1),
    LRC_WF_VARIANT(64, 12, 1), LRC_WF_VARIANT(128, 6, 5), LRC_WF_VARIANT(128, 8, 5), LRC_WF_VARIANT(128, 8, 6),
    LRC_WF_VARIANT(128, 4, 4), LRC_WF_VARIANT(128, 8, 4),
};
#undef LRC_WF_VARIANT
static_assert(sizeof(kWfVariants) / sizeof(kWfVariants[0]) > LRC_WAVEFRONT_DEFAULT_VARIANT &&
              LRC_WAVEFRONT_DEFAULT_VARIANT == 9, "the default shape is (128, 8, 4)");
size_t a256(size_t x) { return (x + 255) / 256 * 256; }
}  // namespace

int wf_variants() { return (int)(sizeof(kWfVariants) / sizeof(kWfVariants[0])); }

int wf_variant_shape(int v, int *block, int *minb) {
    if (v < 0 || v >= wf_variants()) return -1;
    *block = kWfVariants[v].block;
    *minb = kWfVariants[v].minb;
    int n = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, kWfVariants[v].isect, kWfVariants[v].block, 0)) return -1;
    return n;
}

size_t wf_bytes(uint32_t M) {
    const size_t m = M;
    return a256(m * 8) + 5 * a256(m * 4) + a256(m * 8) + 10 * a256(m * 16) + a256(m * 16) + a256(m * 2) + a256(m * 4) +
           2 * a256(m * 2 * 16) + 256 + 256 + 256;
}

WfState wf_carve(void *base, uint32_t M) {
    const size_t m = M;
    char *p = reinterpret_cast<char *>((reinterpret_cast<uintptr_t>(base) + 255) / 256 * 256);
    auto take = [&](size_t bytes) {
        char *q = p;
        p += a256(bytes);
        return q;
    };
    WfState W{};
    W.M = M;
    W.task = reinterpret_cast<unsigned long long *>(take(m * 8));
    W.job = reinterpret_cast<uint32_t *>(take(m * 4));
    W.kk = reinterpret_cast<uint32_t *>(take(m * 4));
    W.trays = reinterpret_cast<uint32_t *>(take(m * 4));
    W.flags = reinterpret_cast<uint32_t *>(take(m * 4));
    W.rq = reinterpret_cast<uint32_t *>(take(m * 4));
    W.xy = reinterpret_cast<uint2 *>(take(m * 8));
    W.sum = reinterpret_cast<float4 *>(take(m * 16));
    W.ro = reinterpret_cast<float4 *>(take(m * 16));
    W.rd = reinterpret_cast<float4 *>(take(m * 16));
    W.thr = reinterpret_cast<float4 *>(take(m * 16));
    W.rad = reinterpret_cast<float4 *>(take(m * 16));
    W.hit = reinterpret_cast<float4 *>(take(m * 16));
    W.nthr = reinterpret_cast<float4 *>(take(m * 16));
    W.nvl = reinterpret_cast<float4 *>(take(m * 16));
    W.nve = reinterpret_cast<float4 *>(take(m * 16));
    W.rng = reinterpret_cast<ulonglong2 *>(take(m * 16));
    W.mom = reinterpret_cast<float4 *>(take(m * 16));
    W.vis = reinterpret_cast<uint8_t *>(take(m * 2));
    take(m * 4);    // (spare)
    W.sq_o = reinterpret_cast<float4 *>(take(m * 2 * 16));
    W.sq_d = reinterpret_cast<float4 *>(take(m * 2 * 16));
    W.ctl = reinterpret_cast<uint32_t *>(take(64));
    W.next = reinterpret_cast<unsigned long long *>(take(64));
    W.run = reinterpret_cast<unsigned long long *>(take(64));
    return W;
}

cudaError_t wf_set_run(const WfState &W, const unsigned long long *h_run4, cudaStream_t st) {
    return cudaMemcpyAsync(W.run, h_run4, 32, cudaMemcpyHostToDevice, st);
}

cudaError_t wf_capture_loop(const BatchJob *d_jobs, const WfState &W, uint32_t *d_status, int variant, bool instances,
                            int num_sms, cudaStream_t st, cudaStream_t body_st) {
    if (variant < 0 || variant >= wf_variants() || W.M == 0 || W.M % pt::ADV_BLOCK) return cudaErrorInvalidValue;
    cudaStreamCaptureStatus cs;
    cudaGraph_t g = nullptr;
    const cudaGraphNode_t *deps = nullptr;
    size_t nd = 0;
    cudaError_t e = cudaStreamGetCaptureInfo(st, &cs, nullptr, &g, &deps, &nd);
    if (e) return e;
    if (cs != cudaStreamCaptureStatusActive) return cudaErrorStreamCaptureUnmatched;
    pt::wf_clear_kernel<<<(W.M + 255) / 256, 256, 0, st>>>(W);
    e = cudaGetLastError();
    if (e) return e;
    e = cudaStreamGetCaptureInfo(st, &cs, nullptr, &g, &deps, &nd);
    if (e) return e;
    cudaGraphConditionalHandle cond;
    e = cudaGraphConditionalHandleCreate(&cond, g, 1, cudaGraphCondAssignDefault);
    if (e) return e;
    cudaGraphNodeParams cp{};
    cp.type = cudaGraphNodeTypeConditional;
    cp.conditional.handle = cond;
    cp.conditional.type = cudaGraphCondTypeWhile;
    cp.conditional.size = 1;
    cudaGraphNode_t node;
    e = cudaGraphAddNode(&node, g, deps, nd, &cp);
    if (e) return e;
    cudaGraph_t body = cp.conditional.phGraph_out[0];
    e = cudaStreamBeginCaptureToGraph(body_st, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal);
    if (e) return e;
    const WfVariant &V = kWfVariants[variant];
    const void *isect = instances ? V.isect : V.isect_world, *shadow = instances ? V.shadow : V.shadow_world;
    int per_sm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, isect, V.block, 0);
    const int grid = std::max(per_sm, 1) * num_sms;
    int shade_per_sm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&shade_per_sm, V.shade, pt::SHADE_BLOCK, 0);
    const int shade_grid = std::max(shade_per_sm, 1) * num_sms;
    WfState w = W;
    pt::wf_advance_kernel<<<W.M / pt::ADV_BLOCK, pt::ADV_BLOCK, 0, body_st>>>(d_jobs, w);
    int use_cond = 1;
    void *iargs[] = {(void *)&d_jobs, (void *)&w, (void *)&d_status, (void *)&cond, (void *)&use_cond};
    e = cudaLaunchKernel(isect, dim3(grid), dim3(V.block), iargs, 0, body_st);
    if (!e) {
        void *hargs[] = {(void *)&d_jobs, (void *)&w, (void *)&d_status};
        e = cudaLaunchKernel(V.shade, dim3(shade_grid), dim3(pt::SHADE_BLOCK), hargs, 0, body_st);
    }
    if (!e) {
        void *sargs[] = {(void *)&d_jobs, (void *)&w, (void *)&d_status};
        e = cudaLaunchKernel(shadow, dim3(grid), dim3(V.block), sargs, 0, body_st);
    }
    if (!e) e = cudaGetLastError();
    cudaGraph_t out = nullptr;
    cudaError_t e2 = cudaStreamEndCapture(body_st, &out);
    if (e) return e;
    if (e2) return e2;
    return cudaStreamUpdateCaptureDependencies(st, &node, 1, cudaStreamSetCaptureDependencies);
}

cudaError_t wf_run_stepped(const BatchJob *d_jobs, uint32_t njobs, unsigned long long ntasks, const WfState &W,
                           uint32_t *d_status, int variant, bool instances, int num_sms, uint32_t max_passes,
                           cudaStream_t st, WfStepStats *stats, bool count) {
    if (variant < 0 || variant >= wf_variants() || W.M == 0 || W.M % pt::ADV_BLOCK) return cudaErrorInvalidValue;
    const WfVariant &V = kWfVariants[variant];
    const void *isect = instances ? V.isect : V.isect_world, *shadow = instances ? V.shadow : V.shadow_world;
    if (stats && count && V.block == 128 && V.minb == 4)   // (the counting kernels: two of the shapes)
        isect = instances ? (const void *)pt::wf_intersect_kernel<128, 4, true, true>
                          : (const void *)pt::wf_intersect_kernel<128, 4, false, true>;
    else if (stats && count && V.block == 128 && V.minb == 8)
        isect = instances ? (const void *)pt::wf_intersect_kernel<128, 8, true, true>
                          : (const void *)pt::wf_intersect_kernel<128, 8, false, true>;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    if (stats) {
        *stats = WfStepStats{};
        if (cudaEventCreate(&e0) || cudaEventCreate(&e1)) return cudaGetLastError();
    }
    int per_sm = 0, shade_per_sm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, isect, V.block, 0);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&shade_per_sm, V.shade, pt::SHADE_BLOCK, 0);
    const int grid = std::max(per_sm, 1) * num_sms, shade_grid = std::max(shade_per_sm, 1) * num_sms;
    WfState w = W;
    cudaGraphConditionalHandle cond = 0;
    int use_cond = 0;
    const unsigned long long run[4] = {ntasks, njobs, max_passes, 0};
    cudaError_t e = cudaMemcpyAsync(W.run, run, 32, cudaMemcpyHostToDevice, st);   // (pageable: staged before it returns)
    if (!e) {
        pt::wf_clear_kernel<<<(W.M + 255) / 256, 256, 0, st>>>(w);
        e = cudaGetLastError();
    }
    for (uint32_t pass = 0; !e && pass <= max_passes; pass++) {
        pt::wf_advance_kernel<<<W.M / pt::ADV_BLOCK, pt::ADV_BLOCK, 0, st>>>(d_jobs, w);
        void *iargs[] = {(void *)&d_jobs, (void *)&w, (void *)&d_status, (void *)&cond, (void *)&use_cond};
        if (stats) cudaEventRecord(e0, st);
        e = cudaLaunchKernel(isect, dim3(grid), dim3(V.block), iargs, 0, st);
        if (stats) cudaEventRecord(e1, st);
        if (e) break;
        void *hargs[] = {(void *)&d_jobs, (void *)&w, (void *)&d_status};
        e = cudaLaunchKernel(V.shade, dim3(shade_grid), dim3(pt::SHADE_BLOCK), hargs, 0, st);
        if (e) break;
        void *sargs[] = {(void *)&d_jobs, (void *)&w, (void *)&d_status};
        e = cudaLaunchKernel(shadow, dim3(grid), dim3(V.block), sargs, 0, st);
        uint32_t queued = 0;
        if (!e) e = cudaMemcpyAsync(&queued, &W.ctl[5], 4, cudaMemcpyDeviceToHost, st);
        if (!e) e = cudaStreamSynchronize(st);
        if (!e && stats) {
            float ms = 0;
            cudaEventElapsedTime(&ms, e0, e1);
            stats->isect_ms += ms;
            stats->isect_rays += queued;
            stats->isect_launches++;
            stats->launches += 4;
        }
        if (!e && queued == 0) break;
    }
    if (stats) {
        unsigned long long c[2] = {0, 0};
        if (!e) e = cudaMemcpy(c, &W.next[2], 16, cudaMemcpyDeviceToHost);
        stats->box_tests = c[0];
        stats->tri_tests = c[1];
        stats->launches += 1;
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
    }
    return e;
}

}  // namespace lrc
