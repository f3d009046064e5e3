// caustics.cu - light-traced caustics on sm_100a: the reference's light_trace_caustics
// (engine/rt/tracer.c:553-665), which its WGSL `ltrace` restates per light path
// (engine/gpu/shaders/trace/trace.wgsl:1415-1511).
//
// A light path leaves a uniform point of the lamp quad in a cosine-distributed direction with
// power Le * area * pi, passes mirrors / glass (its first vertex must be one: lamp -> rough is the
// path tracer's, by next event estimation) and, at every rough vertex after the first, is joined
// to the pinhole camera by a shadow ray; the contribution beta * f * corr * |cos_o| / (dist^2 *
// pixel_area * cos_c^3) goes to the pixel the vertex projects to. Contributions are summed as
// 32.32 fixed-point integers (value * 2^32 / photons, rounded) with 64-bit atomic adds: integer
// addition does not depend on the order, so the image is the same for any launch shape, thread
// count or scheduling, and a batched run gives the plain one's sums to the bit.
//
// Random streams, as the path tracer's two modes:
//   exact: one PCG32 stream per 4096 light paths, seeded as light_trace_caustics seeds its
//          batches (seed ^ b * golden, stream 2b + 1), the paths of a batch in order: the CPU's
//          sums up to transcendental rounding (the parity mode);
//   fast:  one stream per light path (batches of 1), its seed hashed from (seed, path) as the
//          path tracer's fast mode hashes its per-sample seeds.
// Each thread owns a run of streams and regenerates: when its path ends it starts the next one
// at the top of the same bounce loop, so the lanes of a warp keep executing the same code
// (path regeneration) instead of waiting for the warp's longest path.

#include "pt_device.cuh"
#include <algorithm>
#include <cooperative_groups.h>

namespace cg = cooperative_groups;

namespace lrc {
namespace pt {

constexpr unsigned long long LT_BATCH = 4096;   // light paths per random stream in exact mode

// the camera as camera_project (engine/scene/camera.h:48-59) and camera_screen_area (:62) use it
struct LtView {
    V3 origin, fw, horizontal, vertical;
    float hh, vv, pix_area;
    int W, H;
};

__device__ __forceinline__ LtView lt_view(const PtParams &P) {
    LtView c;
    c.origin = P.origin;
    c.horizontal = P.horizontal;
    c.vertical = P.vertical;
    V3 center = vadd(P.upper_left, vsub(vscale(P.horizontal, 0.5f), vscale(P.vertical, 0.5f)));
    c.fw = vsub(center, P.origin);
    c.hh = vdot(P.horizontal, P.horizontal);
    c.vv = vdot(P.vertical, P.vertical);
    c.pix_area = dvd(mul(vlen(P.horizontal), vlen(P.vertical)), mul((float)P.W, (float)P.H));
    c.W = P.W;
    c.H = P.H;
    return c;
}

// camera_project: the point's screen coordinates (s right, t down, [0, 1) on the image) and the
// cosine between the view axis and the direction to it; false behind the eye
__device__ __forceinline__ bool camera_project(const LtView &c, V3 p, float &s, float &t, float &cos_axis) {
    V3 q = vsub(p, c.origin);
    float z = vdot(q, c.fw);
    if (z <= 0.0f) return false;
    V3 e = vsub(vscale(q, dvd(1.0f, z)), c.fw);
    s = add(0.5f, dvd(vdot(e, c.horizontal), c.hh));
    t = sub(0.5f, dvd(vdot(e, c.vertical), c.vv));
    cos_axis = dvd(z, vlen(q));
    return true;
}

// one contribution into the 32.32 sums: per channel value * scale rounded to an integer, left out
// when it is NaN, not positive or absurd (above 1.8e19, the float build's constant)
__device__ __forceinline__ void splat(unsigned long long *__restrict__ sums, uint32_t pix, V3 c, double scale) {
    const float ch[3] = {c.x, c.y, c.z};
#pragma unroll
    for (int k = 0; k < 3; k++) {
        const double cc = __dmul_rn((double)ch[k], scale);
        if (!(cc > 0.0) || cc > (double)1.8e19f) continue;
        atomicAdd(&sums[(size_t)pix * 3 + k], (unsigned long long)__dadd_rn(cc, 0.5));
    }
}

// stream b's generator: exact mode light_trace_caustics' batch seeding, fast mode a hashed seed
__device__ __forceinline__ void lt_stream(Rng &rng, uint64_t seed, unsigned long long b, bool exact) {
    if (exact) rng_seed(rng, seed ^ (b * 0x9E3779B97F4A7C15ull), b * 2 + 1);
    else rng_seed(rng, mix64(seed ^ (b * 0x9E3779B97F4A7C15ull)), b);
}

// the next stream for each lane of the warp that asks: one atomic add per warp
__device__ __forceinline__ unsigned long long fetch_stream(unsigned long long *next) {
    cg::coalesced_group g = cg::coalesced_threads();
    unsigned long long base = 0;
    if (g.thread_rank() == 0) base = atomicAdd(next, (unsigned long long)g.size());
    return g.shfl(base, 0) + g.thread_rank();
}

// Persistent threads (one wave of blocks): each takes streams from the counter `next` (zeroed
// before the launch) as its light paths end; stream b holds light paths [b * per, min((b + 1) *
// per, photons)). INST = false: the world alone (no two-level walk compiled in). MINB: the
// register cap's blocks per SM.
template <bool INST, int MINB>
__global__ void __launch_bounds__(128, MINB) caustics_kernel(PtScene S, PtParams P, unsigned long long photons,
                                                             unsigned long long per, uint64_t seed, double scale,
                                                             unsigned long long *__restrict__ sums,
                                                             unsigned long long *next, unsigned long long *ray_count,
                                                             uint32_t *err) {
    const LtView cam = lt_view(P);
    const Lamp L = load_lamp(S);
    const unsigned long long streams = (photons + per - 1) / per;
    unsigned long long k = 0, end = 0;   // the stream's next light path and its end
    Rng rng;
    V3 ro = v3(0, 0, 0), rd = v3(0, 0, 0), beta = v3(0, 0, 0), thr = v3(0, 0, 0);
    int depth = 0;
    bool alive = false;
    uint32_t rays = 0;
    const bool exact = per > 1;
    for (;;) {
        if (!alive) {
            if (k == end) {                          // the stream is done: the thread's next one
                const unsigned long long b = fetch_stream(next);
                if (b >= streams) break;
                lt_stream(rng, seed, b, exact);
                k = b * per;
                end = min(k + per, photons);
            }
            // emit: a uniform point on the lamp (the v coordinate drawn first, as the C code's
            // argument evaluation draws it), a cosine-distributed direction
            const float a = rng_real(rng), c = rng_real(rng);
            ro = vadd(L.q, vadd(vscale(L.u, c), vscale(L.v, a)));
            const float u1 = rng_real(rng), u2 = rng_real(rng);
            rd = cosine_hemisphere(L.normal, u1, u2);
            beta = vscale(L.le, mul(L.area, PIF));   // Le cos / (pdf_area pdf_dir)
            thr = v3(1, 1, 1);
            depth = 0;
            alive = true;
            k++;
        }
        if (depth >= P.max_depth) {
            alive = false;
            continue;
        }
        Hit h;
        rays++;
        float t;
        int id, inst, tri;
        scene_find<INST>(S, ro, rd, RT_EPS, 1e30f, t, id, inst, tri, err);
        if (S.nvol) {                                // a scattering in a medium: the path tracer's
            float ts;
            int which;
            if (scene_medium_collision(S.vols, S.nvol, ro, rd, 0.0f, id >= 0 || inst >= 0 ? t : 1e30f, rng, ts, which, err)) {
                alive = false;
                continue;
            }
        }
        if (!make_hit(S, ro, rd, t, id, inst, tri, h)) {
            alive = false;
            continue;
        }
        Mat m = load_mat(S.mats, hit_material(S, h) & 63);
        if (textured(m)) m = hit_shading(S, h, ro, rd, vneg(rd), m);
        if (m.type == MAT_LIGHT) {
            alive = false;
            continue;
        }
        Bsdf bsdf = bsdf_make(m, h.front, S.tab);
        const V3 wi = vneg(rd);                      // towards where the light came from
        const float cg = fabsf(vdot(h.ng, wi)), cs = fabsf(vdot(h.n, wi));
        const float corr = cg > 0.0f ? dvd(cs, cg) : 0.0f;   // smooth normals: the adjoint BSDF
        // 1. the rough part to the camera (not at the first vertex)
        if (depth > 0 && bsdf_rough_part(bsdf)) {
            const V3 to_cam = vsub(P.origin, h.p);
            const float dist2 = vdot(to_cam, to_cam), dist = __fsqrt_rn(dist2);
            const V3 wo = vscale(to_cam, dvd(1.0f, dist));
            const float cos_o = vdot(h.ng, wo);      // > 0: the camera on the light's side
            Bsdf bc = cos_o > 0.0f ? bsdf : bsdf_make(m, !h.front, S.tab);
            const V3 nc = cos_o > 0.0f ? h.n : vneg(h.n);
            float pdf;
            const V3 f = cos_o != 0.0f && vdot(nc, wo) > 0.0f ? bsdf_eval(bc, nc, wo, wi, pdf) : v3(0, 0, 0);
            float sx, sy, cos_c;
            if (vmax3(f) > 0.0f && camera_project(cam, h.p, sx, sy, cos_c) && sx >= 0.0f && sy >= 0.0f && sx < 1.0f &&
                sy < 1.0f) {
                const int px = (int)mul(sx, (float)cam.W), py = (int)mul(sy, (float)cam.H);
                if (px < cam.W && py < cam.H) {
                    rays++;
                    if (!scene_occluded<INST>(S, h.p, wo, RT_EPS, mul(dist, sub(1.0f, 1e-4f)), err)) {
                        const float tr = S.nvol ? scene_medium_transmittance(S.vols, S.nvol, h.p, wo, 0.0f, dist, rng, err) : 1.0f;
                        const float wgt = dvd(mul(mul(corr, fabsf(cos_o)), tr),
                                              mul(mul(mul(mul(dist2, cam.pix_area), cos_c), cos_c), cos_c));
                        splat(sums, (uint32_t)py * (uint32_t)cam.W + (uint32_t)px, vscale(vmul(beta, f), wgt), scale);
                    }
                }
            }
        }
        // 2. bounce on, in a direction drawn from the BSDF seen from the light's side
        const float ul = rng_real(rng), v1 = rng_real(rng), v2 = rng_real(rng);
        const float cv = vdot(wi, h.n);
        BsdfSample bs;
        if (cv <= 0.0f) {                            // bsdf_sample: the light below the surface
            alive = false;
            continue;
        }
        bsdf_view(bsdf, cv);
        if (!bsdf_sample_lobe(bsdf, bsdf_pick(bsdf, ul), h.n, wi, v1, v2, bs) || (depth == 0 && !bs.delta)) {
            alive = false;
            continue;
        }
        const float og = vdot(h.ng, bs.l), os = vdot(h.n, bs.l);
        if (!bs.delta && (bs.through ? og >= 0.0f : og <= 0.0f)) {
            alive = false;
            continue;
        }
        V3 fb = bs.w;
        if (!bs.delta) fb = vscale(fb, os != 0.0f ? mul(corr, fabsf(dvd(og, os))) : 0.0f);
        if (bs.through) fb = vscale(fb, mul(bsdf.eta, bsdf.eta));
        beta = vmul(beta, fb);
        thr = vmul(thr, fb);
        if (depth >= RR_START) {
            const float p = rmin(vmax3(thr), 0.95f);
            if (rng_real(rng) >= p) {
                alive = false;
                continue;
            }
            beta = vscale(beta, dvd(1.0f, p));
            thr = vscale(thr, dvd(1.0f, p));
        }
        ro = h.p;
        rd = vnorm(bs.l);
        depth++;
    }
    if (ray_count) {
        unsigned long long r = rays;
        for (int o = 16; o > 0; o >>= 1) r += __shfl_xor_sync(0xffffffffu, r, o);
        if ((threadIdx.x & 31) == 0 && r) atomicAdd(ray_count, r);
    }
}

// image += sums / 2^32 per channel: the sum converted to float (the float build divides the
// 64-bit integer by a float constant), then scaled by 2^-32 (exact) and added
__global__ void caustics_resolve_kernel(const unsigned long long *__restrict__ sums, float *__restrict__ image,
                                        size_t n) {
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        image[i] = __fadd_rn(image[i], __fmul_rn(__ull2float_rn(sums[i]), 2.3283064365386963e-10f));
}

}  // namespace pt

namespace {

using LtKernel = void (*)(PtScene, PtParams, unsigned long long, unsigned long long, uint64_t, double,
                          unsigned long long *, unsigned long long *, unsigned long long *, uint32_t *);
struct LtVariant {
    int minb;
    LtKernel world, inst;
};
const LtVariant kLtVariants[] = {
    {4, pt::caustics_kernel<false, 4>, pt::caustics_kernel<true, 4>},
    {5, pt::caustics_kernel<false, 5>, pt::caustics_kernel<true, 5>},
    {6, pt::caustics_kernel<false, 6>, pt::caustics_kernel<true, 6>},
    {7, pt::caustics_kernel<false, 7>, pt::caustics_kernel<true, 7>},
    {8, pt::caustics_kernel<false, 8>, pt::caustics_kernel<true, 8>},
    {10, pt::caustics_kernel<false, 10>, pt::caustics_kernel<true, 10>},
};
constexpr int kLtDefault = 4;   // the fastest on the plain render's caustics (1M light paths)

}  // namespace

int lt_variants() { return (int)(sizeof kLtVariants / sizeof kLtVariants[0]); }

cudaError_t lt_trace(const PtScene &S, const PtParams &P, unsigned long long photons, uint64_t seed,
                     unsigned long long *d_sums, unsigned long long *d_next, unsigned long long *d_rays,
                     uint32_t *d_status, int num_sms, int variant, cudaStream_t st) {
    if (!photons) return cudaSuccess;
    const LtVariant &V = kLtVariants[variant >= 0 && variant < lt_variants() ? variant : kLtDefault];
    const LtKernel kern = S.ninst ? V.inst : V.world;
    const unsigned long long per = P.exact ? pt::LT_BATCH : 1ull;
    const unsigned long long streams = (photons + per - 1) / per;
    // one wave of persistent blocks (as many as fit at once), fewer when there are few streams
    int fit = 0;
    cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&fit, kern, 128, 0);
    if (e) return e;
    const unsigned long long wave = (unsigned long long)std::max(num_sms, 1) * std::max(fit, 1);
    const unsigned blocks = (unsigned)std::min<unsigned long long>((streams + 127) / 128, wave);
    const double scale = 4294967296.0 / (double)photons;
    e = cudaMemsetAsync(d_next, 0, 8, st);
    if (e) return e;
    kern<<<blocks, 128, 0, st>>>(S, P, photons, per, seed, scale, d_sums, d_next, d_rays, d_status);
    return cudaGetLastError();
}

cudaError_t lt_resolve(const unsigned long long *d_sums, float *d_image, size_t n, int num_sms, cudaStream_t st) {
    if (!n) return cudaSuccess;
    const unsigned blocks = (unsigned)std::min<size_t>((n + 255) / 256, (size_t)std::max(num_sms, 1) * 8);
    pt::caustics_resolve_kernel<<<blocks, 256, 0, st>>>(d_sums, d_image, n);
    return cudaGetLastError();
}

}  // namespace lrc

// ---- the C ABI ------------------------------------------------------------------------------
#include "api_internal.cuh"

using namespace lrcapi;

namespace {

lrc::PtParams lt_params(const lrc_trace_params *p) {
    lrc::PtParams P{};
    P.W = p->width; P.H = p->height; P.y0 = 0; P.rows = p->height;
    P.max_depth = p->max_depth; P.exact = p->exact;
    P.origin = {p->origin[0], p->origin[1], p->origin[2]};
    P.upper_left = {p->upper_left[0], p->upper_left[1], p->upper_left[2]};
    P.horizontal = {p->horizontal[0], p->horizontal[1], p->horizontal[2]};
    P.vertical = {p->vertical[0], p->vertical[1], p->vertical[2]};
    return P;
}

// checks, then traces into d_sums (device, zeroed by the caller when wanted); *skip: nothing to
// trace (no photons, no lamp or nothing perfectly smooth)
int lt_check(lrc_scene *s, const lrc_trace_params *p, uint64_t photons, bool *skip) {
    lrc_ctx *c = s->ctx;
    if (!s->built_n && !s->tlas_n) return fail(c, LRC_E_INVALID, "the scene has nothing built (lrc_scene_build)");
    if (s->ninst && s->tlas_n != s->ninst) return fail(c, LRC_E_INVALID, "instances changed: lrc_scene_build_instances");
    if (!s->d_mats || !s->nmats) return fail(c, LRC_E_INVALID, "the scene has no materials (lrc_scene_set_materials)");
    if (s->light >= (int32_t)s->nprims) return fail(c, LRC_E_INVALID, "the light is not one of the primitives");
    *skip = photons == 0 || s->light < 0 || !s->specular;
    if (!*skip && !s->tables) return lrc_scene_set_tables(s, nullptr, nullptr);
    return LRC_OK;
}

int lt_run(lrc_scene *s, const lrc_trace_params *p, uint64_t photons, uint64_t seed, unsigned long long *d_sums,
           uint64_t *rays) {
    lrc_ctx *c = s->ctx;
    cudaError_t e = cudaSuccess;
    if (!s->d_rays) e = cudaMalloc(&s->d_rays, 256);
    if (!e) e = cudaMemsetAsync(s->d_rays, 0, 8, c->st);
    if (e) return cuda_status(c, e, "ray counter");
    c->timer.begin(LRC_TS_LIGHT, c->st);
    e = lrc::lt_trace(pt_scene(s), lt_params(p), photons, seed, d_sums, s->d_rays + 1, rays ? s->d_rays : nullptr,
                      c->d_status, c->num_sms, c->lt_variant, c->st);
    c->timer.end(c->st);
    return cuda_status(c, e, "light tracing");
}

bool lt_valid(const lrc_scene *s, const lrc_trace_params *p, const void *out) {
    return s && p && out && p->width > 0 && p->height > 0 && p->max_depth >= 0;
}

}  // namespace

extern "C" {

int lrc_caustics_variant(lrc_ctx *c, int variant) {
    if (!c || variant >= lrc::lt_variants()) return LRC_E_INVALID;
    c->lt_variant = variant < 0 ? -1 : variant;
    return lrc::lt_variants();
}

int lrc_caustics(lrc_scene *s, const lrc_trace_params *p, uint64_t photons, uint64_t seed, float *image,
                 uint64_t *rays, unsigned flags) {
    if (!lt_valid(s, p, image)) return LRC_E_INVALID;
    lrc_ctx *c = s->ctx;
    DeviceGuard g(c->device);
    bool skip = false;
    int rc = lt_check(s, p, photons, &skip);
    if (rc) return rc;
    if (rays) *rays = 0;
    if (skip) return LRC_OK;
    const size_t n = (size_t)p->width * p->height * 3;
    cudaError_t e = reserve(&s->d_caus, &s->caus_cap, n * 8);
    if (e) return cuda_status(c, e, "caustic sums");
    auto *d_sums = static_cast<unsigned long long *>(s->d_caus);
    e = cudaMemsetAsync(d_sums, 0, n * 8, c->st);
    float *d_img = image;
    if (!e && !(flags & LRC_DEVICE)) {
        e = reserve(&c->stage, &c->stage_cap, n * 4);
        d_img = static_cast<float *>(c->stage);
        if (!e) e = cudaMemcpyAsync(d_img, image, n * 4, cudaMemcpyHostToDevice, c->st);
    }
    if (e) return cuda_status(c, e, "lrc_caustics");
    rc = lt_run(s, p, photons, seed, d_sums, rays);
    if (rc) return rc;
    e = lrc::lt_resolve(d_sums, d_img, n, c->num_sms, c->st);
    if (!e && !(flags & LRC_DEVICE)) e = cudaMemcpyAsync(image, d_img, n * 4, cudaMemcpyDeviceToHost, c->st);
    unsigned long long nr = 0;
    if (!e && rays) e = cudaMemcpyAsync(&nr, s->d_rays, 8, cudaMemcpyDeviceToHost, c->st);
    if (e) return cuda_status(c, e, "lrc_caustics");
    rc = (flags & LRC_DEVICE) && !rays ? LRC_OK : check_status(c);
    if (rays) *rays = nr;
    return rc;
}

int lrc_caustics_sums(lrc_scene *s, const lrc_trace_params *p, uint64_t photons, uint64_t seed, uint64_t *sums,
                      uint64_t *rays, unsigned flags) {
    if (!lt_valid(s, p, sums)) return LRC_E_INVALID;
    lrc_ctx *c = s->ctx;
    DeviceGuard g(c->device);
    bool skip = false;
    int rc = lt_check(s, p, photons, &skip);
    if (rc) return rc;
    if (rays) *rays = 0;
    if (skip) return LRC_OK;
    const size_t n = (size_t)p->width * p->height * 3;
    auto *d_sums = reinterpret_cast<unsigned long long *>(sums);
    cudaError_t e = cudaSuccess;
    if (!(flags & LRC_DEVICE)) {
        e = reserve(&s->d_caus, &s->caus_cap, n * 8);
        d_sums = static_cast<unsigned long long *>(s->d_caus);
        if (!e) e = cudaMemcpyAsync(d_sums, sums, n * 8, cudaMemcpyHostToDevice, c->st);
    }
    if (e) return cuda_status(c, e, "lrc_caustics_sums");
    rc = lt_run(s, p, photons, seed, d_sums, rays);
    if (rc) return rc;
    if (!(flags & LRC_DEVICE)) e = cudaMemcpyAsync(sums, d_sums, n * 8, cudaMemcpyDeviceToHost, c->st);
    unsigned long long nr = 0;
    if (!e && rays) e = cudaMemcpyAsync(&nr, s->d_rays, 8, cudaMemcpyDeviceToHost, c->st);
    if (e) return cuda_status(c, e, "lrc_caustics_sums");
    rc = (flags & LRC_DEVICE) && !rays ? LRC_OK : check_status(c);
    if (rays) *rays = nr;
    return rc;
}

}  // extern "C"
