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
#include "lrc_internal.cuh"
#include "bsdf.cuh"
#include <algorithm>

namespace lrc {
namespace pt {

constexpr float RT_EPS = 2e-3f;
constexpr float RT_SHADOW_MARGIN = 2e-2f;
constexpr int RR_START = 3;
constexpr int PT_STACK = 64;

struct Hit {
    float t;
    V3 p, n, ng;
    int front;
    int prim;
    int inst;
};

__device__ __forceinline__ float4 ld4(const float4 *p) { return __ldg(p); }

// ---- shape tests (engine/rt/intersect.h:66-112), rounded as the C code rounds them -----------
__device__ __forceinline__ bool hit_sphere_t(V3 c, float radius, V3 o, V3 d, float tmin, float tmax, float &tout) {
    V3 oc = vsub(c, o);
    float a = vdot(d, d);
    float hh = vdot(d, oc);
    float cc = sub(vdot(oc, oc), mul(radius, radius));
    float disc = sub(mul(hh, hh), mul(a, cc));
    if (disc < 0.0f) return false;
    float sq = __fsqrt_rn(disc);
    float t = dvd(sub(hh, sq), a);
    if (t <= tmin || t >= tmax) {
        t = dvd(add(hh, sq), a);
        if (t <= tmin || t >= tmax) return false;
    }
    tout = t;
    return true;
}
__device__ __forceinline__ bool hit_quad_t(const float4 *pr, V3 o, V3 d, float tmin, float tmax, float &tout) {
    float4 q = ld4(pr + 1), u = ld4(pr + 2), v = ld4(pr + 3), nd = ld4(pr + 4), w = ld4(pr + 5);
    V3 nrm = v3(nd.x, nd.y, nd.z);
    float denom = vdot(nrm, d);
    if (fabsf(denom) < 1e-12f) return false;
    float t = dvd(sub(nd.w, vdot(nrm, o)), denom);
    if (t <= tmin || t >= tmax) return false;
    V3 p = vadd(o, vscale(d, t));
    V3 rel = vsub(p, v3(q.x, q.y, q.z));
    V3 ww = v3(w.x, w.y, w.z);
    float a = vdot(ww, vcross(rel, v3(v.x, v.y, v.z)));
    float b = vdot(ww, vcross(v3(u.x, u.y, u.z), rel));
    if (a < 0.0f || a > 1.0f || b < 0.0f || b > 1.0f) return false;
    tout = t;
    return true;
}
__device__ __forceinline__ bool hit_tri_t(const float4 *tp, V3 o, V3 d, float tmin, float tmax, float &tout) {
    float4 q = ld4(tp), u = ld4(tp + 1), v = ld4(tp + 2);
    V3 vv = v3(v.x, v.y, v.z), uu = v3(u.x, u.y, u.z);
    V3 pvec = vcross(d, vv);
    float det = vdot(uu, pvec);
    if (fabsf(det) < 1e-12f) return false;
    float inv = dvd(1.0f, det);
    V3 tvec = vsub(o, v3(q.x, q.y, q.z));
    float b1 = mul(vdot(tvec, pvec), inv);
    if (b1 < 0.0f || b1 > 1.0f) return false;
    V3 qvec = vcross(tvec, uu);
    float b2 = mul(vdot(d, qvec), inv);
    if (b2 < 0.0f || add(b1, b2) > 1.0f) return false;
    float t = mul(vdot(vv, qvec), inv);
    if (t <= tmin || t >= tmax) return false;
    tout = t;
    return true;
}

// shape `id` (primitives, then triangles) against the ray
__device__ __forceinline__ bool shape_test(const PtScene &S, uint32_t id, V3 o, V3 d, float tmin, float tmax, float &t) {
    if (id < S.nprims) {
        const float4 *pr = S.prims + 6 * (size_t)id;
        float4 c = ld4(pr), qf = ld4(pr + 1);
        if (qf.w == 0.0f) return hit_sphere_t(v3(c.x, c.y, c.z), c.w, o, d, tmin, tmax, t);
        return hit_quad_t(pr, o, d, tmin, tmax, t);
    }
    return hit_tri_t(S.tris + 3 * (size_t)(id - S.nprims), o, d, tmin, tmax, t);
}

struct RayBox {
    float ix, iy, iz, ax, ay, az;
};
__device__ __forceinline__ RayBox ray_box(V3 o, V3 d) {
    auto inv = [](float x) { return 1.0f / (fabsf(x) < 1e-20f ? copysignf(1e-20f, x) : x); };
    RayBox r;
    r.ix = inv(d.x); r.iy = inv(d.y); r.iz = inv(d.z);
    r.ax = o.x * r.ix; r.ay = o.y * r.iy; r.az = o.z * r.iz;
    return r;
}
// conservative slab test (boxes are padded by 1e-3): entry distance or +inf
__device__ __forceinline__ float slab(const RayBox &r, float4 lo, float4 hi, float tmin, float tmax) {
    float x0 = fmaf(lo.x, r.ix, -r.ax), x1 = fmaf(hi.x, r.ix, -r.ax);
    float y0 = fmaf(lo.y, r.iy, -r.ay), y1 = fmaf(hi.y, r.iy, -r.ay);
    float z0 = fmaf(lo.z, r.iz, -r.az), z1 = fmaf(hi.z, r.iz, -r.az);
    float tn = fmaxf(fmaxf(fminf(x0, x1), fminf(y0, y1)), fmaxf(fminf(z0, z1), tmin));
    float tf = fminf(fminf(fmaxf(x0, x1), fmaxf(y0, y1)), fminf(fmaxf(z0, z1), tmax));
    return tn <= tf ? tn : __int_as_float(0x7f800000);
}

// The closest (ANY = false) or any (ANY = true) shape of one BVH in (tmin, best): the shape id,
// or -1. A leaf's entries are tested in order; a hit at the same t as the best is not taken
// (t >= tmax rejects), as the CPU's walk does.
template <bool ANY>
__device__ int32_t walk(const PtScene &S, const float4 *nodes, uint32_t root, uint32_t nnodes, const uint32_t *aux,
                        uint32_t naux, V3 o, V3 d, float tmin, float &best, uint32_t *err) {
    RayBox rb = ray_box(o, d);
    float4 r0 = ld4(&nodes[2 * (size_t)root]), r1 = ld4(&nodes[2 * (size_t)root + 1]);
    if (!(slab(rb, r0, r1, tmin, best) <= best)) return -1;
    uint2 stack[PT_STACK];
    int sp = 0;
    int32_t hit = -1;
    uint32_t a = __float_as_uint(r0.w), b = __float_as_uint(r1.w);
    while (true) {
        if (b & LEAF_BIT) {
            const uint32_t count = b & ~LEAF_BIT;
            if (a >= naux || count > naux - a) { atomicOr(err, ST_BAD_TREE); return -1; }
            for (uint32_t k = 0; k < count; k++) {
                uint32_t id = __ldg(&aux[a + k]);
                if (id >= S.nprims + S.ntris) { atomicOr(err, ST_BAD_TREE); return -1; }
                float t;
                if (shape_test(S, id, o, d, tmin, best, t)) {
                    best = t;
                    hit = (int32_t)id;
                    if (ANY) return hit;
                }
            }
        } else {
            if (a >= nnodes || b >= nnodes) { atomicOr(err, ST_BAD_TREE); return -1; }
            float4 l0 = ld4(&nodes[2 * (size_t)a]), l1 = ld4(&nodes[2 * (size_t)a + 1]);
            float4 h0 = ld4(&nodes[2 * (size_t)b]), h1 = ld4(&nodes[2 * (size_t)b + 1]);
            float t0 = slab(rb, l0, l1, tmin, best), t1 = slab(rb, h0, h1, tmin, best);
            bool c0 = t0 <= best, c1 = t1 <= best;
            if (c0 && c1) {
                bool first0 = t0 <= t1;
                if (sp < PT_STACK) stack[sp++] = first0 ? make_uint2(__float_as_uint(h0.w), __float_as_uint(h1.w))
                                                        : make_uint2(__float_as_uint(l0.w), __float_as_uint(l1.w));
                else { atomicOr(err, ST_STACK_OVERFLOW); return -1; }
                a = first0 ? __float_as_uint(l0.w) : __float_as_uint(h0.w);
                b = first0 ? __float_as_uint(l1.w) : __float_as_uint(h1.w);
                continue;
            }
            if (c0) { a = __float_as_uint(l0.w); b = __float_as_uint(l1.w); continue; }
            if (c1) { a = __float_as_uint(h0.w); b = __float_as_uint(h1.w); continue; }
        }
        if (sp == 0) break;
        uint2 e = stack[--sp];
        a = e.x;
        b = e.y;
    }
    return hit;
}

// set_hit (intersect.c): point, the normal facing the ray, front_face
__device__ __forceinline__ void set_hit(Hit &h, V3 o, V3 d, float t, V3 outward) {
    h.t = t;
    h.p = vadd(o, vscale(d, t));
    h.front = vdot(d, outward) < 0.0f;
    h.n = h.front ? outward : vneg(outward);
    h.ng = h.n;
}
// shape_hit (intersect.c): the Hit of the shape kept
__device__ __forceinline__ void shape_hit(const PtScene &S, int id, V3 o, V3 d, float t, Hit &h) {
    if ((uint32_t)id < S.nprims) {
        const float4 *pr = S.prims + 6 * (size_t)id;
        float4 c = ld4(pr), qf = ld4(pr + 1);
        if (qf.w == 0.0f) {
            V3 p = vadd(o, vscale(d, t));
            V3 n = vscale(vsub(p, v3(c.x, c.y, c.z)), dvd(1.0f, c.w));
            set_hit(h, o, d, t, n);
        } else {
            float4 nd = ld4(pr + 4);
            set_hit(h, o, d, t, v3(nd.x, nd.y, nd.z));
        }
    } else {
        const float4 *tp = S.tris + 3 * (size_t)(id - S.nprims);
        float4 u = ld4(tp + 1), v = ld4(tp + 2), q = ld4(tp);
        V3 uu = v3(u.x, u.y, u.z), vv = v3(v.x, v.y, v.z);
        set_hit(h, o, d, t, vnorm(vcross(uu, vv)));
        uint32_t n0 = __float_as_uint(q.w);
        if (n0 != 0xffffffffu && S.normals) {
            // smooth: the vertex normals blended by the barycentrics (finish_triangle)
            V3 pvec = vcross(d, vv);
            float inv = dvd(1.0f, vdot(uu, pvec));
            V3 tvec = vsub(o, v3(q.x, q.y, q.z));
            float b1 = mul(vdot(tvec, pvec), inv);
            float b2 = mul(vdot(d, vcross(tvec, uu)), inv);
            uint32_t n1 = __float_as_uint(u.w), n2 = __float_as_uint(v.w) & 0x03ffffffu;
            auto N = [&](uint32_t k) { return v3(__ldg(&S.normals[3 * k]), __ldg(&S.normals[3 * k + 1]), __ldg(&S.normals[3 * k + 2])); };
            V3 ns = vnorm(vadd(vadd(vscale(N(n0), sub(sub(1.0f, b1), b2)), vscale(N(n1), b1)), vscale(N(n2), b2)));
            if (vdot(ns, h.n) < 0.0f) ns = vneg(ns);
            if (vdot(ns, ns) > 0.5f) h.n = ns;
        }
    }
    h.prim = id;
    h.inst = -1;
}

// scene_intersect: the closest hit in (tmin, tmax)
__device__ __forceinline__ bool scene_intersect(const PtScene &S, V3 o, V3 d, float tmin, float tmax, Hit &h, uint32_t *err) {
    float best = tmax;
    int32_t id = walk<false>(S, S.nodes, S.root, S.nnodes, S.aux, S.naux, o, d, tmin, best, err);
    if (id < 0) return false;
    shape_hit(S, id, o, d, best, h);
    return true;
}
// scene_occluded: any hit in (tmin, tmax)
__device__ __forceinline__ bool scene_occluded(const PtScene &S, V3 o, V3 d, float tmin, float tmax, uint32_t *err) {
    float best = tmax;
    return walk<true>(S, S.nodes, S.root, S.nnodes, S.aux, S.naux, o, d, tmin, best, err) >= 0;
}

__device__ __forceinline__ float power_heuristic(float pa, float pb) {
    float a = mul(pa, pa), b = mul(pb, pb);
    return add(a, b) > 0.0f ? dvd(a, add(a, b)) : 0.0f;
}

// the lamp (Scene.light: a quad primitive) and its emission
struct Lamp {
    V3 q, u, v, normal, le;
    float area;
    int prim;
};
__device__ __forceinline__ Lamp load_lamp(const PtScene &S) {
    Lamp L;
    L.prim = S.light;
    const float4 *pr = S.prims + 6 * (size_t)S.light;
    float4 q = ld4(pr + 1), u = ld4(pr + 2), v = ld4(pr + 3), nd = ld4(pr + 4);
    L.q = v3(q.x, q.y, q.z);
    L.u = v3(u.x, u.y, u.z);
    L.v = v3(v.x, v.y, v.z);
    L.normal = v3(nd.x, nd.y, nd.z);
    L.area = v.w;
    Mat m = load_mat(S.mats, (int)u.w);
    L.le = m.emission;
    return L;
}
__device__ __forceinline__ float light_pdf(const Lamp &L, float dist2, float cos_light) {
    return dvd(dist2, mul(cos_light, L.area));
}

// sample_direct_light (tracer.c:56-84)
__device__ __forceinline__ V3 direct_light(const PtScene &S, const Lamp &L, const Hit &h, Bsdf &b, V3 v, int mis, float ua,
                                           float ub, uint32_t *err, uint32_t &rays) {
    V3 xl = vadd(L.q, vadd(vscale(L.u, ua), vscale(L.v, ub)));
    V3 to = vsub(xl, h.p);
    float dist2 = vdot(to, to);
    float dist = __fsqrt_rn(dist2);
    V3 wi = vscale(to, dvd(1.0f, dist));
    float cos_surf = vdot(h.n, wi);
    float cos_light = -vdot(L.normal, wi);
    if (cos_light <= 0.0f) return v3(0, 0, 0);
    float pdf;
    V3 f = bsdf_eval(b, h.n, v, wi, pdf);
    if (!(vmax3(f) > 0.0f)) return v3(0, 0, 0);
    rays++;
    if (scene_occluded(S, h.p, wi, RT_EPS, sub(dist, RT_SHADOW_MARGIN), err)) return v3(0, 0, 0);
    float g = dvd(mul(mul(fabsf(cos_surf), cos_light), L.area), dist2);
    if (mis) g = mul(g, power_heuristic(light_pdf(L, dist2, cos_light), pdf));
    return vscale(vmul(f, L.le), g);
}

enum { EMIT_FULL, EMIT_NONE, EMIT_MIS };

// trace_path_sampled (tracer.c:364-545) without media, textures, sky and glowing-shape sampling
// (none in these scenes: each is a step of its own), counting the rays it traces
__device__ V3 trace_path(const PtScene &S, const PtParams &P, V3 ro, V3 rd, Sampler &sm, uint32_t *err, uint32_t &rays) {
    const int max_depth = P.max_depth, mis = P.mis;
    V3 radiance = v3(0, 0, 0), thr = v3(1, 1, 1);
    int emit = EMIT_FULL;
    float bounce_pdf = 0.0f;
    const bool have_lamp = S.light >= 0;
    Lamp L;
    if (have_lamp) L = load_lamp(S);
    if (mis) rd = vnorm(rd);
    for (int depth = 0;; depth++) {
        Hit h;
        rays++;
        bool found = scene_intersect(S, ro, rd, RT_EPS, 1e30f, h, err);
        if (!found) break;                           // escaped: black without a sky
        const int mi = h.prim < (int)S.nprims ? (int)ld4(S.prims + 6 * (size_t)h.prim + 2).w
                                              : (int)(__float_as_uint(ld4(S.tris + 3 * (size_t)(h.prim - S.nprims) + 2).w) >> 26);
        const Mat m = load_mat(S.mats, mi);
        if (m.type == MAT_LIGHT) {
            if (h.front) {
                if (emit == EMIT_FULL) {
                    radiance = vadd(radiance, vmul(thr, m.emission));
                } else if (emit == EMIT_MIS && h.inst < 0 && h.prim == S.light) {
                    float cos_light = -vdot(L.normal, rd);
                    if (cos_light > 0.0f) {
                        float w = power_heuristic(bounce_pdf, light_pdf(L, mul(h.t, h.t), cos_light));
                        radiance = vadd(radiance, vmul(thr, vscale(m.emission, w)));
                    }
                }
            }
            break;
        }
        if (glows(m)) radiance = vadd(radiance, vmul(thr, m.emission));   // (no glowing shapes sampled)
        if (depth >= max_depth) break;
        V3 v = vneg(vnorm(rd));
        Bsdf b = bsdf_make(m, h.front, S.tab);
        if (bsdf_rough_part(b) && have_lamp) {
            float la, lb;
            sampler_2d(sm, SAMPLE_LIGHT(depth), la, lb);
            radiance = vadd(radiance, vmul(thr, direct_light(S, L, h, b, v, mis, lb, la, err, rays)));
        }
        bsdf_view(b, vdot(v, h.n));
        float ur = 0.0f, ul = 0.0f, da = 0.0f, db = 0.0f;
        if (depth >= RR_START || bsdf_nlobes(b) > 1) sampler_2d(sm, SAMPLE_MISC(depth), ur, ul);
        int lobe = bsdf_pick(b, ul);
        if (lobe >= 0 && !bsdf_lobe_delta(b, lobe)) sampler_2d(sm, SAMPLE_DIR(depth), da, db);
        BsdfSample bs;
        if (!bsdf_sample_lobe(b, lobe, h.n, v, da, db, bs)) break;
        thr = vmul(thr, bs.w);
        if (bs.delta) {
            emit = EMIT_FULL;
        } else {
            bounce_pdf = bs.pdf;
            emit = mis ? EMIT_MIS : EMIT_NONE;
        }
        if (depth >= RR_START) {                     // russian_roulette_u
            float p = rmin(vmax3(thr), 0.95f);
            if (ur >= p) break;
            thr = vscale(thr, dvd(1.0f, p));
        }
        ro = h.p;
        rd = mis ? vnorm(bs.l) : bs.l;
    }
    return radiance;
}

// camera_ray (camera.h:38-42)
__device__ __forceinline__ void camera_ray(const PtParams &P, float s, float t, V3 &o, V3 &d) {
    V3 target = vsub(vadd(P.upper_left, vscale(P.horizontal, s)), vscale(P.vertical, t));
    o = P.origin;
    d = vnorm(vsub(target, P.origin));
}

__device__ __forceinline__ bool is_number(V3 c) { return c.x == c.x && c.y == c.y && c.z == c.z; }

__device__ __forceinline__ V3 clamp_sample(V3 c, float clamp) {
    if (clamp > 0.0f && vmax3(c) > clamp) c = vscale(c, dvd(clamp, vmax3(c)));
    return c;
}

// exact mode: one thread per pixel of rows [y0, y0 + rows), samples [0, spp) in order from the
// CPU's per-pixel stream (trace_image, tracer.c:337-353)
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
        for (int k = 0; k < P.spp; k++) {
            Sampler sm{&rng, (uint32_t)k, (uint32_t)P.seed * 0x9e3779b9u, (int)x, (int)y, P.sampler_on, S.mask};
            float jx, jy;
            sampler_2d(sm, 0, jx, jy);
            float u = dvd(add((float)x, jx), (float)P.W), v = dvd(add((float)y, jy), (float)P.H);
            V3 o, d;
            camera_ray(P, u, v, o, d);
            V3 c = trace_path(S, P, o, d, sm, err, rays);
            if (!is_number(c)) continue;
            c = clamp_sample(c, P.clamp);
            sum = vadd(sum, c);
        }
        float4 a = accum[pixel];
        accum[pixel] = make_float4(a.x + sum.x, a.y + sum.y, a.z + sum.z, a.w + (float)P.spp);
    }
    if (ray_count) {
        unsigned long long r = rays;
        for (int o = 16; o > 0; o >>= 1) r += __shfl_xor_sync(0xffffffffu, r, o);
        if ((threadIdx.x & 31) == 0 && r) atomicAdd(ray_count, r);
    }
}

__device__ __forceinline__ uint64_t mix64(uint64_t z) {
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    return z ^ (z >> 31);
}

// fast mode: P.group lanes (a power of 2 dividing 32) per pixel, lane s tracing samples s, s + g,
// s + 2g, ... of [spp0, spp0 + spp), each from its own PCG32 stream; the group's sums are then added
// in a fixed order (deterministic)
__global__ void __launch_bounds__(128) fast_kernel(PtScene S, PtParams P, float4 *accum, unsigned long long *ray_count,
                                                   uint32_t *err) {
    const uint32_t g = P.group;
    const uint64_t tid = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const uint64_t pix_local = tid / g;
    const uint32_t lane_s = (uint32_t)(tid % g);
    const uint64_t npix = (uint64_t)P.W * P.rows;
    uint32_t rays = 0;
    V3 c = v3(0, 0, 0);
    float cnt = 0.0f;
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
            V3 s = trace_path(S, P, o, d, sm, err, rays);
            s = is_number(s) ? clamp_sample(s, P.clamp) : v3(0, 0, 0);
            c = vadd(c, s);
            cnt += 1.0f;
        }
    }
    for (uint32_t o = 1; o < g; o <<= 1) {               // fixed-order tree sum over the group
        c.x += __shfl_down_sync(0xffffffffu, c.x, o, g);
        c.y += __shfl_down_sync(0xffffffffu, c.y, o, g);
        c.z += __shfl_down_sync(0xffffffffu, c.z, o, g);
        cnt += __shfl_down_sync(0xffffffffu, cnt, o, g);
    }
    if (live && lane_s == 0) {
        float4 a = accum[pixel];
        accum[pixel] = make_float4(a.x + c.x, a.y + c.y, a.z + c.z, a.w + cnt);
    }
    if (ray_count) {
        unsigned long long r = rays;
        for (int o = 16; o > 0; o >>= 1) r += __shfl_xor_sync(0xffffffffu, r, o);
        if ((threadIdx.x & 31) == 0 && r) atomicAdd(ray_count, r);
    }
}

// closest hits over shape ids (primitives, then triangles): lrc_scene_intersect for world scenes
__global__ void __launch_bounds__(128) shapes_closest_kernel(PtScene S, const float *__restrict__ orig,
                                                             const float *__restrict__ dir, uint64_t n, float tmin, float tmax,
                                                             int32_t *__restrict__ prim, float *__restrict__ tout, uint32_t *err) {
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    V3 o = v3(orig[3 * i], orig[3 * i + 1], orig[3 * i + 2]), d = v3(dir[3 * i], dir[3 * i + 1], dir[3 * i + 2]);
    float best = tmax;
    int32_t id = walk<false>(S, S.nodes, S.root, S.nnodes, S.aux, S.naux, o, d, tmin, best, err);
    prim[i] = id;
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
    if (P.exact) {
        const uint64_t threads = (uint64_t)P.W * P.rows;
        pt::exact_kernel<<<(unsigned)((threads + 127) / 128), 128, 0, st>>>(S, P, acc, d_rays, d_status);
    } else {
        const uint64_t threads = (uint64_t)P.W * P.rows * P.group;
        pt::fast_kernel<<<(unsigned)((threads + 127) / 128), 128, 0, st>>>(S, P, acc, d_rays, d_status);
    }
    return cudaGetLastError();
}

cudaError_t pt_intersect(const PtScene &S, const float *d_orig, const float *d_dir, uint64_t n, float tmin, float tmax,
                         int32_t *d_prim, float *d_t, uint32_t *d_status, cudaStream_t st) {
    if (!n) return cudaSuccess;
    pt::shapes_closest_kernel<<<(unsigned)((n + 127) / 128), 128, 0, st>>>(S, d_orig, d_dir, n, tmin, tmax, d_prim, d_t,
                                                                           d_status);
    return cudaGetLastError();
}

}  // namespace lrc
