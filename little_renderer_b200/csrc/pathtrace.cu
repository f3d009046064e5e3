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

// One BVH walk in (tmin, best): nodes and aux as the reference lays them out, root its root node.
// leaf(entry) tests one leaf entry (an aux value), lowering best on a hit, and returns true to
// end the walk (an any-hit found). Entries of a leaf in order; a hit at the same t as the best is
// not taken (t >= tmax rejects), as the CPU's walk does. Returns true if a leaf ended it.
template <typename Leaf>
__device__ bool bvh_walk(const float4 *nodes, uint32_t root, uint32_t nnodes, const uint32_t *aux, uint32_t naux, V3 o,
                         V3 d, float tmin, float &best, uint32_t *err, Leaf &&leaf) {
    RayBox rb = ray_box(o, d);
    float4 r0 = ld4(&nodes[2 * (size_t)root]), r1 = ld4(&nodes[2 * (size_t)root + 1]);
    if (!(slab(rb, r0, r1, tmin, best) <= best)) return false;
    uint2 stack[PT_STACK];
    int sp = 0;
    uint32_t a = __float_as_uint(r0.w), b = __float_as_uint(r1.w);
    while (true) {
        if (b & LEAF_BIT) {
            const uint32_t count = b & ~LEAF_BIT;
            if (a >= naux || count > naux - a) { atomicOr(err, ST_BAD_TREE); return false; }
            for (uint32_t k = 0; k < count; k++)
                if (leaf(__ldg(&aux[a + k]))) return true;
        } else {
            if (a >= nnodes || b >= nnodes) { atomicOr(err, ST_BAD_TREE); return false; }
            float4 l0 = ld4(&nodes[2 * (size_t)a]), l1 = ld4(&nodes[2 * (size_t)a + 1]);
            float4 h0 = ld4(&nodes[2 * (size_t)b]), h1 = ld4(&nodes[2 * (size_t)b + 1]);
            float t0 = slab(rb, l0, l1, tmin, best), t1 = slab(rb, h0, h1, tmin, best);
            bool c0 = t0 <= best, c1 = t1 <= best;
            if (c0 && c1) {
                bool first0 = t0 <= t1;
                if (sp < PT_STACK) stack[sp++] = first0 ? make_uint2(__float_as_uint(h0.w), __float_as_uint(h1.w))
                                                        : make_uint2(__float_as_uint(l0.w), __float_as_uint(l1.w));
                else { atomicOr(err, ST_STACK_OVERFLOW); return false; }
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
    return false;
}

// the closest (ANY = false) or any world shape (primitives, then triangles) in (tmin, best), or -1
template <bool ANY>
__device__ int32_t walk(const PtScene &S, const float4 *nodes, uint32_t root, uint32_t nnodes, const uint32_t *aux,
                        uint32_t naux, V3 o, V3 d, float tmin, float &best, uint32_t *err) {
    int32_t hit = -1;
    bvh_walk(nodes, root, nnodes, aux, naux, o, d, tmin, best, err, [&](uint32_t id) {
        if (id >= S.nprims + S.ntris) { atomicOr(err, ST_BAD_TREE); return true; }
        float t;
        if (shape_test(S, id, o, d, tmin, best, t)) {
            best = t;
            hit = (int32_t)id;
            return ANY;
        }
        return false;
    });
    return hit;
}

// ---- instances (scene.h:202-209; intersect_instances, accel.c:77-150) ---------------------------
// An instance record: 8 float4 (the object -> world transform's rows, the inverse's rows, the
// world box's lo with the mesh index's bits, hi with the material's bits: -1 the triangles' own)
__device__ __forceinline__ V3 xpoint(const float4 *m, V3 p) {     // xform_point (scene.h)
    float4 r0 = ld4(m), r1 = ld4(m + 1), r2 = ld4(m + 2);
    return v3(add(add(add(mul(r0.x, p.x), mul(r0.y, p.y)), mul(r0.z, p.z)), r0.w),
              add(add(add(mul(r1.x, p.x), mul(r1.y, p.y)), mul(r1.z, p.z)), r1.w),
              add(add(add(mul(r2.x, p.x), mul(r2.y, p.y)), mul(r2.z, p.z)), r2.w));
}
__device__ __forceinline__ V3 xdir(const float4 *m, V3 d) {       // xform_dir
    float4 r0 = ld4(m), r1 = ld4(m + 1), r2 = ld4(m + 2);
    return v3(add(add(mul(r0.x, d.x), mul(r0.y, d.y)), mul(r0.z, d.z)),
              add(add(mul(r1.x, d.x), mul(r1.y, d.y)), mul(r1.z, d.z)),
              add(add(mul(r2.x, d.x), mul(r2.y, d.y)), mul(r2.z, d.z)));
}
__device__ __forceinline__ V3 xnormal(const float4 *inv, V3 n) {  // xform_normal: by the inverse's transpose
    float4 r0 = ld4(inv), r1 = ld4(inv + 1), r2 = ld4(inv + 2);
    return vnorm(v3(add(add(mul(r0.x, n.x), mul(r1.x, n.y)), mul(r2.x, n.z)),
                    add(add(mul(r0.y, n.x), mul(r1.y, n.y)), mul(r2.y, n.z)),
                    add(add(mul(r0.z, n.x), mul(r1.z, n.y)), mul(r2.z, n.z))));
}

// The closest (ANY = false) or any hit on the instances in (tmin, best): the instance and the
// triangle's index in its mesh; false if none. The top level's leaves are instances; each is
// entered with the ray in its own space (o' = inv o, d' = inv d: the same t) and its mesh's BVH walked.
template <bool ANY>
__device__ bool walk_instances(const PtScene &S, V3 o, V3 d, float tmin, float &best, int &inst, int &tri, uint32_t *err) {
    bool found = false;
    bvh_walk(S.tlas_nodes, 0, S.tlas_nnodes, S.tlas_aux, S.ninst, o, d, tmin, best, err, [&](uint32_t i) {
        if (i >= S.ninst) { atomicOr(err, ST_BAD_TREE); return true; }
        const float4 *rec = S.inst + 8 * (size_t)i;
        const uint32_t mesh = __float_as_uint(ld4(rec + 6).w);
        if (mesh >= S.nmeshes) return false;                       // (shapes: not in these scenes)
        const uint4 mi = __ldg(&S.mesh_info[mesh]);                // root node, first triangle, triangles
        V3 ro = xpoint(rec + 3, o), rd = xdir(rec + 3, d);
        return bvh_walk(S.mnodes, mi.x, S.mnnodes, S.maux, S.mnaux, ro, rd, tmin, best, err, [&](uint32_t g) {
            if (g >= S.nmtris) { atomicOr(err, ST_BAD_TREE); return true; }
            float t;
            if (hit_tri_t(S.mtris + 3 * (size_t)g, ro, rd, tmin, best, t)) {
                best = t;
                inst = (int)i;
                tri = (int)(g - mi.y);
                found = true;
                return ANY;
            }
            return false;
        });
    });
    return found;
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

// the Hit of an instance's triangle (intersect_instance, accel.c:98-105): made in the instance's
// space (finish_triangle with the object ray), the point in the world, the normals turned back
__device__ __forceinline__ void instance_hit(const PtScene &S, int inst, int tri, V3 o, V3 d, float t, Hit &h) {
    const float4 *rec = S.inst + 8 * (size_t)inst;
    const uint4 mi = __ldg(&S.mesh_info[__float_as_uint(ld4(rec + 6).w)]);
    V3 ro = xpoint(rec + 3, o), rd = xdir(rec + 3, d);
    const float4 *tp = S.mtris + 3 * (size_t)(mi.y + tri);
    float4 u = ld4(tp + 1), v = ld4(tp + 2);
    set_hit(h, ro, rd, t, vnorm(vcross(v3(u.x, u.y, u.z), v3(v.x, v.y, v.z))));
    h.p = vadd(o, vscale(d, t));
    h.n = xnormal(rec + 3, h.n);
    h.ng = xnormal(rec + 3, h.ng);
    h.prim = tri;
    h.inst = inst;
}

// scene_intersect (accel.c:252): the world's closest hit, then the instances' closer than it
__device__ __forceinline__ bool scene_intersect(const PtScene &S, V3 o, V3 d, float tmin, float tmax, Hit &h, uint32_t *err) {
    float best = tmax;
    bool found = false;
    if (S.nnodes) {
        int32_t id = walk<false>(S, S.nodes, S.root, S.nnodes, S.aux, S.naux, o, d, tmin, best, err);
        if (id >= 0) {
            shape_hit(S, id, o, d, best, h);
            found = true;
        }
    }
    if (S.ninst) {
        int inst = -1, tri = -1;
        if (walk_instances<false>(S, o, d, tmin, best, inst, tri, err)) {
            instance_hit(S, inst, tri, o, d, best, h);
            found = true;
        }
    }
    return found;
}
// scene_occluded (accel.c:280): any hit in (tmin, tmax), the instances first
__device__ __forceinline__ bool scene_occluded(const PtScene &S, V3 o, V3 d, float tmin, float tmax, uint32_t *err) {
    float best = tmax;
    if (S.ninst) {
        int inst, tri;
        if (walk_instances<true>(S, o, d, tmin, best, inst, tri, err)) return true;
    }
    return S.nnodes && walk<true>(S, S.nodes, S.root, S.nnodes, S.aux, S.naux, o, d, tmin, best, err) >= 0;
}

// ---- the sky (engine/scene/env.c: env_eval, env_sample, env_pdf) --------------------------------
// rgbp: the map's radiance and each pixel's probability (env_pixel_prob), w x h; cond: each row's
// cumulative distribution (w + 1 per row); marg: the rows' (h + 1)
__device__ __forceinline__ void map_uv(V3 d, float &u, float &v) {
    float y = d.y < -1.0f ? -1.0f : (d.y > 1.0f ? 1.0f : d.y);
    float uu = add(0.5f, mul(atan2f(d.x, d.z), dvd(0.5f, PIF)));
    u = sub(uu, floorf(uu));
    v = mul(acosf(y), dvd(1.0f, PIF));
}
__device__ __forceinline__ V3 map_dir(float u, float v) {
    float ph = mul(sub(u, 0.5f), mul(2.0f, PIF)), th = mul(v, PIF);
    float st = sinf(th);
    return v3(mul(st, sinf(ph)), cosf(th), mul(st, cosf(ph)));
}
__device__ __forceinline__ V3 env_bilerp(const PtScene &S, float u, float v) {
    const int w = S.env_w, h = S.env_h;
    float x = sub(mul(u, (float)w), 0.5f), y = sub(mul(v, (float)h), 0.5f);
    int x0 = (int)floorf(x), y0 = (int)floorf(y);
    float fx = sub(x, (float)x0), fy = sub(y, (float)y0);
    int y1 = y0 + 1;
    if (y0 < 0) y0 = 0;
    if (y1 > h - 1) y1 = h - 1;
    if (y0 > h - 1) y0 = h - 1;
    int xa = x0 < 0 ? x0 + w : (x0 >= w ? x0 - w : x0);
    if (xa < 0 || xa >= w) xa = ((xa % w) + w) % w;
    int xb = xa + 1 == w ? 0 : xa + 1;
    float4 a = ld4(&S.env_rgbp[(size_t)y0 * w + xa]), b = ld4(&S.env_rgbp[(size_t)y0 * w + xb]);
    float4 c = ld4(&S.env_rgbp[(size_t)y1 * w + xa]), dd = ld4(&S.env_rgbp[(size_t)y1 * w + xb]);
    float gx = sub(1.0f, fx), gy = sub(1.0f, fy);
    return v3(add(mul(gy, add(mul(gx, a.x), mul(fx, b.x))), mul(fy, add(mul(gx, c.x), mul(fx, dd.x)))),
              add(mul(gy, add(mul(gx, a.y), mul(fx, b.y))), mul(fy, add(mul(gx, c.y), mul(fx, dd.y)))),
              add(mul(gy, add(mul(gx, a.z), mul(fx, b.z))), mul(fy, add(mul(gx, c.z), mul(fx, dd.z)))));
}
__device__ __forceinline__ V3 env_eval(const PtScene &S, V3 d) {
    float u, v;
    map_uv(d, u, v);
    return vscale(env_bilerp(S, u, v), S.env_scale);
}
__device__ __forceinline__ int upper_bound(const float *c, int n, float x) {
    int lo = 0, hi = n;
    while (hi - lo > 1) {
        int mid = (lo + hi) / 2;
        if (__ldg(&c[mid]) <= x) lo = mid;
        else hi = mid;
    }
    return lo;
}
__device__ __forceinline__ float env_density(const PtScene &S, int x, int y, float st) {
    float prob = ld4(&S.env_rgbp[(size_t)y * S.env_w + x]).w;
    return dvd(mul(mul(prob, (float)S.env_w), (float)S.env_h), mul(mul(mul(2.0f, PIF), PIF), st));
}
__device__ __forceinline__ V3 env_sample(const PtScene &S, float u1, float u2, V3 &d, float &pdf) {
    pdf = 0.0f;
    if (!S.env_weighted) return v3(0, 0, 0);
    const int w = S.env_w, h = S.env_h;
    int y = upper_bound(S.env_marg, h, u2);
    float m0 = __ldg(&S.env_marg[y]), m1 = __ldg(&S.env_marg[y + 1]);
    float dv = m1 > m0 ? dvd(sub(u2, m0), sub(m1, m0)) : 0.5f;
    const float *c = S.env_cond + (size_t)y * (w + 1);
    int x = upper_bound(c, w, u1);
    float c0 = __ldg(&c[x]), c1 = __ldg(&c[x + 1]);
    float du = c1 > c0 ? dvd(sub(u1, c0), sub(c1, c0)) : 0.5f;
    if (dv > 0.9999f) dv = 0.9999f;
    if (du > 0.9999f) du = 0.9999f;
    float u = dvd(add((float)x, du), (float)w), v = dvd(add((float)y, dv), (float)h);
    float st = sinf(mul(v, PIF));
    if (st < 1e-6f) return v3(0, 0, 0);
    d = map_dir(u, v);
    pdf = env_density(S, x, y, st);
    return env_eval(S, d);
}
__device__ __forceinline__ float env_pdf(const PtScene &S, V3 d) {
    if (!S.env_weighted) return 0.0f;
    float u, v;
    map_uv(d, u, v);
    float st = sinf(mul(v, PIF));
    if (st < 1e-6f) return 0.0f;
    int x = (int)mul(u, (float)S.env_w), y = (int)mul(v, (float)S.env_h);
    if (x > S.env_w - 1) x = S.env_w - 1;
    if (y > S.env_h - 1) y = S.env_h - 1;
    return env_density(S, x, y, st);
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

// sample_direct_env (tracer.c:87-101): a sky direction by its luminance, the light along it if
// nothing is in the way, weighted against the BSDF's own sampling
__device__ __forceinline__ V3 direct_env(const PtScene &S, const Hit &h, Bsdf &b, V3 v, int mis, float ua, float ub,
                                         uint32_t *err, uint32_t &rays) {
    V3 wi = v3(0, 0, 0);
    float pdf;
    V3 le = env_sample(S, ua, ub, wi, pdf);
    if (!(pdf > 0.0f) || !(vmax3(le) > 0.0f)) return v3(0, 0, 0);
    float bpdf;
    V3 f = bsdf_eval(b, h.n, v, wi, bpdf);
    if (!(vmax3(f) > 0.0f)) return v3(0, 0, 0);
    rays++;
    if (scene_occluded(S, h.p, wi, RT_EPS, 1e30f, err)) return v3(0, 0, 0);
    float g = dvd(fabsf(vdot(h.n, wi)), pdf);
    if (mis) g = mul(g, power_heuristic(pdf, bpdf));
    return vscale(vmul(f, le), g);
}

// the material of what was hit (hit_material, intersect.h:23-25; scene_instance_material)
__device__ __forceinline__ int hit_material(const PtScene &S, const Hit &h) {
    if (h.inst >= 0) {
        const float4 *rec = S.inst + 8 * (size_t)h.inst;
        int m = __float_as_int(ld4(rec + 7).w);
        if (m >= 0) return m;
        const uint4 mi = __ldg(&S.mesh_info[__float_as_uint(ld4(rec + 6).w)]);
        return (int)(__float_as_uint(ld4(S.mtris + 3 * (size_t)(mi.y + h.prim) + 2).w) >> 26);
    }
    if (h.prim < (int)S.nprims) return (int)ld4(S.prims + 6 * (size_t)h.prim + 2).w;
    return (int)(__float_as_uint(ld4(S.tris + 3 * (size_t)(h.prim - S.nprims) + 2).w) >> 26);
}

enum { EMIT_FULL, EMIT_NONE, EMIT_MIS };

// The state trace_path_sampled (tracer.c:364-545) carries from one bounce to the next: the ray,
// the throughput, the radiance gathered so far, how the next emitter hit counts and the pdf of
// the bounce that led to it. With the Rng (and the sample index the Sampler is made from) it is
// all a path needs to resume, so a thread can hold one path per lane and start the next sample
// the moment its path ends (path regeneration in the batch kernel).
struct PathState {
    V3 ro, rd, thr, radiance;
    float bounce_pdf;
    int depth, emit;
};

__device__ __forceinline__ void path_begin(int mis, V3 ro, V3 rd, PathState &ps) {
    ps.ro = ro;
    ps.rd = mis ? vnorm(rd) : rd;
    ps.thr = v3(1, 1, 1);
    ps.radiance = v3(0, 0, 0);
    ps.bounce_pdf = 0.0f;
    ps.depth = 0;
    ps.emit = EMIT_FULL;
}

// One pass of trace_path_sampled's bounce loop (without media, textures and glowing-shape
// sampling: none in these scenes), counting the rays it traces. Returns false when the path has
// ended; ps.radiance is then its value.
__device__ __forceinline__ bool path_bounce(const PtScene &S, int max_depth, int mis, PathState &ps, Sampler &sm,
                                            uint32_t *err, uint32_t &rays) {
    const int depth = ps.depth;
    const bool have_lamp = S.light >= 0;
    Hit h;
    rays++;
    bool found = scene_intersect(S, ps.ro, ps.rd, RT_EPS, 1e30f, h, err);
    if (!found) {                                    // escaped: the sky (black without one)
        if (S.has_env && ps.emit != EMIT_NONE) {
            V3 le = env_eval(S, ps.rd);
            if (ps.emit == EMIT_MIS) le = vscale(le, power_heuristic(ps.bounce_pdf, env_pdf(S, ps.rd)));
            ps.radiance = vadd(ps.radiance, vmul(ps.thr, le));
        }
        return false;
    }
    const Mat m = load_mat(S.mats, hit_material(S, h) & 63);   // (MAX_MATS 64: the buffer's size)
    if (m.type == MAT_LIGHT) {
        if (h.front) {
            if (ps.emit == EMIT_FULL) {
                ps.radiance = vadd(ps.radiance, vmul(ps.thr, m.emission));
            } else if (ps.emit == EMIT_MIS && h.inst < 0 && h.prim == S.light) {
                const Lamp L = load_lamp(S);
                float cos_light = -vdot(L.normal, ps.rd);
                if (cos_light > 0.0f) {
                    float w = power_heuristic(ps.bounce_pdf, light_pdf(L, mul(h.t, h.t), cos_light));
                    ps.radiance = vadd(ps.radiance, vmul(ps.thr, vscale(m.emission, w)));
                }
            }
        }
        return false;
    }
    if (glows(m)) ps.radiance = vadd(ps.radiance, vmul(ps.thr, m.emission));   // (no glowing shapes sampled)
    if (depth >= max_depth) return false;
    V3 v = vneg(vnorm(ps.rd));
    Bsdf b = bsdf_make(m, h.front, S.tab);
    if (bsdf_rough_part(b)) {
        float la, lb;
        if (have_lamp) {
            const Lamp L = load_lamp(S);
            sampler_2d(sm, SAMPLE_LIGHT(depth), la, lb);
            ps.radiance = vadd(ps.radiance, vmul(ps.thr, direct_light(S, L, h, b, v, mis, lb, la, err, rays)));
        }
        if (S.has_env) {
            // env_numbers (tracer.c:209-213): the lamp's pair when there is no lamp, else plain ones
            if (!have_lamp) sampler_2d(sm, SAMPLE_LIGHT(depth), la, lb);
            else {
                la = rng_real(*sm.rng);
                lb = rng_real(*sm.rng);
            }
            ps.radiance = vadd(ps.radiance, vmul(ps.thr, direct_env(S, h, b, v, mis, la, lb, err, rays)));
        }
    }
    bsdf_view(b, vdot(v, h.n));
    float ur = 0.0f, ul = 0.0f, da = 0.0f, db = 0.0f;
    if (depth >= RR_START || bsdf_nlobes(b) > 1) sampler_2d(sm, SAMPLE_MISC(depth), ur, ul);
    int lobe = bsdf_pick(b, ul);
    if (lobe >= 0 && !bsdf_lobe_delta(b, lobe)) sampler_2d(sm, SAMPLE_DIR(depth), da, db);
    BsdfSample bs;
    if (!bsdf_sample_lobe(b, lobe, h.n, v, da, db, bs)) return false;
    ps.thr = vmul(ps.thr, bs.w);
    if (bs.delta) {
        ps.emit = EMIT_FULL;
    } else {
        ps.bounce_pdf = bs.pdf;
        ps.emit = mis ? EMIT_MIS : EMIT_NONE;
    }
    if (depth >= RR_START) {                         // russian_roulette_u
        float p = rmin(vmax3(ps.thr), 0.95f);
        if (ur >= p) return false;
        ps.thr = vscale(ps.thr, dvd(1.0f, p));
    }
    ps.ro = h.p;
    ps.rd = mis ? vnorm(bs.l) : bs.l;
    ps.depth = depth + 1;
    return true;
}

// trace_path_sampled (tracer.c:364-545): the bounces of one path
__device__ V3 trace_path(const PtScene &S, const PtParams &P, V3 ro, V3 rd, Sampler &sm, uint32_t *err, uint32_t &rays) {
    PathState ps;
    path_begin(P.mis, ro, rd, ps);
    while (path_bounce(S, P.max_depth, P.mis, ps, sm, err, rays)) {
    }
    return ps.radiance;
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

// ---- the batch: one persistent kernel over the tasks of many jobs --------------------------------
// the job holding task t (jobs in task order; binary search over task0)
__device__ __forceinline__ uint32_t batch_job_of(const BatchJob *__restrict__ jobs, uint32_t njobs, unsigned long long t) {
    uint32_t lo = 0, hi = njobs - 1;
    while (lo < hi) {
        uint32_t mid = (lo + hi + 1) >> 1;
        if (__ldg(&jobs[mid].task0) <= t) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

// Each lane holds one task (a pixel's lane slot) and one path of it at a time. A loop pass is
// one bounce for every lane with a path; a lane whose path ends adds it to its task's sum and
// starts the task's next sample, and a lane whose task is done writes it out and takes the next
// task of the queue (one atomic per warp and pass for all such lanes). The lanes thus stay busy
// however the path lengths and the samples per task differ, within a job and across jobs, and
// the grid drains the queue with no launch per job and no tail per job.
template <int BLOCK, int MINB>
__global__ void __launch_bounds__(BLOCK, MINB) batch_kernel(const BatchJob *__restrict__ jobs, uint32_t njobs,
                                                      unsigned long long ntasks, unsigned long long *next, uint32_t *err) {
    const uint32_t lane = threadIdx.x & 31;
    const uint32_t lt_mask = (1u << lane) - 1u;
    int j = -1;                       // the job of the lane's task (-1: none)
    unsigned long long task = 0;
    uint64_t pixel = 0;               // the pixel's index in its image
    uint32_t x = 0, y = 0, slot = 0, kk = 0, kend = 0, g = 1, rays = 0;
    V3 c = v3(0, 0, 0);
    float cnt = 0.0f;
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
            path_begin(J.P.mis, o, d, ps);
            active = true;
        }
        if (!path_bounce(J.S, J.P.max_depth, J.P.mis, ps, sm, err, rays)) {
            V3 s = is_number(ps.radiance) ? clamp_sample(ps.radiance, J.P.clamp) : v3(0, 0, 0);
            c = vadd(c, s);
            cnt += 1.0f;
            active = false;
            kk += g;
        }
    }
}

// one thread per pixel of all the batch's bands: the pixel's slots summed in the fast kernel's
// shuffle order (pairs, then pairs of pairs, ...) and added to its image, its rays to its job
__global__ void __launch_bounds__(128) batch_resolve_kernel(const BatchJob *__restrict__ jobs, uint32_t njobs,
                                                            unsigned long long npix) {
    const unsigned long long i = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x;
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
        float4 *a = J.accum + (uint64_t)y * (uint32_t)J.P.W + x;
        float4 av = *a;
        *a = make_float4(av.x + v[0].x, av.y + v[0].y, av.z + v[0].z, av.w + v[0].w);
    }
    // the rays of the warp's pixels, one atomic per job present
    const uint32_t peers = __match_any_sync(0xffffffffu, jj);
    const uint32_t sum = __reduce_add_sync(peers, (uint32_t)r);
    if (jj != 0xffffffffu && (threadIdx.x & 31) == (uint32_t)(__ffs(peers) - 1) && sum)
        atomicAdd(jobs[jj].rays, (unsigned long long)sum);
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
    if (P.exact) {
        const uint64_t threads = (uint64_t)P.W * P.rows;
        pt::exact_kernel<<<(unsigned)((threads + 127) / 128), 128, 0, st>>>(S, P, acc, d_rays, d_status);
    } else {
        const uint64_t threads = (uint64_t)P.W * P.rows * P.group;
        pt::fast_kernel<<<(unsigned)((threads + 127) / 128), 128, 0, st>>>(S, P, acc, d_rays, d_status);
    }
    return cudaGetLastError();
}

// the batch kernel's launch shapes: threads per block and the blocks per SM its registers are
// capped for (65536 / (threads x blocks) registers a thread)
namespace {
using BatchFn = void (*)(const BatchJob *, uint32_t, unsigned long long, unsigned long long *, uint32_t *);
struct BatchVariant {
    int block, minb;
    BatchFn fn;
};
const BatchVariant kBatchVariants[] = {
    {128, 4, pt::batch_kernel<128, 4>}, {128, 3, pt::batch_kernel<128, 3>}, {128, 5, pt::batch_kernel<128, 5>},
    {256, 2, pt::batch_kernel<256, 2>}, {64, 8, pt::batch_kernel<64, 8>},   {256, 3, pt::batch_kernel<256, 3>},
};
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
                        uint32_t *d_status, int variant, int grid, cudaStream_t st) {
    if (!njobs || !ntasks) return cudaSuccess;
    if (grid < 1 || variant < 0 || variant >= batch_variants()) return cudaErrorInvalidValue;
    void *args[] = {(void *)&d_jobs, (void *)&njobs, (void *)&ntasks, (void *)&d_next, (void *)&d_status};
    return cudaLaunchKernel((const void *)kBatchVariants[variant].fn, dim3(grid), dim3(kBatchVariants[variant].block), args,
                            0, st);
}

cudaError_t batch_resolve(const BatchJob *d_jobs, uint32_t njobs, unsigned long long npix, cudaStream_t st) {
    if (!njobs || !npix) return cudaSuccess;
    pt::batch_resolve_kernel<<<(unsigned)((npix + 127) / 128), 128, 0, st>>>(d_jobs, njobs, npix);
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
