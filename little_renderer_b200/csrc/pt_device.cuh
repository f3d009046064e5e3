// pt_device.cuh - the path tracer's device code, shared by the plain kernels (pathtrace.cu) and
// the wavefront batch (wavefront.cu): the light transport of the reference's trace_path_sampled
// (engine/rt/tracer.c:364-545), which its WGSL megakernel restates (trace.wgsl:1125-1316).
#pragma once
#include "lrc_internal.cuh"
#include "bsdf.cuh"
#include "media.cuh"

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
// COUNT: cnt[0] += the boxes tested (32-byte node records read), cnt[1] += the leaf entries tested
// (a kernel compiled with it measures the walk's algorithmic bytes; the others never carry it)
template <bool COUNT = false, typename Leaf>
__device__ bool bvh_walk(const float4 *nodes, uint32_t root, uint32_t nnodes, const uint32_t *aux, uint32_t naux, V3 o,
                         V3 d, float tmin, float &best, uint32_t *err, Leaf &&leaf, uint32_t *cnt = nullptr) {
    RayBox rb = ray_box(o, d);
    float4 r0 = ld4(&nodes[2 * (size_t)root]), r1 = ld4(&nodes[2 * (size_t)root + 1]);
    if constexpr (COUNT) cnt[0] += 1;
    if (!(slab(rb, r0, r1, tmin, best) <= best)) return false;
    uint2 stack[PT_STACK];
    int sp = 0;
    uint32_t a = __float_as_uint(r0.w), b = __float_as_uint(r1.w);
    while (true) {
        if (b & LEAF_BIT) {
            const uint32_t count = b & ~LEAF_BIT;
            if (a >= naux || count > naux - a) { atomicOr(err, ST_BAD_TREE); return false; }
            for (uint32_t k = 0; k < count; k++) {
                if constexpr (COUNT) cnt[1] += 1;
                if (leaf(__ldg(&aux[a + k]))) return true;
            }
        } else {
            if (a >= nnodes || b >= nnodes) { atomicOr(err, ST_BAD_TREE); return false; }
            float4 l0 = ld4(&nodes[2 * (size_t)a]), l1 = ld4(&nodes[2 * (size_t)a + 1]);
            float4 h0 = ld4(&nodes[2 * (size_t)b]), h1 = ld4(&nodes[2 * (size_t)b + 1]);
            if constexpr (COUNT) cnt[0] += 2;
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
template <bool ANY, bool COUNT = false>
__device__ int32_t walk(const PtScene &S, const float4 *nodes, uint32_t root, uint32_t nnodes, const uint32_t *aux,
                        uint32_t naux, V3 o, V3 d, float tmin, float &best, uint32_t *err, uint32_t *cnt = nullptr) {
    int32_t hit = -1;
    bvh_walk<COUNT>(nodes, root, nnodes, aux, naux, o, d, tmin, best, err, [&](uint32_t id) {
        if (id >= S.nprims + S.ntris) { atomicOr(err, ST_BAD_TREE); return true; }
        float t;
        if (shape_test(S, id, o, d, tmin, best, t)) {
            best = t;
            hit = (int32_t)id;
            return ANY;
        }
        return false;
    }, cnt);
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
// entered with the ray in its own space (o' = inv o, d' = inv d: the same t) and its mesh's BVH
// walked. One loop walks both levels: a top-level node and a mesh's node take the same box-test
// code (the level picks the node array and the ray), so the lanes of a warp that are in different
// levels still run together (walking each mesh in a walk of its own, nested in the top level's
// leaf, left 2 of 32 lanes active per instruction). Entering an instance pushes a mark that
// brings the walk back to the top level when its mesh is done, and a leaf's further instances
// wait on the stack in order, so the instances, their nodes and their triangles are visited in the
// nested walk's order: the same hits and the same ties. COUNT as bvh_walk's.
template <bool ANY, bool COUNT = false>
__device__ bool walk_instances(const PtScene &S, V3 o, V3 d, float tmin, float &best, int &inst, int &tri, uint32_t *err,
                               uint32_t *cnt = nullptr) {
    constexpr uint32_t MARK = 0xffffffffu, ENTER = 0xfffffffeu;   // (stack entries' first word; node indices are smaller)
    const RayBox rw = ray_box(o, d);
    const float4 *tn = S.tlas_nodes;
    float4 r0 = ld4(&tn[0]), r1 = ld4(&tn[1]);
    if constexpr (COUNT) cnt[0] += 1;
    if (!(slab(rw, r0, r1, tmin, best) <= best)) return false;
    uint2 stack[PT_STACK];
    int sp = 0;
    bool found = false, in_mesh = false;
    RayBox rb = rw;
    V3 ro = o, rd = d;
    uint32_t cur = 0, first = 0;
    const float4 *nodes = tn;
    uint32_t nn = S.tlas_nnodes;
    uint32_t a = __float_as_uint(r0.w), b = __float_as_uint(r1.w);
    // instance i entered: its mesh's root box against the ray in its space; true with (a, b) its
    // root's record when the walk goes into the mesh; sp = -1: the walk ends (a bad index, a full stack)
    auto enter = [&](uint32_t i) -> bool {
        if (i >= S.ninst) { atomicOr(err, ST_BAD_TREE); sp = -1; return false; }
        const float4 *rec = S.inst + 8 * (size_t)i;
        const uint32_t mesh = __float_as_uint(ld4(rec + 6).w);
        if (mesh >= S.nmeshes) return false;                        // (shapes: not in these scenes)
        const uint4 mi = __ldg(&S.mesh_info[mesh]);                 // root node, first triangle, triangles
        const V3 io = xpoint(rec + 3, o), id = xdir(rec + 3, d);
        const RayBox ib = ray_box(io, id);
        const float4 m0 = ld4(&S.mnodes[2 * (size_t)mi.x]), m1 = ld4(&S.mnodes[2 * (size_t)mi.x + 1]);
        if constexpr (COUNT) cnt[0] += 1;
        if (!(slab(ib, m0, m1, tmin, best) <= best)) return false;
        if (sp >= PT_STACK) { atomicOr(err, ST_STACK_OVERFLOW); sp = -1; return false; }
        stack[sp++] = make_uint2(MARK, 0u);
        in_mesh = true;
        ro = io; rd = id; rb = ib;
        nodes = S.mnodes;
        nn = S.mnnodes;
        cur = i;
        first = mi.y;
        a = __float_as_uint(m0.w);
        b = __float_as_uint(m1.w);
        return true;
    };
    while (true) {
        if (b & LEAF_BIT) {
            const uint32_t count = b & ~LEAF_BIT;
            if (!in_mesh) {
                if (a >= S.ninst || count > S.ninst - a) { atomicOr(err, ST_BAD_TREE); return found; }
                if (count) {
                    for (uint32_t k = count - 1; k >= 1; k--) {             // the leaf's later instances wait
                        if (sp >= PT_STACK) { atomicOr(err, ST_STACK_OVERFLOW); return found; }
                        stack[sp++] = make_uint2(ENTER, __ldg(&S.tlas_aux[a + k]));
                    }
                    if constexpr (COUNT) cnt[1] += 1;
                    const bool in = enter(__ldg(&S.tlas_aux[a]));
                    if (sp < 0) return found;
                    if (in) continue;
                }
            } else {
                if (a >= S.mnaux || count > S.mnaux - a) { atomicOr(err, ST_BAD_TREE); return found; }
                for (uint32_t k = 0; k < count; k++) {
                    if constexpr (COUNT) cnt[1] += 1;
                    const uint32_t g = __ldg(&S.maux[a + k]);
                    if (g >= S.nmtris) { atomicOr(err, ST_BAD_TREE); return found; }
                    float t;
                    if (hit_tri_t(S.mtris + 3 * (size_t)g, ro, rd, tmin, best, t)) {
                        best = t;
                        inst = (int)cur;
                        tri = (int)(g - first);
                        found = true;
                        if (ANY) return true;
                    }
                }
            }
        } else {
            if (a >= nn || b >= nn) { atomicOr(err, ST_BAD_TREE); return found; }
            float4 l0 = ld4(&nodes[2 * (size_t)a]), l1 = ld4(&nodes[2 * (size_t)a + 1]);
            float4 h0 = ld4(&nodes[2 * (size_t)b]), h1 = ld4(&nodes[2 * (size_t)b + 1]);
            if constexpr (COUNT) cnt[0] += 2;
            float t0 = slab(rb, l0, l1, tmin, best), t1 = slab(rb, h0, h1, tmin, best);
            bool c0 = t0 <= best, c1 = t1 <= best;
            if (c0 && c1) {
                bool first0 = t0 <= t1;
                if (sp >= PT_STACK) { atomicOr(err, ST_STACK_OVERFLOW); return found; }
                stack[sp++] = first0 ? make_uint2(__float_as_uint(h0.w), __float_as_uint(h1.w))
                                     : make_uint2(__float_as_uint(l0.w), __float_as_uint(l1.w));
                a = first0 ? __float_as_uint(l0.w) : __float_as_uint(h0.w);
                b = first0 ? __float_as_uint(l1.w) : __float_as_uint(h1.w);
                continue;
            }
            if (c0) { a = __float_as_uint(l0.w); b = __float_as_uint(l1.w); continue; }
            if (c1) { a = __float_as_uint(h0.w); b = __float_as_uint(h1.w); continue; }
        }
        // the next entry: a node of this level, a mark (back to the top level) or an instance to enter
        bool next = false;
        while (!next) {
            if (sp == 0) return found;
            const uint2 e = stack[--sp];
            if (e.x == MARK) {
                in_mesh = false;
                ro = o; rd = d; rb = rw;
                nodes = tn;
                nn = S.tlas_nnodes;
            } else if (e.x == ENTER) {
                if constexpr (COUNT) cnt[1] += 1;
                next = enter(e.y);
                if (sp < 0) return found;
            } else {
                a = e.x;
                b = e.y;
                next = true;
            }
        }
    }
}

}  // namespace pt
}  // namespace lrc
#include "textures.cuh"
namespace lrc {
namespace pt {

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
// scene_occluded (accel.c:280): any hit in (tmin, tmax), the instances first. INST = false: a
// scene known to have no instances (the walk of the two levels not compiled in: fewer registers)
template <bool INST = true>
__device__ __forceinline__ bool scene_occluded(const PtScene &S, V3 o, V3 d, float tmin, float tmax, uint32_t *err) {
    float best = tmax;
    if (INST && S.ninst) {
        int inst, tri;
        if (walk_instances<true>(S, o, d, tmin, best, inst, tri, err)) return true;
    }
    return S.nnodes && walk<true>(S, S.nodes, S.root, S.nnodes, S.aux, S.naux, o, d, tmin, best, err) >= 0;
}

// The any-hit query compiled once (not inlined) for the kernels that trace media: with the
// in-medium next event estimation they query from four places, and four inlined walks beside
// the media's tracking overflowed the instruction cache.
static __device__ __noinline__ bool scene_occluded_once(const PtScene &S, V3 o, V3 d, float tmin, float tmax, uint32_t *err) {
    return scene_occluded<true>(S, o, d, tmin, tmax, err);
}
template <bool ONCE>
__device__ __forceinline__ bool occluded(const PtScene &S, V3 o, V3 d, float tmin, float tmax, uint32_t *err) {
    return ONCE ? scene_occluded_once(S, o, d, tmin, tmax, err) : scene_occluded(S, o, d, tmin, tmax, err);
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

// sample_direct_light (tracer.c:56-84) up to its shadow ray: the contribution V if nothing is in
// the way, the ray's direction and length. False: no ray is traced and the contribution is 0.
// (M: the pieces a medium's transmittance goes between: f * Le, the geometry term before the MIS
// weight, that weight, and the lamp's distance; V = fle * (g0 * w), or fle * g0 without MIS)
struct NeeParts {
    V3 fle;
    float g0, w, dist;
};
__device__ __forceinline__ bool direct_light_ray(const Lamp &L, const Hit &h, Bsdf &b, V3 v, int mis, float ua, float ub,
                                                 V3 &V, V3 &wi, float &tmax, NeeParts &M) {
    V3 xl = vadd(L.q, vadd(vscale(L.u, ua), vscale(L.v, ub)));
    V3 to = vsub(xl, h.p);
    float dist2 = vdot(to, to);
    float dist = __fsqrt_rn(dist2);
    wi = vscale(to, dvd(1.0f, dist));
    float cos_surf = vdot(h.n, wi);
    float cos_light = -vdot(L.normal, wi);
    if (cos_light <= 0.0f) return false;
    float pdf;
    V3 f = bsdf_eval(b, h.n, v, wi, pdf);
    if (!(vmax3(f) > 0.0f)) return false;
    float g = dvd(mul(mul(fabsf(cos_surf), cos_light), L.area), dist2);
    M.g0 = g;
    M.w = mis ? power_heuristic(light_pdf(L, dist2, cos_light), pdf) : 1.0f;
    if (mis) g = mul(g, M.w);
    M.fle = vmul(f, L.le);
    M.dist = dist;
    V = vscale(M.fle, g);
    tmax = sub(dist, RT_SHADOW_MARGIN);
    return true;
}
// the contribution with a medium's transmittance tr: g0 * tr, then the MIS weight (tracer.c:77-79)
__device__ __forceinline__ V3 nee_through(const NeeParts &M, int mis, float tr) {
    float g = mul(M.g0, tr);
    if (mis) g = mul(g, M.w);
    return vscale(M.fle, g);
}

// sample_direct_env (tracer.c:87-101) up to its shadow ray: a sky direction by its luminance,
// weighted against the BSDF's own sampling. False: no ray is traced and the contribution is 0.
__device__ __forceinline__ bool direct_env_ray(const PtScene &S, const Hit &h, Bsdf &b, V3 v, int mis, float ua, float ub,
                                               V3 &V, V3 &wi, NeeParts &M) {
    wi = v3(0, 0, 0);
    float pdf;
    V3 le = env_sample(S, ua, ub, wi, pdf);
    if (!(pdf > 0.0f) || !(vmax3(le) > 0.0f)) return false;
    float bpdf;
    V3 f = bsdf_eval(b, h.n, v, wi, bpdf);
    if (!(vmax3(f) > 0.0f)) return false;
    float g = dvd(fabsf(vdot(h.n, wi)), pdf);
    M.g0 = g;
    M.w = mis ? power_heuristic(pdf, bpdf) : 1.0f;
    if (mis) g = mul(g, M.w);
    M.fle = vmul(f, le);
    M.dist = 1e6f;
    V = vscale(M.fle, g);
    return true;
}

// sample_light_in_medium (tracer.c:267-288): the lamp seen from a point p in a medium reached
// along d, through the media (the phase function in place of the BSDF), its shadow ray traced
__device__ __forceinline__ V3 light_in_medium(const PtScene &S, const Lamp &L, V3 p, V3 d, float g, int mis, float ua,
                                              float ub, Rng &rng, uint32_t *err, uint32_t &rays) {
    V3 xl = vadd(L.q, vadd(vscale(L.u, ua), vscale(L.v, ub)));
    V3 to = vsub(xl, p);
    float dist2 = vdot(to, to);
    float dist = __fsqrt_rn(dist2);
    V3 wi = vscale(to, dvd(1.0f, dist));
    float cos_light = -vdot(L.normal, wi);
    if (cos_light <= 0.0f) return v3(0, 0, 0);
    rays++;
    if (scene_occluded_once(S, p, wi, RT_EPS, sub(dist, RT_SHADOW_MARGIN), err)) return v3(0, 0, 0);
    float tr = scene_medium_transmittance(S.vols, S.nvol, p, wi, 0.0f, dist, rng, err);
    if (tr <= 0.0f) return v3(0, 0, 0);
    float ph = phase_hg(vdot(d, wi), g);
    float w = dvd(mul(mul(mul(ph, tr), cos_light), L.area), dist2);
    if (mis) w = mul(w, power_heuristic(light_pdf(L, dist2, cos_light), ph));
    return vscale(L.le, w);
}

// sample_env_in_medium (tracer.c:104-118): the sky from a point in a medium
__device__ __forceinline__ V3 env_in_medium(const PtScene &S, V3 p, V3 d, float g, int mis, float ua, float ub, Rng &rng,
                                            uint32_t *err, uint32_t &rays) {
    V3 wi;
    float pdf;
    V3 le = env_sample(S, ua, ub, wi, pdf);
    if (!(pdf > 0.0f) || !(vmax3(le) > 0.0f)) return v3(0, 0, 0);
    rays++;
    if (scene_occluded_once(S, p, wi, RT_EPS, 1e30f, err)) return v3(0, 0, 0);
    float tr = scene_medium_transmittance(S.vols, S.nvol, p, wi, 0.0f, 1e6f, rng, err);
    if (tr <= 0.0f) return v3(0, 0, 0);
    float ph = phase_hg(vdot(d, wi), g);
    float w = dvd(mul(ph, tr), pdf);
    if (mis) w = mul(w, power_heuristic(pdf, ph));
    return vscale(le, w);
}

// One bounce's next event estimation with its shadow rays not yet traced (the wavefront batch):
// the throughput the contributions are weighted by, the lamp's and the sky's contribution if
// their ray is unoccluded, the rays (from p) and which of it there is.
enum { NEE_L = 1, NEE_E = 2, NEE_RL = 4, NEE_RE = 8, NEE_ROUGH = 16 };   // ROUGH: their indirect cap is on
struct Nee {
    V3 thr, vl, ve, p, wl, we;
    float tl;
    uint32_t flags;
};

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
// the moment its path ends (path regeneration), or a path can wait in memory between the
// kernels of a wavefront.
// skip_caustics' state (tracer.c:371-375): CAUS_CHAIN the camera saw a rough surface first,
// CAUS_SPEC a mirror / glass vertex since the last rough one; a path with both that reaches the
// lamp is light tracing's (lrc_caustics), not counted here. CAUS_SKIP: the job leaves them out.
// CAUS_ROUGH (the same bits): a rough bounce (or a medium's) so far, so that from then on what the
// path brings is indirect light, each part held to the job's indirect clamp (tracer.c:376-378).
enum { CAUS_CHAIN = 1, CAUS_SPEC = 2, CAUS_SKIP = 4, CAUS_ROUGH = 8 };

struct PathState {
    V3 ro, rd, thr, radiance;
    float bounce_pdf;
    float icap;                                      // TraceParams.indirect_clamp (0: off)
    int depth, emit, caus;
};

// (norm: MIS or media, whose distances and pdfs need a unit direction: tracer.c:380)
__device__ __forceinline__ void path_begin(int norm, V3 ro, V3 rd, PathState &ps, int skip_caustics, float icap) {
    ps.ro = ro;
    ps.rd = norm ? vnorm(rd) : rd;
    ps.thr = v3(1, 1, 1);
    ps.radiance = v3(0, 0, 0);
    ps.bounce_pdf = 0.0f;
    ps.icap = icap;
    ps.depth = 0;
    ps.emit = EMIT_FULL;
    ps.caus = skip_caustics ? CAUS_SKIP : 0;
}

// indirect_cap (tracer.c:358-362): a contribution c after a rough bounce (on) held to k by its
// largest channel, c scaled by k / max
__device__ __forceinline__ V3 indirect_cap(V3 c, bool on, float k) {
    const float m = vmax3(c);
    return on && k > 0.0f && m > k ? vscale(c, dvd(k, m)) : c;
}
// radiance += indirect_cap(c, the path is past a rough bounce)
__device__ __forceinline__ void path_add(PathState &ps, V3 c) {
    ps.radiance = vadd(ps.radiance, indirect_cap(c, (ps.caus & CAUS_ROUGH) != 0, ps.icap));
}

// scene_intersect's search alone: the closest t, the world shape (or -1) and the instance and its
// triangle (or -1); make_hit then gives the Hit scene_intersect gives. INST as scene_occluded's.
template <bool INST = true, bool COUNT = false>
__device__ __forceinline__ void scene_find(const PtScene &S, V3 o, V3 d, float tmin, float tmax, float &t, int &id, int &inst,
                                           int &tri, uint32_t *err, uint32_t *cnt = nullptr) {
    float best = tmax;
    id = -1;
    inst = -1;
    tri = -1;
    if (S.nnodes) id = walk<false, COUNT>(S, S.nodes, S.root, S.nnodes, S.aux, S.naux, o, d, tmin, best, err, cnt);
    if (INST && S.ninst) {
        int ii = -1, tt = -1;
        if (walk_instances<false, COUNT>(S, o, d, tmin, best, ii, tt, err, cnt)) {
            inst = ii;
            tri = tt;
        }
    }
    t = best;
}
__device__ __forceinline__ bool make_hit(const PtScene &S, V3 o, V3 d, float t, int id, int inst, int tri, Hit &h) {
    if (inst >= 0) instance_hit(S, inst, tri, o, d, t, h);
    else if (id >= 0) shape_hit(S, id, o, d, t, h);
    else return false;
    return true;
}

// The bounce after its closest hit (found, h): what trace_path_sampled's loop does with it
// (without media, textures and glowing-shape sampling: none in these scenes), counting the shadow
// rays it traces. DEFER = false traces the shadow rays here and adds their contributions; DEFER =
// true leaves them in nee (the caller adds vmul(nee.thr, V or 0) for the lamp, then the sky,
// before the next bounce, which is what this order of additions gives). Returns false when the
// path has ended (after nee's contributions, if any).
template <bool DEFER, bool MEDIA = false>
__device__ __forceinline__ bool path_shade(const PtScene &S, int max_depth, int mis, PathState &ps, bool found, const Hit &hit,
                                           Sampler &sm, uint32_t *err, uint32_t &rays, Nee &nee) {
    Hit h = hit;                                     // (a normal map bends its shading normal)
    const int depth = ps.depth;
    const bool have_lamp = S.light >= 0;
    if (DEFER) nee.flags = 0;
    // In a medium the ray may scatter before the surface (delta tracking, tracer.c:384-420): that
    // point replaces the hit for this bounce. (Media are traced with their shadow rays in place:
    // their transmittance draws random numbers only when the shadow ray gets through.)
    if (MEDIA && !DEFER && S.nvol) {
        float ts;
        int which;
        if (scene_medium_collision(S.vols, S.nvol, ps.ro, ps.rd, 0.0f, found ? h.t : 1e30f, *sm.rng, ts, which, err)) {
            if (depth >= max_depth) return false;
            const VolDev &vol = S.vols[which];
            const V3 p = vadd(ps.ro, vscale(ps.rd, ts));
            ps.thr = vmul(ps.thr, v3(vol.albedo[0], vol.albedo[1], vol.albedo[2]));
            float la, lb;
            if (have_lamp) {
                const Lamp L = load_lamp(S);
                sampler_2d(sm, SAMPLE_LIGHT(depth), la, lb);
                path_add(ps, vmul(ps.thr, light_in_medium(S, L, p, ps.rd, vol.g, mis, lb, la, *sm.rng, err, rays)));
            }
            if (S.has_env) {
                if (!have_lamp) sampler_2d(sm, SAMPLE_LIGHT(depth), la, lb);
                else {
                    la = rng_real(*sm.rng);
                    lb = rng_real(*sm.rng);
                }
                path_add(ps, vmul(ps.thr, env_in_medium(S, p, ps.rd, vol.g, mis, la, lb, *sm.rng, err, rays)));
            }
            float da, db;
            sampler_2d(sm, SAMPLE_DIR(depth), da, db);
            const V3 nd = sample_phase_u(ps.rd, vol.g, da, db);
            ps.bounce_pdf = phase_hg(vdot(ps.rd, nd), vol.g);
            ps.ro = p;
            ps.rd = nd;
            ps.emit = mis ? EMIT_MIS : EMIT_NONE;
            ps.caus = (ps.caus & ~CAUS_CHAIN) | CAUS_ROUGH;
            if (depth >= RR_START) {                 // russian_roulette (tracer.c:302-304)
                const float u = sampler_1d(sm, SAMPLE_MISC(depth), 0);
                const float pr = rmin(vmax3(ps.thr), 0.95f);
                if (u >= pr) return false;
                ps.thr = vscale(ps.thr, dvd(1.0f, pr));
            }
            ps.depth = depth + 1;
            return true;
        }
    }
    if (!found) {                                    // escaped: the sky (black without one)
        if (S.has_env && ps.emit != EMIT_NONE) {
            V3 le = env_eval(S, ps.rd);
            if (ps.emit == EMIT_MIS) le = vscale(le, power_heuristic(ps.bounce_pdf, env_pdf(S, ps.rd)));
            path_add(ps, vmul(ps.thr, le));
        }
        return false;
    }
    Mat m = load_mat(S.mats, hit_material(S, h) & 63);   // (MAX_MATS 64: the buffer's size)
    if (textured(m)) m = hit_shading(S, h, ps.ro, ps.rd, vneg(vnorm(ps.rd)), m);
    if (m.type == MAT_LIGHT) {
        if (h.front && (ps.caus & (CAUS_CHAIN | CAUS_SPEC)) != (CAUS_CHAIN | CAUS_SPEC)) {
            if (ps.emit == EMIT_FULL) {
                path_add(ps, vmul(ps.thr, m.emission));
            } else if (ps.emit == EMIT_MIS && h.inst < 0 && h.prim == S.light) {
                const Lamp L = load_lamp(S);
                float cos_light = -vdot(L.normal, ps.rd);
                if (cos_light > 0.0f) {
                    float w = power_heuristic(ps.bounce_pdf, light_pdf(L, mul(h.t, h.t), cos_light));
                    path_add(ps, vmul(ps.thr, vscale(m.emission, w)));
                }
            }
        }
        return false;
    }
    if (glows(m)) path_add(ps, vmul(ps.thr, m.emission));   // (no glowing shapes sampled)
    if (depth >= max_depth) return false;
    V3 v = vneg(vnorm(ps.rd));
    Bsdf b = bsdf_make(m, h.front, S.tab);
    if (bsdf_rough_part(b)) {
        float la, lb;
        if (DEFER) {
            nee.thr = ps.thr;
            nee.p = h.p;
            if ((ps.caus & CAUS_ROUGH) && ps.icap > 0.0f) nee.flags |= NEE_ROUGH;
        }
        if (have_lamp) {
            const Lamp L = load_lamp(S);
            sampler_2d(sm, SAMPLE_LIGHT(depth), la, lb);
            V3 V = v3(0, 0, 0), wi;
            float tmax = 0.0f;
            NeeParts M;
            const bool ray = direct_light_ray(L, h, b, v, mis, lb, la, V, wi, tmax, M);
            if (ray) rays++;
            if (DEFER) {
                nee.flags |= NEE_L | (ray ? NEE_RL : 0);
                nee.vl = V;
                nee.wl = wi;
                nee.tl = tmax;
            } else {
                if (ray && occluded<MEDIA>(S, h.p, wi, RT_EPS, tmax, err)) V = v3(0, 0, 0);
                else if (MEDIA && ray && S.nvol) V = nee_through(M, mis, scene_medium_transmittance(S.vols, S.nvol, h.p, wi, 0.0f, M.dist, *sm.rng, err));
                path_add(ps, vmul(ps.thr, ray ? V : v3(0, 0, 0)));
            }
        }
        if (S.has_env) {
            // env_numbers (tracer.c:209-213): the lamp's pair when there is no lamp, else plain ones
            if (!have_lamp) sampler_2d(sm, SAMPLE_LIGHT(depth), la, lb);
            else {
                la = rng_real(*sm.rng);
                lb = rng_real(*sm.rng);
            }
            V3 V = v3(0, 0, 0), wi;
            NeeParts M;
            const bool ray = direct_env_ray(S, h, b, v, mis, la, lb, V, wi, M);
            if (ray) rays++;
            if (DEFER) {
                nee.flags |= NEE_E | (ray ? NEE_RE : 0);
                nee.ve = V;
                nee.we = wi;
            } else {
                if (ray && occluded<MEDIA>(S, h.p, wi, RT_EPS, 1e30f, err)) V = v3(0, 0, 0);
                else if (MEDIA && ray && S.nvol) V = nee_through(M, mis, scene_medium_transmittance(S.vols, S.nvol, h.p, wi, 0.0f, M.dist, *sm.rng, err));
                path_add(ps, vmul(ps.thr, ray ? V : v3(0, 0, 0)));
            }
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
        ps.caus |= CAUS_SPEC;
    } else {
        ps.bounce_pdf = bs.pdf;
        ps.emit = mis ? EMIT_MIS : EMIT_NONE;
        if (depth == 0 && (ps.caus & CAUS_SKIP)) ps.caus |= CAUS_CHAIN;
        ps.caus = (ps.caus & ~CAUS_SPEC) | CAUS_ROUGH;
    }
    if (depth >= RR_START) {                         // russian_roulette_u
        float p = rmin(vmax3(ps.thr), 0.95f);
        if (ur >= p) return false;
        ps.thr = vscale(ps.thr, dvd(1.0f, p));
    }
    ps.ro = h.p;
    ps.rd = mis || (MEDIA && S.nvol) ? vnorm(bs.l) : bs.l;
    ps.depth = depth + 1;
    return true;
}

// One pass of trace_path_sampled's bounce loop: the closest hit, then the rest of the bounce with
// its shadow rays traced in place. Returns false when the path has ended (ps.radiance its value).
template <bool MEDIA = false>
__device__ __forceinline__ bool path_bounce(const PtScene &S, int max_depth, int mis, PathState &ps, Sampler &sm,
                                            uint32_t *err, uint32_t &rays) {
    Hit h;
    rays++;
    bool found = scene_intersect(S, ps.ro, ps.rd, RT_EPS, 1e30f, h, err);
    Nee unused;
    return path_shade<false, MEDIA>(S, max_depth, mis, ps, found, h, sm, err, rays, unused);
}

// trace_path_sampled (tracer.c:364-545): the bounces of one path
// (MEDIA: the scene's media traced; a kernel compiled without them serves the scenes that have none)
template <bool MEDIA = false>
__device__ __forceinline__ V3 trace_path(const PtScene &S, const PtParams &P, V3 ro, V3 rd, Sampler &sm, uint32_t *err,
                                         uint32_t &rays) {
    PathState ps;
    path_begin(P.mis || (MEDIA && S.nvol), ro, rd, ps, P.skip_caustics, P.indirect_clamp);
    while (path_bounce<MEDIA>(S, P.max_depth, P.mis, ps, sm, err, rays)) {
    }
    return ps.radiance;
}

// camera_ray (camera.h:38-42)
__device__ __forceinline__ void camera_ray(const PtParams &P, float s, float t, V3 &o, V3 &d) {
    V3 target = vsub(vadd(P.upper_left, vscale(P.horizontal, s)), vscale(P.vertical, t));
    o = P.origin;
    d = vnorm(vsub(target, P.origin));
}

// a sample's luminance for the denoiser's moments: over the guide's albedo on a rough surface
// (kind 0), else as it is (trace.wgsl:1300-1305)
__device__ __forceinline__ float sample_luma(V3 c, float4 ga) {
    const float kind = ga.w - 4.0f * floorf(ga.w * 0.25f);
    if (kind == 0.0f) c = v3(c.x / fmaxf(ga.x, 1e-3f), c.y / fmaxf(ga.y, 1e-3f), c.z / fmaxf(ga.z, 1e-3f));
    return 0.2126f * c.x + 0.7152f * c.y + 0.0722f * c.z;
}

__device__ __forceinline__ bool is_number(V3 c) { return c.x == c.x && c.y == c.y && c.z == c.z; }

__device__ __forceinline__ V3 clamp_sample(V3 c, float clamp) {
    if (clamp > 0.0f && vmax3(c) > clamp) c = vscale(c, dvd(clamp, vmax3(c)));
    return c;
}

__device__ __forceinline__ uint64_t mix64(uint64_t z) {
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    return z ^ (z >> 31);
}

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

}  // namespace pt
}  // namespace lrc
