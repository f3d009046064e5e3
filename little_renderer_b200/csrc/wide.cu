// wide.cu - the ray queries' walk over 8-wide nodes with quantised child boxes, made on the device
// from a binary tree (the walk's tree: the reference's topology with tight boxes). The node is the
// compressed wide node of Ylitie, Karras and Laine ("Efficient incoherent ray traversal on GPUs
// through compressed wide BVHs", HPG 2017) in a layout of our own: 80 bytes for up to 8 children
// (a binary walk reads 64 bytes for 2), so a ray's walk fetches fewer bytes and makes fewer
// dependent loads.
//
// Node (5 x 16 bytes): the grid origin p (the node box's lo) and the three axes' scale exponents
// (scale = a power of two, its float exponent field), the first inner child, the first triangle
// entry, one byte per slot (0 empty, 1 + k the k-th inner child, 0x80 | k the k-th triangle
// entry), then the slots' boxes as bytes: lo = p + q_lo scale rounded down, hi = p + q_hi scale
// rounded up, so a decoded box holds the box it was made from.
//
// Collapse (top down, one level of wide nodes per launch): a wide node takes its binary node's two
// children and opens the inner one with the largest surface area while fewer than 8 slots are
// used; a leaf of several triangles opens into one slot per triangle (each slot the triangle's own
// box, widened as the walk's tree widens leaves). No kernel waits on another; a leaf too large for
// the slots left is reported (ST_BAD_TREE) and the caller keeps the binary walk.
#include "lrc_internal.cuh"

namespace lrc {

namespace {

constexpr int WD_THREADS = 128;
constexpr int WD_SSTACK = 8;                // stack entries per thread in shared memory
constexpr int WD_LSTACK = 120;              // then in local memory

__device__ __forceinline__ float area(const float lo[3], const float hi[3]) {
    const float dx = hi[0] - lo[0], dy = hi[1] - lo[1], dz = hi[2] - lo[2];
    return dx * dy + dy * dz + dz * dx;
}

// the scale exponent field for an axis of extent ext: the smallest power of two s with ext / s <= 255
__device__ __forceinline__ uint32_t scale_bits(float ext) {
    const float x = __fdiv_ru(fmaxf(ext, 0x1p-120f), 255.0f);
    const uint32_t e = (__float_as_uint(x) >> 23) & 0xffu;  // x < 2^(e - 126)
    return min(e + 1u, 254u);
}

struct Slot {
    float lo[3], hi[3];
    uint32_t ref;                            // inner: binary node index; triangle: triangle id
    bool inner;
};

// one wide node per item of this level: items[i] = (binary node, wide node); the next level's items
// appended at next[]; counts: [0] wide nodes made, [1] triangle entries, [2] next level's items
__global__ void __launch_bounds__(128) collapse_kernel(const Node *__restrict__ bin, uint32_t nn, const uint32_t *__restrict__ aux,
                                                       uint32_t naux, const float4 *__restrict__ tris, uint32_t ntris, float pad,
                                                       const uint2 *__restrict__ items, const uint32_t *__restrict__ nitems,
                                                       uint2 *__restrict__ next, uint32_t *counts, float4 *wnodes,
                                                       uint32_t wcap, uint32_t *wrefs, uint32_t rcap, uint32_t *err) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= *nitems) return;
    const uint2 it = items[i];
    Slot s[8];
    int n = 0;
    bool bad = false;
    auto triangle_slot = [&](uint32_t id, Slot &o) {
        if (id >= ntris) { bad = true; return; }
        const float4 q = __ldg(&tris[3 * (size_t)id]), u = __ldg(&tris[3 * (size_t)id + 1]), v = __ldg(&tris[3 * (size_t)id + 2]);
        const float cx[3] = {q.x, q.x + u.x, q.x + v.x}, cy[3] = {q.y, q.y + u.y, q.y + v.y},
                    cz[3] = {q.z, q.z + u.z, q.z + v.z};
        o.lo[0] = fminf(fminf(cx[0], cx[1]), cx[2]) - pad; o.hi[0] = fmaxf(fmaxf(cx[0], cx[1]), cx[2]) + pad;
        o.lo[1] = fminf(fminf(cy[0], cy[1]), cy[2]) - pad; o.hi[1] = fmaxf(fmaxf(cy[0], cy[1]), cy[2]) + pad;
        o.lo[2] = fminf(fminf(cz[0], cz[1]), cz[2]) - pad; o.hi[2] = fmaxf(fmaxf(cz[0], cz[1]), cz[2]) + pad;
        o.ref = id;
        o.inner = false;
    };
    // a binary child into slots: inner -> one slot; a leaf -> one slot per triangle (room permitting)
    auto add = [&](uint32_t c) {
        if (c >= nn) { bad = true; return; }
        const Node &m = bin[c];
        if (m.b & LEAF_BIT) {
            const uint32_t cnt = m.b & ~LEAF_BIT;
            if (m.a >= naux || cnt > naux - m.a || n + (int)cnt > 8) { bad = true; return; }
            for (uint32_t k = 0; k < cnt && !bad; k++) triangle_slot(__ldg(&aux[m.a + k]), s[n++]);
        } else {
            if (n >= 8) { bad = true; return; }
            Slot &o = s[n++];
            for (int a = 0; a < 3; a++) { o.lo[a] = m.lo[a]; o.hi[a] = m.hi[a]; }
            o.ref = c;
            o.inner = true;
        }
    };
    if (it.x >= nn) {
        atomicOr(err, ST_BAD_TREE);
        return;
    }
    const Node &r = bin[it.x];
    if (r.b & LEAF_BIT) {                                      // (a root that is a leaf)
        const uint32_t cnt = r.b & ~LEAF_BIT;
        if (r.a >= naux || cnt > naux - r.a || cnt > 8) bad = true;
        for (uint32_t k = 0; k < cnt && !bad; k++) triangle_slot(__ldg(&aux[r.a + k]), s[n++]);
    } else {
        add(r.a);
        if (!bad) add(r.b);
    }
    // open the largest inner slot while there is room (a bounded number of times: a slot is opened
    // at most once, and at most 8 can be)
    for (int opened = 0; !bad && n < 8 && opened < 16; opened++) {
        int best = -1;
        float ba = -1.0f;
        for (int k = 0; k < n; k++)
            if (s[k].inner) {
                const float a = area(s[k].lo, s[k].hi);
                if (a > ba) { ba = a; best = k; }
            }
        if (best < 0) break;
        const Node &m = bin[s[best].ref];
        const uint32_t ca = m.a, cb = m.b;
        // the slots the two children take; a child that does not fit leaves the slot unopened
        uint32_t need = 0;
        for (uint32_t c : {ca, cb}) {
            if (c >= nn) { need = 99u; break; }
            const Node &x = bin[c];
            need += (x.b & LEAF_BIT) ? (x.b & ~LEAF_BIT) : 1u;
        }
        if (need > 8u || n - 1 + (int)need > 8) break;
        s[best] = s[n - 1];                                   // (the opened slot's place: the last slot)
        n--;
        add(ca);
        if (!bad) add(cb);
    }
    if (bad || n == 0) {
        atomicOr(err, ST_BAD_TREE);
        return;
    }
    // the node's box, the grid, the slots' bytes
    float lo[3] = {s[0].lo[0], s[0].lo[1], s[0].lo[2]}, hi[3] = {s[0].hi[0], s[0].hi[1], s[0].hi[2]};
    int ninner = 0, ntri = 0;
    for (int k = 0; k < n; k++) {
        for (int a = 0; a < 3; a++) { lo[a] = fminf(lo[a], s[k].lo[a]); hi[a] = fmaxf(hi[a], s[k].hi[a]); }
        if (s[k].inner) ninner++;
        else ntri++;
    }
    uint32_t eb[3];
    float scale[3];
    for (int a = 0; a < 3; a++) {
        eb[a] = scale_bits(__fsub_ru(hi[a], lo[a]));
        scale[a] = __uint_as_float(eb[a] << 23);
    }
    const uint32_t child0 = ninner ? atomicAdd(&counts[0], (uint32_t)ninner) : 0u;
    const uint32_t tri0 = ntri ? atomicAdd(&counts[1], (uint32_t)ntri) : 0u;
    if (child0 + ninner > wcap || tri0 + ntri > rcap) {
        atomicOr(err, ST_BAD_TREE);
        return;
    }
    const uint32_t next0 = ninner ? atomicAdd(&counts[2], (uint32_t)ninner) : 0u;
    uint8_t meta[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    uint8_t q[6][8];
    for (int k = 0; k < 8; k++)
        for (int a = 0; a < 6; a++) q[a][k] = 0;
    int ki = 0, kt = 0;
    for (int k = 0; k < n; k++) {
        for (int a = 0; a < 3; a++) {
            const float l = floorf(__fdiv_rd(__fsub_rd(s[k].lo[a], lo[a]), scale[a]));
            const float h = ceilf(__fdiv_ru(__fsub_ru(s[k].hi[a], lo[a]), scale[a]));
            q[a][k] = (uint8_t)fminf(fmaxf(l, 0.0f), 255.0f);
            q[3 + a][k] = (uint8_t)fminf(fmaxf(h, 0.0f), 255.0f);
        }
        if (s[k].inner) {
            meta[k] = (uint8_t)(1 + ki);
            next[next0 + ki] = make_uint2(s[k].ref, child0 + ki);
            ki++;
        } else {
            meta[k] = (uint8_t)(0x80 | kt);
            wrefs[tri0 + kt] = s[k].ref;
            kt++;
        }
    }
    auto pack4 = [](const uint8_t *b) { return (uint32_t)b[0] | (uint32_t)b[1] << 8 | (uint32_t)b[2] << 16 | (uint32_t)b[3] << 24; };
    float4 *o = wnodes + 5 * (size_t)it.y;
    o[0] = make_float4(lo[0], lo[1], lo[2], __uint_as_float(eb[0] | eb[1] << 8 | eb[2] << 16 | (uint32_t)n << 24));
    o[1] = make_float4(__uint_as_float(child0), __uint_as_float(tri0), __uint_as_float(pack4(meta)), __uint_as_float(pack4(meta + 4)));
    o[2] = make_float4(__uint_as_float(pack4(q[0])), __uint_as_float(pack4(q[0] + 4)), __uint_as_float(pack4(q[1])),
                       __uint_as_float(pack4(q[1] + 4)));
    o[3] = make_float4(__uint_as_float(pack4(q[2])), __uint_as_float(pack4(q[2] + 4)), __uint_as_float(pack4(q[3])),
                       __uint_as_float(pack4(q[3] + 4)));
    o[4] = make_float4(__uint_as_float(pack4(q[4])), __uint_as_float(pack4(q[4] + 4)), __uint_as_float(pack4(q[5])),
                       __uint_as_float(pack4(q[5] + 4)));
}

__global__ void root_item_kernel(uint2 *items, uint32_t *nitems, uint32_t *counts) {
    items[0] = make_uint2(0u, 0u);
    *nitems = 1;
    counts[0] = 1;                                      // (the root is wide node 0)
    counts[1] = 0;
    counts[2] = 0;
}

__global__ void next_level_kernel(uint32_t *nitems, uint32_t *counts) {
    *nitems = counts[2];
    counts[2] = 0;
}

// ---- the walk ---------------------------------------------------------------------------------
struct WRay {
    float ox, oy, oz, dx, dy, dz, ix, iy, iz, ax, ay, az;
};
__device__ __forceinline__ float inv_safe(float d) {
    const float eps = 1e-20f;
    return 1.0f / (fabsf(d) < eps ? copysignf(eps, d) : d);
}
__device__ __forceinline__ WRay wray(const float *o, const float *d) {
    WRay r;
    r.ox = o[0]; r.oy = o[1]; r.oz = o[2];
    r.dx = d[0]; r.dy = d[1]; r.dz = d[2];
    r.ix = inv_safe(r.dx); r.iy = inv_safe(r.dy); r.iz = inv_safe(r.dz);
    r.ax = r.ox * r.ix; r.ay = r.oy * r.iy; r.az = r.oz * r.iz;
    return r;
}

// Moller-Trumbore rounded as the reference rounds it (intersect.h:96-112), as the binary walk's
__device__ __forceinline__ bool tri_hit(const WRay &r, float4 q, float4 u, float4 v, float tmin, float tmax, float &tout) {
    float px = fsub(fmul(r.dy, v.z), fmul(r.dz, v.y));
    float py = fsub(fmul(r.dz, v.x), fmul(r.dx, v.z));
    float pz = fsub(fmul(r.dx, v.y), fmul(r.dy, v.x));
    float det = fadd(fadd(fmul(u.x, px), fmul(u.y, py)), fmul(u.z, pz));
    if (fabsf(det) < 1e-12f) return false;
    float inv = __fdiv_rn(1.0f, det);
    float tx = fsub(r.ox, q.x), ty = fsub(r.oy, q.y), tz = fsub(r.oz, q.z);
    float b1 = fmul(fadd(fadd(fmul(tx, px), fmul(ty, py)), fmul(tz, pz)), inv);
    if (b1 < 0.0f || b1 > 1.0f) return false;
    float qx = fsub(fmul(ty, u.z), fmul(tz, u.y));
    float qy = fsub(fmul(tz, u.x), fmul(tx, u.z));
    float qz = fsub(fmul(tx, u.y), fmul(ty, u.x));
    float b2 = fmul(fadd(fadd(fmul(r.dx, qx), fmul(r.dy, qy)), fmul(r.dz, qz)), inv);
    if (b2 < 0.0f || fadd(b1, b2) > 1.0f) return false;
    float t = fmul(fadd(fadd(fmul(v.x, qx), fmul(v.y, qy)), fmul(v.z, qz)), inv);
    if (t <= tmin || t >= tmax) return false;
    tout = t;
    return true;
}

__device__ __forceinline__ uint32_t byte_of(uint32_t lo4, uint32_t hi4, int k) {
    return ((k < 4 ? lo4 : hi4) >> (8 * (k & 3))) & 0xffu;
}
__device__ __forceinline__ void cswap(float &ta, uint32_t &ca, float &tb, uint32_t &cb) {
    if (tb < ta) {
        float t = ta; ta = tb; tb = t;
        uint32_t c = ca; ca = cb; cb = c;
    }
}

struct WStack {
    uint32_t (*sh)[WD_THREADS];
    uint32_t loc[WD_LSTACK];
    int sp;
    __device__ __forceinline__ bool push(uint32_t e) {
        if (sp < WD_SSTACK) sh[sp][threadIdx.x] = e;
        else if (sp < WD_SSTACK + WD_LSTACK) loc[sp - WD_SSTACK] = e;
        else return false;
        sp++;
        return true;
    }
    __device__ __forceinline__ uint32_t pop() {
        sp--;
        return sp < WD_SSTACK ? sh[sp][threadIdx.x] : loc[sp - WD_SSTACK];
    }
};

// closest (ANY = false) or any hit of one ray over the wide tree; the triangle id or -1, best its t.
// A node's children are all tested at once: its triangles at their slots, its inner children hit
// visited nearest first (the others wait on the stack). Every child index is higher than its
// node's (the collapse hands indices out level by level), so the walk ends. COUNT: cnt[0] += the
// nodes fetched (80 bytes each), cnt[1] += the triangle tests
template <bool ANY, bool COUNT = false>
__device__ __forceinline__ int32_t wide_walk(const WideTables &wt, const WRay &r, float tmin, float &best, WStack &stk,
                                             uint32_t *err, uint32_t *cnt = nullptr) {
    stk.sp = 0;
    int32_t hit = -1;
    uint32_t node = 0;
    while (true) {
        if (node >= wt.nnodes) { atomicOr(err, ST_BAD_TREE); return -1; }
        const float4 *np = wt.nodes + 5 * (size_t)node;
        const float4 n0 = __ldg(np), n1 = __ldg(np + 1), n2 = __ldg(np + 2), n3 = __ldg(np + 3), n4 = __ldg(np + 4);
        if constexpr (COUNT) cnt[0]++;
        const uint32_t ex = __float_as_uint(n0.w);
        const float sx = __uint_as_float((ex & 0xffu) << 23), sy = __uint_as_float(((ex >> 8) & 0xffu) << 23),
                    sz = __uint_as_float(((ex >> 16) & 0xffu) << 23);
        const uint32_t child0 = __float_as_uint(n1.x), tri0 = __float_as_uint(n1.y);
        const uint32_t m0 = __float_as_uint(n1.z), m1 = __float_as_uint(n1.w);
        const uint32_t qlx0 = __float_as_uint(n2.x), qlx1 = __float_as_uint(n2.y), qly0 = __float_as_uint(n2.z),
                       qly1 = __float_as_uint(n2.w), qlz0 = __float_as_uint(n3.x), qlz1 = __float_as_uint(n3.y),
                       qhx0 = __float_as_uint(n3.z), qhx1 = __float_as_uint(n3.w), qhy0 = __float_as_uint(n4.x),
                       qhy1 = __float_as_uint(n4.y), qhz0 = __float_as_uint(n4.z), qhz1 = __float_as_uint(n4.w);
        float tk[8];
        uint32_t ck[8];
#pragma unroll
        for (int k = 0; k < 8; k++) {
            tk[k] = __int_as_float(0x7f800000);
            ck[k] = 0;
            const uint32_t m = byte_of(m0, m1, k);
            if (!m) continue;
            const float lx = __fmaf_rd((float)byte_of(qlx0, qlx1, k), sx, n0.x);
            const float ly = __fmaf_rd((float)byte_of(qly0, qly1, k), sy, n0.y);
            const float lz = __fmaf_rd((float)byte_of(qlz0, qlz1, k), sz, n0.z);
            const float hx = __fmaf_ru((float)byte_of(qhx0, qhx1, k), sx, n0.x);
            const float hy = __fmaf_ru((float)byte_of(qhy0, qhy1, k), sy, n0.y);
            const float hz = __fmaf_ru((float)byte_of(qhz0, qhz1, k), sz, n0.z);
            const float x0 = fmaf(lx, r.ix, -r.ax), x1 = fmaf(hx, r.ix, -r.ax);
            const float y0 = fmaf(ly, r.iy, -r.ay), y1 = fmaf(hy, r.iy, -r.ay);
            const float z0 = fmaf(lz, r.iz, -r.az), z1 = fmaf(hz, r.iz, -r.az);
            const float tn = fmaxf(fmaxf(fminf(x0, x1), fminf(y0, y1)), fmaxf(fminf(z0, z1), tmin));
            const float tf = fminf(fminf(fmaxf(x0, x1), fmaxf(y0, y1)), fminf(fmaxf(z0, z1), best));
            if (!(tn <= tf)) continue;
            if (m & 0x80u) {                                   // a triangle: tested at once
                const uint32_t e = tri0 + (m & 7u);
                if (e >= wt.nrefs) { atomicOr(err, ST_BAD_TREE); return -1; }
                const uint32_t id = __ldg(&wt.refs[e]);
                if (id >= wt.ntris) { atomicOr(err, ST_BAD_TREE); return -1; }
                const float4 *tp = wt.tris + 3 * (size_t)id;
                if constexpr (COUNT) cnt[1]++;
                float t;
                if (tri_hit(r, __ldg(tp), __ldg(tp + 1), __ldg(tp + 2), tmin, best, t)) {
                    best = t;
                    hit = (int32_t)id;
                    if (ANY) return hit;
                }
            } else {
                tk[k] = tn;
                ck[k] = child0 + m - 1u;
            }
        }
        // the inner children hit, nearest first: sorted by entry distance (Batcher's network of 19)
        cswap(tk[0], ck[0], tk[1], ck[1]); cswap(tk[2], ck[2], tk[3], ck[3]);
        cswap(tk[4], ck[4], tk[5], ck[5]); cswap(tk[6], ck[6], tk[7], ck[7]);
        cswap(tk[0], ck[0], tk[2], ck[2]); cswap(tk[1], ck[1], tk[3], ck[3]);
        cswap(tk[4], ck[4], tk[6], ck[6]); cswap(tk[5], ck[5], tk[7], ck[7]);
        cswap(tk[1], ck[1], tk[2], ck[2]); cswap(tk[5], ck[5], tk[6], ck[6]);
        cswap(tk[0], ck[0], tk[4], ck[4]); cswap(tk[3], ck[3], tk[7], ck[7]);
        cswap(tk[1], ck[1], tk[5], ck[5]); cswap(tk[2], ck[2], tk[6], ck[6]);
        cswap(tk[1], ck[1], tk[4], ck[4]); cswap(tk[3], ck[3], tk[6], ck[6]);
        cswap(tk[2], ck[2], tk[4], ck[4]); cswap(tk[3], ck[3], tk[5], ck[5]);
        cswap(tk[3], ck[3], tk[4], ck[4]);
        // (an entry farther than the best hit found meanwhile is still walked: as the binary walk)
#pragma unroll
        for (int k = 7; k >= 1; k--)
            if (tk[k] <= best && !stk.push(ck[k])) { atomicOr(err, ST_STACK_OVERFLOW); return -1; }
        if (tk[0] <= best) {
            node = ck[0];
            continue;
        }
        if (stk.sp == 0) break;
        node = stk.pop();
    }
    return hit;
}

__global__ void __launch_bounds__(WD_THREADS) wide_closest_kernel(WideTables wt, const float *__restrict__ orig,
                                                                  const float *__restrict__ dir, uint64_t nrays, float tmin,
                                                                  float tmax, int32_t *__restrict__ prim,
                                                                  float *__restrict__ tout, uint32_t *err) {
    __shared__ uint32_t sstack[WD_SSTACK][WD_THREADS];
    const uint64_t i = (uint64_t)blockIdx.x * WD_THREADS + threadIdx.x;
    if (i >= nrays) return;
    const WRay r = wray(orig + 3 * i, dir + 3 * i);
    WStack stk;
    stk.sh = sstack;
    float best = tmax;
    const int32_t h = wide_walk<false>(wt, r, tmin, best, stk, err);
    prim[i] = h;
    tout[i] = h >= 0 ? best : -1.0f;
}

__global__ void __launch_bounds__(WD_THREADS) wide_any_kernel(WideTables wt, const float *__restrict__ orig,
                                                              const float *__restrict__ dir, const float *__restrict__ tmaxs,
                                                              uint64_t nrays, float tmin, uint8_t *__restrict__ out,
                                                              uint32_t *err) {
    __shared__ uint32_t sstack[WD_SSTACK][WD_THREADS];
    const uint64_t i = (uint64_t)blockIdx.x * WD_THREADS + threadIdx.x;
    if (i >= nrays) return;
    const WRay r = wray(orig + 3 * i, dir + 3 * i);
    WStack stk;
    stk.sh = sstack;
    float best = tmaxs[i];
    out[i] = wide_walk<true>(wt, r, tmin, best, stk, err) >= 0 ? 1 : 0;
}

__global__ void __launch_bounds__(WD_THREADS) wide_count_kernel(WideTables wt, const float *__restrict__ orig,
                                                                const float *__restrict__ dir, uint64_t nrays, float tmin,
                                                                float tmax, unsigned long long *stats, uint32_t *err) {
    __shared__ uint32_t sstack[WD_SSTACK][WD_THREADS];
    const uint64_t i = (uint64_t)blockIdx.x * WD_THREADS + threadIdx.x;
    uint32_t cnt[2] = {0, 0};
    if (i < nrays) {
        const WRay r = wray(orig + 3 * i, dir + 3 * i);
        WStack stk;
        stk.sh = sstack;
        float best = tmax;
        wide_walk<false, true>(wt, r, tmin, best, stk, err, cnt);
    }
    unsigned long long a = cnt[0], b = cnt[1];
    for (int o = 16; o > 0; o >>= 1) {
        a += __shfl_xor_sync(0xffffffffu, a, o);
        b += __shfl_xor_sync(0xffffffffu, b, o);
    }
    if ((threadIdx.x & 31) == 0 && (a | b)) {
        atomicAdd(&stats[0], a);
        atomicAdd(&stats[1], b);
    }
}

}  // namespace

size_t wide_node_cap(uint32_t naux) { return naux ? naux : 1; }   // (no more wide nodes than binary leaves)

size_t wide_scratch_bytes(uint32_t naux) { return 2 * wide_node_cap(naux) * 8 + 256; }

cudaError_t wide_build(const Node *d_bin, uint32_t nn, const uint32_t *d_aux, uint32_t naux, const float *d_tris,
                       uint32_t ntris, float4 *d_wnodes, uint32_t wcap, uint32_t *d_wrefs, uint32_t rcap, void *scratch,
                       size_t scratch_bytes, uint32_t *d_status, cudaStream_t st, uint32_t *nwide) {
    if (!nn) return cudaErrorInvalidValue;
    if (scratch_bytes < wide_scratch_bytes(naux)) return cudaErrorInvalidValue;
    const size_t cap = wide_node_cap(naux);
    char *s = static_cast<char *>(scratch);
    uint2 *items = reinterpret_cast<uint2 *>(s), *next = items + cap;
    uint32_t *small = reinterpret_cast<uint32_t *>(next + cap);   // [0..2] counts, [3] items this level
    // the widening of the triangle slots (the walk's tree's rule): from the root box
    Node root;
    cudaError_t e = cudaMemcpyAsync(&root, d_bin, sizeof(Node), cudaMemcpyDeviceToHost, st);
    if (!e) e = cudaStreamSynchronize(st);
    if (e) return e;
    const float m = fmaxf(fmaxf(fmaxf(fabsf(root.lo[0]), fabsf(root.lo[1])), fmaxf(fabsf(root.lo[2]), fabsf(root.hi[0]))),
                          fmaxf(fabsf(root.hi[1]), fabsf(root.hi[2])));
    const float pad = fminf(1e-3f, m * 0x1p-17f);
    root_item_kernel<<<1, 1, 0, st>>>(items, small + 3, small);
    // level by level: each launch makes the wide nodes of one level and lists the next
    uint32_t level_items = 1;
    for (uint32_t level = 0; level < 256 && level_items; level++) {
        const uint32_t blocks = (level_items + 127) / 128;
        collapse_kernel<<<blocks, 128, 0, st>>>(d_bin, nn, d_aux, naux, reinterpret_cast<const float4 *>(d_tris), ntris, pad,
                                                items, small + 3, next, small, d_wnodes, wcap, d_wrefs, rcap, d_status);
        next_level_kernel<<<1, 1, 0, st>>>(small + 3, small);
        std::swap(items, next);
        e = cudaMemcpyAsync(&level_items, small + 3, 4, cudaMemcpyDeviceToHost, st);
        if (!e) e = cudaStreamSynchronize(st);
        if (e) return e;
    }
    uint32_t counts[2] = {0, 0};
    e = cudaMemcpyAsync(counts, small, 8, cudaMemcpyDeviceToHost, st);
    if (!e) e = cudaStreamSynchronize(st);
    if (nwide) *nwide = counts[0];
    return e ? e : cudaGetLastError();
}

cudaError_t wide_intersect(const WideTables &wt, const float *d_orig, const float *d_dir, uint64_t nrays, float tmin,
                           float tmax, int32_t *d_prim, float *d_t, uint32_t *d_status, cudaStream_t st) {
    if (!nrays) return cudaSuccess;
    const uint64_t blocks = (nrays + WD_THREADS - 1) / WD_THREADS;
    wide_closest_kernel<<<(unsigned)blocks, WD_THREADS, 0, st>>>(wt, d_orig, d_dir, nrays, tmin, tmax, d_prim, d_t, d_status);
    return cudaGetLastError();
}

cudaError_t wide_occluded(const WideTables &wt, const float *d_orig, const float *d_dir, const float *d_tmax, uint64_t nrays,
                          float tmin, uint8_t *d_out, uint32_t *d_status, cudaStream_t st) {
    if (!nrays) return cudaSuccess;
    const uint64_t blocks = (nrays + WD_THREADS - 1) / WD_THREADS;
    wide_any_kernel<<<(unsigned)blocks, WD_THREADS, 0, st>>>(wt, d_orig, d_dir, d_tmax, nrays, tmin, d_out, d_status);
    return cudaGetLastError();
}

cudaError_t wide_count(const WideTables &wt, const float *d_orig, const float *d_dir, uint64_t nrays, float tmin, float tmax,
                       unsigned long long *d_stats, uint32_t *d_status, cudaStream_t st) {
    cudaError_t e = cudaMemsetAsync(d_stats, 0, 16, st);
    if (e || !nrays) return e;
    const uint64_t blocks = (nrays + WD_THREADS - 1) / WD_THREADS;
    wide_count_kernel<<<(unsigned)blocks, WD_THREADS, 0, st>>>(wt, d_orig, d_dir, nrays, tmin, tmax, d_stats, d_status);
    return cudaGetLastError();
}

}  // namespace lrc
