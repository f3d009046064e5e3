// traverse.cu - ray queries through a binary BVH in the reference's node layout (trace.wgsl:2;
// put_nodes, trace_gpu.c:883-896), triangles in its GPU layout (trace.wgsl Tri; put_tris,
// trace_gpu.c:898-911). Closest hit (scene_intersect, engine/rt/accel.c:252) and any hit
// (scene_occluded, accel.c:280).
//
// Latency-bound pointer chasing: one thread per ray, the two children of a node fetched as four
// 16-byte loads through the read-only path, the stack of (children, entry distance) in local
// memory (L1), entries popped only while they can still hold a closer hit. The box test is the
// fast fused-multiply-add slab test (conservative: leaf boxes are padded by 1e-3, triangle_bounds,
// scene.c:65-74); the triangle test is the reference's Moller-Trumbore (intersect.h:96-112) with
// every operation rounded as the C code rounds it (no contraction), so t and the hit are the
// CPU's to the bit. A stack that would overflow sets a status bit; nothing is dropped silently.
#include "lrc_internal.cuh"
#include <algorithm>

namespace lrc {

constexpr int TR_STACK = 96;
constexpr int TR_THREADS = 128;

struct RayCtx {
    float ox, oy, oz, dx, dy, dz;
    float ix, iy, iz;          // 1 / d (a zero component made tiny first)
    float ax, ay, az;          // o / d
};

__device__ __forceinline__ float safe_inv(float d) {
    const float eps = 1e-20f;
    return 1.0f / (fabsf(d) < eps ? copysignf(eps, d) : d);
}

// slab test against [tmin, tmax]: entry distance, or +inf when missed
__device__ __forceinline__ float box_enter(const RayCtx &r, float4 lo, float4 hi, float tmin, float tmax) {
    float x0 = fmaf(lo.x, r.ix, -r.ax), x1 = fmaf(hi.x, r.ix, -r.ax);
    float y0 = fmaf(lo.y, r.iy, -r.ay), y1 = fmaf(hi.y, r.iy, -r.ay);
    float z0 = fmaf(lo.z, r.iz, -r.az), z1 = fmaf(hi.z, r.iz, -r.az);
    float tn = fmaxf(fmaxf(fminf(x0, x1), fminf(y0, y1)), fmaxf(fminf(z0, z1), tmin));
    float tf = fminf(fminf(fmaxf(x0, x1), fmaxf(y0, y1)), fminf(fmaxf(z0, z1), tmax));
    return tn <= tf ? tn : __int_as_float(0x7f800000);
}

// Moller-Trumbore as lr_hit_triangle_t (intersect.h:96-112): v_cross, v_dot left to right,
// inv = 1 / det, every product and sum rounded on its own
__device__ __forceinline__ bool tri_test(const RayCtx &r, float4 q, float4 u, float4 v, float tmin, float tmax, float &tout) {
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

struct StackEntry {
    uint32_t a, b;
    float t;
};

// closest hit (ANY = false) or any hit (ANY = true) of one ray; returns the triangle (aux value)
// or -1, best = its t. COUNT: box tests into cnt[0], triangle tests into cnt[1].
template <bool ANY, bool COUNT = false>
__device__ __forceinline__ int32_t trace_one(const TraceTables &tt, const RayCtx &r, float tmin, float &best, uint32_t *err,
                                             uint32_t *cnt = nullptr) {
    StackEntry stack[TR_STACK];
    int sp = 0;
    int32_t hit = -1;
    const float4 *nodes = reinterpret_cast<const float4 *>(tt.nodes);
    // the root: its own box first (as bvh_intersect), then its record's children
    float4 r0 = __ldg(&nodes[2 * (size_t)tt.root]), r1 = __ldg(&nodes[2 * (size_t)tt.root + 1]);
    float te = box_enter(r, r0, r1, tmin, best);
    if (COUNT) cnt[0]++;
    if (!(te <= best)) return -1;
    uint32_t a = __float_as_uint(r0.w), b = __float_as_uint(r1.w);
    while (true) {
        if (b & LEAF_BIT) {
            const uint32_t count = b & ~LEAF_BIT;
            if (a >= tt.naux || count > tt.naux - a) { atomicOr(err, ST_BAD_TREE); return -1; }
            for (uint32_t k = 0; k < count; k++) {
                const uint32_t id = __ldg(&tt.aux[a + k]);
                if (id >= tt.ntris) { atomicOr(err, ST_BAD_TREE); return -1; }
                const float4 *tp = tt.tris + 3 * (size_t)id;
                float t;
                if (COUNT) cnt[1]++;
                if (tri_test(r, __ldg(tp), __ldg(tp + 1), __ldg(tp + 2), tmin, best, t)) {
                    best = t;
                    hit = (int32_t)id;
                    if (ANY) return hit;
                }
            }
        } else {
            if (a >= tt.nnodes || b >= tt.nnodes) { atomicOr(err, ST_BAD_TREE); return -1; }
            const float4 *c0 = &nodes[2 * (size_t)a], *c1 = &nodes[2 * (size_t)b];
            float4 l0 = __ldg(c0), l1 = __ldg(c0 + 1), h0 = __ldg(c1), h1 = __ldg(c1 + 1);
            float t0 = box_enter(r, l0, l1, tmin, best), t1 = box_enter(r, h0, h1, tmin, best);
            if (COUNT) cnt[0] += 2;
            bool hit0 = t0 <= best, hit1 = t1 <= best;
            if (hit0 && hit1) {
                // the nearer first; the farther waits on the stack
                bool first0 = t0 <= t1;
                uint32_t fa = first0 ? __float_as_uint(h0.w) : __float_as_uint(l0.w);
                uint32_t fb = first0 ? __float_as_uint(h1.w) : __float_as_uint(l1.w);
                if (sp < TR_STACK) stack[sp++] = {fa, fb, first0 ? t1 : t0};
                else atomicOr(err, ST_STACK_OVERFLOW);
                a = first0 ? __float_as_uint(l0.w) : __float_as_uint(h0.w);
                b = first0 ? __float_as_uint(l1.w) : __float_as_uint(h1.w);
                continue;
            }
            if (hit0) { a = __float_as_uint(l0.w); b = __float_as_uint(l1.w); continue; }
            if (hit1) { a = __float_as_uint(h0.w); b = __float_as_uint(h1.w); continue; }
        }
        // pop the next entry that can still hold a closer hit
        bool found = false;
        while (sp > 0) {
            StackEntry e = stack[--sp];
            if (e.t <= best) { a = e.a; b = e.b; found = true; break; }
        }
        if (!found) break;
    }
    return hit;
}

__device__ __forceinline__ RayCtx make_ray(const float *o, const float *d) {
    RayCtx r;
    r.ox = o[0]; r.oy = o[1]; r.oz = o[2];
    r.dx = d[0]; r.dy = d[1]; r.dz = d[2];
    r.ix = safe_inv(r.dx); r.iy = safe_inv(r.dy); r.iz = safe_inv(r.dz);
    r.ax = r.ox * r.ix; r.ay = r.oy * r.iy; r.az = r.oz * r.iz;
    return r;
}

__global__ void __launch_bounds__(TR_THREADS) closest_kernel(TraceTables tt, const float *__restrict__ orig,
                                                             const float *__restrict__ dir, uint64_t nrays, float tmin,
                                                             float tmax, int32_t *__restrict__ prim, float *__restrict__ tout,
                                                             uint32_t *err) {
    const uint64_t i = (uint64_t)blockIdx.x * TR_THREADS + threadIdx.x;
    if (i >= nrays) return;
    RayCtx r = make_ray(orig + 3 * i, dir + 3 * i);
    float best = tmax;
    int32_t h = trace_one<false>(tt, r, tmin, best, err);
    prim[i] = h;
    tout[i] = h >= 0 ? best : -1.0f;
}

__global__ void __launch_bounds__(TR_THREADS) any_kernel(TraceTables tt, const float *__restrict__ orig,
                                                         const float *__restrict__ dir, const float *__restrict__ tmaxs,
                                                         uint64_t nrays, float tmin, uint8_t *__restrict__ out, uint32_t *err) {
    const uint64_t i = (uint64_t)blockIdx.x * TR_THREADS + threadIdx.x;
    if (i >= nrays) return;
    RayCtx r = make_ray(orig + 3 * i, dir + 3 * i);
    float best = tmaxs[i];
    out[i] = trace_one<true>(tt, r, tmin, best, err) >= 0 ? 1 : 0;
}

// the same walk as closest_kernel, counting: totals of box tests and triangle tests into stats[0..1]
__global__ void __launch_bounds__(TR_THREADS) count_kernel(TraceTables tt, const float *__restrict__ orig,
                                                           const float *__restrict__ dir, uint64_t nrays, float tmin, float tmax,
                                                           unsigned long long *stats, uint32_t *err) {
    const uint64_t i = (uint64_t)blockIdx.x * TR_THREADS + threadIdx.x;
    uint32_t cnt[2] = {0, 0};
    if (i < nrays) {
        RayCtx r = make_ray(orig + 3 * i, dir + 3 * i);
        float best = tmax;
        trace_one<false, true>(tt, r, tmin, best, err, cnt);
    }
    unsigned long long a = cnt[0], b = cnt[1];
    for (int o = 16; o > 0; o >>= 1) {
        a += __shfl_xor_sync(0xffffffffu, a, o);
        b += __shfl_xor_sync(0xffffffffu, b, o);
    }
    if ((threadIdx.x & 31) == 0) {
        atomicAdd(&stats[0], a);
        atomicAdd(&stats[1], b);
    }
}

cudaError_t count_device(const TraceTables &tt, const float *d_orig, const float *d_dir, uint64_t nrays, float tmin,
                         float tmax, unsigned long long *d_stats, uint32_t *d_status, cudaStream_t st) {
    cudaError_t e = cudaMemsetAsync(d_stats, 0, 16, st);
    if (e || !nrays) return e;
    uint64_t blocks = (nrays + TR_THREADS - 1) / TR_THREADS;
    count_kernel<<<(unsigned)blocks, TR_THREADS, 0, st>>>(tt, d_orig, d_dir, nrays, tmin, tmax, d_stats, d_status);
    return cudaGetLastError();
}

cudaError_t intersect_device(const TraceTables &tt, const float *d_orig, const float *d_dir, uint64_t nrays, float tmin,
                             float tmax, int32_t *d_prim, float *d_t, uint32_t *d_status, cudaStream_t st, int) {
    if (!nrays) return cudaSuccess;
    uint64_t blocks = (nrays + TR_THREADS - 1) / TR_THREADS;
    closest_kernel<<<(unsigned)blocks, TR_THREADS, 0, st>>>(tt, d_orig, d_dir, nrays, tmin, tmax, d_prim, d_t, d_status);
    return cudaGetLastError();
}

cudaError_t occluded_device(const TraceTables &tt, const float *d_orig, const float *d_dir, const float *d_tmax,
                            uint64_t nrays, float tmin, uint8_t *d_out, uint32_t *d_status, cudaStream_t st) {
    if (!nrays) return cudaSuccess;
    uint64_t blocks = (nrays + TR_THREADS - 1) / TR_THREADS;
    any_kernel<<<(unsigned)blocks, TR_THREADS, 0, st>>>(tt, d_orig, d_dir, d_tmax, nrays, tmin, d_out, d_status);
    return cudaGetLastError();
}

}  // namespace lrc
