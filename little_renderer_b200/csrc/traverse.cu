// traverse.cu - ray queries through a binary BVH in the reference's node layout (trace.wgsl:2;
// put_nodes, trace_gpu.c:883-896), triangles in its GPU layout (trace.wgsl Tri; put_tris,
// trace_gpu.c:898-911). Closest hit (scene_intersect, engine/rt/accel.c:252) and any hit
// (scene_occluded, accel.c:280).
//
// Latency-bound pointer chasing. One thread per ray; a node's two children are fetched as four
// 16-byte loads through the read-only path. The walk's stack of pending far children (their child
// pairs, 8 bytes) lives in shared memory, entry i of thread t at [i][t] (a warp's threads touch
// consecutive words), with a local-memory overflow area behind it: the stack in local memory alone
// thrashed L1 (16 % hits, 3 useful bytes per 32-byte sector). Large batches of rays are first
// reordered by a 30-bit key (where the ray enters the tree's root box, and its direction; 5 bits per
// dimension, interleaved) so that the rays of a warp walk the same nodes; the results go back to
// the callers' order.
//
// The box test is the fused-multiply-add slab test (conservative: leaf boxes are padded by 1e-3,
// triangle_bounds, scene.c:65-74); the triangle test is the reference's Moller-Trumbore
// (intersect.h:96-112) with every operation rounded as the C code rounds it (no contraction), so t
// and the hit are the CPU's to the bit. A stack that would overflow sets a status bit; tree indices
// out of range are reported, not followed.
#include "lrc_internal.cuh"
#include <algorithm>

namespace lrc {

constexpr int TR_THREADS = 128;
constexpr int TR_SSTACK = 8;               // entries per thread in shared memory (8 KB per block)
constexpr int TR_LSTACK = 88;              // then in local memory
constexpr uint64_t SORT_RAYS_FROM = 1u << 18;

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

// The walk's stack: TR_SSTACK entries in shared memory, then TR_LSTACK in local memory.
struct Stack {
    uint2 (*sh)[TR_THREADS];
    uint2 loc[TR_LSTACK];
    int sp;
    __device__ __forceinline__ bool push(uint2 e) {
        if (sp < TR_SSTACK) sh[sp][threadIdx.x] = e;
        else if (sp < TR_SSTACK + TR_LSTACK) loc[sp - TR_SSTACK] = e;
        else return false;
        sp++;
        return true;
    }
    __device__ __forceinline__ uint2 pop() {
        sp--;
        return sp < TR_SSTACK ? sh[sp][threadIdx.x] : loc[sp - TR_SSTACK];
    }
};

// closest hit (ANY = false) or any hit (ANY = true) of one ray; returns the triangle (aux value)
// or -1, best = its t. COUNT: box tests into cnt[0], triangle tests into cnt[1].
template <bool ANY, bool COUNT = false>
__device__ __forceinline__ int32_t trace_one(const TraceTables &tt, const RayCtx &r, float tmin, float &best, Stack &stk,
                                             uint32_t *err, uint32_t *cnt = nullptr) {
    stk.sp = 0;
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
                uint2 far = first0 ? make_uint2(__float_as_uint(h0.w), __float_as_uint(h1.w))
                                   : make_uint2(__float_as_uint(l0.w), __float_as_uint(l1.w));
                if (!stk.push(far)) { atomicOr(err, ST_STACK_OVERFLOW); return -1; }
                a = first0 ? __float_as_uint(l0.w) : __float_as_uint(h0.w);
                b = first0 ? __float_as_uint(l1.w) : __float_as_uint(h1.w);
                continue;
            }
            if (hit0) { a = __float_as_uint(l0.w); b = __float_as_uint(l1.w); continue; }
            if (hit1) { a = __float_as_uint(h0.w); b = __float_as_uint(h1.w); continue; }
        }
        if (stk.sp == 0) break;
        uint2 e = stk.pop();
        a = e.x;
        b = e.y;
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

// the ray thread i works on: perm[i] when the rays were reordered
__device__ __forceinline__ uint64_t ray_index(const uint32_t *perm, uint64_t i) { return perm ? (uint64_t)__ldg(&perm[i]) : i; }

__global__ void __launch_bounds__(TR_THREADS) closest_kernel(TraceTables tt, const float *__restrict__ orig,
                                                             const float *__restrict__ dir, const uint32_t *__restrict__ perm,
                                                             uint64_t nrays, float tmin, float tmax, int32_t *__restrict__ prim,
                                                             float *__restrict__ tout, uint32_t *err) {
    __shared__ uint2 sstack[TR_SSTACK][TR_THREADS];
    const uint64_t i = (uint64_t)blockIdx.x * TR_THREADS + threadIdx.x;
    if (i >= nrays) return;
    const uint64_t ri = ray_index(perm, i);
    if (ri >= nrays) {                                           // (a reordering whose look-back ran out)
        atomicOr(err, ST_TIMEOUT_SORT);
        return;
    }
    RayCtx r = make_ray(orig + 3 * ri, dir + 3 * ri);
    Stack stk;
    stk.sh = sstack;
    float best = tmax;
    int32_t h = trace_one<false>(tt, r, tmin, best, stk, err);
    prim[ri] = h;
    tout[ri] = h >= 0 ? best : -1.0f;
}

__global__ void __launch_bounds__(TR_THREADS) any_kernel(TraceTables tt, const float *__restrict__ orig,
                                                         const float *__restrict__ dir, const float *__restrict__ tmaxs,
                                                         uint64_t nrays, float tmin, uint8_t *__restrict__ out, uint32_t *err) {
    __shared__ uint2 sstack[TR_SSTACK][TR_THREADS];
    const uint64_t i = (uint64_t)blockIdx.x * TR_THREADS + threadIdx.x;
    if (i >= nrays) return;
    RayCtx r = make_ray(orig + 3 * i, dir + 3 * i);
    Stack stk;
    stk.sh = sstack;
    float best = tmaxs[i];
    out[i] = trace_one<true>(tt, r, tmin, best, stk, err) >= 0 ? 1 : 0;
}

// the same walk as closest_kernel, counting: totals of box tests and triangle tests into stats[0..1]
__global__ void __launch_bounds__(TR_THREADS) count_kernel(TraceTables tt, const float *__restrict__ orig,
                                                           const float *__restrict__ dir, uint64_t nrays, float tmin, float tmax,
                                                           unsigned long long *stats, uint32_t *err) {
    __shared__ uint2 sstack[TR_SSTACK][TR_THREADS];
    const uint64_t i = (uint64_t)blockIdx.x * TR_THREADS + threadIdx.x;
    uint32_t cnt[2] = {0, 0};
    if (i < nrays) {
        RayCtx r = make_ray(orig + 3 * i, dir + 3 * i);
        Stack stk;
        stk.sh = sstack;
        float best = tmax;
        trace_one<false, true>(tt, r, tmin, best, stk, err, cnt);
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

// ---- reordering of large ray batches -----------------------------------------------------------
__device__ __forceinline__ uint32_t spread5x6(uint32_t v, int slot) {
    // bit k of v (k < 5) to bit 6 k + slot
    uint32_t x = 0;
#pragma unroll
    for (int k = 0; k < 5; k++) x |= ((v >> k) & 1u) << (6 * k + slot);
    return x;
}
__device__ __forceinline__ uint32_t q5(float x) { return (uint32_t)fminf(fmaxf(x * 32.0f, 0.0f), 31.0f); }

// key of each ray: where it enters the root box (its origin if inside; the box's far corner's cell
// when it misses) and its direction, 5 bits each, interleaved; the 4 radix passes' histograms
__global__ void __launch_bounds__(256) ray_key_kernel(TraceTables tt, const float *__restrict__ orig,
                                                      const float *__restrict__ dir, uint64_t nrays, float tmin, float tmax,
                                                      uint32_t *__restrict__ keys, uint32_t *__restrict__ hist) {
    __shared__ uint32_t sh[4 * 256];
    for (int i = threadIdx.x; i < 4 * 256; i += 256) sh[i] = 0;
    const float4 *nodes = reinterpret_cast<const float4 *>(tt.nodes);
    const float4 lo = __ldg(&nodes[2 * (size_t)tt.root]), hi = __ldg(&nodes[2 * (size_t)tt.root + 1]);
    const float sx = 1.0f / fmaxf(hi.x - lo.x, 1e-30f), sy = 1.0f / fmaxf(hi.y - lo.y, 1e-30f),
                sz = 1.0f / fmaxf(hi.z - lo.z, 1e-30f);
    __syncthreads();
    for (uint64_t i = (uint64_t)blockIdx.x * 256 + threadIdx.x; i < nrays; i += (uint64_t)gridDim.x * 256) {
        RayCtx r = make_ray(orig + 3 * i, dir + 3 * i);
        float te = box_enter(r, lo, hi, tmin, tmax);
        uint32_t key = 0xffffffffu >> 2;
        if (te <= tmax) {
            float px = fmaf(te, r.dx, r.ox), py = fmaf(te, r.dy, r.oy), pz = fmaf(te, r.dz, r.oz);
            float inv = rsqrtf(fmaxf(r.dx * r.dx + r.dy * r.dy + r.dz * r.dz, 1e-30f));
            key = spread5x6(q5((px - lo.x) * sx), 5) | spread5x6(q5((py - lo.y) * sy), 4) | spread5x6(q5((pz - lo.z) * sz), 3) |
                  spread5x6(q5(0.5f + 0.5f * r.dx * inv), 2) | spread5x6(q5(0.5f + 0.5f * r.dy * inv), 1) |
                  spread5x6(q5(0.5f + 0.5f * r.dz * inv), 0);
        }
        keys[i] = key;
#pragma unroll
        for (int p = 0; p < 4; p++) atomicAdd(&sh[p * 256 + ((key >> (8 * p)) & 255u)], 1u);
    }
    __syncthreads();
    for (int i = threadIdx.x; i < 4 * 256; i += 256)
        if (sh[i]) atomicAdd(&hist[i], sh[i]);
}

size_t intersect_scratch_bytes(uint64_t nrays) { return nrays >= SORT_RAYS_FROM ? sort_u32_scratch_bytes(nrays) : 0; }

cudaError_t count_device(const TraceTables &tt, const float *d_orig, const float *d_dir, uint64_t nrays, float tmin,
                         float tmax, unsigned long long *d_stats, uint32_t *d_status, cudaStream_t st) {
    cudaError_t e = cudaMemsetAsync(d_stats, 0, 16, st);
    if (e || !nrays) return e;
    uint64_t blocks = (nrays + TR_THREADS - 1) / TR_THREADS;
    count_kernel<<<(unsigned)blocks, TR_THREADS, 0, st>>>(tt, d_orig, d_dir, nrays, tmin, tmax, d_stats, d_status);
    return cudaGetLastError();
}

cudaError_t intersect_device(const TraceTables &tt, const float *d_orig, const float *d_dir, uint64_t nrays, float tmin,
                             float tmax, int32_t *d_prim, float *d_t, uint32_t *d_status, cudaStream_t st, int num_sms,
                             void *scratch, size_t scratch_bytes) {
    if (!nrays) return cudaSuccess;
    const uint32_t *perm = nullptr;
    // (reordering gave no gain on incoherent batches: the rays of a warp still part within a few
    // levels of the root; it runs only when asked for with scratch)
    if (scratch && nrays >= SORT_RAYS_FROM && nrays < (1ull << 30) && scratch_bytes >= sort_u32_scratch_bytes(nrays)) {
        SortU32 S = sort_u32_carve(scratch, nrays);
        cudaError_t e = sort_u32_clear(S, st);
        if (e) return e;
        int grid = (int)std::min<uint64_t>((nrays + 255) / 256, (uint64_t)num_sms * 8);
        ray_key_kernel<<<grid, 256, 0, st>>>(tt, d_orig, d_dir, nrays, tmin, tmax, S.keys, S.hist);
        e = sort_u32_run(S, d_status, st, &perm);
        if (e) return e;
    }
    uint64_t blocks = (nrays + TR_THREADS - 1) / TR_THREADS;
    closest_kernel<<<(unsigned)blocks, TR_THREADS, 0, st>>>(tt, d_orig, d_dir, perm, nrays, tmin, tmax, d_prim, d_t, d_status);
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
