// build.cu - the BVH builders on sm_100a: LBVH (Karras 2012) and PLOC (Meister & Bittner 2018),
// producing node for node and bit for bit the trees of the reference's WGSL builders
// (engine/gpu/shaders/trace/trace_build.wgsl, trace_ploc.wgsl; host: engine/gpu/trace_gpu.c:587-764).
//
// The pipeline (HBM-bound integer work; no tensor cores):
//   tri_boxes     triangle_bounds of each triangle + the mesh box, one pass over the triangles
//   morton_hist   Morton codes of the box centres (30-bit as the reference, or 63-bit), fused with
//                 the digit histograms of every radix pass (the onesweep "upsweep")
//   onesweep      one kernel per 8-bit digit: tile ranking with warp match, decoupled look-back
//                 over the tiles' digit counts, scatter through shared memory. A stable LSD sort of
//                 (code, item) starting in item order gives exactly the order of the reference's
//                 bitonic sort of unique (code, index) pairs.
//   lbvh          one kernel, bottom-up: leaf threads climb, the second child to reach a split
//                 makes the parent (Apetrei 2014) and numbers it as Karras does (a left child sits
//                 at its range's right end, a right child at its left end, the root at 0); boxes
//                 are made on the way up (min/max: the same bits as the reference's passes up).
//   ploc          one cooperative persistent kernel: every round is one pass of tiles (nearest in
//                 +-16 with the reference's tie rule, mutual pairs, decoupled look-back over the
//                 tiles' keep/merge counts, merges and compaction), rounds separated by a grid
//                 barrier; the last rounds in one block.
// Every spin-wait is bounded (SPIN_LIMIT) and reports through the status word instead of hanging.
#include "lrc_internal.cuh"
#include <cooperative_groups.h>
#include <algorithm>

namespace lrc {

// ---- Morton codes ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t spread10(uint32_t v) {
    uint32_t x = v & 1023u;
    x = (x | (x << 16)) & 0x030000ffu;
    x = (x | (x << 8)) & 0x0300f00fu;
    x = (x | (x << 4)) & 0x030c30c3u;
    x = (x | (x << 2)) & 0x09249249u;
    return x;
}
__device__ __forceinline__ uint64_t spread21(uint32_t v) {
    uint64_t x = v & 0x1fffffu;
    x = (x | (x << 32)) & 0x001f00000000ffffull;
    x = (x | (x << 16)) & 0x001f0000ff0000ffull;
    x = (x | (x << 8)) & 0x100f00f00f00f00full;
    x = (x | (x << 4)) & 0x10c30c30c30c30c3ull;
    x = (x | (x << 2)) & 0x1249249249249249ull;
    return x;
}

// the quantised box centre on one axis (trace_build.wgsl:30-32): c = (lo + hi) * 0.5,
// clamp((c - lo_b) * ext, 0, 0.999) * scale, truncated
__device__ __forceinline__ uint32_t quantise(float blo, float bhi, float plo, float pext, float scale) {
    float c = fmul(fadd(blo, bhi), 0.5f);
    float x = fmul(fsub(c, plo), pext);
    x = wmin(wmax(x, 0.0f), 0.999f);
    return __float2uint_rz(fmul(x, scale));
}

template <typename K> struct KeyTraits;
template <> struct KeyTraits<uint32_t> { static constexpr int PASSES = 4; };
template <> struct KeyTraits<uint64_t> { static constexpr int PASSES = 8; };

constexpr int MH_THREADS = 256;

// codes of n items, and the 256-bin histogram of every radix pass's digit into hist[pass][256]
template <typename K>
__global__ void __launch_bounds__(MH_THREADS) morton_hist_kernel(const float4 *__restrict__ boxes, uint32_t n,
                                                                 float3 plo, float3 pext, const float *__restrict__ dlo_ext,
                                                                 K *__restrict__ codes, uint32_t *__restrict__ hist) {
    constexpr int P = KeyTraits<K>::PASSES;
    __shared__ uint32_t sh[P * 256];
    for (int i = threadIdx.x; i < P * 256; i += MH_THREADS) sh[i] = 0;
    if (dlo_ext) {
        plo = make_float3(dlo_ext[0], dlo_ext[1], dlo_ext[2]);
        pext = make_float3(dlo_ext[3], dlo_ext[4], dlo_ext[5]);
    }
    __syncthreads();
    for (uint32_t i = blockIdx.x * MH_THREADS + threadIdx.x; i < n; i += gridDim.x * MH_THREADS) {
        float4 lo = __ldg(&boxes[2 * (size_t)i]), hi = __ldg(&boxes[2 * (size_t)i + 1]);
        K code;
        if constexpr (sizeof(K) == 4) {
            uint32_t qx = quantise(lo.x, hi.x, plo.x, pext.x, 1024.0f);
            uint32_t qy = quantise(lo.y, hi.y, plo.y, pext.y, 1024.0f);
            uint32_t qz = quantise(lo.z, hi.z, plo.z, pext.z, 1024.0f);
            code = (spread10(qx) << 2) | (spread10(qy) << 1) | spread10(qz);
        } else {
            uint32_t qx = quantise(lo.x, hi.x, plo.x, pext.x, 2097152.0f);
            uint32_t qy = quantise(lo.y, hi.y, plo.y, pext.y, 2097152.0f);
            uint32_t qz = quantise(lo.z, hi.z, plo.z, pext.z, 2097152.0f);
            code = (spread21(qx) << 2) | (spread21(qy) << 1) | spread21(qz);
        }
        codes[i] = code;
#pragma unroll
        for (int p = 0; p < P; p++) atomicAdd(&sh[p * 256 + (uint32_t)((code >> (8 * p)) & 255u)], 1u);
    }
    __syncthreads();
    for (int i = threadIdx.x; i < P * 256; i += MH_THREADS)
        if (sh[i]) atomicAdd(&hist[i], sh[i]);
}

// ---- block scan (THREADS threads, one value each) ----------------------------------------------
template <int THREADS, typename T>
__device__ __forceinline__ T block_excl_scan(T v, T *s_warp, T &total) {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    T x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        T y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) s_warp[w] = x;
    __syncthreads();
    if (w == 0) {
        T t = lane < THREADS / 32 ? s_warp[lane] : T(0);
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            T y = __shfl_up_sync(0xffffffffu, t, o);
            if (lane >= o) t += y;
        }
        if (lane < THREADS / 32) s_warp[lane] = t;
    }
    __syncthreads();
    T excl = (w ? s_warp[w - 1] : T(0)) + x - v;
    total = s_warp[THREADS / 32 - 1];
    __syncthreads();
    return excl;
}

// ---- onesweep radix sort ---------------------------------------------------------------------
constexpr int OS_THREADS = 512;                     // (the first 256 threads also own one digit each)
constexpr int OS_WARPS = OS_THREADS / 32;
constexpr int OS_ITEMS = 16;
constexpr int OS_TILE = OS_THREADS * OS_ITEMS;      // 8192 keys per tile
constexpr int OS_MINB = 2;                          // blocks per SM (64 registers a thread)
constexpr uint32_t FLAG_AGG = 1u << 30, FLAG_PRE = 2u << 30, VAL_MASK = (1u << 30) - 1;

template <typename K>
struct OsShared {
    uint32_t warp_hist[OS_WARPS][256];
    uint32_t digit_start[256];
    uint32_t global_excl[256];
    uint32_t scan[OS_WARPS];
    uint32_t tile;
    K key_stage[OS_TILE];
    uint32_t val_stage[OS_TILE];
};

__device__ __forceinline__ uint32_t ld_volatile(const uint32_t *p) { return *(const volatile uint32_t *)p; }
__device__ __forceinline__ void st_volatile(uint32_t *p, uint32_t v) { *(volatile uint32_t *)p = v; }

// One radix pass over bits [shift, shift + 8). first: the values are the items' indices.
// A tile's keys are ranked warp by warp (the lanes holding one digit: one ballot per digit bit; the
// group's leader takes the group's places from the warp's counter with one shared atomic - the
// warp's items in order, so the ranks are stable - results read after all 16 are issued), staged in
// digit order in shared memory with their values (read only then, so that the ranking keeps its
// registers), and written out at their digit's global offset: the tiles before it (decoupled
// look-back over posted counts / prefixes) plus the digits before it (the pass's histogram). A
// full tile (all but the last) ranks without bounds checks and without the validity ballot.
template <typename K, bool FIRST>
__global__ void __launch_bounds__(OS_THREADS, OS_MINB) onesweep_kernel(const K *__restrict__ keys_in,
                                                                 const uint32_t *__restrict__ vals_in,
                                                                 K *__restrict__ keys_out, uint32_t *__restrict__ vals_out,
                                                                 uint32_t n, int shift, const uint32_t *__restrict__ hist,
                                                                 uint32_t *status, uint32_t *tile_counter, uint32_t *err) {
    extern __shared__ __align__(16) unsigned char os_smem[];
    OsShared<K> &S = *reinterpret_cast<OsShared<K> *>(os_smem);
    const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
    if (tid == 0) S.tile = atomicAdd(tile_counter, 1u);
    for (int i = tid; i < OS_WARPS * 256; i += OS_THREADS) (&S.warp_hist[0][0])[i] = 0;
    __syncthreads();
    const uint32_t tile = S.tile;
    const uint32_t tile0 = tile * OS_TILE;
    const uint32_t in_tile = min((uint32_t)OS_TILE, n - tile0);
    const bool full = in_tile == (uint32_t)OS_TILE;

    K key[OS_ITEMS];
    uint32_t rank[OS_ITEMS];   // rank: the leader's base | leader << 16 | lanes before << 24, then the rank
    const uint32_t lt_mask = (1u << lane) - 1u;
    const uint32_t idx0 = tile0 + w * (32 * OS_ITEMS) + lane;
#pragma unroll
    for (int k = 0; k < OS_ITEMS; k++) {
        const uint32_t idx = idx0 + k * 32;
        key[k] = (full || idx < n) ? keys_in[idx] : K(0);
    }
    if (full) {
#pragma unroll
        for (int k = 0; k < OS_ITEMS; k++) {
            const uint32_t d = (uint32_t)((key[k] >> shift) & 255u);
            // the lanes with this lane's digit: one ballot per digit bit
            uint32_t peers = 0xffffffffu;
#pragma unroll
            for (int bit = 0; bit < 8; bit++) {
                const bool on = (d >> bit) & 1u;
                const uint32_t bal = __ballot_sync(0xffffffffu, on);
                peers &= on ? bal : ~bal;
            }
            const int leader = __ffs(peers) - 1;
            uint32_t base = 0;
            if (lane == leader) base = atomicAdd(&S.warp_hist[w][d], (uint32_t)__popc(peers));
            rank[k] = base | (uint32_t)leader << 16 | (uint32_t)__popc(peers & lt_mask) << 24;
        }
    } else {
#pragma unroll
        for (int k = 0; k < OS_ITEMS; k++) {
            const uint32_t idx = idx0 + k * 32;
            const uint32_t d = idx < n ? (uint32_t)((key[k] >> shift) & 255u) : 0x100u;
            // (and one ballot for validity)
            uint32_t peers = 0xffffffffu;
#pragma unroll
            for (int bit = 0; bit < 9; bit++) {
                const bool on = (d >> bit) & 1u;
                const uint32_t bal = __ballot_sync(0xffffffffu, on);
                peers &= on ? bal : ~bal;
            }
            const int leader = __ffs(peers) - 1;
            uint32_t base = 0;
            if (d < 256 && lane == leader) base = atomicAdd(&S.warp_hist[w][d], (uint32_t)__popc(peers));
            rank[k] = base | (uint32_t)leader << 16 | (uint32_t)__popc(peers & lt_mask) << 24;
        }
    }
#pragma unroll
    for (int k = 0; k < OS_ITEMS; k++)
        rank[k] = (__shfl_sync(0xffffffffu, rank[k], (rank[k] >> 16) & 31u) & 0xffffu) + (rank[k] >> 24);
    __syncthreads();
    // this thread's digit (the first 256 threads): the warps' offsets, the tile's count - posted at
    // once for the tiles after
    const bool dig = tid < 256;
    const uint32_t d = dig ? (uint32_t)tid : 0u;
    uint32_t count = 0;
    if (dig) {
#pragma unroll
        for (int ww = 0; ww < OS_WARPS; ww++) {
            uint32_t c = S.warp_hist[ww][d];
            S.warp_hist[ww][d] = count;
            count += c;
        }
        if (tile) st_volatile(&status[(size_t)tile * 256 + d], FLAG_AGG | count);
    }
    uint32_t tot;
    const uint32_t dstart = block_excl_scan<OS_THREADS>(count, S.scan, tot);
    if (dig) S.digit_start[d] = dstart;
    __syncthreads();
    // stage the tile in digit order (stable: warp, then item, then lane order), the values read now
#pragma unroll
    for (int k = 0; k < OS_ITEMS; k++) {
        const uint32_t idx = idx0 + k * 32;
        if (full || idx < n) {
            const uint32_t dk = (uint32_t)((key[k] >> shift) & 255u);
            const uint32_t pos = S.digit_start[dk] + S.warp_hist[w][dk] + rank[k];
            S.key_stage[pos] = key[k];
            S.val_stage[pos] = FIRST ? idx : vals_in[idx];
        }
    }
    // decoupled look-back: tile t's prefix of digit d over the tiles before it
    uint32_t excl = 0;
    if (tile == 0) {
        excl = block_excl_scan<OS_THREADS>(dig ? hist[d] : 0u, S.scan, tot);   // the digits before d, all keys
        if (dig) st_volatile(&status[d], FLAG_PRE | (excl + count));
    } else if (dig) {
        excl = 0;
        // the tiles before, nearest first, LB_WIDE statuses read at once (independent loads): their
        // counts summed up to the first inclusive prefix; a status not yet posted is waited for
        constexpr int LB_WIDE = 8;
        int64_t t = (int64_t)tile - 1;
        bool done = false;
        while (t >= 0 && !done) {
            uint32_t s[LB_WIDE];
#pragma unroll
            for (int j = 0; j < LB_WIDE; j++) s[j] = t - j >= 0 ? ld_volatile(&status[(size_t)(t - j) * 256 + d]) : 0u;
#pragma unroll
            for (int j = 0; j < LB_WIDE; j++) {
                if (done || t - j < 0) continue;
                uint32_t v = s[j];
                uint32_t spins = 0;
                while ((v & ~VAL_MASK) == 0) {
                    if (++spins > SPIN_LIMIT) { atomicOr(err, ST_TIMEOUT_SORT); break; }
                    __nanosleep(32);
                    v = ld_volatile(&status[(size_t)(t - j) * 256 + d]);
                }
                excl += v & VAL_MASK;
                if ((v & ~VAL_MASK) != FLAG_AGG) done = true;   // a prefix (or a timeout): done
            }
            t -= LB_WIDE;
        }
        st_volatile(&status[(size_t)tile * 256 + d], FLAG_PRE | (excl + count));
    }
    if (dig) S.global_excl[d] = excl;
    __syncthreads();
    for (uint32_t i = tid; i < in_tile; i += OS_THREADS) {
        K kk = S.key_stage[i];
        uint32_t dk = (uint32_t)((kk >> shift) & 255u);
        uint32_t g = S.global_excl[dk] + (i - S.digit_start[dk]);
        if (g >= n) {                                            // only after a look-back that ran out
            atomicOr(err, ST_TIMEOUT_SORT);
            continue;
        }
        keys_out[g] = kk;
        vals_out[g] = S.val_stage[i];
    }
}

// ---- LBVH: Karras's tree, made bottom-up in one pass -----------------------------------------
template <typename K>
__device__ __forceinline__ int delta_at(const K *__restrict__ codes, uint32_t i, uint32_t j) {
    K a = __ldg(&codes[i]), b = __ldg(&codes[j]);
    if constexpr (sizeof(K) == 4) {
        if (a == b) return 32 + __clz(i ^ j);
        return __clz(a ^ b);
    } else {
        if (a == b) return 64 + __clz(i ^ j);
        return __clzll((long long)(a ^ b));
    }
}
// a node over [l, r] is its parent's left child (the parent splits at r) or right child (at l - 1)
template <typename K>
__device__ __forceinline__ bool is_left_child(const K *codes, uint32_t l, uint32_t r, uint32_t n) {
    return l == 0 || (r != n - 1 && delta_at(codes, r, r + 1) > delta_at(codes, l - 1, l));
}

__device__ __forceinline__ void store_node(Node *p, float lx, float ly, float lz, uint32_t a, float hx, float hy, float hz,
                                           uint32_t b) {
    float4 *q = reinterpret_cast<float4 *>(p);
    q[0] = make_float4(lx, ly, lz, __uint_as_float(a));
    q[1] = make_float4(hx, hy, hz, __uint_as_float(b));
}

template <typename K>
__global__ void __launch_bounds__(256) lbvh_kernel(const K *__restrict__ codes, const uint32_t *__restrict__ items,
                                                   const float4 *__restrict__ boxes, uint32_t n, uint32_t node0,
                                                   uint32_t ref0, uint32_t ref_add, Node *nodes, uint32_t *__restrict__ aux,
                                                   uint32_t *other, uint32_t *err) {
    const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n) return;
    uint32_t item = __ldg(&items[j]);
    if (item >= n) {                                            // (a sort that went wrong: said, not followed)
        atomicOr(err, ST_TIMEOUT_SORT);
        item = 0;
    }
    float4 lo = __ldg(&boxes[2 * (size_t)item]), hi = __ldg(&boxes[2 * (size_t)item + 1]);
    float bl[3] = {lo.x, lo.y, lo.z}, bh[3] = {hi.x, hi.y, hi.z};
    uint32_t cur = n - 1 + j;                                   // relative to node0
    store_node(&nodes[cur], bl[0], bl[1], bl[2], ref0 + j, bh[0], bh[1], bh[2], LEAF_BIT | 1u);
    aux[j] = item + ref_add;
    if (n == 1) return;
    uint32_t l = j, r = j;
    bool left = is_left_child(codes, l, r, n);
    while (true) {
        const uint32_t split = left ? r : l - 1;
        __threadfence();                                        // our node before the exchange
        const uint32_t got = atomicExch(&other[split], left ? l : r);
        if (got == 0xffffffffu) return;                         // the sibling makes the parent
        __threadfence();
        uint32_t L, R, lc, rc;
        if (left) { L = l; R = got; lc = cur; rc = got == split + 1 ? n + split : split + 1; }
        else { L = got; R = r; rc = cur; lc = got == split ? n - 1 + split : split; }
        const uint32_t sib = left ? rc : lc;
        const float4 *sp = reinterpret_cast<const float4 *>(&nodes[sib]);
        float4 s0 = __ldcg(sp), s1 = __ldcg(sp + 1);
        float al[3], ah[3], cl[3], ch[3];                        // left child's box, right child's
        if (left) {
            al[0] = bl[0]; al[1] = bl[1]; al[2] = bl[2]; ah[0] = bh[0]; ah[1] = bh[1]; ah[2] = bh[2];
            cl[0] = s0.x; cl[1] = s0.y; cl[2] = s0.z; ch[0] = s1.x; ch[1] = s1.y; ch[2] = s1.z;
        } else {
            al[0] = s0.x; al[1] = s0.y; al[2] = s0.z; ah[0] = s1.x; ah[1] = s1.y; ah[2] = s1.z;
            cl[0] = bl[0]; cl[1] = bl[1]; cl[2] = bl[2]; ch[0] = bh[0]; ch[1] = bh[1]; ch[2] = bh[2];
        }
#pragma unroll
        for (int k = 0; k < 3; k++) { bl[k] = wmin(al[k], cl[k]); bh[k] = wmax(ah[k], ch[k]); }
        const bool root = L == 0 && R == n - 1;
        bool pleft = false;
        uint32_t pidx = 0;
        if (!root) {
            pleft = is_left_child(codes, L, R, n);
            pidx = pleft ? R : L;
        }
        store_node(&nodes[pidx], bl[0], bl[1], bl[2], node0 + lc, bh[0], bh[1], bh[2], node0 + rc);
        if (root) return;
        cur = pidx; l = L; r = R; left = pleft;
    }
}

// ---- PLOC -------------------------------------------------------------------------------------
constexpr int PL_THREADS = 256;
constexpr int PL_PER = 4;                          // clusters per thread
constexpr int PL_TILE = PL_THREADS * PL_PER;       // 1024 clusters per tile
constexpr int PL_R = 16;                           // the search radius (trace_ploc.wgsl R)
constexpr int PL_WIN = PL_TILE + 4 * PL_R;         // the tile's clusters with their neighbours' neighbours
constexpr int PL_NN = PL_TILE + 2 * PL_R;          // the clusters whose nearest the tile needs

// a cluster: its box and id (internal k 0..n-2, leaf j at n - 1 + j), laid out as a Node
struct __align__(16) Cl {
    float lo[3];
    uint32_t id;
    float hi[3];
    uint32_t pad;
};

struct PlocState {
    uint32_t nc_next;
    uint32_t bar_count;
    uint32_t bar_gen;
    uint32_t pad;
};

struct PlocShared {
    Cl win[PL_WIN];
    uint32_t nn[PL_NN];
    uint32_t scan[PL_THREADS / 32];
    uint64_t prefix;         // (keep, merge) of the tiles before this one
    uint32_t keep_total;
};

// area (trace_ploc.wgsl:18) of the two clusters' joined box, the reference's order of operations
__device__ __forceinline__ float joined_area(const Cl &a, const Cl &b) {
    float ex = fsub(wmax(a.hi[0], b.hi[0]), wmin(a.lo[0], b.lo[0]));
    float ey = fsub(wmax(a.hi[1], b.hi[1]), wmin(a.lo[1], b.lo[1]));
    float ez = fsub(wmax(a.hi[2], b.hi[2]), wmin(a.lo[2], b.lo[2]));
    return fadd(fadd(fmul(ex, ey), fmul(ey, ez)), fmul(ez, ex));
}
// nearer (trace_ploc.wgsl:60-66)
__device__ __forceinline__ bool nearer(float d, uint32_t i, uint32_t j, float bd, uint32_t bj) {
    if (bj == 0xffffffffu || d < bd) return true;
    if (d > bd) return false;
    uint32_t mn = min(i, j), bmn = min(i, bj);
    return mn < bmn || (mn == bmn && max(i, j) < max(i, bj));
}

__device__ __forceinline__ void final_node(const Cl &c, uint32_t n, uint32_t node0, uint32_t ref0, Node *out) {
    uint32_t x = c.id, a, b;
    if (x < n - 1) { a = node0 + 1 + 2 * x; b = node0 + 2 + 2 * x; }
    else { a = ref0 + x - (n - 1); b = LEAF_BIT | 1u; }
    store_node(out, c.lo[0], c.lo[1], c.lo[2], a, c.hi[0], c.hi[1], c.hi[2], b);
}

__device__ __forceinline__ uint64_t ld_volatile64(const uint64_t *p) { return *(const volatile uint64_t *)p; }
__device__ __forceinline__ void st_volatile64(uint64_t *p, uint64_t v) { *(volatile uint64_t *)p = v; }

constexpr uint64_t PF_AGG = 1ull << 62, PF_PRE = 2ull << 62, PF_MASK = 3ull << 62;
__device__ __forceinline__ uint64_t pack_km(uint64_t keep, uint64_t merge) { return (keep << 31) | merge; }

// A grid barrier for a cooperative launch (all blocks resident), bounded: after SPIN_LIMIT polls it
// flags ST_TIMEOUT_BARRIER and lets the block go on (the result is then wrong, and said to be).
__device__ void grid_barrier(PlocState *st, uint32_t *err) {
    __syncthreads();
    if (threadIdx.x == 0) {
        volatile uint32_t *gen = &st->bar_gen;
        uint32_t g = *gen;
        __threadfence();
        if (atomicAdd(&st->bar_count, 1u) == gridDim.x - 1) {
            atomicExch(&st->bar_count, 0u);
            __threadfence();
            atomicAdd(&st->bar_gen, 1u);
        } else if (!(ld_volatile(err) & ST_TIMEOUT_BARRIER)) {
            uint32_t spins = 0;
            while (*gen == g) {
                if (++spins > SPIN_LIMIT) { atomicOr(err, ST_TIMEOUT_BARRIER); break; }
                __nanosleep(64);
            }
        }
        __threadfence();
    }
    __syncthreads();
}

// One tile of one round: nearest, keep/merge, prefix (look-back when lookback), merges, compaction.
// Returns (to thread 0's caller through S.keep_total) the clusters the tile keeps.
__device__ void ploc_tile(PlocShared &S, const Cl *__restrict__ Lp, Cl *__restrict__ Lq, uint32_t nc, uint32_t tile,
                          uint32_t ntiles, uint32_t n, uint32_t node0, uint32_t ref0, Node *nodes, uint64_t *stat,
                          bool lookback, PlocState *st, uint32_t *err) {
    const int tid = threadIdx.x;
    const int64_t base = (int64_t)tile * PL_TILE;
    const int64_t w0 = base - 2 * PL_R;                          // the window's first position
    // the window: clusters w0 .. w0 + PL_WIN - 1 that exist
    for (int i = tid; i < PL_WIN; i += PL_THREADS) {
        int64_t g = w0 + i;
        if (g >= 0 && g < (int64_t)nc) {
            const float4 *src = reinterpret_cast<const float4 *>(&Lp[g]);
            float4 *dst = reinterpret_cast<float4 *>(&S.win[i]);
            dst[0] = __ldcg(src);
            dst[1] = __ldcg(src + 1);
        }
    }
    __syncthreads();
    // nearest of the clusters base - R .. base + TILE + R
    for (int i = tid; i < PL_NN; i += PL_THREADS) {
        int64_t p = base - PL_R + i;
        if (p < 0 || p >= (int64_t)nc) continue;
        const uint32_t pi = (uint32_t)p;
        const uint32_t j0 = pi > PL_R ? pi - PL_R : 0u;
        const uint32_t j1 = min(pi + PL_R, nc - 1);
        const Cl &c = S.win[p - w0];
        float bd = 0.0f;
        uint32_t bj = 0xffffffffu;
        for (uint32_t j = j0; j <= j1; j++) {
            if (j == pi) continue;
            float d = joined_area(c, S.win[(int64_t)j - w0]);
            if (nearer(d, pi, j, bd, bj)) { bd = d; bj = j; }
        }
        S.nn[i] = bj;
    }
    __syncthreads();
    // keep / merge of this thread's clusters base + tid * PER + k
    uint32_t keepm = 0, mergem = 0;
#pragma unroll
    for (int k = 0; k < PL_PER; k++) {
        int64_t i = base + tid * PL_PER + k;
        if (i >= (int64_t)nc) continue;
        uint32_t j = S.nn[i - (base - PL_R)];
        bool mu = j < nc && S.nn[(int64_t)j - (base - PL_R)] == (uint32_t)i;
        if (!(mu && (uint32_t)i > j)) keepm |= 1u << k;
        if (mu && (uint32_t)i < j) mergem |= 1u << k;
    }
    uint32_t tot;
    const uint32_t packed = __popc(keepm) | (__popc(mergem) << 16);
    const uint32_t excl = block_excl_scan<PL_THREADS>(packed, S.scan, tot);
    const uint32_t tile_keep = tot & 0xffffu, tile_merge = tot >> 16;
    if (tid == 0) {
        uint64_t pre = 0;
        if (lookback) {
            if (tile == 0) st_volatile64(&stat[0], PF_PRE | pack_km(tile_keep, tile_merge));
            else {
                st_volatile64(&stat[tile], PF_AGG | pack_km(tile_keep, tile_merge));
                int64_t t = (int64_t)tile - 1;
                uint64_t kk = 0, mm = 0;
                while (t >= 0) {
                    uint64_t s = ld_volatile64(&stat[t]);
                    uint32_t spins = 0;
                    while ((s & PF_MASK) == 0) {
                        if (++spins > SPIN_LIMIT) { atomicOr(err, ST_TIMEOUT_PLOC); break; }
                        __nanosleep(32);
                        s = ld_volatile64(&stat[t]);
                    }
                    kk += (s >> 31) & 0x7fffffffull;
                    mm += s & 0x7fffffffull;
                    if ((s & PF_MASK) != PF_AGG) break;
                    t--;
                }
                pre = pack_km(kk, mm);
                st_volatile64(&stat[tile], PF_PRE | pack_km(kk + tile_keep, mm + tile_merge));
            }
            if (tile == ntiles - 1) st->nc_next = (uint32_t)((pre >> 31) & 0x7fffffffull) + tile_keep;
        }
        S.prefix = pre;
        S.keep_total = tile_keep;
    }
    __syncthreads();
    uint32_t dest = (uint32_t)((S.prefix >> 31) & 0x7fffffffull) + (excl & 0xffffu);
    uint32_t m = (uint32_t)(S.prefix & 0x7fffffffull) + (excl >> 16);
#pragma unroll
    for (int k = 0; k < PL_PER; k++) {
        if (!((keepm >> k) & 1u)) continue;
        int64_t i = base + tid * PL_PER + k;
        const Cl &c = S.win[i - w0];
        Cl out = c;
        if (dest >= nc || m + 1 >= nc) {                         // only after a look-back that ran out
            atomicOr(err, ST_TIMEOUT_PLOC);
            break;
        }
        if ((mergem >> k) & 1u) {
            uint32_t j = S.nn[i - (base - PL_R)];
            const Cl &dd = S.win[(int64_t)j - w0];
            uint32_t kid = nc - 2 - m;                           // (n - 2) - (merges before it)
            m++;
#pragma unroll
            for (int q = 0; q < 3; q++) { out.lo[q] = wmin(c.lo[q], dd.lo[q]); out.hi[q] = wmax(c.hi[q], dd.hi[q]); }
            out.id = kid;
            final_node(c, n, node0, ref0, &nodes[1 + 2 * kid]);
            final_node(dd, n, node0, ref0, &nodes[2 + 2 * kid]);
            if (kid == 0)
                store_node(&nodes[0], out.lo[0], out.lo[1], out.lo[2], node0 + 1, out.hi[0], out.hi[1], out.hi[2], node0 + 2);
        }
        float4 *dst = reinterpret_cast<float4 *>(&Lq[dest]);
        dst[0] = make_float4(out.lo[0], out.lo[1], out.lo[2], __uint_as_float(out.id));
        dst[1] = make_float4(out.hi[0], out.hi[1], out.hi[2], 0.0f);
        dest++;
    }
}

__global__ void __launch_bounds__(PL_THREADS) ploc_kernel(Cl *listA, Cl *listB, uint32_t n, uint32_t node0, uint32_t ref0,
                                                          Node *nodes, uint64_t *stat0, uint64_t *stat1, PlocState *st,
                                                          uint32_t *err) {
    extern __shared__ __align__(16) unsigned char pl_smem[];
    PlocShared &S = *reinterpret_cast<PlocShared *>(pl_smem);
    uint32_t nc = n, r = 0;
    Cl *Lp = listA, *Lq = listB;
    while (nc > 1) {
        const uint32_t ntiles = (nc + PL_TILE - 1) / PL_TILE;
        if (ntiles == 1) {                                       // the rest in one block
            if (blockIdx.x != 0) return;
            while (nc > 1) {
                ploc_tile(S, Lp, Lq, nc, 0, 1, n, node0, ref0, nodes, nullptr, false, st, err);
                __syncthreads();
                const uint32_t next = S.keep_total;
                if (next >= nc) {                                // every round merges at least one pair
                    if (threadIdx.x == 0) atomicOr(err, ST_TIMEOUT_PLOC);
                    return;
                }
                nc = next;
                Cl *t = Lp; Lp = Lq; Lq = t;
                __threadfence_block();
                __syncthreads();
            }
            return;
        }
        uint64_t *stat = (r & 1) ? stat1 : stat0, *other = (r & 1) ? stat0 : stat1;
        for (uint32_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
            ploc_tile(S, Lp, Lq, nc, tile, ntiles, n, node0, ref0, nodes, stat, true, st, err);
            __syncthreads();
        }
        for (uint32_t i = blockIdx.x * PL_THREADS + threadIdx.x; i < ntiles; i += gridDim.x * PL_THREADS) other[i] = 0;
        __threadfence();
        grid_barrier(st, err);
        const uint32_t next = ld_volatile(&st->nc_next);
        if (next >= nc || (ld_volatile(err) & (ST_TIMEOUT_PLOC | ST_TIMEOUT_BARRIER))) {
            if (threadIdx.x == 0) atomicOr(err, ST_TIMEOUT_PLOC);
            return;                                              // (every block sees the same: all leave)
        }
        nc = next;
        Cl *t = Lp; Lp = Lq; Lq = t;
        r++;
    }
}

// the first clusters: the leaves in sorted order, and aux (the reference's `leaves` in PLOC mode;
// the leaf nodes themselves are all overwritten by the merges, so they are not written)
__global__ void ploc_leaves_kernel(const uint32_t *__restrict__ items, const float4 *__restrict__ boxes, uint32_t n,
                                   uint32_t ref0, uint32_t ref_add, Cl *__restrict__ list, uint32_t *__restrict__ aux,
                                   uint32_t *err) {
    const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n) return;
    uint32_t item = __ldg(&items[j]);
    if (item >= n) {
        atomicOr(err, ST_TIMEOUT_SORT);
        item = 0;
    }
    float4 lo = __ldg(&boxes[2 * (size_t)item]), hi = __ldg(&boxes[2 * (size_t)item + 1]);
    float4 *dst = reinterpret_cast<float4 *>(&list[j]);
    dst[0] = make_float4(lo.x, lo.y, lo.z, __uint_as_float(n - 1 + j));
    dst[1] = make_float4(hi.x, hi.y, hi.z, 0.0f);
    aux[j] = item + ref_add;
}

// ---- triangle boxes and the mesh box ----------------------------------------------------------
// a float's bits as an unsigned key in the float order
__device__ __forceinline__ uint32_t fkey(float f) {
    uint32_t u = __float_as_uint(f);
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__device__ __forceinline__ float fkey_inv(uint32_t k) {
    return __uint_as_float((k & 0x80000000u) ? (k & 0x7fffffffu) : ~k);
}

__global__ void __launch_bounds__(256) tri_boxes_kernel(const float4 *__restrict__ tris, uint32_t n, float4 *__restrict__ boxes,
                                                        uint32_t *__restrict__ bkeys) {
    float mlo[3] = {1e30f, 1e30f, 1e30f}, mhi[3] = {-1e30f, -1e30f, -1e30f};
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        float4 q = __ldg(&tris[3 * (size_t)i]), u = __ldg(&tris[3 * (size_t)i + 1]), v = __ldg(&tris[3 * (size_t)i + 2]);
        float p0[3] = {q.x, q.y, q.z};
        float p1[3] = {fadd(q.x, u.x), fadd(q.y, u.y), fadd(q.z, u.z)};
        float p2[3] = {fadd(q.x, v.x), fadd(q.y, v.y), fadd(q.z, v.z)};
        float lo[3], hi[3];
#pragma unroll
        for (int k = 0; k < 3; k++) {
            // triangle_bounds (scene.c:65-74): from q, grown by q + u then q + v (r_fmin / r_fmax), padded by 1e-3
            lo[k] = rfmin(rfmin(p0[k], p1[k]), p2[k]);
            hi[k] = rfmax(rfmax(p0[k], p1[k]), p2[k]);
            mlo[k] = rfmin(mlo[k], lo[k]);
            mhi[k] = rfmax(mhi[k], hi[k]);
            lo[k] = fsub(lo[k], 1e-3f);
            hi[k] = fadd(hi[k], 1e-3f);
        }
        boxes[2 * (size_t)i] = make_float4(lo[0], lo[1], lo[2], 0.0f);
        boxes[2 * (size_t)i + 1] = make_float4(hi[0], hi[1], hi[2], 0.0f);
    }
    // the mesh box (mesh_bounds, scene.c:638-646): min / max of all corners, order-free
#pragma unroll
    for (int k = 0; k < 3; k++) {
        uint32_t a = fkey(mlo[k]), b = fkey(mhi[k]);
        for (int o = 16; o > 0; o >>= 1) {
            a = min(a, __shfl_xor_sync(0xffffffffu, a, o));
            b = max(b, __shfl_xor_sync(0xffffffffu, b, o));
        }
        if ((threadIdx.x & 31) == 0) { atomicMin(&bkeys[k], a); atomicMax(&bkeys[3 + k], b); }
    }
}

// the mesh box's keys -> bounds (6 floats) and build_queue's lo / ext (trace_gpu.c:605-611)
__global__ void bounds_params_kernel(const uint32_t *bkeys, float *bounds6, float *lo_ext) {
    if (threadIdx.x != 0) return;
    for (int k = 0; k < 3; k++) {
        float lo = fkey_inv(bkeys[k]), hi = fkey_inv(bkeys[3 + k]);
        if (bounds6) { bounds6[k] = lo; bounds6[3 + k] = hi; }
        if (lo_ext) {
            float e = fsub(hi, lo);
            lo_ext[k] = lo;
            lo_ext[3 + k] = e > 0.0f ? __fdiv_rn(1.0f, e) : 0.0f;
        }
    }
}

// ---- host orchestration -----------------------------------------------------------------------
static size_t align256(size_t x) { return (x + 255) / 256 * 256; }

// kernel attributes set once per device (a context is used from one host thread at a time, as the
// reference's Gpu is: engine/gpu/gpu.h:32-42)
struct DevCache {
    bool os_attr[2];
    int ploc_per_sm;
};
static DevCache g_dev_cache[64];
static DevCache &dev_cache() {
    int d = 0;
    cudaGetDevice(&d);
    return g_dev_cache[d & 63];
}

// Every pass of a stable LSD radix sort of n keys (values: the keys' positions to start with), the
// passes' 256-bin histograms already in hist[pass][256], look-back status words zeroed. On return
// kin / vin hold the sorted keys and the permutation (the buffers swap roles pass by pass).
template <typename K>
static void onesweep_passes(K *&kin, K *&kout, uint32_t *&vin, uint32_t *&vout, uint32_t n, const uint32_t *hist,
                            uint32_t *status, uint32_t *counters, uint32_t tiles, uint32_t *d_status, cudaStream_t st) {
    constexpr int P = KeyTraits<K>::PASSES;
    const size_t smem = sizeof(OsShared<K>);
    DevCache &dc = dev_cache();
    if (!dc.os_attr[sizeof(K) == 8]) {
        cudaFuncSetAttribute(onesweep_kernel<K, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        cudaFuncSetAttribute(onesweep_kernel<K, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        dc.os_attr[sizeof(K) == 8] = true;
    }
    for (int pass = 0; pass < P; pass++) {
        uint32_t *stp = status + (size_t)pass * tiles * 256;
        if (pass == 0)
            onesweep_kernel<K, true><<<tiles, OS_THREADS, smem, st>>>(kin, nullptr, kout, vout, n, 8 * pass, hist + pass * 256,
                                                                      stp, counters + pass, d_status);
        else
            onesweep_kernel<K, false><<<tiles, OS_THREADS, smem, st>>>(kin, vin, kout, vout, n, 8 * pass, hist + pass * 256,
                                                                       stp, counters + pass, d_status);
        std::swap(kin, kout);
        std::swap(vin, vout);
    }
}

struct BuildLayout {
    size_t codes_a, codes_b, vals_a, vals_b, hist, status, counters, other, list_a, list_b, stat0, stat1, pstate, total;
    uint32_t tiles;
};
static BuildLayout layout_for(uint32_t n, int key_bits, int builder);

// ---- a sort of 32-bit keys for other users (the ray reordering) ----------------------------
size_t sort_u32_scratch_bytes(uint64_t n) { return layout_for((uint32_t)n, 30, 0).total; }

SortU32 sort_u32_carve(void *scratch, uint64_t n) {
    BuildLayout L = layout_for((uint32_t)n, 30, 0);
    char *s = reinterpret_cast<char *>((reinterpret_cast<uintptr_t>(scratch) + 255) / 256 * 256);
    SortU32 r;
    r.keys = reinterpret_cast<uint32_t *>(s + L.codes_a);
    r.hist = reinterpret_cast<uint32_t *>(s + L.hist);
    r.base = s;
    r.n = (uint32_t)n;
    return r;
}

cudaError_t sort_u32_clear(const SortU32 &S, cudaStream_t st) {
    BuildLayout L = layout_for(S.n, 30, 0);
    return cudaMemsetAsync(S.base + L.hist, 0, L.counters + 4 * 4 - L.hist, st);
}

cudaError_t sort_u32_run(const SortU32 &S, uint32_t *d_status, cudaStream_t st, const uint32_t **perm_out) {
    BuildLayout L = layout_for(S.n, 30, 0);
    uint32_t *ka = reinterpret_cast<uint32_t *>(S.base + L.codes_a), *kb = reinterpret_cast<uint32_t *>(S.base + L.codes_b);
    uint32_t *va = reinterpret_cast<uint32_t *>(S.base + L.vals_a), *vb = reinterpret_cast<uint32_t *>(S.base + L.vals_b);
    onesweep_passes<uint32_t>(ka, kb, va, vb, S.n, reinterpret_cast<uint32_t *>(S.base + L.hist),
                              reinterpret_cast<uint32_t *>(S.base + L.status), reinterpret_cast<uint32_t *>(S.base + L.counters),
                              L.tiles, d_status, st);
    *perm_out = va;
    return cudaGetLastError();
}

static BuildLayout layout_for(uint32_t n, int key_bits, int builder) {
    BuildLayout L{};
    const size_t K = key_bits == 63 ? 8 : 4;
    const int passes = key_bits == 63 ? 8 : 4;
    const size_t nn = n ? n : 1;
    L.tiles = (uint32_t)((nn + OS_TILE - 1) / OS_TILE);
    size_t off = 0;
    auto put = [&](size_t bytes) { size_t at = off; off += align256(bytes); return at; };
    L.codes_a = put(nn * K);
    L.codes_b = put(nn * K);
    L.vals_a = put(nn * 4);
    L.vals_b = put(nn * 4);
    // zeroed together: histograms, look-back status, tile counters
    L.hist = put((size_t)passes * 256 * 4);
    L.status = put((size_t)passes * L.tiles * 256 * 4);
    L.counters = put((size_t)passes * 4);
    if (builder == 1) {
        const size_t pt = (nn + PL_TILE - 1) / PL_TILE;
        L.list_a = put(nn * sizeof(Cl));
        L.list_b = put(nn * sizeof(Cl));
        L.stat0 = put(pt * 8);
        L.stat1 = put(pt * 8);
        L.pstate = put(sizeof(PlocState));
        L.other = 0;
    } else {
        L.other = put(nn * 4);
    }
    L.total = off + 256;
    return L;
}

size_t build_scratch_bytes(uint32_t n, int key_bits, int builder) {
    return layout_for(n, key_bits, builder == 1 && n > 2 ? 1 : 0).total;
}

template <typename K>
static cudaError_t build_typed(const lrc_build_params &p, const float *d_boxes, Node *d_nodes, uint32_t *d_aux,
                               char *scratch, const BuildLayout &L, uint32_t *d_status, int num_sms, cudaStream_t st,
                               const float *dlo_ext, bool ploc, uint32_t *d_sorted_codes_out, StageTimer *tm) {
    constexpr int P = KeyTraits<K>::PASSES;
    const uint32_t n = p.n;
    K *ca = reinterpret_cast<K *>(scratch + L.codes_a), *cb = reinterpret_cast<K *>(scratch + L.codes_b);
    uint32_t *va = reinterpret_cast<uint32_t *>(scratch + L.vals_a), *vb = reinterpret_cast<uint32_t *>(scratch + L.vals_b);
    uint32_t *hist = reinterpret_cast<uint32_t *>(scratch + L.hist);
    uint32_t *status = reinterpret_cast<uint32_t *>(scratch + L.status);
    uint32_t *counters = reinterpret_cast<uint32_t *>(scratch + L.counters);
    if (tm) tm->begin(LRC_TS_MORTON, st);
    cudaError_t e = cudaMemsetAsync(scratch + L.hist, 0, L.counters + (size_t)P * 4 - L.hist, st);
    if (e) return e;
    const float4 *boxes = reinterpret_cast<const float4 *>(d_boxes);
    {
        int grid = (int)std::min<uint64_t>(((uint64_t)n + MH_THREADS - 1) / MH_THREADS, (uint64_t)num_sms * 8);
        morton_hist_kernel<K><<<std::max(grid, 1), MH_THREADS, 0, st>>>(
            boxes, n, make_float3(p.lo[0], p.lo[1], p.lo[2]), make_float3(p.ext[0], p.ext[1], p.ext[2]), dlo_ext, ca, hist);
    }
    if (tm) tm->begin(LRC_TS_SORT, st);
    K *kin = ca, *kout = cb;
    uint32_t *vin = va, *vout = vb;
    onesweep_passes<K>(kin, kout, vin, vout, n, hist, status, counters, L.tiles, d_status, st);
    // sorted: codes in kin, items in vin
    if (d_sorted_codes_out)
        cudaMemcpyAsync(d_sorted_codes_out, kin, (size_t)n * sizeof(K), cudaMemcpyDeviceToDevice, st);
    const uint32_t blocks = (n + 255) / 256;
    if (tm) tm->begin(LRC_TS_HIERARCHY, st);
    if (!ploc) {
        uint32_t *other = reinterpret_cast<uint32_t *>(scratch + L.other);
        if (n > 1) cudaMemsetAsync(other, 0xff, (size_t)(n - 1) * 4, st);
        lbvh_kernel<K><<<blocks, 256, 0, st>>>(kin, vin, boxes, n, p.node0, p.ref0, p.ref_add, d_nodes, d_aux, other, d_status);
        if (tm) tm->end(st);
        return cudaGetLastError();
    }
    Cl *la = reinterpret_cast<Cl *>(scratch + L.list_a), *lb = reinterpret_cast<Cl *>(scratch + L.list_b);
    uint64_t *s0 = reinterpret_cast<uint64_t *>(scratch + L.stat0), *s1 = reinterpret_cast<uint64_t *>(scratch + L.stat1);
    PlocState *ps = reinterpret_cast<PlocState *>(scratch + L.pstate);
    ploc_leaves_kernel<<<blocks, 256, 0, st>>>(vin, boxes, n, p.ref0, p.ref_add, la, d_aux, d_status);
    e = cudaMemsetAsync(scratch + L.stat0, 0, L.pstate + sizeof(PlocState) - L.stat0, st);
    if (e) return e;
    const int psmem = (int)sizeof(PlocShared);
    int &per_sm = dev_cache().ploc_per_sm;
    if (per_sm <= 0) {
        cudaFuncSetAttribute(ploc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, psmem);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, ploc_kernel, PL_THREADS, psmem);
        if (per_sm < 1) per_sm = 1;
    }
    const uint32_t want = (n + PL_TILE - 1) / PL_TILE;
    uint32_t grid = std::min<uint32_t>((uint32_t)(per_sm * num_sms), std::max<uint32_t>(want, 1));
    uint32_t node0 = p.node0, ref0 = p.ref0, nn_ = n;
    void *args[] = {&la, &lb, &nn_, &node0, &ref0, &d_nodes, &s0, &s1, &ps, &d_status};
    e = cudaLaunchCooperativeKernel((void *)ploc_kernel, dim3(grid), dim3(PL_THREADS), args, psmem, st);
    if (tm) tm->end(st);
    if (e) return e;
    return cudaGetLastError();
}

cudaError_t build_device(const lrc_build_params &p, const float *d_boxes, Node *d_nodes, uint32_t *d_aux, void *d_scratch,
                         size_t scratch_bytes, uint32_t *d_status, int num_sms, cudaStream_t st,
                         uint32_t *d_sorted_codes_out) {
    return build_device_ext(p, d_boxes, nullptr, d_nodes, d_aux, d_scratch, scratch_bytes, d_status, num_sms, st,
                            d_sorted_codes_out, nullptr);
}

cudaError_t build_device_ext(const lrc_build_params &p, const float *d_boxes, const float *d_lo_ext, Node *d_nodes,
                             uint32_t *d_aux, void *d_scratch, size_t scratch_bytes, uint32_t *d_status, int num_sms,
                             cudaStream_t st, uint32_t *d_sorted_codes_out, StageTimer *tm) {
    if (p.n == 0) return cudaSuccess;
    const bool ploc = p.builder == 1 && p.n > 2;
    BuildLayout L = layout_for(p.n, p.key_bits, ploc ? 1 : 0);
    if (scratch_bytes < L.total) return cudaErrorInvalidValue;
    char *scratch = reinterpret_cast<char *>((reinterpret_cast<uintptr_t>(d_scratch) + 255) / 256 * 256);
    if (p.key_bits == 63)
        return build_typed<uint64_t>(p, d_boxes, d_nodes, d_aux, scratch, L, d_status, num_sms, st, d_lo_ext, ploc,
                                     d_sorted_codes_out, tm);
    return build_typed<uint32_t>(p, d_boxes, d_nodes, d_aux, scratch, L, d_status, num_sms, st, d_lo_ext, ploc,
                                 d_sorted_codes_out, tm);
}

__global__ void bkeys_init_kernel(uint32_t *bkeys) {
    if (threadIdx.x < 6) bkeys[threadIdx.x] = threadIdx.x < 3 ? 0xffffffffu : 0u;
}

cudaError_t triangle_boxes(const uint32_t *d_tris, uint32_t n, float *d_boxes, uint32_t *d_bkeys, cudaStream_t st,
                           int num_sms) {
    bkeys_init_kernel<<<1, 32, 0, st>>>(d_bkeys);
    if (n) {
        int grid = (int)std::min<uint64_t>(((uint64_t)n + 255) / 256, (uint64_t)num_sms * 8);
        tri_boxes_kernel<<<grid, 256, 0, st>>>(reinterpret_cast<const float4 *>(d_tris), n,
                                               reinterpret_cast<float4 *>(d_boxes), d_bkeys);
    }
    return cudaGetLastError();
}

// the union of n boxes (their padded corners) into the bound keys
__global__ void __launch_bounds__(256) boxes_bounds_kernel(const float4 *__restrict__ boxes, uint32_t n, uint32_t *bkeys) {
    uint32_t a[3] = {0xffffffffu, 0xffffffffu, 0xffffffffu}, b[3] = {0u, 0u, 0u};
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        float4 lo = __ldg(&boxes[2 * (size_t)i]), hi = __ldg(&boxes[2 * (size_t)i + 1]);
        a[0] = min(a[0], fkey(lo.x)); a[1] = min(a[1], fkey(lo.y)); a[2] = min(a[2], fkey(lo.z));
        b[0] = max(b[0], fkey(hi.x)); b[1] = max(b[1], fkey(hi.y)); b[2] = max(b[2], fkey(hi.z));
    }
#pragma unroll
    for (int k = 0; k < 3; k++) {
        for (int o = 16; o > 0; o >>= 1) {
            a[k] = min(a[k], __shfl_xor_sync(0xffffffffu, a[k], o));
            b[k] = max(b[k], __shfl_xor_sync(0xffffffffu, b[k], o));
        }
        if ((threadIdx.x & 31) == 0) { atomicMin(&bkeys[k], a[k]); atomicMax(&bkeys[3 + k], b[k]); }
    }
}

cudaError_t boxes_bounds(const float *d_boxes, uint32_t n, uint32_t *d_bkeys, cudaStream_t st, int num_sms, bool init) {
    if (init) bkeys_init_kernel<<<1, 32, 0, st>>>(d_bkeys);
    if (n) {
        int grid = (int)std::min<uint64_t>(((uint64_t)n + 255) / 256, (uint64_t)num_sms * 8);
        boxes_bounds_kernel<<<grid, 256, 0, st>>>(reinterpret_cast<const float4 *>(d_boxes), n, d_bkeys);
    }
    return cudaGetLastError();
}

cudaError_t bounds_params(const uint32_t *d_bkeys, float *d_bounds6, float *d_lo_ext, cudaStream_t st) {
    bounds_params_kernel<<<1, 32, 0, st>>>(d_bkeys, d_bounds6, d_lo_ext);
    return cudaGetLastError();
}

}  // namespace lrc
