// refit.cu - a built tree's boxes made again for moved items, on the topology as built: the
// reference's bvh_refit_boxes (engine/rt/bvh.c:471-485), which its top level uses for instances
// that only moved (build_tlas, engine/rt/accel.c:154-173; scene_update_instances :197-207).
//
// bvh_refit_boxes walks the nodes from the last back (children after parents in its preorder
// layout). The GPU trees have no such order, so the refit climbs instead: one thread per leaf sets
// the leaf's box from its items' boxes and walks up; at every inner node the first child to arrive
// stops and the second (the one that sees the other's box, published before its atomic) unions the
// two children and goes on. Union as bvh.c's box_add_box: left child's box, then the right's, with
// mn(a, b) = a < b ? a : b - exact, so the boxes are bvh_refit_boxes' to the bit.
#include "lrc_internal.cuh"

namespace lrc {

namespace {

__device__ __forceinline__ float mn(float a, float b) { return a < b ? a : b; }
__device__ __forceinline__ float mx(float a, float b) { return a > b ? a : b; }

// parent[i] of every node (the root's: ~0); a child index out of range is reported, not followed
__global__ void parent_kernel(const Node *__restrict__ nodes, uint32_t nn, uint32_t *__restrict__ parent, uint32_t *err) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nn) return;
    if (i == 0) parent[0] = ~0u;
    const uint32_t a = nodes[i].a, b = nodes[i].b;
    if (b & LEAF_BIT) return;
    if (a >= nn || b >= nn || a == 0 || b == 0) {
        atomicOr(err, ST_BAD_TREE);
        return;
    }
    parent[a] = i;
    parent[b] = i;
}

// from parent p up: at every inner node the first child to arrive stops, the second unions the
// two children (left, then right) and goes on
__device__ __forceinline__ void climb(Node *nodes, uint32_t nn, uint32_t p, const uint32_t *__restrict__ parent,
                                      uint32_t *flags, uint32_t *err) {
    for (uint32_t steps = 0; p != ~0u; steps++) {
        if (steps >= nn || p >= nn) {              // (no tree is that deep: a broken parent chain)
            atomicOr(err, ST_BAD_TREE);
            return;
        }
        __threadfence();                           // this child's box before the count the sibling reads
        if (atomicAdd(&flags[p], 1u) == 0) return; // the other child finishes this node
        __threadfence();
        const Node *q = &nodes[p];
        const Node *L = &nodes[q->a], *R = &nodes[q->b];
        float l0 = __ldcg(&L->lo[0]), l1 = __ldcg(&L->lo[1]), l2 = __ldcg(&L->lo[2]);
        float h0 = __ldcg(&L->hi[0]), h1 = __ldcg(&L->hi[1]), h2 = __ldcg(&L->hi[2]);
        l0 = mn(l0, __ldcg(&R->lo[0])); l1 = mn(l1, __ldcg(&R->lo[1])); l2 = mn(l2, __ldcg(&R->lo[2]));
        h0 = mx(h0, __ldcg(&R->hi[0])); h1 = mx(h1, __ldcg(&R->hi[1])); h2 = mx(h2, __ldcg(&R->hi[2]));
        Node *w = &nodes[p];
        w->lo[0] = l0; w->lo[1] = l1; w->lo[2] = l2;
        w->hi[0] = h0; w->hi[1] = h1; w->hi[2] = h2;
        p = parent[p];
    }
}

// items' boxes: item k's lo at box[k * stride + lo_at], hi at box[k * stride + lo_at + 1] (float4s)
__global__ void refit_kernel(Node *nodes, const uint32_t *__restrict__ aux, uint32_t nn, uint32_t naux, uint32_t ref_add,
                             const float4 *__restrict__ box, uint32_t nitems, uint32_t stride, uint32_t lo_at,
                             const uint32_t *__restrict__ parent, uint32_t *flags, uint32_t *err) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nn) return;
    const uint32_t a = nodes[i].a, b = nodes[i].b;
    if (!(b & LEAF_BIT)) return;
    const uint32_t count = b & ~LEAF_BIT;
    if (a >= naux || count > naux - a) {
        atomicOr(err, ST_BAD_TREE);
        return;
    }
    float lo[3] = {__int_as_float(0x7f800000), __int_as_float(0x7f800000), __int_as_float(0x7f800000)};
    float hi[3] = {-lo[0], -lo[1], -lo[2]};
    for (uint32_t k = 0; k < count; k++) {
        const uint32_t item = aux[a + k] - ref_add;
        if (item >= nitems) {
            atomicOr(err, ST_BAD_TREE);
            return;
        }
        const float4 l = __ldg(&box[(size_t)item * stride + lo_at]), h = __ldg(&box[(size_t)item * stride + lo_at + 1]);
        lo[0] = mn(lo[0], l.x); lo[1] = mn(lo[1], l.y); lo[2] = mn(lo[2], l.z);
        hi[0] = mx(hi[0], h.x); hi[1] = mx(hi[1], h.y); hi[2] = mx(hi[2], h.z);
    }
    Node *n = &nodes[i];
    n->lo[0] = lo[0]; n->lo[1] = lo[1]; n->lo[2] = lo[2];
    n->hi[0] = hi[0]; n->hi[1] = hi[1]; n->hi[2] = hi[2];
    climb(nodes, nn, parent[i], parent, flags, err);
}

// the walk's tree: leaf i's box from its triangles' corners (q, q + u, q + v) widened by pad on
// every side - pad = 2^-17 of the largest coordinate m of the source tree's root box, at most the
// reference's 1e-3 (triangle_bounds, scene.c:65-74) - then the climb. The slab test's bounds are
// off by at most about (m + |origin|) 2^-23 in units of t, so every hit stays inside its leaf's
// box (and its ancestors') for ray origins within about 60 m of the origin: the margin the
// reference's 1e-3 gives at its own 555-unit scene scale.
__global__ void walk_leaf_kernel(Node *nodes, const Node *__restrict__ src_root, const uint32_t *__restrict__ aux,
                                 uint32_t nn, uint32_t naux, const float4 *__restrict__ tris, uint32_t ntris,
                                 const uint32_t *__restrict__ parent, uint32_t *flags, uint32_t *err) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nn) return;
    const uint32_t a = nodes[i].a, b = nodes[i].b;
    if (!(b & LEAF_BIT)) return;
    const uint32_t count = b & ~LEAF_BIT;
    if (a >= naux || count > naux - a) {
        atomicOr(err, ST_BAD_TREE);
        return;
    }
    const Node &r = *src_root;
    float m = fmaxf(fmaxf(fmaxf(fabsf(r.lo[0]), fabsf(r.lo[1])), fmaxf(fabsf(r.lo[2]), fabsf(r.hi[0]))),
                    fmaxf(fabsf(r.hi[1]), fabsf(r.hi[2])));
    const float pad = fminf(1e-3f, m * 0x1p-17f);
    float lo[3] = {__int_as_float(0x7f800000), __int_as_float(0x7f800000), __int_as_float(0x7f800000)};
    float hi[3] = {-lo[0], -lo[1], -lo[2]};
    for (uint32_t k = 0; k < count; k++) {
        const uint32_t id = aux[a + k];
        if (id >= ntris) {
            atomicOr(err, ST_BAD_TREE);
            return;
        }
        const float4 q = __ldg(&tris[3 * (size_t)id]), u = __ldg(&tris[3 * (size_t)id + 1]),
                     v = __ldg(&tris[3 * (size_t)id + 2]);
        const float cx[3] = {q.x, q.x + u.x, q.x + v.x}, cy[3] = {q.y, q.y + u.y, q.y + v.y},
                    cz[3] = {q.z, q.z + u.z, q.z + v.z};
#pragma unroll
        for (int j = 0; j < 3; j++) {
            lo[0] = mn(lo[0], cx[j]); lo[1] = mn(lo[1], cy[j]); lo[2] = mn(lo[2], cz[j]);
            hi[0] = mx(hi[0], cx[j]); hi[1] = mx(hi[1], cy[j]); hi[2] = mx(hi[2], cz[j]);
        }
    }
    Node *n = &nodes[i];
    n->lo[0] = lo[0] - pad; n->lo[1] = lo[1] - pad; n->lo[2] = lo[2] - pad;
    n->hi[0] = hi[0] + pad; n->hi[1] = hi[1] + pad; n->hi[2] = hi[2] + pad;
    climb(nodes, nn, parent[i], parent, flags, err);
}

// the tree's SAH cost as bvh_cost (engine/rt/bvh.c:463-468) reckons it - the nodes' surface areas
// over the root's - summed in double in one fixed order (one block), so that it is the same on
// every run
__global__ void cost_kernel(const Node *__restrict__ nodes, uint32_t nn, double *out) {
    __shared__ double part[256];
    double sum = 0.0;
    for (uint32_t i = threadIdx.x; i < nn; i += 256) {
        const Node &n = nodes[i];
        const double dx = (double)n.hi[0] - n.lo[0], dy = (double)n.hi[1] - n.lo[1], dz = (double)n.hi[2] - n.lo[2];
        if (!(dx < 0 || dy < 0 || dz < 0)) sum += 2.0 * (dx * dy + dy * dz + dz * dx);
    }
    part[threadIdx.x] = sum;
    __syncthreads();
    for (int o = 128; o > 0; o >>= 1) {
        if ((int)threadIdx.x < o) part[threadIdx.x] += part[threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        const Node &r = nodes[0];
        const double dx = (double)r.hi[0] - r.lo[0], dy = (double)r.hi[1] - r.lo[1], dz = (double)r.hi[2] - r.lo[2];
        const double root = (dx < 0 || dy < 0 || dz < 0) ? 0.0 : 2.0 * (dx * dy + dy * dz + dz * dx);
        out[0] = root > 0 ? part[0] / root : 0.0;
    }
}

}  // namespace

size_t refit_scratch_bytes(uint32_t n) { return n ? (2 * (size_t)n - 1) * 8 + 256 : 256; }

cudaError_t refit_device(Node *d_nodes, const uint32_t *d_aux, uint32_t n, uint32_t ref_add, const float *d_boxes,
                         uint32_t stride4, uint32_t lo_at, void *scratch, size_t scratch_bytes, uint32_t *d_status,
                         cudaStream_t st) {
    if (!n) return cudaSuccess;
    if (scratch_bytes < refit_scratch_bytes(n)) return cudaErrorInvalidValue;
    const uint32_t nn = 2 * n - 1;
    uint32_t *parent = static_cast<uint32_t *>(scratch), *flags = parent + nn;
    cudaError_t e = cudaMemsetAsync(flags, 0, (size_t)nn * 4, st);
    if (e) return e;
    const uint32_t blocks = (nn + 255) / 256;
    parent_kernel<<<blocks, 256, 0, st>>>(d_nodes, nn, parent, d_status);
    refit_kernel<<<blocks, 256, 0, st>>>(d_nodes, d_aux, nn, n, ref_add, reinterpret_cast<const float4 *>(d_boxes), n,
                                         stride4, lo_at, parent, flags, d_status);
    return cudaGetLastError();
}

size_t walk_tree_scratch_bytes(uint32_t nn) { return (size_t)nn * 8 + 256; }

cudaError_t walk_tree_device(const Node *d_src, uint32_t nn, const uint32_t *d_aux, uint32_t naux, const float *d_tris,
                             uint32_t ntris, Node *d_dst, void *scratch, size_t scratch_bytes, uint32_t *d_status,
                             cudaStream_t st) {
    if (!nn) return cudaSuccess;
    if (scratch_bytes < walk_tree_scratch_bytes(nn)) return cudaErrorInvalidValue;
    uint32_t *parent = static_cast<uint32_t *>(scratch), *flags = parent + nn;
    cudaError_t e = cudaMemcpyAsync(d_dst, d_src, (size_t)nn * 32, cudaMemcpyDeviceToDevice, st);
    if (!e) e = cudaMemsetAsync(flags, 0, (size_t)nn * 4, st);
    if (e) return e;
    const uint32_t blocks = (nn + 255) / 256;
    parent_kernel<<<blocks, 256, 0, st>>>(d_dst, nn, parent, d_status);
    walk_leaf_kernel<<<blocks, 256, 0, st>>>(d_dst, d_src, d_aux, nn, naux, reinterpret_cast<const float4 *>(d_tris),
                                             ntris, parent, flags, d_status);
    return cudaGetLastError();
}

cudaError_t tree_cost_device(const Node *d_nodes, uint32_t n, double *d_out, cudaStream_t st) {
    if (!n) return cudaMemsetAsync(d_out, 0, 8, st);
    cost_kernel<<<1, 256, 0, st>>>(d_nodes, 2 * n - 1, d_out);
    return cudaGetLastError();
}

}  // namespace lrc
