// oracle.h - TEST INFRASTRUCTURE. A C restatement of the reference's GPU BVH builders, which
// exist only as WGSL compute shaders (no CPU version in the reference):
//   engine/gpu/shaders/trace/trace_build.wgsl  morton, bsort, hier, leaves, up   (LBVH, Karras 2012)
//   engine/gpu/shaders/trace/trace_ploc.wgsl   init, nn, mark, top, scatter, small (PLOC, Meister & Bittner 2018)
//   engine/gpu/trace_gpu.c:546-641             BuildParams and build_queue (n, p, node0, ref0, ref_add, lo, ext)
// Each function simulates the shader's dispatches one after the other, with the shader's
// semantics (one dispatch's threads do not see each other's writes where the shader relies on
// it). Compiled with -ffp-contract=off: IEEE single precision, no fused multiply-add.
// Parity of this restatement is unpinned: the reference ships no test or golden data for its builders.
#ifndef LR_ORACLE_H
#define LR_ORACLE_H
#include <stdint.h>

// a node as the reference's path tracer reads it (trace.wgsl Node): 32 bytes
typedef struct { float lo[3]; uint32_t a; float hi[3]; uint32_t b; } OrNode;

// build_queue's parameters (trace_gpu.c:605-611): lo = the bounds' low corner, ext = 1 / their
// size per axis (0 where the size is 0), the division in float as the float build does it
void or_params(const float bounds_lo[3], const float bounds_hi[3], float lo[3], float ext[3]);

// morton (trace_build.wgsl:25-33): codes of n items' box centres, keys (code, index) padded
// with (0xffffffff, 0xffffffff) to p = pow2 >= n (p >= 2). keys: 2 * p words.
// bits = 30 (10 per axis, the reference) or 63 (21 per axis; code in 2 words: low, high).
void or_morton(const float *boxes, int n, const float lo[3], const float ext[3], int bits, uint32_t *keys);

// bsort (trace_build.wgsl:35-50), every (k, j) step of the bitonic network over p keys
// (30-bit keys: 2 words each). For 63-bit keys (3 words: code low, code high, index) the same network.
void or_bitonic(uint32_t *keys, uint32_t p, int bits);

// The whole LBVH build of build_queue + gpu_trace_build (trace_gpu.c:587-764): morton, bitonic
// sort, hier, leaves, up passes. nodes: at least node0 + 2n - 1 entries; aux: ref0 + n entries.
// keys_out (optional, p * words): the sorted keys. Returns 0, or -1 when out of memory.
// For bits = 63 (no reference counterpart) delta is 64 + clz(i ^ j) on equal codes and the
// passes up go on until every node is done.
int or_lbvh(const float *boxes, int n, const float lo[3], const float ext[3], int bits, uint32_t node0,
            uint32_t ref0, uint32_t ref_add, OrNode *nodes, uint32_t *aux, uint32_t *keys_out);

// PLOC over the same sorted leaves (build_queue with the builder PLOC: morton, bsort, leaves,
// then init / rounds of nn, mark, top, scatter / small; trace_gpu.c:685-701, 730-734).
// small = the count handled in one workgroup (LR_GPU_PLOC_SMALL, 1024 by default). n >= 3.
int or_ploc(const float *boxes, int n, const float lo[3], const float ext[3], int bits, uint32_t node0,
            uint32_t ref0, uint32_t ref_add, int small, OrNode *nodes, uint32_t *aux);

// check_tree (trace_gpu.c:768-805): 1 if the nodes from node0 are one tree over n leaves, with
// its cost (bvh_cost: sum of node areas over the root's) and depth
int or_check_tree(const OrNode *nodes, int n, uint32_t node0, double *cost, int *depth);

// Closest hit of rays through a built binary tree (1 triangle per leaf, aux -> triangle), by
// the reference's Moller-Trumbore arithmetic (intersect.h:96-112); counts node visits and
// triangle tests (the traversal's algorithmic bytes). tris: 9 floats each (q, u, v).
// prim: the triangle hit (-1: none), t. counts[0] = box tests, counts[1] = triangle tests.
void or_trace_tree(const OrNode *nodes, const uint32_t *aux, uint32_t node0, const float *tris,
                   const float *orig, const float *dir, long long nrays, float tmin, float tmax,
                   int *prim, float *t, long long *counts);
// bvh_refit_boxes on a GPU-layout tree (tree_oracle.c)
int or_refit(OrNode *w, int nn, const uint32_t *aux, uint32_t ref_add, const float *boxes, int nitems);

#endif
