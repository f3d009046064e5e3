// tree_oracle.c - TEST INFRASTRUCTURE (the oracle): checks of a built tree and a counted
// closest-hit walk through it.
//   or_check_tree  restates check_tree (engine/gpu/trace_gpu.c:768-805)
//   or_trace_tree  a binary-tree walk (as bvh_intersect, engine/rt/bvh.c:608-663) with the
//                  reference's slab test (intersect.h:38-51) and Moller-Trumbore arithmetic
//                  (intersect.h:96-112), counting box and triangle tests: the algorithmic bytes
//                  of a traversal through that tree.
#include "oracle.h"
#include <math.h>
#include <stdlib.h>
#include <string.h>

int or_check_tree(const OrNode *w, int n, uint32_t node0, double *cost, int *depth){
    size_t nn = 2 * (size_t)n - 1;
    unsigned char *seen = calloc(nn, 1);
    uint32_t *stack = malloc(nn * 2 * sizeof(uint32_t));
    if (!seen || !stack){ free(seen); free(stack); return 0; }
    double sum = 0, root = 0;
    int leaves = 0, ok = 1, top = 0, deep = 0;
    stack[top++] = 0; stack[top++] = 1;
    seen[0] = 1;
    while (top > 0 && ok){
        uint32_t d = stack[--top], i = stack[--top];
        if ((int)d > deep) deep = (int)d;
        const OrNode *f = &w[node0 + i];
        double ex = (double)f->hi[0] - f->lo[0], ey = (double)f->hi[1] - f->lo[1], ez = (double)f->hi[2] - f->lo[2];
        double area = 2 * (ex * ey + ey * ez + ez * ex);
        if (!(area >= 0)) ok = 0;
        sum += area;
        if (i == 0) root = area;
        if (f->b & 0x80000000u){ leaves++; continue; }
        uint32_t c[2] = {f->a - node0, f->b - node0};
        for (int k = 0; k < 2; k++){
            if (c[k] >= nn || seen[c[k]]){ ok = 0; break; }
            seen[c[k]] = 1;
            const OrNode *g = &w[node0 + c[k]];
            for (int x = 0; x < 3; x++)
                if (g->lo[x] < f->lo[x] - 1e-3f * (1 + fabsf(f->lo[x])) || g->hi[x] > f->hi[x] + 1e-3f * (1 + fabsf(f->hi[x]))) ok = 0;
            stack[top++] = c[k]; stack[top++] = d + 1;
        }
    }
    free(seen);
    free(stack);
    *cost = root > 0 ? sum / root : 0;
    *depth = deep;
    return ok && leaves == n;
}

// r_fmin / r_fmax (lrmath.h): the other number when one is a NaN
static inline float rmin(float a, float b){ return b != b ? a : (a < b ? a : b); }
static inline float rmax(float a, float b){ return b != b ? a : (a > b ? a : b); }

static int box_hit(const OrNode *b, const float o[3], const float inv[3], float tmin, float tmax, float *te){
    for (int k = 0; k < 3; k++){
        float t0 = (b->lo[k] - o[k]) * inv[k], t1 = (b->hi[k] - o[k]) * inv[k];
        if (inv[k] < 0){ float t = t0; t0 = t1; t1 = t; }
        tmin = rmax(t0, tmin); tmax = rmin(t1, tmax);
    }
    if (tmax < tmin) return 0;
    *te = tmin;
    return 1;
}

static inline float dot3(const float *a, const float *b){ return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }
static inline void cross3(const float *a, const float *b, float *r){
    r[0] = a[1] * b[2] - a[2] * b[1];
    r[1] = a[2] * b[0] - a[0] * b[2];
    r[2] = a[0] * b[1] - a[1] * b[0];
}
static int tri_hit(const float *tr, const float o[3], const float d[3], float tmin, float tmax, float *tout){
    const float *q = tr, *u = tr + 3, *v = tr + 6;
    float pvec[3], tvec[3], qvec[3];
    cross3(d, v, pvec);
    float det = dot3(u, pvec);
    if (fabsf(det) < 1e-12f) return 0;
    float inv = 1.0f / det;
    tvec[0] = o[0] - q[0]; tvec[1] = o[1] - q[1]; tvec[2] = o[2] - q[2];
    float b1 = dot3(tvec, pvec) * inv;
    if (b1 < 0 || b1 > 1) return 0;
    cross3(tvec, u, qvec);
    float b2 = dot3(d, qvec) * inv;
    if (b2 < 0 || b1 + b2 > 1) return 0;
    float t = dot3(v, qvec) * inv;
    if (t <= tmin || t >= tmax) return 0;
    *tout = t;
    return 1;
}

void or_trace_tree(const OrNode *nodes, const uint32_t *aux, uint32_t node0, const float *tris,
                   const float *orig, const float *dir, long long nrays, float tmin, float tmax,
                   int *prim, float *tout, long long *counts){
    long long boxes = 0, tests = 0;
#pragma omp parallel for schedule(dynamic, 1024) reduction(+:boxes, tests)
    for (long long r = 0; r < nrays; r++){
        const float *o = orig + 3 * r, *d = dir + 3 * r;
        float inv[3] = {1.0f / d[0], 1.0f / d[1], 1.0f / d[2]};
        struct { uint32_t node; float t; } stack[256];
        int sp = 0, hit = -1;
        float best = tmax, te;
        boxes++;
        if (box_hit(&nodes[node0], o, inv, tmin, best, &te)){ stack[sp].node = node0; stack[sp].t = te; sp++; }
        while (sp > 0){
            sp--;
            if (stack[sp].t > best) continue;
            const OrNode *nd = &nodes[stack[sp].node];
            if (nd->b & 0x80000000u){
                uint32_t cnt = nd->b & 0x7fffffffu;
                for (uint32_t k = 0; k < cnt; k++){
                    uint32_t id = aux[nd->a + k];
                    float t;
                    tests++;
                    if (tri_hit(tris + 9 * (size_t)id, o, d, tmin, best, &t)){ best = t; hit = (int)id; }
                }
                continue;
            }
            float tl = 0, trr = 0;
            boxes += 2;
            int hl = box_hit(&nodes[nd->a], o, inv, tmin, best, &tl);
            int hr = box_hit(&nodes[nd->b], o, inv, tmin, best, &trr);
            if (sp + 2 > 256) continue;           // (deeper than any tree here: never taken in the tests)
            if (hl && hr){
                uint32_t nr = tl <= trr ? nd->a : nd->b, fr = tl <= trr ? nd->b : nd->a;
                stack[sp].node = fr; stack[sp].t = rmax(tl, trr); sp++;
                stack[sp].node = nr; stack[sp].t = rmin(tl, trr); sp++;
            } else if (hl){ stack[sp].node = nd->a; stack[sp].t = tl; sp++; }
            else if (hr){ stack[sp].node = nd->b; stack[sp].t = trr; sp++; }
        }
        prim[r] = hit;
        tout[r] = hit >= 0 ? best : -1;
    }
    counts[0] = boxes;
    counts[1] = tests;
}

// bvh_refit_boxes (engine/rt/bvh.c:471-485) on a tree in the GPU layout (root at node 0, nn
// nodes): every leaf's box the union of its items' boxes (aux = item + ref_add; boxes 8 floats
// each), every inner node's its left child's box with the right's added (box_add_box, bvh.c:20,
// mn / mx: a < b ? a : b), children before parents (an explicit postorder walk).
static inline float or_mn(float a, float b){ return a < b ? a : b; }
static inline float or_mx(float a, float b){ return a > b ? a : b; }
int or_refit(OrNode *w, int nn, const uint32_t *aux, uint32_t ref_add, const float *boxes, int nitems){
    uint32_t *stack = malloc((size_t)nn * 2 * sizeof(uint32_t));
    if (!stack) return 0;
    int top = 0, ok = 1;
    stack[top++] = 0; stack[top++] = 0;             // (node, children done)
    while (top > 0 && ok){
        uint32_t done = stack[--top], i = stack[--top];
        OrNode *f = &w[i];
        if (f->b & 0x80000000u){
            float lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
            uint32_t cnt = f->b & 0x7fffffffu;
            for (uint32_t k = 0; k < cnt; k++){
                uint32_t item = aux[f->a + k] - ref_add;
                if ((int)item >= nitems){ ok = 0; break; }
                const float *b = boxes + 8 * (size_t)item;
                for (int x = 0; x < 3; x++){ lo[x] = or_mn(lo[x], b[x]); hi[x] = or_mx(hi[x], b[4 + x]); }
            }
            for (int x = 0; x < 3; x++){ f->lo[x] = lo[x]; f->hi[x] = hi[x]; }
            continue;
        }
        if ((int)f->a >= nn || (int)f->b >= nn){ ok = 0; break; }
        if (!done){
            stack[top++] = i; stack[top++] = 1;
            stack[top++] = f->b; stack[top++] = 0;
            stack[top++] = f->a; stack[top++] = 0;
            continue;
        }
        const OrNode *l = &w[f->a], *r = &w[f->b];
        for (int x = 0; x < 3; x++){ f->lo[x] = or_mn(l->lo[x], r->lo[x]); f->hi[x] = or_mx(l->hi[x], r->hi[x]); }
    }
    free(stack);
    return ok;
}
