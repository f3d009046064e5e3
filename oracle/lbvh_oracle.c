// lbvh_oracle.c - TEST INFRASTRUCTURE (the oracle): the reference's LBVH builder restated in C.
// Follows engine/gpu/shaders/trace/trace_build.wgsl (morton :25-33, bsort :35-50, delta/hier
// :52-96, leaves :98-107, up :109-122) and the host side of engine/gpu/trace_gpu.c (BuildParams
// and build_queue :546-641, up_passes :560, sort_passes :567), dispatch after dispatch.
// Build flags: -ffp-contract=off (no fused multiply-add), IEEE single precision.
#include "oracle.h"
#include <math.h>
#include <stdlib.h>
#include <string.h>

// WGSL min / max: e2 if e2 < e1 (e2 > e1), else e1
static inline float wmin(float a, float b){ return b < a ? b : a; }
static inline float wmax(float a, float b){ return b > a ? b : a; }
static inline int clz32(uint32_t x){ return x ? __builtin_clz(x) : 32; }
static inline int clz64(uint64_t x){ return x ? __builtin_clzll(x) : 64; }

void or_params(const float blo[3], const float bhi[3], float lo[3], float ext[3]){
    for (int k = 0; k < 3; k++){
        float e = bhi[k] - blo[k];                 // v_sub(bounds.hi, bounds.lo) in float
        lo[k] = blo[k];
        ext[k] = e > 0 ? 1.0f / e : 0.0f;          // (float)(1.0 / ext.x): a float division
    }
}

// spread (trace_build.wgsl:16-23): 10 bits to every third bit
static uint32_t spread10(uint32_t v){
    uint32_t x = v & 1023u;
    x = (x | (x << 16)) & 0x030000ffu;
    x = (x | (x << 8)) & 0x0300f00fu;
    x = (x | (x << 4)) & 0x030c30c3u;
    x = (x | (x << 2)) & 0x09249249u;
    return x;
}
// the 63-bit extension: 21 bits to every third bit of a 64-bit word
static uint64_t spread21(uint32_t v){
    uint64_t x = v & 0x1fffffu;
    x = (x | (x << 32)) & 0x001f00000000ffffull;
    x = (x | (x << 16)) & 0x001f0000ff0000ffull;
    x = (x | (x << 8)) & 0x100f00f00f00f00full;
    x = (x | (x << 4)) & 0x10c30c30c30c30c3ull;
    x = (x | (x << 2)) & 0x1249249249249249ull;
    return x;
}

static uint32_t pow2_at_least(uint32_t n){ uint32_t p = 2; while (p < n) p <<= 1; return p; }
static int up_passes(int n){ int k = 0; while ((1 << k) < n) k++; return n > 1 ? 34 + k : 0; }
static int words(int bits){ return bits == 63 ? 3 : 2; }

// the quantised centre of item i on each axis: clamp((c - lo) * ext, 0, 0.999) * scale, truncated
static void quantise(const float *boxes, int i, const float lo[3], const float ext[3], float scale, uint32_t q[3]){
    const float *b = boxes + 8 * (size_t)i;
    for (int k = 0; k < 3; k++){
        float c = (b[k] + b[4 + k]) * 0.5f;
        float x = (c - lo[k]) * ext[k];
        x = wmin(wmax(x, 0.0f), 0.999f) * scale;
        q[k] = (uint32_t)x;
    }
}

void or_morton(const float *boxes, int n, const float lo[3], const float ext[3], int bits, uint32_t *keys){
    uint32_t p = pow2_at_least((uint32_t)n);
    int w = words(bits);
    for (uint32_t i = 0; i < p; i++){
        uint32_t *k = keys + (size_t)w * i;
        if (i >= (uint32_t)n){ for (int j = 0; j < w; j++) k[j] = 0xffffffffu; continue; }
        uint32_t q[3];
        if (bits == 63){
            quantise(boxes, (int)i, lo, ext, 2097152.0f, q);
            uint64_t c = (spread21(q[0]) << 2) | (spread21(q[1]) << 1) | spread21(q[2]);
            k[0] = (uint32_t)c; k[1] = (uint32_t)(c >> 32); k[2] = i;
        } else {
            quantise(boxes, (int)i, lo, ext, 1024.0f, q);
            k[0] = (spread10(q[0]) << 2) | (spread10(q[1]) << 1) | spread10(q[2]);
            k[1] = i;
        }
    }
}

static int key_gt(const uint32_t *a, const uint32_t *b, int bits){
    if (bits == 63){
        uint64_t ca = ((uint64_t)a[1] << 32) | a[0], cb = ((uint64_t)b[1] << 32) | b[0];
        return ca > cb || (ca == cb && a[2] > b[2]);
    }
    return a[0] > b[0] || (a[0] == b[0] && a[1] > b[1]);
}

void or_bitonic(uint32_t *keys, uint32_t p, int bits){
    int w = words(bits);
    uint32_t tmp[3];
    for (uint32_t kk = 2; kk <= p; kk <<= 1)
        for (uint32_t j = kk >> 1; j > 0; j >>= 1)
            for (uint32_t i = 0; i < p; i++){           // one dispatch: disjoint pairs
                uint32_t q = i ^ j;
                if (q <= i) continue;
                uint32_t *a = keys + (size_t)w * i, *b = keys + (size_t)w * q;
                int ascending = (i & kk) == 0;
                if (key_gt(a, b, bits) == ascending){
                    memcpy(tmp, a, 4 * w); memcpy(a, b, 4 * w); memcpy(b, tmp, 4 * w);
                }
            }
}

typedef struct { const uint32_t *keys; int n, bits; } Sorted;

// delta (trace_build.wgsl:52-58): the common prefix of keys i and j, their positions breaking ties
static int delta(const Sorted *s, int i, int j){
    if (j < 0 || j >= s->n) return -1;
    if (s->bits == 63){
        const uint32_t *a = s->keys + 3 * (size_t)i, *b = s->keys + 3 * (size_t)j;
        uint64_t ca = ((uint64_t)a[1] << 32) | a[0], cb = ((uint64_t)b[1] << 32) | b[0];
        if (ca == cb) return 64 + clz32((uint32_t)i ^ (uint32_t)j);
        return clz64(ca ^ cb);
    }
    uint32_t a = s->keys[2 * (size_t)i], b = s->keys[2 * (size_t)j];
    if (a == b) return 32 + clz32((uint32_t)i ^ (uint32_t)j);
    return clz32(a ^ b);
}

// hier (trace_build.wgsl:60-96): internal node ii's children (absolute node indices)
static void hier(const Sorted *s, int ii, uint32_t node0, OrNode *nodes){
    const int n = s->n, i = ii;
    int d = delta(s, i, i + 1) > delta(s, i, i - 1) ? 1 : -1;
    int dmin = delta(s, i, i - d);
    int lmax = 2;
    for (int g = 0; g < 32; g++){
        if (lmax >= 2 * n || delta(s, i, i + lmax * d) <= dmin) break;
        lmax *= 2;
    }
    int l = 0, t = lmax / 2;
    for (int g = 0; g < 32; g++){
        if (t < 1) break;
        if (delta(s, i, i + (l + t) * d) > dmin) l += t;
        t /= 2;
    }
    int j = i + l * d;
    int dnode = delta(s, i, j);
    int sp = 0, div = 2;
    for (int g = 0; g < 32; g++){
        int st = (l + div - 1) / div;
        if (delta(s, i, i + (sp + st) * d) > dnode) sp += st;
        if (st <= 1) break;
        div *= 2;
    }
    int gam = i + sp * d + (d < 0 ? d : 0);
    int mn = i < j ? i : j, mx = i > j ? i : j;
    int left = mn == gam ? n - 1 + gam : gam;
    int right = mx == gam + 1 ? n + gam : gam + 1;
    nodes[node0 + (uint32_t)ii].a = node0 + (uint32_t)left;
    nodes[node0 + (uint32_t)ii].b = node0 + (uint32_t)right;
}

// leaves (trace_build.wgsl:98-107) for the sorted keys
static void leaves(const float *boxes, const Sorted *s, uint32_t node0, uint32_t ref0, uint32_t ref_add,
                   OrNode *nodes, uint32_t *aux, uint32_t *flags){
    const int n = s->n, w = words(s->bits);
    for (int j = 0; j < n; j++){
        uint32_t item = s->keys[(size_t)w * j + (w - 1)];
        OrNode *o = &nodes[node0 + (uint32_t)(n - 1 + j)];
        const float *b = boxes + 8 * (size_t)item;
        memcpy(o->lo, b, 12);
        memcpy(o->hi, b + 4, 12);
        o->a = ref0 + (uint32_t)j;
        o->b = 0x80000001u;
        aux[ref0 + (uint32_t)j] = item + ref_add;
        if (flags) flags[n - 1 + j] = 1;
    }
}

// morton + sort into keys (p * words), returning p
static uint32_t sorted_keys(const float *boxes, int n, const float lo[3], const float ext[3], int bits, uint32_t **out){
    uint32_t p = pow2_at_least((uint32_t)n);
    uint32_t *keys = malloc((size_t)p * words(bits) * 4);
    if (!keys) return 0;
    or_morton(boxes, n, lo, ext, bits, keys);
    or_bitonic(keys, p, bits);
    *out = keys;
    return p;
}

int or_lbvh(const float *boxes, int n, const float lo[3], const float ext[3], int bits, uint32_t node0,
            uint32_t ref0, uint32_t ref_add, OrNode *nodes, uint32_t *aux, uint32_t *keys_out){
    if (n <= 0) return 0;
    uint32_t *keys = NULL;
    uint32_t p = sorted_keys(boxes, n, lo, ext, bits, &keys);
    if (!p) return -1;
    uint32_t *flags = calloc((size_t)2 * n, 4);
    if (!flags){ free(keys); return -1; }
    Sorted s = {keys, n, bits};
    for (int i = 0; i + 1 < n; i++){ hier(&s, i, node0, nodes); flags[i] = 0; }
    leaves(boxes, &s, node0, ref0, ref_add, nodes, aux, flags);
    // up: pass u finishes the nodes whose children were both finished before it (flags: the
    // pass a node was finished in + 1; leaves 1). 63-bit keys: until nothing is left.
    int passes = bits == 63 ? 64 + 64 : up_passes(n);
    for (uint32_t u = 1; u <= (uint32_t)passes && n > 1; u++){
        int left = 0;
        for (int i = 0; i + 1 < n; i++){
            if (flags[i] != 0) continue;
            OrNode *nd = &nodes[node0 + (uint32_t)i];
            uint32_t fl = flags[nd->a - node0], fr = flags[nd->b - node0];
            if (fl == 0 || fr == 0 || fl > u || fr > u){ left = 1; continue; }
            const OrNode *a = &nodes[nd->a], *b = &nodes[nd->b];
            for (int k = 0; k < 3; k++){ nd->lo[k] = wmin(a->lo[k], b->lo[k]); nd->hi[k] = wmax(a->hi[k], b->hi[k]); }
            flags[i] = u + 1;
        }
        if (!left && bits == 63) break;
    }
    if (keys_out) memcpy(keys_out, keys, (size_t)p * words(bits) * 4);
    free(flags);
    free(keys);
    return 0;
}

// ---- the PLOC builder (trace_ploc.wgsl), after morton, bsort and leaves ----------------------
#define PL_R 16
#define PL_WG 256

typedef struct {
    int n, small;
    uint32_t node0, ref0;
    uint32_t cnt[4];           // pl[0..3]: the lists' counts, the list in use, its count
    uint32_t *list[2];         // cl(p, i)
    uint32_t *nn, *sc, *bk, *bm;
    float *bx;                 // 8 floats per cluster (lo.xyz, -, hi.xyz, -)
    OrNode *nodes;
} Ploc;

// area (trace_ploc.wgsl:18): e.x*e.y + e.y*e.z + e.z*e.x, left to right, no fused multiply-add
static inline float area3(const float lo[3], const float hi[3]){
    float ex = hi[0] - lo[0], ey = hi[1] - lo[1], ez = hi[2] - lo[2];
    return ex * ey + ey * ez + ez * ex;
}
static inline int nearer(float d, uint32_t i, uint32_t j, float bd, uint32_t bj){
    if (bj == 0xffffffffu || d < bd) return 1;
    if (d > bd) return 0;
    uint32_t mn = i < j ? i : j, bmn = i < bj ? i : bj;
    uint32_t mx = i > j ? i : j, bmx = i > bj ? i : bj;
    return mn < bmn || (mn == bmn && mx < bmx);
}
static uint32_t nearest(const Ploc *P, uint32_t p, uint32_t i, uint32_t nc){
    const float *ci = P->bx + 8 * (size_t)P->list[p][i];
    uint32_t j0 = i > PL_R ? i - PL_R : 0, j1 = i + PL_R < nc - 1 ? i + PL_R : nc - 1;
    float bd = 0.0f;
    uint32_t bj = 0xffffffffu;
    for (uint32_t j = j0; j <= j1; j++){
        if (j == i) continue;
        const float *cj = P->bx + 8 * (size_t)P->list[p][j];
        float lo[3], hi[3];
        for (int k = 0; k < 3; k++){ lo[k] = wmin(ci[k], cj[k]); hi[k] = wmax(ci[4 + k], cj[4 + k]); }
        float d = area3(lo, hi);
        if (nearer(d, i, j, bd, bj)){ bd = d; bj = j; }
    }
    return bj;
}
static void keep_merge(const Ploc *P, uint32_t i, uint32_t nc, uint32_t *keep, uint32_t *merge){
    uint32_t j = P->nn[i];
    int mu = j < nc && P->nn[j] == i;
    *keep = mu && i > j ? 0 : 1;
    *merge = mu && i < j ? 1 : 0;
}
static void final_node(const Ploc *P, uint32_t x, OrNode *o){
    const uint32_t n = (uint32_t)P->n;
    const float *b = P->bx + 8 * (size_t)x;
    memcpy(o->lo, b, 12);
    memcpy(o->hi, b + 4, 12);
    if (x < n - 1){ o->a = P->node0 + 1 + 2 * x; o->b = P->node0 + 2 + 2 * x; }
    else { o->a = P->ref0 + x - (n - 1); o->b = 0x80000001u; }
}
static void merge(Ploc *P, uint32_t k, uint32_t c, uint32_t d){
    float *bk = P->bx + 8 * (size_t)k;
    const float *bc = P->bx + 8 * (size_t)c, *bd = P->bx + 8 * (size_t)d;
    float lo[3], hi[3];
    for (int q = 0; q < 3; q++){ lo[q] = wmin(bc[q], bd[q]); hi[q] = wmax(bc[4 + q], bd[4 + q]); }
    memcpy(bk, lo, 12); memcpy(bk + 4, hi, 12);
    final_node(P, c, &P->nodes[P->node0 + 1 + 2 * k]);
    final_node(P, d, &P->nodes[P->node0 + 2 + 2 * k]);
    if (k == 0){
        OrNode *r = &P->nodes[P->node0];
        memcpy(r->lo, lo, 12); memcpy(r->hi, hi, 12);
        r->a = P->node0 + 1; r->b = P->node0 + 2;
    }
}
static void leaf_in(Ploc *P, uint32_t i){
    uint32_t x = (uint32_t)P->n - 1 + i;
    const OrNode *nd = &P->nodes[P->node0 + x];
    float *b = P->bx + 8 * (size_t)x;
    memcpy(b, nd->lo, 12); memcpy(b + 4, nd->hi, 12);
}
static uint32_t live(const Ploc *P, uint32_t nc){ return nc <= (uint32_t)P->small ? 0 : nc; }

// one round of four dispatches (nn, mark, top, scatter; trace_ploc.wgsl:119-234), round r
static void ploc_round(Ploc *P, uint32_t r){
    const uint32_t p = r & 1, n = (uint32_t)P->n;
    uint32_t nc = live(P, P->cnt[p]);
    for (uint32_t i = 0; i < nc; i++) P->nn[i] = nearest(P, p, i, nc);                  // nn
    uint32_t nb = (nc + PL_WG - 1) / PL_WG;                                                // mark
    for (uint32_t blk = 0; blk < nb; blk++){
        uint32_t sk = 0, sm = 0;
        for (uint32_t l = 0; l < PL_WG; l++){
            uint32_t i = blk * PL_WG + l, kx = 0, mx = 0;
            if (i < nc) keep_merge(P, i, nc, &kx, &mx);
            if (i < nc) P->sc[i] = sk | (sm << 9) | (kx << 18) | (mx << 19);
            sk += kx; sm += mx;
        }
        P->bk[blk] = sk; P->bm[blk] = sm;
    }
    uint32_t ck = 0, cm = 0;                                                               // top
    for (uint32_t b = 0; b < nb; b++){
        uint32_t vk = P->bk[b], vm = P->bm[b];
        P->bk[b] = ck; P->bm[b] = cm;
        ck += vk; cm += vm;
    }
    uint32_t q = 1 - p, next = P->cnt[p];
    if (P->cnt[p] > (uint32_t)P->small){ next = ck; P->cnt[2] = q; P->cnt[3] = ck; }
    for (uint32_t i = 0; i < nc; i++){                                                    // scatter
        uint32_t s = P->sc[i];
        if (((s >> 18) & 1u) == 0) continue;
        uint32_t blk = i / PL_WG;
        uint32_t dest = P->bk[blk] + (s & 0x1ffu);
        uint32_t c = P->list[p][i], out = c;
        if ((s >> 19) & 1u){
            uint32_t d = P->list[p][P->nn[i]];
            uint32_t k = (n - 2) - (n - nc + P->bm[blk] + ((s >> 9) & 0x1ffu));
            merge(P, k, c, d);
            out = k;
        }
        P->list[q][dest] = out;
    }
    P->cnt[q] = next;
}

// small (trace_ploc.wgsl:238-301): every remaining round in one workgroup
static void ploc_small(Ploc *P, int whole){
    const uint32_t n = (uint32_t)P->n;
    uint32_t p = 0, nc;
    if (whole){
        for (uint32_t i = 0; i < n; i++){ leaf_in(P, i); P->list[0][i] = n - 1 + i; }
        nc = n;
    } else { p = P->cnt[2]; nc = P->cnt[3]; }
    while (nc > 1){
        for (uint32_t i = 0; i < nc; i++) P->nn[i] = nearest(P, p, i, nc);
        uint32_t q = 1 - p, dk = 0, dm = 0;
        for (uint32_t i = 0; i < nc; i++){
            uint32_t kx, mx;
            keep_merge(P, i, nc, &kx, &mx);
            if (!kx) continue;
            uint32_t c = P->list[p][i], out = c;
            if (mx){
                uint32_t d = P->list[p][P->nn[i]];
                uint32_t k = (n - 2) - (n - nc + dm);
                dm++;
                merge(P, k, c, d);
                out = k;
            }
            P->list[q][dk++] = out;
        }
        nc = dk;
        p = q;
    }
}

static int ploc_rounds(int n, int small){ int r = 0; for (int64_t m = n; m > small; m = m * 5 / 6) r++; return r ? r + 2 : 0; }

int or_ploc(const float *boxes, int n, const float lo[3], const float ext[3], int bits, uint32_t node0,
            uint32_t ref0, uint32_t ref_add, int small, OrNode *nodes, uint32_t *aux){
    if (n < 3) return -1;
    uint32_t *keys = NULL;
    if (!sorted_keys(boxes, n, lo, ext, bits, &keys)) return -1;
    Sorted s = {keys, n, bits};
    leaves(boxes, &s, node0, ref0, ref_add, nodes, aux, NULL);
    free(keys);
    Ploc P;
    memset(&P, 0, sizeof(P));
    P.n = n; P.small = small > 0 ? small : 1024; P.node0 = node0; P.ref0 = ref0; P.nodes = nodes;
    uint32_t nb = ((uint32_t)n + PL_WG - 1) / PL_WG;
    P.list[0] = malloc((size_t)n * 4); P.list[1] = malloc((size_t)n * 4);
    P.nn = malloc((size_t)n * 4); P.sc = malloc((size_t)n * 4);
    P.bk = malloc((size_t)nb * 4); P.bm = malloc((size_t)nb * 4);
    P.bx = malloc((size_t)(2 * n - 1) * 32);
    int ok = P.list[0] && P.list[1] && P.nn && P.sc && P.bk && P.bm && P.bx;
    if (ok){
        if (n <= P.small) ploc_small(&P, 1);
        else {
            for (uint32_t i = 0; i < (uint32_t)n; i++){ leaf_in(&P, i); P.list[0][i] = (uint32_t)n - 1 + i; }   // init
            P.cnt[0] = (uint32_t)n; P.cnt[1] = 0; P.cnt[2] = 0; P.cnt[3] = (uint32_t)n;
            int rounds = ploc_rounds(n, P.small);
            for (int r = 0; r < rounds; r++) ploc_round(&P, (uint32_t)r);
            ploc_small(&P, 0);
        }
    }
    free(P.list[0]); free(P.list[1]); free(P.nn); free(P.sc); free(P.bk); free(P.bm); free(P.bx);
    return ok ? 0 : -1;
}
