// gpu_cuda.c - a `cuda` GPU backend for little_renderer: the engine's public GPU headers
// (engine/gpu/gpu.h and the path-tracing part of engine/gpu/view_gpu.h) implemented on the CUDA
// library's C ABI (include/lrc.h), so that the engine's programs (engine/app/gpu_frame.c:
// gpu_frame_open / gpu_frame_trace / gpu_frame_close, the viewer's trace calls) path trace on a
// B200 instead of through WebGPU. It is compiled against the engine's own headers and replaces
// engine/gpu/gpu.c, view_gpu.c and trace_gpu.c in a build, as NOGPU=1 swaps in their stubs
// (view_gpu.c:5-46): the functions this backend does not take over keep the stubs' answers
// ("this GPU cannot": the engine then draws or traces on the CPU).
//
// What it does (the reference's behaviour, view_gpu.h:49-176):
//   gpu_create            a context on CUDA device 0 (offscreen only: no canvas, no window)
//   gpu_view_trace_start  the scene to the device: primitives and triangles in the GPU layouts
//                         (upload_world, put_tris: trace_gpu.c:898-911, 1145-1154), vertex normals,
//                         materials, the lamp, the sky (upload_sky :1522-1569) and the scene's OWN
//                         BVH (scene_bvh: the 4-wide SAH tree's binary form in put_nodes' layout,
//                         :883-896, as upload_world traces it, :1103-1112; a scene without one
//                         gets one built on the device); a new image
//   gpu_view_trace_more   the band scheduler (view_gpu.c:1081-1190): whole-image passes, as many
//                         per call as the time budget allows (at most 16), or a band of rows when
//                         one pass is slower than the budget; never past gpu_view_trace_limit.
//                         Every pass adds one sample per pixel, in sample order, so an image's
//                         sums do not depend on how its passes were cut into calls
//   gpu_view_trace_read   the sums and counts read back, the callback delivered by gpu_poll /
//                         gpu_wait on the thread that owns the Gpu (gpu.h:32-42)
// Scenes it cannot hold yet (instances, media, textures, a rotated sky, light-traced photons)
// make gpu_view_trace_start return 0, as a scene too big for a GPU does: the caller path traces
// on the CPU.
#include "gpu/gpu.h"
#include "gpu/view_gpu.h"
#include "rt/accel.h"
#include "rt/bvh.h"
#include "scene/env.h"
#include "lrc.h"

#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

#define SHIM_MAX_READS 4
#define SHIM_MAX_REPEATS 16
#define SHIM_BUDGET_MS 40.0          // a call's GPU time when none is set (the reference's bands: 12-45 ms)

typedef struct {
    GpuTraceReadFn fn;
    void *user;
    float *data;                     // NULL: the read failed (fn gets NULL)
    int w, h;
} ShimRead;

struct Gpu {
    lrc_ctx *ctx;
    GpuState state;
    int offscreen, timing;
    char msg[256];
    ShimRead reads[SHIM_MAX_READS];
    int nreads;
};

static int g_timing_asked;

static double now_ms(void) {
    struct timespec t;
    clock_gettime(CLOCK_MONOTONIC, &t);
    return t.tv_sec * 1e3 + t.tv_nsec * 1e-6;
}

int gpu_available(void) { return 1; }

static Gpu *shim_gpu(int offscreen) {
    Gpu *g = calloc(1, sizeof *g);
    if (!g) return NULL;
    g->offscreen = offscreen;
    if (!offscreen) {
        g->state = GPU_FAILED;
        snprintf(g->msg, sizeof g->msg, "the CUDA backend draws offscreen only (no canvas or window)");
        return g;
    }
    int rc = lrc_open(0, &g->ctx);
    if (rc) {
        g->state = GPU_FAILED;
        snprintf(g->msg, sizeof g->msg, "no CUDA device (lrc_open: %d)", rc);
        g->ctx = NULL;
        return g;
    }
    g->state = GPU_READY;
    g->timing = g_timing_asked;
    lrc_set_timing(g->ctx, g->timing);
    snprintf(g->msg, sizeof g->msg, "CUDA (lrc, %d SMs)", lrc_num_sms(g->ctx));
    return g;
}

Gpu *gpu_create(const char *canvas, int width, int height) {
    (void)width;
    (void)height;
    return shim_gpu(canvas == NULL);
}

Gpu *gpu_create_window(void *display, uintptr_t window, int width, int height) {
    (void)display;
    (void)window;
    (void)width;
    (void)height;
    return shim_gpu(0);
}

// the reads whose data is there: their callbacks, in the order they were asked for
void gpu_poll(Gpu *g) {
    if (!g) return;
    int n = g->nreads;
    g->nreads = 0;
    ShimRead rs[SHIM_MAX_READS];
    memcpy(rs, g->reads, sizeof rs);
    for (int i = 0; i < n; i++) {
        rs[i].fn(rs[i].user, rs[i].data, rs[i].w, rs[i].h);
        free(rs[i].data);
    }
}

static void shim_lost(Gpu *g, const char *what) {
    if (g->state == GPU_FAILED) return;
    g->state = GPU_FAILED;
    snprintf(g->msg, sizeof g->msg, "%s: %s", what, g->ctx ? lrc_message(g->ctx) : "no context");
    // reads that will not come: their callbacks with NULL (once a read was accepted, fn is called)
    for (int i = 0; i < g->nreads; i++) {
        free(g->reads[i].data);
        g->reads[i].data = NULL;
    }
    gpu_poll(g);
}

void gpu_wait(Gpu *g) {
    if (!g) return;
    if (g->state == GPU_READY && lrc_sync(g->ctx)) shim_lost(g, "the CUDA device failed");
    gpu_poll(g);
}

GpuState gpu_state(Gpu *g) {
    if (!g) return GPU_FAILED;
    if (g->state == GPU_READY) gpu_poll(g);
    return g->state;
}

const char *gpu_message(const Gpu *g) { return g ? g->msg : "no GPU"; }
int gpu_offscreen(const Gpu *g) { return g ? g->offscreen : 1; }
int gpu_software(const Gpu *g) { (void)g; return 0; }
int gpu_rt_offered(const Gpu *g) { (void)g; return 0; }

void gpu_destroy(Gpu *g) {
    if (!g) return;
    for (int i = 0; i < g->nreads; i++) free(g->reads[i].data);
    if (g->ctx) lrc_close(g->ctx);
    free(g);
}

void gpu_set_timing(int on) { g_timing_asked = on; }
int gpu_timing(const Gpu *g) { return g ? g->timing : 0; }
void gpu_set_vsync(int on) { (void)on; }
void gpu_set_async_views(int on) { (void)on; }
void gpu_resize(Gpu *g, int width, int height) { (void)g; (void)width; (void)height; }

// ---- the view: the path tracer's image and its scene ------------------------------------------
struct GpuView {
    Gpu *g;
    int w, h;
    lrc_scene *scene;
    const Scene *src;                // the scene last uploaded, and what says it changed
    unsigned tris_version;
    const void *accel;
    int nprims, nmats, light;
    float *d_accum;                  // w x h x (sum rgb, count), device
    int started;
    lrc_trace_params tp;
    int passes;                      // whole passes done (samples per pixel)
    int next_row;                    // the band scheduler's next row of the pass under way
    int limit;
    double budget_ms, budget_live_ms, budget_pass_ms;
    double pass_ms;                  // the last measured time of one whole pass (0: none yet)
    int rows, reps;                  // the last call's band
    double t_submit;                 // host clock when the last call's work was submitted
    int submitted_rows, submitted_reps, busy;
    double work;
    uint64_t images;
    double gpu_total_ms;
};

GpuView *gpu_view_create(Gpu *g, int width, int height) {
    if (!g || g->state != GPU_READY || width <= 0 || height <= 0) return NULL;
    GpuView *v = calloc(1, sizeof *v);
    if (!v) return NULL;
    v->g = g;
    v->w = width;
    v->h = height;
    if (lrc_scene_create(g->ctx, &v->scene) ||
        lrc_device_alloc(g->ctx, (size_t)width * height * 16, (void **)&v->d_accum)) {
        if (v->scene) lrc_scene_destroy(v->scene);
        free(v);
        return NULL;
    }
    return v;
}

void gpu_view_destroy(GpuView *v) {
    if (!v) return;
    lrc_sync(v->g->ctx);
    lrc_device_free(v->g->ctx, v->d_accum);
    lrc_scene_destroy(v->scene);
    free(v);
}

int gpu_view_ready(GpuView *v) { return v ? 1 : -1; }

static void put3(float *o, Vec3 a, float w) {
    o[0] = (float)a.x;
    o[1] = (float)a.y;
    o[2] = (float)a.z;
    o[3] = w;
}
static float bits_f(uint32_t u) {
    float f;
    memcpy(&f, &u, 4);
    return f;
}

// what this backend holds: a world of primitives and triangles (vertex normals), materials
// without textures, one lamp, an unrotated sky
static int shim_can_hold(const Scene *s, const GpuTraceParams *tp) {
    if (s->ninsts > 0 || s->nvolumes > 0 || s->ntexmaps > 0 || s->nemitters > 0) return 0;
    if (s->env && s->env->rot != 0) return 0;
    if (tp->photons > 0 || tp->photon_cache) return 0;
    if (s->nprims + s->ntris == 0) return 0;
    for (int m = 0; m < s->nmats; m++) {
        const Material *mt = &s->mats[m];
        if (mt->tex_base || mt->tex_mr || mt->tex_normal || mt->tex_emissive) return 0;
    }
    return 1;
}

// the scene's shapes, materials, lamp, sky and tree into the lrc scene
static int shim_upload(GpuView *v, const Scene *s) {
    lrc_scene *sc = v->scene;
    int rc = 0;
    // primitives: upload_world's 24 floats
    float *pr = malloc((size_t)(s->nprims ? s->nprims : 1) * 96);
    uint32_t *tr = malloc((size_t)(s->ntris ? s->ntris : 1) * 48);
    float *nr = malloc((size_t)(s->nnormals ? s->nnormals : 1) * 12);
    float *mt = calloc(64, 64);
    if (!pr || !tr || !nr || !mt) rc = LRC_RETRY;
    for (int i = 0; !rc && i < s->nprims; i++) {
        const Primitive *p = &s->prims[i];
        float *o = pr + 24 * (size_t)i;
        put3(o, p->center, (float)p->radius);
        put3(o + 4, p->q, p->type == PRIM_QUAD ? 1.0f : 0.0f);
        put3(o + 8, p->u, (float)p->material);
        put3(o + 12, p->v, (float)p->area);
        put3(o + 16, p->normal, (float)p->plane_d);
        put3(o + 20, p->w, 0.0f);
    }
    // triangles: put_tris' 12 words (normal indices as they are: the world's normals start at 0)
    for (int i = 0; !rc && i < s->ntris; i++) {
        const Triangle *q = &s->tris[i];
        uint32_t *o = tr + 12 * (size_t)i;
        float a[4];
        put3(a, q->q, 0);
        memcpy(o, a, 12);
        put3(a, q->u, 0);
        memcpy(o + 4, a, 12);
        put3(a, q->v, 0);
        memcpy(o + 8, a, 12);
        const int smooth = q->n[0] >= 0;
        o[3] = smooth ? (uint32_t)q->n[0] : 0xffffffffu;
        o[7] = smooth ? (uint32_t)q->n[1] : 0;
        o[11] = ((uint32_t)(q->material & 63) << 26) | (smooth ? ((uint32_t)q->n[2] & 0x03ffffffu) : 0);
    }
    for (int i = 0; !rc && i < s->nnormals; i++) {
        nr[3 * i] = (float)s->normals[i].x;
        nr[3 * i + 1] = (float)s->normals[i].y;
        nr[3 * i + 2] = (float)s->normals[i].z;
    }
    // materials: albedo, type | emission | ior, metallic, roughness, transmission | (no textures)
    const int nm = s->nmats < 64 ? s->nmats : 64;
    for (int m = 0; !rc && m < nm; m++) {
        const Material *M = &s->mats[m];
        float *o = mt + 16 * m;
        put3(o, M->albedo, bits_f((uint32_t)M->type));
        put3(o + 4, M->emission, 0.0f);
        o[8] = (float)M->ior;
        o[9] = (float)M->metallic;
        o[10] = (float)M->roughness;
        o[11] = (float)M->transmission;
    }
    if (!rc) rc = lrc_scene_set_prims(sc, pr, (uint32_t)s->nprims, 0);
    if (!rc) rc = lrc_scene_set_triangles(sc, tr, (uint32_t)s->ntris, 0);
    if (!rc) rc = lrc_scene_set_normals(sc, nr, (uint32_t)s->nnormals, 0);
    if (!rc) rc = lrc_scene_set_materials(sc, mt, (uint32_t)(nm ? nm : 1));
    if (!rc) rc = lrc_scene_set_light(sc, s->light);
    if (!rc) rc = lrc_scene_set_tables(sc, NULL, NULL);
    if (!rc) {
        const Env *e = s->env;
        rc = e ? lrc_scene_set_sky(sc, e->rgb, e->w, e->h, NULL, NULL, NULL, (float)e->scale)
               : lrc_scene_set_sky(sc, NULL, 0, 0, NULL, NULL, NULL, 1.0f);
    }
    free(pr);
    free(tr);
    free(nr);
    free(mt);
    if (rc) return rc;
    // the tree: the scene's own (put_nodes: lo, a, hi, b; a leaf's a its first ref, b its count
    // with the top bit; an inner node's a and b its children), or one built on the device
    const Bvh *b = scene_bvh(s);
    if (!b || b->nnodes == 0) return lrc_scene_build(sc, 1, 30);
    uint32_t *nd = malloc((size_t)b->nnodes * 32);
    uint32_t *ax = malloc((size_t)(b->nrefs ? b->nrefs : 1) * 4);
    if (!nd || !ax) {
        free(nd);
        free(ax);
        return LRC_RETRY;
    }
    for (int i = 0; i < b->nnodes; i++) {
        const BvhNode *n = &b->nodes[i];
        uint32_t *o = nd + 8 * (size_t)i;
        float lo[4], hi[4];
        put3(lo, n->box.lo, 0);
        put3(hi, n->box.hi, 0);
        memcpy(o, lo, 12);
        memcpy(o + 4, hi, 12);
        o[3] = n->count > 0 ? (uint32_t)n->start : (uint32_t)n->left;
        o[7] = n->count > 0 ? (0x80000000u | (uint32_t)n->count) : (uint32_t)n->right;
    }
    for (int i = 0; i < b->nrefs; i++) ax[i] = (uint32_t)b->refs[i];
    rc = lrc_scene_set_tree(sc, nd, (uint32_t)b->nnodes, ax, (uint32_t)b->nrefs, 0);
    free(nd);
    free(ax);
    return rc;
}

int gpu_view_trace_start(GpuView *v, const Scene *s, const GpuTraceParams *tp) {
    if (!v || !s || !tp || v->g->state != GPU_READY) return 0;
    if (!shim_can_hold(s, tp)) return 0;
    lrc_sync(v->g->ctx);
    const int same = v->src == s && v->tris_version == s->tris_version && v->accel == s->accel &&
                     v->nprims == s->nprims && v->nmats == s->nmats && v->light == s->light;
    if (!same) {
        if (shim_upload(v, s)) {
            v->src = NULL;
            return 0;
        }
        v->src = s;
        v->tris_version = s->tris_version;
        v->accel = s->accel;
        v->nprims = s->nprims;
        v->nmats = s->nmats;
        v->light = s->light;
    }
    lrc_trace_params *p = &v->tp;
    memset(p, 0, sizeof *p);
    const Camera *c = &tp->cam;
    const Vec3 cv[4] = {c->origin, c->upper_left, c->horizontal, c->vertical};
    float *dst[4] = {p->origin, p->upper_left, p->horizontal, p->vertical};
    for (int k = 0; k < 4; k++) {
        dst[k][0] = (float)cv[k].x;
        dst[k][1] = (float)cv[k].y;
        dst[k][2] = (float)cv[k].z;
    }
    p->width = v->w;
    p->height = v->h;
    p->max_depth = tp->max_depth;
    p->mis = tp->mis;
    p->sampler = !tp->random;
    p->exact = 0;                    // a stream per sample: a pixel's samples independent of the passes
    p->seed = v->images++;
    p->clamp = (float)tp->clamp;
    p->skip_caustics = 0;
    p->indirect_clamp = (float)tp->indirect_clamp;
    if (lrc_device_zero(v->g->ctx, v->d_accum, (size_t)v->w * v->h * 16)) return 0;
    v->started = 1;
    v->passes = 0;
    v->next_row = 0;
    v->busy = 0;
    return 1;
}

int gpu_view_trace_failed(const GpuView *v) { (void)v; return 0; }
void gpu_view_trace_prepare(GpuView *v) { (void)v; }

// (no reprojection through this backend yet: a move starts a new image)
int gpu_view_trace_move(GpuView *v, const Scene *s, const GpuTraceParams *tp, int history) {
    (void)history;
    return gpu_view_trace_start(v, s, tp);
}
int gpu_view_trace_reads_tlas(const GpuView *v, const Scene *s) { (void)v; (void)s; return 0; }

// the time the last call took, from when it was submitted to now (its work done)
static void shim_settle(GpuView *v) {
    if (!v->busy) return;
    if (lrc_sync(v->g->ctx)) {
        shim_lost(v->g, "the CUDA device failed");
        v->busy = 0;
        return;
    }
    const double ms = now_ms() - v->t_submit;
    const double pass_part = (double)v->submitted_rows / v->h * v->submitted_reps;
    if (pass_part > 0) v->pass_ms = ms / pass_part;
    v->gpu_total_ms += ms;
    v->busy = 0;
}

int gpu_view_trace_more(GpuView *v, const Scene *s, const RenderParams *p, const MarchParams *mp) {
    (void)s;
    (void)p;
    (void)mp;
    if (!v || !v->started || v->g->state != GPU_READY) return 0;
    if (lrc_query(v->g->ctx) == 0) return 1;          // the previous band is still running
    shim_settle(v);
    if (v->g->state != GPU_READY) return 0;
    if (v->limit > 0 && v->passes >= v->limit) return 1;
    const double budget = v->budget_ms > 0 ? v->budget_ms : SHIM_BUDGET_MS;
    int rows = v->h, reps = 1;
    if (v->pass_ms > 0 && v->next_row == 0) {
        // whole passes that fit the budget (at least one when asked for), up to 16
        reps = (int)(budget / v->pass_ms);
        if (v->budget_pass_ms > 0 && reps < 1) reps = 1;
        if (reps > SHIM_MAX_REPEATS) reps = SHIM_MAX_REPEATS;
        if (reps < 1) {                               // a pass is slower than the budget: a band
            reps = 1;
            rows = (int)(v->h * budget / v->pass_ms);
            if (rows < 1) rows = 1;
        }
    } else if (v->next_row > 0) {
        rows = v->pass_ms > 0 ? (int)(v->h * budget / v->pass_ms) : v->h;
        if (rows < 1) rows = 1;
    }
    if (v->limit > 0 && reps > v->limit - v->passes) reps = v->limit - v->passes;
    if (rows > v->h - v->next_row) rows = v->h - v->next_row;
    v->t_submit = now_ms();
    for (int r = 0; r < reps; r++) {
        // one sample of every pixel of the band, sample number passes (+ r for whole passes)
        const int rc = lrc_trace(v->scene, &v->tp, v->next_row, rows, (uint32_t)(v->passes + r), 1, v->d_accum, NULL,
                                 LRC_DEVICE);
        if (rc) {
            shim_lost(v->g, "gpu_view_trace_more");
            return 0;
        }
    }
    v->rows = rows;
    v->reps = reps;
    v->submitted_rows = rows;
    v->submitted_reps = reps;
    v->busy = 1;
    v->next_row += rows;
    v->work += (double)rows / v->h * reps;
    if (v->next_row >= v->h) {
        v->next_row = 0;
        v->passes += reps;
    }
    return 1;
}

void gpu_view_trace_limit(GpuView *v, int spp) { if (v) v->limit = spp > 0 ? spp : 0; }
void gpu_view_trace_budget(GpuView *v, double ms) { if (v) v->budget_ms = ms > 0 ? ms : 0; }
void gpu_view_trace_budget_pass(GpuView *v, double max_ms) { if (v) v->budget_pass_ms = max_ms > 0 ? max_ms : 0; }
void gpu_view_trace_budget_live(GpuView *v, double ms) { if (v) v->budget_live_ms = ms > 0 ? ms : 0; }
int gpu_view_trace_passes(const GpuView *v) { return v ? v->passes : 0; }
double gpu_view_trace_work(const GpuView *v) { return v ? v->work : 0; }
int gpu_view_trace_busy(const GpuView *v) { return v && v->busy && lrc_query(v->g->ctx) == 0; }
int gpu_view_trace_compiling(const GpuView *v) { (void)v; return 0; }
double gpu_view_trace_pass_ms(const GpuView *v) { return v ? v->pass_ms : 0; }

void gpu_view_trace_band(const GpuView *v, int *rows, int *reps, double *budget_ms) {
    *rows = v ? v->rows : 0;
    *reps = v ? v->reps : 0;
    *budget_ms = v ? (v->budget_ms > 0 ? v->budget_ms : SHIM_BUDGET_MS) : 0;
}

int gpu_view_trace_read(GpuView *v, GpuTraceReadFn fn, void *user) {
    if (!v || !fn || !v->started || v->g->state != GPU_READY) return 0;
    Gpu *g = v->g;
    for (int i = 0; i < g->nreads; i++)
        if (g->reads[i].user == user && g->reads[i].fn == fn) return 0;   // one on its way already
    if (g->nreads >= SHIM_MAX_READS) return 0;
    shim_settle(v);
    ShimRead *r = &g->reads[g->nreads++];
    r->fn = fn;
    r->user = user;
    r->w = v->w;
    r->h = v->h;
    r->data = malloc((size_t)v->w * v->h * 16);
    if (r->data && lrc_device_copy(g->ctx, r->data, v->d_accum, (size_t)v->w * v->h * 16, LRC_COPY_D2H)) {
        free(r->data);
        r->data = NULL;              // (the callback gets NULL: the read failed)
    }
    return 1;
}

// ---- the rest of view_gpu.h: not taken over (the stubs' answers; the engine stays on the CPU) ---
void gpu_view_present(GpuView *v, const Framebuffer *fb, const Scene *s, const RenderParams *p, const MarchParams *mp,
                      int volumes) {
    (void)v; (void)fb; (void)s; (void)p; (void)mp; (void)volumes;
}
void gpu_view_hud(GpuView *v, const uint32_t *argb, int w, int h, int x, int y) {
    (void)v; (void)argb; (void)w; (void)h; (void)x; (void)y;
}
int gpu_view_present_scene(GpuView *v, const Scene *s, const RenderParams *p, const MarchParams *mp, int volumes) {
    (void)v; (void)s; (void)p; (void)mp; (void)volumes;
    return 0;
}
int gpu_view_volumes_fit(GpuView *v, const Scene *s, const MarchParams *mp) {
    (void)v; (void)mp;
    return s && s->nvolumes == 0;
}
void gpu_view_aa(GpuView *v, int on) { (void)v; (void)on; }
void gpu_view_trace_wavefront(GpuView *v, int on) { (void)v; (void)on; }   // (lrc_trace picks its engine by size)
void gpu_view_trace_raster_guide(GpuView *v, int mode) { (void)v; (void)mode; }
void gpu_view_trace_gradients(GpuView *v, int history_max) { (void)v; (void)history_max; }
void gpu_view_trace_edited(GpuView *v, int on) { (void)v; (void)on; }
int gpu_view_trace_has_gradients(const GpuView *v) { (void)v; return 0; }
int gpu_view_trace_raster_guided(const GpuView *v) { (void)v; return 0; }
int gpu_view_trace_planes_read(GpuView *v, int first, int n, float *out) {
    (void)first;
    if (!v || n != 1 || first != 0 || !out) return 0;        // plane 0 (the samples) only
    shim_settle(v);
    return lrc_device_copy(v->g->ctx, out, v->d_accum, (size_t)v->w * v->h * 16, LRC_COPY_D2H) == 0;
}
int gpu_view_trace_denoise(GpuView *v, int on) { (void)v; (void)on; return 0; }
void gpu_view_trace_denoise_moving(GpuView *v, int passes) { (void)v; (void)passes; }
int gpu_view_present_traced(GpuView *v, const Scene *s, const RenderParams *p, const MarchParams *mp, int volumes) {
    (void)v; (void)s; (void)p; (void)mp; (void)volumes;
    return 0;
}
double gpu_view_gpu_ms(GpuView *v, int what) {
    if (!v || what != 0 || v->passes == 0) return 0;
    return v->pass_ms;
}
void gpu_view_gpu_totals(GpuView *v, double ms[8]) {
    for (int k = 0; k < 8; k++) ms[k] = 0;
    if (v) ms[0] = v->gpu_total_ms;
}
void gpu_view_gpu_ms_reset(GpuView *v) { if (v) v->gpu_total_ms = 0; }
double gpu_view_bench_denoise(GpuView *v, int n) { (void)v; (void)n; return -1; }
int gpu_view_capture(GpuView *v, GpuCaptureFn fn, void *user) { (void)v; (void)fn; (void)user; return 0; }
