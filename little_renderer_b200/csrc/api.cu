// api.cu - the C ABI (include/lrc.h) over the builder and traversal kernels.
//
// A context owns a CUDA stream, a device status word (bits of bounded waits that ran out and of
// traversal stacks that would have overflowed) and one growing scratch arena, as the reference's
// GpuTrace owns its builder's keys/flags/lists buffers (trace_gpu.c:736-741, gpu_buffer_reserve).
// Calls with host arrays stage them through a second growing device arena, run, copy back and
// synchronise; calls with LRC_DEVICE only enqueue (lrc_sync waits and reports).
#include "api_internal.cuh"
#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <new>
#include <vector>

using namespace lrcapi;
using lrc::Node;

namespace lrcapi {

int scene_build_on(lrc_scene *s, int builder, int key_bits, void **scratch, size_t *scratch_cap, cudaStream_t st,
                   lrc::StageTimer *timer, bool no_alloc) {
    lrc_ctx *c = s->ctx;
    if (key_bits != 30 && key_bits != 63) return fail(c, LRC_E_INVALID, "key_bits must be 30 or 63");
    if (builder != 0 && builder != 1) return fail(c, LRC_E_INVALID, "builder must be 0 (LBVH) or 1 (PLOC)");
    if ((uint64_t)s->ntris + s->nprims >= (1u << 30)) return fail(c, LRC_E_INVALID, "more than 2^30 - 1 shapes");
    DeviceGuard g(c->device);
    // the shapes: primitives, then triangles (their ids as the reference's, scene.h:101-106)
    const uint32_t n = s->ntris + s->nprims;
    if (!no_alloc) s->built_n = 0;
    s->tree_nnodes = s->tree_naux = 0;
    s->walk_ok = false;
    s->wide_ok = false;
    if (!n) return LRC_OK;
    const size_t need_scratch = lrc::build_scratch_bytes(n, key_bits, builder);
    if (no_alloc) {
        if (s->boxes_cap < (size_t)n * 32 || !s->d_boxes || s->tree_cap < n || *scratch_cap < need_scratch)
            return fail(c, LRC_E_INVALID, "a build to capture needs its buffers sized by an earlier run");
    }
    cudaError_t e = reserve(reinterpret_cast<void **>(&s->d_boxes), &s->boxes_cap, (size_t)n * 32);
    if (!e && s->tree_cap < n) {
        cudaFree(s->d_nodes);
        cudaFree(s->d_aux);
        s->d_nodes = nullptr;
        s->d_aux = nullptr;
        s->tree_cap = 0;
        e = cudaMalloc(&s->d_nodes, (2 * (size_t)n - 1) * 32);
        if (!e) e = cudaMalloc(&s->d_aux, (size_t)n * 4);
        if (!e) s->tree_cap = n;
    }
    if (!e) e = reserve(scratch, scratch_cap, need_scratch);
    if (e) return cuda_status(c, e, "scene build memory");
    uint32_t *keys = s->d_small;
    float *bounds = reinterpret_cast<float *>(s->d_small + 8), *lo_ext = reinterpret_cast<float *>(s->d_small + 16);
    if (timer) timer->begin(LRC_TS_BOXES, st);
    float *tri_boxes = s->d_boxes + 8 * (size_t)s->nprims;
    e = lrc::triangle_boxes(s->d_tris, s->ntris, tri_boxes, keys, st, c->num_sms);
    if (!e && s->nprims) {
        // a world with primitives: their boxes (primitive_bounds) first, the bounds over all shapes' boxes
        e = lrc::pt_prim_boxes(s->d_prims, s->nprims, s->d_boxes, st);
        if (!e) e = lrc::boxes_bounds(s->d_boxes, n, keys, st, c->num_sms, true);
    }
    if (!e) e = lrc::bounds_params(keys, bounds, lo_ext, st);
    lrc_build_params p{};
    p.n = n;
    p.key_bits = key_bits;
    p.builder = builder;
    if (!e) e = lrc::build_device_ext(p, s->d_boxes, lo_ext, s->d_nodes, s->d_aux, *scratch, *scratch_cap, c->d_status,
                                      c->num_sms, st, nullptr, timer);
    if (e) return cuda_status(c, e, "lrc_scene_build");
    s->built_n = n;
    return LRC_OK;
}

// the top level over n instances (records at d_inst): LBVH over their world boxes, 30-bit keys,
// bounds their union (upload_instances, trace_gpu.c:1415-1463) into d_nodes / d_aux; d_boxes
// (n x 8 floats) and d_small (64 words) are scratch, as is the build scratch
cudaError_t build_tlas_on(lrc_ctx *c, const float *d_inst, uint32_t n, Node *d_nodes, uint32_t *d_aux, float *d_boxes,
                          uint32_t *d_small, void *scratch, size_t scratch_cap, cudaStream_t st, lrc::StageTimer *timer) {
    uint32_t *keys = d_small;
    float *bounds = reinterpret_cast<float *>(d_small + 8), *lo_ext = reinterpret_cast<float *>(d_small + 16);
    cudaError_t e = lrc::pt_inst_boxes(d_inst, n, d_boxes, st);
    if (!e) e = lrc::boxes_bounds(d_boxes, n, keys, st, c->num_sms, true);
    if (!e) e = lrc::bounds_params(keys, bounds, lo_ext, st);
    lrc_build_params p{};
    p.n = n; p.key_bits = 30; p.builder = 0;
    if (!e) e = lrc::build_device_ext(p, d_boxes, lo_ext, d_nodes, d_aux, scratch, scratch_cap, c->d_status, c->num_sms,
                                      st, nullptr, timer);
    return e;
}

// the walk's tree of a triangle scene (no primitives): its tree's topology with tight boxes, for
// the closest- and any-hit queries; the path tracer walks the tree as built
int make_walk(lrc_scene *s) {
    s->walk_ok = false;
    s->wide_ok = false;
    if (!s->walk_mode || s->nprims || !s->built_n || !s->ntris) return LRC_OK;
    lrc_ctx *c = s->ctx;
    const size_t nn = s->tree_nnodes ? s->tree_nnodes : 2 * (size_t)s->built_n - 1;
    const size_t na = s->tree_nnodes ? s->tree_naux : s->built_n;
    cudaError_t e = cudaSuccess;
    if (s->wnodes_cap < nn) {
        cudaFree(s->d_wnodes);
        s->d_wnodes = nullptr;
        s->wnodes_cap = 0;
        e = cudaMalloc(&s->d_wnodes, nn * 32);
        if (!e) s->wnodes_cap = nn;
    }
    if (!e) e = reserve(&c->scratch, &c->scratch_cap, lrc::walk_tree_scratch_bytes((uint32_t)nn));
    c->timer.begin(LRC_TS_HIERARCHY, c->st);
    if (!e) e = lrc::walk_tree_device(s->d_nodes, (uint32_t)nn, s->d_aux, (uint32_t)na, reinterpret_cast<const float *>(s->d_tris),
                                      s->ntris, s->d_wnodes, c->scratch, c->scratch_cap, c->d_status, c->st);
    c->timer.end(c->st);
    if (e) return cuda_status(c, e, "the walk's tree");
    s->walk_ok = true;
    if (s->walk_mode != 2) return LRC_OK;
    // the 8-wide nodes from it (a tree whose leaves do not fit a node's slots keeps the binary walk)
    const size_t wcap = lrc::wide_node_cap((uint32_t)na);
    if (s->wide_cap < wcap) {
        cudaFree(s->d_wide);
        s->d_wide = nullptr;
        s->wide_cap = 0;
        e = cudaMalloc(&s->d_wide, wcap * 80);
        if (!e) s->wide_cap = wcap;
    }
    if (!e && s->wrefs_cap < wcap) {
        cudaFree(s->d_wrefs);
        s->d_wrefs = nullptr;
        s->wrefs_cap = 0;
        e = cudaMalloc(&s->d_wrefs, wcap * 4);
        if (!e) s->wrefs_cap = wcap;
    }
    if (!e) e = reserve(&c->scratch, &c->scratch_cap, lrc::wide_scratch_bytes((uint32_t)na));
    c->timer.begin(LRC_TS_HIERARCHY, c->st);
    uint32_t nwide = 0;
    if (!e) e = lrc::wide_build(s->d_wnodes, (uint32_t)nn, s->d_aux, (uint32_t)na, reinterpret_cast<const float *>(s->d_tris),
                                s->ntris, s->d_wide, (uint32_t)s->wide_cap, s->d_wrefs, (uint32_t)s->wrefs_cap, c->scratch,
                                c->scratch_cap, c->d_status, c->st, &nwide);
    c->timer.end(c->st);
    if (e) return cuda_status(c, e, "the walk's wide tree");
    uint32_t status = 0;
    e = cudaMemcpy(&status, c->d_status, 4, cudaMemcpyDeviceToHost);
    if (e) return cuda_status(c, e, "the walk's wide tree");
    if (status & lrc::ST_BAD_TREE) {                   // (leaves too large: the binary walk stays)
        cudaMemset(c->d_status, 0, 4);
        return LRC_OK;
    }
    s->nwide = nwide;
    s->wide_ok = nwide > 0;
    return LRC_OK;
}

}  // namespace lrcapi

extern "C" {

int lrc_open(int device, lrc_ctx **out) {
    if (!out) return LRC_E_INVALID;
    *out = nullptr;
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count <= 0) {
        cudaGetLastError();
        return LRC_E_NODEVICE;
    }
    if (device < 0 || device >= count) return LRC_E_INVALID;
    lrc_ctx *c = new (std::nothrow) lrc_ctx;
    if (!c) return LRC_RETRY;
    c->device = device;
    DeviceGuard g(device);
    cudaError_t e = cudaDeviceGetAttribute(&c->num_sms, cudaDevAttrMultiProcessorCount, device);
    if (!e) e = cudaStreamCreateWithFlags(&c->own, cudaStreamNonBlocking);
    if (!e) e = cudaMalloc(&c->d_status, 256);
    if (!e) e = cudaMemset(c->d_status, 0, 256);
    if (e) {
        int rc = cuda_status(c, e, "lrc_open");
        if (c->own) cudaStreamDestroy(c->own);
        if (c->d_status) cudaFree(c->d_status);
        delete c;
        return rc;
    }
    c->st = c->own;
    *out = c;
    return LRC_OK;
}

void lrc_close(lrc_ctx *c) {
    if (!c) return;
    DeviceGuard g(c->device);
    cudaStreamSynchronize(c->st);
    if (c->single) lrc_batch_destroy(c->single);
    if (c->scratch) cudaFree(c->scratch);
    if (c->stage) cudaFree(c->stage);
    if (c->dn) cudaFree(c->dn);
    if (c->d_status) cudaFree(c->d_status);
    if (c->own) cudaStreamDestroy(c->own);
    delete c;
}

const char *lrc_message(const lrc_ctx *c) { return c ? c->msg.c_str() : "no context"; }

int lrc_sync(lrc_ctx *c) {
    if (!c) return LRC_E_INVALID;
    DeviceGuard g(c->device);
    return check_status(c);
}

int lrc_set_stream(lrc_ctx *c, void *stream) {
    if (!c) return LRC_E_INVALID;
    c->st = stream ? reinterpret_cast<cudaStream_t>(stream) : c->own;
    return LRC_OK;
}

uint32_t lrc_status(lrc_ctx *c) {
    if (!c) return 0;
    DeviceGuard g(c->device);
    uint32_t s = 0;
    cudaStreamSynchronize(c->st);
    cudaMemcpy(&s, c->d_status, 4, cudaMemcpyDeviceToHost);
    cudaMemset(c->d_status, 0, 4);
    return s;
}

int lrc_num_sms(const lrc_ctx *c) { return c ? c->num_sms : 0; }

int lrc_set_timing(lrc_ctx *c, int on) {
    if (!c) return LRC_E_INVALID;
    DeviceGuard g(c->device);
    c->timer.end(c->st);
    c->timer.on = on != 0;
    return LRC_OK;
}

int lrc_timings(lrc_ctx *c, double *ms, int *launches) {
    if (!c || !ms) return LRC_E_INVALID;
    DeviceGuard g(c->device);
    c->timer.end(c->st);
    c->timer.collect();
    for (int i = 0; i < LRC_NUM_STAGES; i++) {
        ms[i] = c->timer.ms[i];
        if (launches) launches[i] = c->timer.launches[i];
        c->timer.ms[i] = 0;
        c->timer.launches[i] = 0;
    }
    return LRC_OK;
}

void lrc_params_from_bounds(const float lo[3], const float hi[3], lrc_build_params *p) {
    for (int k = 0; k < 3; k++) {
        volatile float e = hi[k] - lo[k];      // v_sub in float
        p->lo[k] = lo[k];
        p->ext[k] = e > 0 ? 1.0f / e : 0.0f;   // (float)(1.0 / ext.x): a float division
    }
}

size_t lrc_build_scratch_bytes(uint32_t n, int key_bits, int builder) { return lrc::build_scratch_bytes(n, key_bits, builder); }

int lrc_build(lrc_ctx *c, const lrc_build_params *p, const float *boxes, uint32_t *nodes, uint32_t *aux, unsigned flags) {
    if (!c || !p) return LRC_E_INVALID;
    if (p->key_bits != 30 && p->key_bits != 63) return fail(c, LRC_E_INVALID, "key_bits must be 30 or 63");
    if (p->n >= (1u << 30)) return fail(c, LRC_E_INVALID, "more than 2^30 - 1 items");
    if (p->n == 0) return LRC_OK;
    if (!boxes || !nodes || !aux) return fail(c, LRC_E_INVALID, "null array");
    DeviceGuard g(c->device);
    const uint32_t n = p->n;
    const size_t need = lrc::build_scratch_bytes(n, p->key_bits, p->builder);
    cudaError_t e = reserve(&c->scratch, &c->scratch_cap, need);
    if (e) return cuda_status(c, e, "build scratch");
    const size_t nnodes = 2 * (size_t)n - 1;
    if (flags & LRC_DEVICE) {
        e = lrc::build_device(*p, boxes, reinterpret_cast<Node *>(nodes) + p->node0, aux + p->ref0, c->scratch,
                              c->scratch_cap, c->d_status, c->num_sms, c->st);
        return cuda_status(c, e, "lrc_build");
    }
    const size_t b_boxes = al((size_t)n * 32), b_nodes = al(nnodes * 32), b_aux = al((size_t)n * 4);
    e = reserve(&c->stage, &c->stage_cap, b_boxes + b_nodes + b_aux);
    if (e) return cuda_status(c, e, "build staging");
    char *s = static_cast<char *>(c->stage);
    float *d_boxes = reinterpret_cast<float *>(s);
    Node *d_nodes = reinterpret_cast<Node *>(s + b_boxes);
    uint32_t *d_aux = reinterpret_cast<uint32_t *>(s + b_boxes + b_nodes);
    e = cudaMemcpyAsync(d_boxes, boxes, (size_t)n * 32, cudaMemcpyHostToDevice, c->st);
    if (!e) e = lrc::build_device(*p, d_boxes, d_nodes, d_aux, c->scratch, c->scratch_cap, c->d_status, c->num_sms, c->st);
    if (!e) e = cudaMemcpyAsync(reinterpret_cast<Node *>(nodes) + p->node0, d_nodes, nnodes * 32, cudaMemcpyDeviceToHost, c->st);
    if (!e) e = cudaMemcpyAsync(aux + p->ref0, d_aux, (size_t)n * 4, cudaMemcpyDeviceToHost, c->st);
    if (e) return cuda_status(c, e, "lrc_build");
    return check_status(c);
}

int lrc_triangle_boxes(lrc_ctx *c, const uint32_t *tris, uint32_t n, float *boxes, float *bounds6, unsigned flags) {
    if (!c || (n && (!tris || !boxes))) return LRC_E_INVALID;
    DeviceGuard g(c->device);
    const size_t b_tris = al((size_t)n * 48), b_boxes = al((size_t)n * 32);
    cudaError_t e = reserve(&c->stage, &c->stage_cap, b_tris + b_boxes + 256);
    if (e) return cuda_status(c, e, "staging");
    char *s = static_cast<char *>(c->stage);
    uint32_t *keys = reinterpret_cast<uint32_t *>(s + b_tris + b_boxes);
    float *d_bounds = reinterpret_cast<float *>(keys + 8);
    const uint32_t *d_tris = tris;
    float *d_boxes = boxes;
    if (!(flags & LRC_DEVICE)) {
        d_tris = reinterpret_cast<uint32_t *>(s);
        d_boxes = reinterpret_cast<float *>(s + b_tris);
        e = cudaMemcpyAsync(const_cast<uint32_t *>(d_tris), tris, (size_t)n * 48, cudaMemcpyHostToDevice, c->st);
        if (e) return cuda_status(c, e, "copy in");
    }
    e = lrc::triangle_boxes(d_tris, n, d_boxes, keys, c->st, c->num_sms);
    if (!e) e = lrc::bounds_params(keys, (flags & LRC_DEVICE) && bounds6 ? bounds6 : d_bounds, nullptr, c->st);
    if (e) return cuda_status(c, e, "lrc_triangle_boxes");
    if (flags & LRC_DEVICE) return LRC_OK;
    e = cudaMemcpyAsync(boxes, d_boxes, (size_t)n * 32, cudaMemcpyDeviceToHost, c->st);
    if (!e && bounds6) e = cudaMemcpyAsync(bounds6, d_bounds, 24, cudaMemcpyDeviceToHost, c->st);
    if (e) return cuda_status(c, e, "copy out");
    return check_status(c);
}

// ---- scenes -------------------------------------------------------------------------------------
int lrc_scene_create(lrc_ctx *c, lrc_scene **out) {
    if (!c || !out) return LRC_E_INVALID;
    *out = nullptr;
    lrc_scene *s = new (std::nothrow) lrc_scene;
    if (!s) return LRC_RETRY;
    s->ctx = c;
    DeviceGuard g(c->device);
    cudaError_t e = cudaMalloc(&s->d_small, 256);
    if (e) {
        delete s;
        return cuda_status(c, e, "scene");
    }
    *out = s;
    return LRC_OK;
}

void lrc_scene_destroy(lrc_scene *s) {
    if (!s) return;
    DeviceGuard g(s->ctx->device);
    cudaStreamSynchronize(s->ctx->st);
    cudaFree(s->d_tris);
    cudaFree(s->d_nodes);
    cudaFree(s->d_wnodes);
    cudaFree(s->d_wide);
    cudaFree(s->d_wrefs);
    cudaFree(s->d_aux);
    cudaFree(s->d_boxes);
    cudaFree(s->d_small);
    cudaFree(s->d_prims);
    cudaFree(s->d_normals);
    cudaFree(s->d_mats);
    cudaFree(s->d_mask);
    cudaFree(s->d_rays);
    cudaFree(s->d_mtris);
    cudaFree(s->d_mnodes);
    cudaFree(s->d_maux);
    cudaFree(s->d_mesh_info);
    cudaFree(s->d_inst);
    cudaFree(s->d_tlas_nodes);
    cudaFree(s->d_tlas_aux);
    cudaFree(s->d_env);
    cudaFree(s->d_caus);
    cudaFree(s->d_vols);
    cudaFree(s->d_tex);
    cudaFree(s->d_uv);
    delete s;
}

int lrc_scene_set_triangles(lrc_scene *s, const uint32_t *tris, uint32_t n, unsigned flags) {
    if (!s || (n && !tris)) return LRC_E_INVALID;
    lrc_ctx *c = s->ctx;
    DeviceGuard g(c->device);
    cudaError_t e = reserve(reinterpret_cast<void **>(&s->d_tris), &s->tris_cap, (size_t)(n ? n : 1) * 48);
    if (e) return cuda_status(c, e, "triangles");
    if (n) e = cudaMemcpyAsync(s->d_tris, tris, (size_t)n * 48,
                               (flags & LRC_DEVICE) ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, c->st);
    if (e) return cuda_status(c, e, "triangles");
    s->ntris = n;
    s->built_n = 0;
    s->tree_nnodes = s->tree_naux = 0;
    s->walk_ok = false;
    s->wide_ok = false;
    if (!(flags & LRC_DEVICE)) return check_status(c);   // (the host array may be freed on return)
    return LRC_OK;
}

int lrc_scene_build(lrc_scene *s, int builder, int key_bits) {
    if (!s) return LRC_E_INVALID;
    lrc_ctx *c = s->ctx;
    int rc = scene_build_on(s, builder, key_bits, &c->scratch, &c->scratch_cap, c->st, &c->timer, false);
    return rc ? rc : make_walk(s);
}

int lrc_scene_set_walk(lrc_scene *s, int mode) {
    if (!s || mode < 0 || mode > 2) return LRC_E_INVALID;
    DeviceGuard g(s->ctx->device);
    s->walk_mode = mode;
    return make_walk(s);
}

int lrc_scene_tree(lrc_scene *s, uint32_t *nodes, uint32_t *aux, unsigned flags) {
    if (!s || !s->built_n) return LRC_E_INVALID;
    lrc_ctx *c = s->ctx;
    DeviceGuard g(c->device);
    const size_t nn = s->tree_nnodes ? s->tree_nnodes : 2 * (size_t)s->built_n - 1;
    const size_t na = s->tree_nnodes ? s->tree_naux : s->built_n;
    cudaMemcpyKind k = (flags & LRC_DEVICE) ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
    cudaError_t e = cudaSuccess;
    if (nodes) e = cudaMemcpyAsync(nodes, s->d_nodes, nn * 32, k, c->st);
    if (!e && aux) e = cudaMemcpyAsync(aux, s->d_aux, na * 4, k, c->st);
    if (e) return cuda_status(c, e, "lrc_scene_tree");
    return check_status(c);
}

int lrc_scene_set_tree(lrc_scene *s, const uint32_t *nodes, uint32_t nnodes, const uint32_t *aux, uint32_t naux,
                       unsigned flags) {
    if (!s || !nodes || !aux || !nnodes || !naux) return LRC_E_INVALID;
    lrc_ctx *c = s->ctx;
    const uint64_t shapes = (uint64_t)s->nprims + s->ntris;
    if (!shapes) return fail(c, LRC_E_INVALID, "the scene has no shapes (primitives or triangles) for a tree");
    if (!(flags & LRC_DEVICE)) {
        // a tree the walks can follow: children and leaf ranges inside the arrays, shapes that exist
        for (uint32_t i = 0; i < nnodes; i++) {
            const uint32_t a = nodes[8 * (size_t)i + 3], b = nodes[8 * (size_t)i + 7];
            if (b & lrc::LEAF_BIT) {
                const uint32_t cnt = b & ~lrc::LEAF_BIT;
                if (a >= naux || cnt > naux - a) return fail(c, LRC_E_INVALID, "a leaf's entries lie outside aux");
            } else if (a >= nnodes || b >= nnodes) {
                return fail(c, LRC_E_INVALID, "a node's child lies outside the nodes");
            }
        }
        for (uint32_t i = 0; i < naux; i++)
            if (aux[i] >= shapes) return fail(c, LRC_E_INVALID, "an aux entry names no shape of the scene");
    }
    DeviceGuard g(c->device);
    s->walk_ok = false;
    s->wide_ok = false;
    const size_t cap = std::max<size_t>(naux, ((size_t)nnodes + 1) / 2);   // (2 cap - 1 nodes, cap aux)
    cudaError_t e = cudaSuccess;
    if (s->tree_cap < cap) {
        cudaFree(s->d_nodes);
        cudaFree(s->d_aux);
        s->d_nodes = nullptr;
        s->d_aux = nullptr;
        s->tree_cap = 0;
        e = cudaMalloc(&s->d_nodes, (2 * cap - 1) * 32);
        if (!e) e = cudaMalloc(&s->d_aux, cap * 4);
        if (!e) s->tree_cap = cap;
    }
    const cudaMemcpyKind k = (flags & LRC_DEVICE) ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
    if (!e) e = cudaMemcpyAsync(s->d_nodes, nodes, (size_t)nnodes * 32, k, c->st);
    if (!e) e = cudaMemcpyAsync(s->d_aux, aux, (size_t)naux * 4, k, c->st);
    if (e) return cuda_status(c, e, "lrc_scene_set_tree");
    s->built_n = naux;
    s->tree_nnodes = nnodes;
    s->tree_naux = naux;
    int rc = make_walk(s);
    if (rc) return rc;
    return (flags & LRC_DEVICE) ? LRC_OK : check_status(c);
}

int lrc_device_alloc(lrc_ctx *c, size_t bytes, void **out) {
    if (!c || !out) return LRC_E_INVALID;
    *out = nullptr;
    DeviceGuard g(c->device);
    cudaError_t e = cudaMalloc(out, bytes ? bytes : 1);
    if (e == cudaErrorMemoryAllocation) {
        cudaGetLastError();
        return fail(c, LRC_RETRY, "out of device memory");
    }
    return cuda_status(c, e, "lrc_device_alloc");
}

void lrc_device_free(lrc_ctx *c, void *p) {
    if (!c || !p) return;
    DeviceGuard g(c->device);
    cudaStreamSynchronize(c->st);
    cudaFree(p);
}

int lrc_device_copy(lrc_ctx *c, void *dst, const void *src, size_t bytes, int kind) {
    if (!c || (bytes && (!dst || !src)) || kind < LRC_COPY_H2D || kind > LRC_COPY_D2D) return LRC_E_INVALID;
    DeviceGuard g(c->device);
    const cudaMemcpyKind k = kind == LRC_COPY_H2D ? cudaMemcpyHostToDevice
                             : kind == LRC_COPY_D2H ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice;
    cudaError_t e = bytes ? cudaMemcpyAsync(dst, src, bytes, k, c->st) : cudaSuccess;
    if (e) return cuda_status(c, e, "lrc_device_copy");
    return check_status(c);
}

int lrc_device_zero(lrc_ctx *c, void *p, size_t bytes) {
    if (!c || (bytes && !p)) return LRC_E_INVALID;
    DeviceGuard g(c->device);
    cudaError_t e = bytes ? cudaMemsetAsync(p, 0, bytes, c->st) : cudaSuccess;
    return cuda_status(c, e, "lrc_device_zero");
}

int lrc_query(lrc_ctx *c) {
    if (!c) return LRC_E_INVALID;
    DeviceGuard g(c->device);
    cudaError_t e = cudaStreamQuery(c->st);
    if (e == cudaErrorNotReady) {
        cudaGetLastError();
        return 0;
    }
    if (e) return cuda_status(c, e, "lrc_query");
    return 1;
}

int lrc_scene_tree_device(lrc_scene *s, const uint32_t **nodes, const uint32_t **aux, uint32_t *n) {
    if (!s) return LRC_E_INVALID;
    if (nodes) *nodes = reinterpret_cast<const uint32_t *>(s->d_nodes);
    if (aux) *aux = s->d_aux;
    if (n) *n = s->built_n;
    return s->built_n ? LRC_OK : LRC_E_INVALID;
}

int lrc_scene_intersect(lrc_scene *s, const float *orig, const float *dir, uint64_t nrays, float tmin, float tmax,
                        int32_t *prim, float *t, unsigned flags) {
    if (!s || (nrays && (!orig || !dir || !prim || !t))) return LRC_E_INVALID;
    if (s->tlas_n) return lrc_scene_intersect_ex(s, orig, dir, nrays, tmin, tmax, prim, nullptr, t, flags);
    lrc_ctx *c = s->ctx;
    if (!s->built_n) return fail(c, LRC_E_INVALID, "the scene has no built BVH (lrc_scene_build)");
    DeviceGuard g(c->device);
    lrc::TraceTables tt = tables(s);
    // LRC_SORT_RAYS: the reordering's scratch (large batches); without it the rays go in their order
    void *sort_scratch = nullptr;
    if ((flags & LRC_SORT_RAYS) && lrc::intersect_scratch_bytes(nrays)) {
        if (reserve(&c->scratch, &c->scratch_cap, lrc::intersect_scratch_bytes(nrays)) == cudaSuccess) sort_scratch = c->scratch;
        else cudaGetLastError();
    }
    // a world with primitives walks shape ids (primitives, then triangles); a mesh, triangles alone
    auto run = [&](const float *o, const float *d, int32_t *p, float *tt_out) {
        if (s->nprims) return lrc::pt_intersect(pt_scene(s), o, d, nrays, tmin, tmax, p, nullptr, tt_out, c->d_status, c->st);
        if (s->wide_ok) return lrc::wide_intersect(wide_tables(s), o, d, nrays, tmin, tmax, p, tt_out, c->d_status, c->st);
        return lrc::intersect_device(tt, o, d, nrays, tmin, tmax, p, tt_out, c->d_status, c->st, c->num_sms, sort_scratch,
                                     c->scratch_cap);
    };
    if (flags & LRC_DEVICE) {
        c->timer.begin(LRC_TS_TRACE, c->st);
        cudaError_t e = run(orig, dir, prim, t);
        c->timer.end(c->st);
        return cuda_status(c, e, "lrc_scene_intersect");
    }
    const size_t b_ray = al(nrays * 12);
    cudaError_t e = reserve(&c->stage, &c->stage_cap, 2 * b_ray + 2 * al(nrays * 4));
    if (e) return cuda_status(c, e, "ray staging");
    char *st = static_cast<char *>(c->stage);
    float *d_o = reinterpret_cast<float *>(st), *d_d = reinterpret_cast<float *>(st + b_ray);
    int32_t *d_p = reinterpret_cast<int32_t *>(st + 2 * b_ray);
    float *d_t = reinterpret_cast<float *>(st + 2 * b_ray + al(nrays * 4));
    e = cudaMemcpyAsync(d_o, orig, nrays * 12, cudaMemcpyHostToDevice, c->st);
    if (!e) e = cudaMemcpyAsync(d_d, dir, nrays * 12, cudaMemcpyHostToDevice, c->st);
    c->timer.begin(LRC_TS_TRACE, c->st);
    if (!e) e = run(d_o, d_d, d_p, d_t);
    c->timer.end(c->st);
    if (!e) e = cudaMemcpyAsync(prim, d_p, nrays * 4, cudaMemcpyDeviceToHost, c->st);
    if (!e) e = cudaMemcpyAsync(t, d_t, nrays * 4, cudaMemcpyDeviceToHost, c->st);
    if (e) return cuda_status(c, e, "lrc_scene_intersect");
    return check_status(c);
}

int lrc_scene_trace_stats(lrc_scene *s, const float *orig, const float *dir, uint64_t nrays, float tmin, float tmax,
                          uint64_t *stats, unsigned flags) {
    if (!s || !stats || (nrays && (!orig || !dir))) return LRC_E_INVALID;
    lrc_ctx *c = s->ctx;
    if (!s->built_n) return fail(c, LRC_E_INVALID, "the scene has no built BVH (lrc_scene_build)");
    DeviceGuard g(c->device);
    lrc::TraceTables tt = tables(s);
    const size_t b_ray = al(nrays * 12);
    cudaError_t e = reserve(&c->stage, &c->stage_cap, 2 * b_ray + 256);
    if (e) return cuda_status(c, e, "ray staging");
    char *st = static_cast<char *>(c->stage);
    const float *d_o = orig, *d_d = dir;
    unsigned long long *d_stats = reinterpret_cast<unsigned long long *>(st + 2 * b_ray);
    if (!(flags & LRC_DEVICE)) {
        float *o = reinterpret_cast<float *>(st), *d = reinterpret_cast<float *>(st + b_ray);
        e = cudaMemcpyAsync(o, orig, nrays * 12, cudaMemcpyHostToDevice, c->st);
        if (!e) e = cudaMemcpyAsync(d, dir, nrays * 12, cudaMemcpyHostToDevice, c->st);
        d_o = o;
        d_d = d;
    }
    if (!e) e = s->wide_ok ? lrc::wide_count(wide_tables(s), d_o, d_d, nrays, tmin, tmax, d_stats, c->d_status, c->st)
                           : lrc::count_device(tt, d_o, d_d, nrays, tmin, tmax, d_stats, c->d_status, c->st);
    if (!e) e = cudaMemcpyAsync(stats, d_stats, 16, cudaMemcpyDeviceToHost, c->st);
    if (e) return cuda_status(c, e, "lrc_scene_trace_stats");
    const int rc = check_status(c);
    if (!rc && s->wide_ok) stats[0] = (stats[0] * 5 + 1) / 2;   // (an 80-byte wide node: 2.5 records of 32 bytes)
    return rc;
}

int lrc_scene_occluded(lrc_scene *s, const float *orig, const float *dir, const float *tmax, uint64_t nrays, float tmin,
                       uint8_t *out, unsigned flags) {
    if (!s || (nrays && (!orig || !dir || !tmax || !out))) return LRC_E_INVALID;
    lrc_ctx *c = s->ctx;
    if (!s->built_n) return fail(c, LRC_E_INVALID, "the scene has no built BVH (lrc_scene_build)");
    DeviceGuard g(c->device);
    lrc::TraceTables tt = tables(s);
    if (flags & LRC_DEVICE) {
        cudaError_t e = s->wide_ok ? lrc::wide_occluded(wide_tables(s), orig, dir, tmax, nrays, tmin, out, c->d_status, c->st)
                                   : lrc::occluded_device(tt, orig, dir, tmax, nrays, tmin, out, c->d_status, c->st);
        return cuda_status(c, e, "lrc_scene_occluded");
    }
    const size_t b_ray = al(nrays * 12);
    cudaError_t e = reserve(&c->stage, &c->stage_cap, 2 * b_ray + al(nrays * 4) + al(nrays));
    if (e) return cuda_status(c, e, "ray staging");
    char *st = static_cast<char *>(c->stage);
    float *d_o = reinterpret_cast<float *>(st), *d_d = reinterpret_cast<float *>(st + b_ray);
    float *d_tm = reinterpret_cast<float *>(st + 2 * b_ray);
    uint8_t *d_out = reinterpret_cast<uint8_t *>(st + 2 * b_ray + al(nrays * 4));
    e = cudaMemcpyAsync(d_o, orig, nrays * 12, cudaMemcpyHostToDevice, c->st);
    if (!e) e = cudaMemcpyAsync(d_d, dir, nrays * 12, cudaMemcpyHostToDevice, c->st);
    if (!e) e = cudaMemcpyAsync(d_tm, tmax, nrays * 4, cudaMemcpyHostToDevice, c->st);
    if (!e) e = s->wide_ok ? lrc::wide_occluded(wide_tables(s), d_o, d_d, d_tm, nrays, tmin, d_out, c->d_status, c->st)
                           : lrc::occluded_device(tt, d_o, d_d, d_tm, nrays, tmin, d_out, c->d_status, c->st);
    if (!e) e = cudaMemcpyAsync(out, d_out, nrays, cudaMemcpyDeviceToHost, c->st);
    if (e) return cuda_status(c, e, "lrc_scene_occluded");
    return check_status(c);
}

// ---- the world besides its triangles, and the path tracer ---------------------------------------
int lrc_scene_set_prims(lrc_scene *s, const float *prims, uint32_t n, unsigned flags) {
    if (!s || (n && !prims)) return LRC_E_INVALID;
    lrc_ctx *c = s->ctx;
    DeviceGuard g(c->device);
    cudaError_t e = reserve(reinterpret_cast<void **>(&s->d_prims), &s->prims_cap, (size_t)(n ? n : 1) * 96);
    if (!e && n)
        e = cudaMemcpyAsync(s->d_prims, prims, (size_t)n * 96, (flags & LRC_DEVICE) ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice,
                            c->st);
    if (e) return cuda_status(c, e, "primitives");
    s->nprims = n;
    s->built_n = 0;
    s->tree_nnodes = s->tree_naux = 0;
    s->walk_ok = false;
    s->wide_ok = false;
    return (flags & LRC_DEVICE) ? LRC_OK : check_status(c);
}

int lrc_scene_set_normals(lrc_scene *s, const float *normals, uint32_t n, unsigned flags) {
    if (!s || (n && !normals)) return LRC_E_INVALID;
    lrc_ctx *c = s->ctx;
    DeviceGuard g(c->device);
    cudaError_t e = reserve(reinterpret_cast<void **>(&s->d_normals), &s->normals_cap, (size_t)(n ? n : 1) * 12);
    if (!e && n)
        e = cudaMemcpyAsync(s->d_normals, normals, (size_t)n * 12,
                            (flags & LRC_DEVICE) ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, c->st);
    if (e) return cuda_status(c, e, "normals");
    s->nnormals = n;
    return (flags & LRC_DEVICE) ? LRC_OK : check_status(c);
}

int lrc_scene_set_materials(lrc_scene *s, const float *mats, uint32_t n) {
    if (!s || n > 64 || (n && !mats)) return LRC_E_INVALID;
    lrc_ctx *c = s->ctx;
    DeviceGuard g(c->device);
    cudaError_t e = cudaSuccess;
    if (!s->d_mats) e = cudaMalloc(&s->d_mats, 64 * 64);
    if (!e && n) e = cudaMemcpyAsync(s->d_mats, mats, (size_t)n * 64, cudaMemcpyHostToDevice, c->st);
    if (e) return cuda_status(c, e, "materials");
    s->nmats = n;
    // scene_has_specular (tracer.c:547-551): material_has_delta (brdf.h:407-410) of any material,
    // the roughness as material_resolved fills it in for the presets
    s->specular = false;
    for (uint32_t i = 0; i < n; i++) {
        const float *m = mats + 16 * (size_t)i;
        int type;
        std::memcpy(&type, m + 3, 4);
        float r = m[10];
        if (type == 3) continue;                  // MAT_LIGHT
        if (type == 0) r = 1.0f;                  // MAT_DIFFUSE
        else if (type == 1 || type == 2) r = 0.0f;   // MAT_MIRROR, MAT_GLASS
        const float c01 = r < 0.0f ? 0.0f : (r > 1.0f ? 1.0f : r);
        if (c01 <= 0.02f) s->specular = true;
        uint32_t mr;                              // (a roughness texture may make any texel smooth)
        std::memcpy(&mr, m + 13, 4);
        if (mr & 0xffu) s->specular = true;
    }
    return check_status(c);
}

int lrc_scene_set_light(lrc_scene *s, int32_t prim) {
    if (!s) return LRC_E_INVALID;
    s->light = prim;
    return LRC_OK;
}

int lrc_scene_set_tables(lrc_scene *s, const uint16_t *blue_noise, const float *bsdf_tables) {
    if (!s) return LRC_E_INVALID;
    lrc_ctx *c = s->ctx;
    DeviceGuard g(c->device);
    std::vector<uint16_t> mask(4096);
    std::vector<float> tab(kBsdfTableFloats);
    if (blue_noise) std::memcpy(mask.data(), blue_noise, 4096 * 2);
    else lrc::default_blue_noise(mask.data());
    if (bsdf_tables) std::memcpy(tab.data(), bsdf_tables, tab.size() * 4);
    else lrc::default_bsdf_tables(tab.data());
    cudaError_t e = cudaSuccess;
    if (!s->d_mask) e = cudaMalloc(&s->d_mask, 4096 * 2 + kBsdfTableFloats * 4 + 256);
    if (e) return cuda_status(c, e, "tables");
    s->d_tab = reinterpret_cast<float *>(s->d_mask + 4096);
    e = cudaMemcpyAsync(s->d_mask, mask.data(), 4096 * 2, cudaMemcpyHostToDevice, c->st);
    if (!e) e = cudaMemcpyAsync(s->d_tab, tab.data(), tab.size() * 4, cudaMemcpyHostToDevice, c->st);
    if (e) return cuda_status(c, e, "tables");
    s->tables = true;
    return check_status(c);
}

int lrc_scene_set_meshes(lrc_scene *s, const uint32_t *tris, const uint32_t *tri_counts, uint32_t nmeshes, unsigned flags) {
    if (!s || (nmeshes && !tri_counts)) return LRC_E_INVALID;
    lrc_ctx *c = s->ctx;
    uint64_t total = 0;
    for (uint32_t m = 0; m < nmeshes; m++) total += tri_counts[m];
    if (total >= (1u << 30)) return fail(c, LRC_E_INVALID, "more than 2^30 - 1 mesh triangles");
    if (total && !tris) return LRC_E_INVALID;
    DeviceGuard g(c->device);
    cudaFree(s->d_mtris);
    cudaFree(s->d_mnodes);
    cudaFree(s->d_maux);
    cudaFree(s->d_mesh_info);
    s->d_mtris = nullptr; s->d_mnodes = nullptr; s->d_maux = nullptr; s->d_mesh_info = nullptr;
    s->meshes_built = false;
    s->mesh_counts.assign(tri_counts, tri_counts + nmeshes);
    s->nmtris = (uint32_t)total;
    size_t nodes = 0;
    for (uint32_t m = 0; m < nmeshes; m++) nodes += tri_counts[m] ? 2 * (size_t)tri_counts[m] - 1 : 0;
    cudaError_t e = cudaMalloc(&s->d_mtris, (size_t)(total ? total : 1) * 48);
    if (!e) e = cudaMalloc(&s->d_mnodes, (nodes ? nodes : 1) * 32);
    if (!e) e = cudaMalloc(&s->d_maux, (size_t)(total ? total : 1) * 4);
    if (!e) e = cudaMalloc(&s->d_mesh_info, (size_t)(nmeshes ? nmeshes : 1) * 16);
    if (!e && total)
        e = cudaMemcpyAsync(s->d_mtris, tris, total * 48, (flags & LRC_DEVICE) ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice,
                            c->st);
    if (e) return cuda_status(c, e, "meshes");
    return (flags & LRC_DEVICE) ? LRC_OK : check_status(c);
}

int lrc_scene_set_instances(lrc_scene *s, const float *records, uint32_t n, unsigned flags) {
    if (!s || (n && !records)) return LRC_E_INVALID;
    lrc_ctx *c = s->ctx;
    if (n >= (1u << 30)) return fail(c, LRC_E_INVALID, "more than 2^30 - 1 instances");
    DeviceGuard g(c->device);
    cudaError_t e = reserve(reinterpret_cast<void **>(&s->d_inst), &s->inst_cap, (size_t)(n ? n : 1) * 128);
    if (!e && n)
        e = cudaMemcpyAsync(s->d_inst, records, (size_t)n * 128,
                            (flags & LRC_DEVICE) ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, c->st);
    if (e) return cuda_status(c, e, "instances");
    s->ninst = n;
    s->tlas_n = 0;
    return (flags & LRC_DEVICE) ? LRC_OK : check_status(c);
}

int lrc_scene_build_instances(lrc_scene *s, int mesh_builder, int key_bits) {
    if (!s) return LRC_E_INVALID;
    lrc_ctx *c = s->ctx;
    if (key_bits != 30 && key_bits != 63) return fail(c, LRC_E_INVALID, "key_bits must be 30 or 63");
    DeviceGuard g(c->device);
    cudaError_t e = cudaSuccess;
    uint32_t *keys = s->d_small;
    float *bounds = reinterpret_cast<float *>(s->d_small + 8), *lo_ext = reinterpret_cast<float *>(s->d_small + 16);
    if (!s->meshes_built) {
        // each mesh's tree as a dynamic mesh's (upload_instances, trace_gpu.c:1497-1512): its triangles'
        // boxes, its corners' box as the bounds; leaves' aux: the triangles' global indices
        std::vector<uint4> info(s->mesh_counts.size());
        uint32_t node0 = 0, tri0 = 0, most = 1;
        for (uint32_t n : s->mesh_counts) most = n > most ? n : most;
        e = reserve(reinterpret_cast<void **>(&s->d_boxes), &s->boxes_cap, (size_t)most * 32);
        if (!e) e = reserve(&c->scratch, &c->scratch_cap, lrc::build_scratch_bytes(most, key_bits, mesh_builder));
        if (e) return cuda_status(c, e, "mesh build memory");
        c->timer.begin(LRC_TS_BOXES, c->st);
        for (size_t m = 0; m < s->mesh_counts.size() && !e; m++) {
            const uint32_t n = s->mesh_counts[m];
            info[m] = make_uint4(node0, tri0, n, 0);
            if (!n) continue;
            e = lrc::triangle_boxes(s->d_mtris + 12 * (size_t)tri0, n, s->d_boxes, keys, c->st, c->num_sms);
            if (!e) e = lrc::bounds_params(keys, bounds, lo_ext, c->st);
            lrc_build_params p{};
            p.n = n; p.node0 = node0; p.ref0 = tri0; p.ref_add = tri0; p.key_bits = key_bits; p.builder = mesh_builder;
            if (!e) e = lrc::build_device_ext(p, s->d_boxes, lo_ext, s->d_mnodes + node0, s->d_maux + tri0, c->scratch,
                                              c->scratch_cap, c->d_status, c->num_sms, c->st, nullptr, &c->timer);
            node0 += 2 * n - 1;
            tri0 += n;
        }
        if (!e && !info.empty())
            e = cudaMemcpyAsync(s->d_mesh_info, info.data(), info.size() * 16, cudaMemcpyHostToDevice, c->st);
        if (e) return cuda_status(c, e, "mesh trees");
        int rc = check_status(c);                        // (the host vector goes out of scope)
        if (rc) return rc;
        s->meshes_built = true;
    }
    s->tlas_n = 0;
    const uint32_t n = s->ninst;
    if (!n) return LRC_OK;
    if (s->tlas_cap < n) {
        cudaFree(s->d_tlas_nodes);
        cudaFree(s->d_tlas_aux);
        s->d_tlas_nodes = nullptr; s->d_tlas_aux = nullptr; s->tlas_cap = 0;
        e = cudaMalloc(&s->d_tlas_nodes, (2 * (size_t)n - 1) * 32);
        if (!e) e = cudaMalloc(&s->d_tlas_aux, (size_t)n * 4);
        if (!e) s->tlas_cap = n;
    }
    if (!e) e = reserve(reinterpret_cast<void **>(&s->d_boxes), &s->boxes_cap, (size_t)n * 32);
    if (!e) e = reserve(&c->scratch, &c->scratch_cap, lrc::build_scratch_bytes(n, 30, 0));
    if (e) return cuda_status(c, e, "top level memory");
    c->timer.begin(LRC_TS_BOXES, c->st);
    e = build_tlas_on(c, s->d_inst, n, s->d_tlas_nodes, s->d_tlas_aux, s->d_boxes, s->d_small, c->scratch, c->scratch_cap,
                      c->st, &c->timer);
    if (e) return cuda_status(c, e, "top level");
    s->tlas_n = n;
    s->tlas_cost = -1.0;
    return LRC_OK;
}

int lrc_scene_move_instances(lrc_scene *s, const float *records, uint32_t n, int mode, unsigned flags) {
    if (!s || !records) return LRC_E_INVALID;
    lrc_ctx *c = s->ctx;
    if (mode < LRC_TLAS_REFIT || mode > LRC_TLAS_AUTO) return fail(c, LRC_E_INVALID, "mode: refit, rebuild or auto");
    if (!s->tlas_n || n != s->ninst) return fail(c, LRC_E_INVALID, "moves the built instances only (same count)");
    DeviceGuard g(c->device);
    cudaError_t e = cudaMemcpyAsync(s->d_inst, records, (size_t)n * 128,
                                    (flags & LRC_DEVICE) ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, c->st);
    if (e) return cuda_status(c, e, "instances");
    if (mode == LRC_TLAS_REBUILD) {
        s->tlas_n = 0;
        e = reserve(&c->scratch, &c->scratch_cap, lrc::build_scratch_bytes(n, 30, 0));
        if (!e) e = build_tlas_on(c, s->d_inst, n, s->d_tlas_nodes, s->d_tlas_aux, s->d_boxes, s->d_small, c->scratch,
                                  c->scratch_cap, c->st, &c->timer);
        if (e) return cuda_status(c, e, "top level");
        s->tlas_n = n;
        s->tlas_cost = -1.0;
        return (flags & LRC_DEVICE) ? LRC_OK : check_status(c);
    }
    if (mode == LRC_TLAS_AUTO && s->tlas_cost < 0) {        // (the cost the refits are held against)
        int rc = lrc_scene_tlas_cost(s, &s->tlas_cost);
        if (rc) return rc;
    }
    e = reserve(&c->scratch, &c->scratch_cap, lrc::refit_scratch_bytes(n));
    if (!e) e = lrc::refit_device(s->d_tlas_nodes, s->d_tlas_aux, n, 0, s->d_inst, 8, 6, c->scratch, c->scratch_cap,
                                  c->d_status, c->st);
    if (e) return cuda_status(c, e, "top level refit");
    if (mode == LRC_TLAS_AUTO) {
        double cost = 0;
        int rc = lrc_scene_tlas_cost(s, &cost);
        if (rc) return rc;
        if (cost > 1.1 * s->tlas_cost) return lrc_scene_move_instances(s, s->d_inst, n, LRC_TLAS_REBUILD, LRC_DEVICE);
    }
    return (flags & LRC_DEVICE) ? LRC_OK : check_status(c);
}

int lrc_scene_tlas_cost(lrc_scene *s, double *cost) {
    if (!s || !cost) return LRC_E_INVALID;
    lrc_ctx *c = s->ctx;
    if (!s->tlas_n) return fail(c, LRC_E_INVALID, "the scene has no top level");
    DeviceGuard g(c->device);
    double *d = reinterpret_cast<double *>(s->d_small + 32);
    cudaError_t e = lrc::tree_cost_device(s->d_tlas_nodes, s->tlas_n, d, c->st);
    if (!e) e = cudaMemcpyAsync(cost, d, 8, cudaMemcpyDeviceToHost, c->st);
    if (e) return cuda_status(c, e, "top level cost");
    return check_status(c);
}

int lrc_refit(lrc_ctx *c, uint32_t *nodes, const uint32_t *aux, uint32_t n, uint32_t ref_add, const float *boxes,
              unsigned flags) {
    if (!c || !nodes || !aux || !boxes) return LRC_E_INVALID;
    if (!n) return LRC_OK;
    if (n >= (1u << 30)) return fail(c, LRC_E_INVALID, "more than 2^30 - 1 items");
    DeviceGuard g(c->device);
    const size_t b_nodes = (2 * (size_t)n - 1) * 32, b_aux = (size_t)n * 4, b_boxes = (size_t)n * 32;
    cudaError_t e = reserve(&c->scratch, &c->scratch_cap, lrc::refit_scratch_bytes(n));
    if (e) return cuda_status(c, e, "refit scratch");
    Node *d_nodes = reinterpret_cast<Node *>(nodes);
    const uint32_t *d_aux = aux;
    const float *d_boxes = boxes;
    if (!(flags & LRC_DEVICE)) {
        e = reserve(&c->stage, &c->stage_cap, al(b_nodes) + al(b_aux) + al(b_boxes));
        if (e) return cuda_status(c, e, "refit staging");
        char *st = static_cast<char *>(c->stage);
        d_nodes = reinterpret_cast<Node *>(st);
        d_aux = reinterpret_cast<const uint32_t *>(st + al(b_nodes));
        d_boxes = reinterpret_cast<const float *>(st + al(b_nodes) + al(b_aux));
        e = cudaMemcpyAsync(d_nodes, nodes, b_nodes, cudaMemcpyHostToDevice, c->st);
        if (!e) e = cudaMemcpyAsync(const_cast<uint32_t *>(d_aux), aux, b_aux, cudaMemcpyHostToDevice, c->st);
        if (!e) e = cudaMemcpyAsync(const_cast<float *>(d_boxes), boxes, b_boxes, cudaMemcpyHostToDevice, c->st);
    }
    if (!e) e = lrc::refit_device(d_nodes, d_aux, n, ref_add, d_boxes, 2, 0, c->scratch, c->scratch_cap, c->d_status, c->st);
    if (!e && !(flags & LRC_DEVICE)) e = cudaMemcpyAsync(nodes, d_nodes, b_nodes, cudaMemcpyDeviceToHost, c->st);
    if (e) return cuda_status(c, e, "lrc_refit");
    return (flags & LRC_DEVICE) ? LRC_OK : check_status(c);
}

int lrc_scene_set_sky(lrc_scene *s, const float *rgb, int32_t w, int32_t h, const float *marg, const float *cond,
                      const float *prob, float scale) {
    if (!s) return LRC_E_INVALID;
    lrc_ctx *c = s->ctx;
    DeviceGuard g(c->device);
    cudaFree(s->d_env);
    s->d_env = nullptr;
    s->env_w = s->env_h = 0;
    if (!rgb) return LRC_OK;
    if (w <= 0 || h <= 0 || h > w) return fail(c, LRC_E_INVALID, "a sky is w x h with h <= w (upload_sky)");
    const size_t np = (size_t)w * h;
    std::vector<float> host(4 * np + (size_t)h * (w + 1) + (h + 1));
    float *rgbp = host.data(), *hc = rgbp + 4 * np, *hm = hc + (size_t)h * (w + 1);
    std::vector<float> own_prob;
    int weighted = 1;
    if (!marg || !cond || !prob) {
        own_prob.resize(np);
        weighted = lrc::env_tables(rgb, w, h, hm, hc, own_prob.data()) ? 1 : 0;
        prob = own_prob.data();
    } else {
        std::memcpy(hm, marg, sizeof(float) * (h + 1));
        std::memcpy(hc, cond, sizeof(float) * (size_t)h * (w + 1));
        weighted = 0;
        for (size_t i = 0; i < np && !weighted; i++) weighted = prob[i] > 0;
    }
    for (size_t i = 0; i < np; i++) {
        rgbp[4 * i] = rgb[3 * i];
        rgbp[4 * i + 1] = rgb[3 * i + 1];
        rgbp[4 * i + 2] = rgb[3 * i + 2];
        rgbp[4 * i + 3] = prob[i];
    }
    cudaError_t e = cudaMalloc(&s->d_env, host.size() * 4);
    if (!e) e = cudaMemcpyAsync(s->d_env, host.data(), host.size() * 4, cudaMemcpyHostToDevice, c->st);
    if (e) return cuda_status(c, e, "sky");
    s->env_w = w;
    s->env_h = h;
    s->env_weighted = weighted;
    s->env_scale = scale;
    return check_status(c);
}

int lrc_scene_intersect_ex(lrc_scene *s, const float *orig, const float *dir, uint64_t nrays, float tmin, float tmax,
                           int32_t *prim, int32_t *inst, float *t, unsigned flags) {
    if (!s || (nrays && (!orig || !dir || !prim || !t))) return LRC_E_INVALID;
    lrc_ctx *c = s->ctx;
    if (!s->built_n && !(s->meshes_built && s->tlas_n)) return fail(c, LRC_E_INVALID, "the scene has nothing built");
    DeviceGuard g(c->device);
    if (flags & LRC_DEVICE) {
        cudaError_t e = lrc::pt_intersect(pt_scene(s), orig, dir, nrays, tmin, tmax, prim, inst, t, c->d_status, c->st);
        return cuda_status(c, e, "lrc_scene_intersect_ex");
    }
    const size_t b_ray = al(nrays * 12), b_out = al(nrays * 4);
    cudaError_t e = reserve(&c->stage, &c->stage_cap, 2 * b_ray + 3 * b_out);
    if (e) return cuda_status(c, e, "ray staging");
    char *st = static_cast<char *>(c->stage);
    float *d_o = reinterpret_cast<float *>(st), *d_d = reinterpret_cast<float *>(st + b_ray);
    int32_t *d_p = reinterpret_cast<int32_t *>(st + 2 * b_ray), *d_i = reinterpret_cast<int32_t *>(st + 2 * b_ray + b_out);
    float *d_t = reinterpret_cast<float *>(st + 2 * b_ray + 2 * b_out);
    e = cudaMemcpyAsync(d_o, orig, nrays * 12, cudaMemcpyHostToDevice, c->st);
    if (!e) e = cudaMemcpyAsync(d_d, dir, nrays * 12, cudaMemcpyHostToDevice, c->st);
    if (!e) e = lrc::pt_intersect(pt_scene(s), d_o, d_d, nrays, tmin, tmax, d_p, d_i, d_t, c->d_status, c->st);
    if (!e) e = cudaMemcpyAsync(prim, d_p, nrays * 4, cudaMemcpyDeviceToHost, c->st);
    if (!e && inst) e = cudaMemcpyAsync(inst, d_i, nrays * 4, cudaMemcpyDeviceToHost, c->st);
    if (!e) e = cudaMemcpyAsync(t, d_t, nrays * 4, cudaMemcpyDeviceToHost, c->st);
    if (e) return cuda_status(c, e, "lrc_scene_intersect_ex");
    return check_status(c);
}

int lrc_trace(lrc_scene *s, const lrc_trace_params *p, int32_t y0, int32_t rows, uint32_t spp0, uint32_t spp, float *accum,
              uint64_t *rays, unsigned flags) {
    if (!s || !p || !accum || p->width <= 0 || p->height <= 0 || y0 < 0 || rows < 0 || y0 + rows > p->height)
        return LRC_E_INVALID;
    lrc_ctx *c = s->ctx;
    if (!s->built_n && !s->tlas_n) return fail(c, LRC_E_INVALID, "the scene has nothing built (lrc_scene_build)");
    if (s->ninst && s->tlas_n != s->ninst) return fail(c, LRC_E_INVALID, "instances changed: lrc_scene_build_instances");
    if (p->exact && spp0 != 0) return fail(c, LRC_E_INVALID, "exact mode starts at each pixel's first sample (spp0 = 0)");
    if (!s->d_mats || !s->nmats) return fail(c, LRC_E_INVALID, "the scene has no materials (lrc_scene_set_materials)");
    if (s->light >= (int32_t)s->nprims) return fail(c, LRC_E_INVALID, "the light is not one of the primitives");
    DeviceGuard g(c->device);
    if (!s->tables) {
        int rc = lrc_scene_set_tables(s, nullptr, nullptr);
        if (rc) return rc;
    }
    cudaError_t e = cudaSuccess;
    if (!s->d_rays) e = cudaMalloc(&s->d_rays, 256);
    if (!e) e = cudaMemsetAsync(s->d_rays, 0, 8, c->st);
    if (e) return cuda_status(c, e, "ray counter");
    lrc::PtParams P{};
    P.W = p->width; P.H = p->height; P.y0 = y0; P.rows = rows; P.spp0 = (int)spp0; P.spp = (int)spp;
    P.max_depth = p->max_depth; P.mis = p->mis; P.sampler_on = p->sampler; P.exact = p->exact;
    int gsz = 1;
    while (gsz * 2 <= (int)spp && gsz < 16) gsz *= 2;
    P.group = gsz;
    P.seed = p->seed;
    P.clamp = p->clamp;
    P.skip_caustics = p->skip_caustics != 0;
    P.indirect_clamp = p->indirect_clamp;
    P.origin = {p->origin[0], p->origin[1], p->origin[2]};
    P.upper_left = {p->upper_left[0], p->upper_left[1], p->upper_left[2]};
    P.horizontal = {p->horizontal[0], p->horizontal[1], p->horizontal[2]};
    P.vertical = {p->vertical[0], p->vertical[1], p->vertical[2]};
    // LRC_TRACE_GUIDED: accum holds the denoiser's 4 planes; the moments go to plane 1
    const bool guided = (flags & LRC_TRACE_GUIDED) != 0;
    const size_t bytes = (size_t)p->width * p->height * (guided ? 64 : 16);
    float *d_acc = accum;
    if (!(flags & LRC_DEVICE)) {
        e = reserve(&c->stage, &c->stage_cap, bytes);
        if (e) return cuda_status(c, e, "image staging");
        d_acc = static_cast<float *>(c->stage);
        e = cudaMemcpyAsync(d_acc, accum, bytes, cudaMemcpyHostToDevice, c->st);
    }
    if (guided) {
        const size_t N = (size_t)p->width * p->height;
        P.moments = reinterpret_cast<float4 *>(d_acc) + N;
        P.guide = reinterpret_cast<const float4 *>(d_acc) + 3 * N;
    }
    // a large image runs as a one-job batch on the wavefront engine: its kernels keep their own
    // registers (the one-kernel path sits at its cap with every bounce's code in one loop), and its
    // image is this call's to the bit (a batch task traces a pixel's samples as the one-kernel
    // path's lanes do and the resolve pass adds them in that path's order)
    const uint64_t paths = (uint64_t)p->width * (uint64_t)rows * spp;
    if (!e && !(flags & LRC_TRACE_MEGAKERNEL) && !s->nvol && rows > 0 && spp > 0 && paths >= LRC_TRACE_WAVEFRONT_PATHS) {
        int rc = LRC_OK;
        if (!c->single) {
            rc = lrc_batch_create(c, &c->single);
            if (rc) return rc;
        }
        rc = lrc_batch_set_wavefront(c->single, paths >= (8u << 20) ? 1u << 22 : 1u << 20,
                                     LRC_WAVEFRONT_DEFAULT_VARIANT);
        if (!rc) rc = lrc_batch_clear(c->single);
        if (!rc) rc = guided ? lrc_batch_add_guided(c->single, s, p, y0, rows, spp0, spp, d_acc, -1, 30)
                             : lrc_batch_add(c->single, s, p, y0, rows, spp0, spp, d_acc, -1, 30);
        c->timer.begin(LRC_TS_SHADE, c->st);
        if (!rc) rc = lrc_batch_run(c->single, 0);
        c->timer.end(c->st);
        if (rc) return rc;
        if (!(flags & LRC_DEVICE)) {
            e = cudaMemcpyAsync(accum, d_acc, bytes, cudaMemcpyDeviceToHost, c->st);
            if (e) return cuda_status(c, e, "lrc_trace");
        }
        if (rays) return lrc_batch_rays(c->single, rays, nullptr);   // (waits)
        return (flags & LRC_DEVICE) ? LRC_OK : check_status(c);
    }
    c->timer.begin(LRC_TS_SHADE, c->st);
    if (!e) e = lrc::pt_trace(pt_scene(s), P, d_acc, s->d_rays, c->d_status, c->st);
    c->timer.end(c->st);
    if (!e && !(flags & LRC_DEVICE)) e = cudaMemcpyAsync(accum, d_acc, bytes, cudaMemcpyDeviceToHost, c->st);
    unsigned long long nr = 0;
    if (!e && rays) e = cudaMemcpyAsync(&nr, s->d_rays, 8, cudaMemcpyDeviceToHost, c->st);
    if (e) return cuda_status(c, e, "lrc_trace");
    int rc = (flags & LRC_DEVICE) && !rays ? LRC_OK : check_status(c);
    if (rays) *rays = nr;
    return rc;
}

}  // extern "C"
