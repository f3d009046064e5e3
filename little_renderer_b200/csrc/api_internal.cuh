// api_internal.cuh - what the C ABI's translation units share: the context and scene objects
// behind include/lrc.h's opaque handles, status helpers and the path tracer's view of a scene.
#pragma once
#include "lrc_internal.cuh"
#include <algorithm>
#include <string>
#include <vector>

using lrc::Node;

struct lrc_ctx {
    int device = 0;
    int num_sms = 0;
    cudaStream_t own = nullptr, st = nullptr;
    uint32_t *d_status = nullptr;
    void *scratch = nullptr;
    size_t scratch_cap = 0;
    void *stage = nullptr;
    size_t stage_cap = 0;
    lrc::StageTimer timer;
    std::string msg;
    int lt_variant = -1;          // the light tracer's launch variant (-1: the default)
    void *dn = nullptr;           // the denoiser's scratch (packed image ping-pong and guide)
    size_t dn_cap = 0;
    lrc_batch *single = nullptr;  // lrc_trace's one-job batch on the wavefront engine (large images)
};

struct lrc_scene {
    lrc_ctx *ctx = nullptr;
    uint32_t *d_tris = nullptr;
    size_t tris_cap = 0;
    uint32_t ntris = 0;
    Node *d_nodes = nullptr;
    uint32_t *d_aux = nullptr;
    size_t tree_cap = 0;          // items the tree buffers hold
    uint32_t built_n = 0;         // items of the built tree (0: none)
    uint32_t tree_nnodes = 0;     // a tree given by lrc_scene_set_tree: its nodes and aux entries
    uint32_t tree_naux = 0;       // (0: the built tree's 2 n - 1 and n)
    Node *d_wnodes = nullptr;     // the walk's copy of a triangle tree with tight boxes (lrc_scene_set_walk)
    size_t wnodes_cap = 0;        // (nodes)
    bool walk_ok = false;         // d_wnodes is the current tree's
    int walk_mode = 1;            // 0 the tree as built, 1 tight boxes, 2 tight 8-wide nodes
    float4 *d_wide = nullptr;     // the walk's 8-wide nodes (walk_mode 2) and their triangle entries
    size_t wide_cap = 0;
    uint32_t *d_wrefs = nullptr;
    size_t wrefs_cap = 0;
    uint32_t nwide = 0;
    bool wide_ok = false;
    float *d_boxes = nullptr;
    size_t boxes_cap = 0;
    uint32_t *d_small = nullptr;  // 6 bound keys, 6 bounds, 6 lo/ext
    // the world besides its triangles (path tracing)
    float *d_prims = nullptr;     // 24 floats per primitive
    size_t prims_cap = 0;
    uint32_t nprims = 0;
    float *d_normals = nullptr;
    size_t normals_cap = 0;
    uint32_t nnormals = 0;
    float *d_mats = nullptr;      // 64 materials x 16 floats
    uint32_t nmats = 0;
    int32_t light = -1;
    uint16_t *d_mask = nullptr;   // 4096 ranks, then the 2112 table floats
    float *d_tab = nullptr;
    bool tables = false;
    unsigned long long *d_rays = nullptr;
    // instances: meshes' triangles and trees, records, the top level
    uint32_t *d_mtris = nullptr;
    uint32_t nmtris = 0;
    std::vector<uint32_t> mesh_counts;
    Node *d_mnodes = nullptr;
    uint32_t *d_maux = nullptr;
    uint4 *d_mesh_info = nullptr;
    bool meshes_built = false;
    float *d_inst = nullptr;
    size_t inst_cap = 0;
    uint32_t ninst = 0;
    Node *d_tlas_nodes = nullptr;
    uint32_t *d_tlas_aux = nullptr;
    size_t tlas_cap = 0;
    uint32_t tlas_n = 0;
    double tlas_cost = -1.0;      // its SAH cost as built (-1: not yet reckoned)
    // the sky
    float *d_env = nullptr;       // rgbp (w x h float4), cond, marg
    int env_w = 0, env_h = 0, env_weighted = 0;
    float env_scale = 1;
    // light tracing: a material with a perfectly smooth part (scene_has_specular), the sums' scratch
    bool specular = false;
    void *d_caus = nullptr;
    size_t caus_cap = 0;
    // participating media: the VolDev table, then each volume's density and brick majorants
    void *d_vols = nullptr;
    uint32_t nvol = 0;
    // textures: the texmap table, the sRGB table, the texels; the triangles' texture coordinates
    void *d_tex = nullptr;
    uint32_t ntex = 0;
    size_t tex_lut_off = 0, texel_off = 0;
    void *d_uv = nullptr;
    uint32_t uv_tris = 0, nuv = 0;
    size_t uv_off = 0, tangent_off = 0;
};

namespace lrcapi {

inline int fail(lrc_ctx *c, int code, const char *what, cudaError_t e = cudaSuccess) {
    if (c) {
        c->msg = what;
        if (e != cudaSuccess) {
            c->msg += ": ";
            c->msg += cudaGetErrorString(e);
        }
    }
    return code;
}

// a CUDA error as a status: out of memory is refusable (retry after a change), the rest fatal
inline int cuda_status(lrc_ctx *c, cudaError_t e, const char *what) {
    if (e == cudaSuccess) return LRC_OK;
    if (e == cudaErrorMemoryAllocation) {
        cudaGetLastError();
        return fail(c, LRC_RETRY, what, e);
    }
    return fail(c, LRC_E_CUDA, what, e);
}

struct DeviceGuard {
    int prev = -1;
    explicit DeviceGuard(int d) {
        cudaGetDevice(&prev);
        if (prev != d) cudaSetDevice(d);
    }
    ~DeviceGuard() {
        int now = -1;
        cudaGetDevice(&now);
        if (prev >= 0 && now != prev) cudaSetDevice(prev);
    }
};

// a device buffer of at least `bytes` (grown by a quarter more; contents not kept)
inline cudaError_t reserve(void **p, size_t *cap, size_t bytes) {
    if (*cap >= bytes && *p) return cudaSuccess;
    if (*p) cudaFree(*p);
    *p = nullptr;
    *cap = 0;
    size_t want = bytes + bytes / 4 + 4096;
    cudaError_t e = cudaMalloc(p, want);
    if (e == cudaSuccess) *cap = want;
    return e;
}

// reads and clears the status word (synchronises the stream first)
inline int check_status(lrc_ctx *c) {
    cudaError_t e = cudaStreamSynchronize(c->st);
    if (e) return cuda_status(c, e, "device work");
    uint32_t s = 0;
    e = cudaMemcpy(&s, c->d_status, 4, cudaMemcpyDeviceToHost);
    if (e) return cuda_status(c, e, "status word");
    if (s) {
        cudaMemset(c->d_status, 0, 4);
        if (s & lrc::ST_STACK_OVERFLOW) return fail(c, LRC_E_STACK, "a traversal stack would have overflowed (tree too deep)");
        if (s & lrc::ST_BAD_TREE) return fail(c, LRC_E_INVALID, "a tree index out of range was met (not followed)");
        if (s & lrc::ST_LOOP) return fail(c, LRC_E_TIMEOUT, "the wavefront loop ran past its bound (stopped)");
        if (s & lrc::ST_MEDIUM) return fail(c, LRC_E_TIMEOUT, "a medium's tracking ran past its step bound (stopped)");
        return fail(c, LRC_E_TIMEOUT, "a bounded device wait ran out (sort look-back, PLOC look-back or grid barrier)");
    }
    return LRC_OK;
}

inline size_t al(size_t x) { return (x + 255) / 256 * 256; }

// the BSDF tables' floats (E 32 x 32, B 32 x 32, E_avg 32, B_avg 32)
constexpr int kBsdfTableFloats = 2112;

// the path tracer's view of a scene
inline lrc::PtScene pt_scene(const lrc_scene *s) {
    lrc::PtScene S{};
    S.nodes = reinterpret_cast<const float4 *>(s->d_nodes);
    S.aux = s->d_aux;
    S.root = 0;
    S.nnodes = s->tree_nnodes ? s->tree_nnodes : (s->built_n ? 2 * s->built_n - 1 : 0);
    S.naux = s->tree_nnodes ? s->tree_naux : s->built_n;
    S.prims = reinterpret_cast<const float4 *>(s->d_prims);
    S.nprims = s->nprims;
    S.tris = reinterpret_cast<const float4 *>(s->d_tris);
    S.ntris = s->ntris;
    S.normals = s->nnormals ? s->d_normals : nullptr;
    S.mats = reinterpret_cast<const float4 *>(s->d_mats);
    S.nmats = s->nmats;
    S.light = s->light;
    S.mask = s->d_mask;
    S.tab = s->d_tab;
    if (s->meshes_built && s->tlas_n == s->ninst && s->ninst) {
        S.inst = reinterpret_cast<const float4 *>(s->d_inst);
        S.ninst = s->ninst;
        S.tlas_nodes = reinterpret_cast<const float4 *>(s->d_tlas_nodes);
        S.tlas_aux = s->d_tlas_aux;
        S.tlas_nnodes = 2 * s->ninst - 1;
        S.mtris = reinterpret_cast<const float4 *>(s->d_mtris);
        S.nmtris = s->nmtris;
        S.mnodes = reinterpret_cast<const float4 *>(s->d_mnodes);
        S.maux = s->d_maux;
        uint32_t nn = 0;
        for (uint32_t c : s->mesh_counts) nn += c ? 2 * c - 1 : 0;
        S.mnnodes = nn;
        S.mnaux = s->nmtris;
        S.mesh_info = s->d_mesh_info;
        S.nmeshes = (uint32_t)s->mesh_counts.size();
    }
    if (s->nvol) {
        S.vols = static_cast<const lrc::VolDev *>(s->d_vols);
        S.nvol = s->nvol;
    }
    if (s->ntex) {
        const char *b = static_cast<const char *>(s->d_tex);
        S.texs = reinterpret_cast<const uint4 *>(b);
        S.srgb = reinterpret_cast<const float *>(b + s->tex_lut_off);
        S.texels = reinterpret_cast<const uint32_t *>(b + s->texel_off);
        S.ntex = s->ntex;
    }
    if (s->d_uv && s->uv_tris == s->ntris) {         // (texture coordinates for other triangles: none)
        const char *b = static_cast<const char *>(s->d_uv);
        S.tri_uv = reinterpret_cast<const int32_t *>(b);
        S.uvs = reinterpret_cast<const float2 *>(b + s->uv_off);
        S.tangents = reinterpret_cast<const float4 *>(b + s->tangent_off);
        S.nuv = s->nuv;
    }
    if (s->d_env) {
        S.env_rgbp = reinterpret_cast<const float4 *>(s->d_env);
        S.env_cond = s->d_env + 4 * (size_t)s->env_w * s->env_h;
        S.env_marg = S.env_cond + (size_t)s->env_h * (s->env_w + 1);
        S.env_w = s->env_w;
        S.env_h = s->env_h;
        S.has_env = 1;
        S.env_weighted = s->env_weighted;
        S.env_scale = s->env_scale;
    }
    return S;
}

// the walk's view of a scene: its tree (root 0), leaves' triangles, and the sizes it checks against
inline lrc::TraceTables tables(const lrc_scene *s) {
    lrc::TraceTables tt{};
    tt.nodes = s->walk_ok ? s->d_wnodes : s->d_nodes;
    tt.aux = s->d_aux;
    tt.tris = reinterpret_cast<const float4 *>(s->d_tris);
    tt.root = 0;
    tt.nnodes = s->tree_nnodes ? s->tree_nnodes : 2 * s->built_n - 1;
    tt.naux = s->tree_nnodes ? s->tree_naux : s->built_n;
    tt.ntris = s->ntris;
    return tt;
}

// the wide walk's view of a scene (walk_mode 2, made)
inline lrc::WideTables wide_tables(const lrc_scene *s) {
    lrc::WideTables wt{};
    wt.nodes = s->d_wide;
    wt.refs = s->d_wrefs;
    wt.tris = reinterpret_cast<const float4 *>(s->d_tris);
    wt.nnodes = s->nwide;
    wt.nrefs = (uint32_t)std::min<size_t>(s->wrefs_cap, 0xffffffffu);
    wt.ntris = s->ntris;
    return wt;
}

// builds the scene's world tree (triangles and primitives) on stream st with the given scratch
// arena; with no_alloc set, a buffer too small is an error instead of a cudaMalloc (the batch's
// graph capture)
int scene_build_on(lrc_scene *s, int builder, int key_bits, void **scratch, size_t *scratch_cap, cudaStream_t st,
                   lrc::StageTimer *timer, bool no_alloc);
// a batch job's own instances: records and their top level (nodes, aux) in place of the scene's
struct InstView {
    const float *inst;
    const void *tlas_nodes;
    const uint32_t *tlas_aux;
};
// lrc_batch_add (no build) with the job's own instances (a server's moving-instance job)
// an event lrc_batch_run records right before it launches the run's trace (null: none)
void batch_set_launch_event(lrc_batch *b, cudaEvent_t e);
// the run buffers sized for up to `tasks` tasks of up to `jobs` jobs now, so that runs within
// those sizes neither allocate nor free device memory (which would wait for the device)
int batch_reserve(lrc_batch *b, unsigned long long tasks, size_t jobs);
// the last run's ray counts per job (h_rays, nj entries) and its wavefront passes, copied to pinned
// host memory on the context's stream, not waited for
cudaError_t batch_counts_async(lrc_batch *b, unsigned long long *h_rays, uint32_t *h_passes);
int batch_add_view(lrc_batch *b, lrc_scene *s, const lrc_trace_params *p, int32_t y0, int32_t rows, uint32_t spp0,
                   uint32_t spp, float *d_accum, const InstView &view, bool guided);
cudaError_t build_tlas_on(lrc_ctx *c, const float *d_inst, uint32_t n, Node *d_nodes, uint32_t *d_aux, float *d_boxes,
                          uint32_t *d_small, void *scratch, size_t scratch_cap, cudaStream_t st, lrc::StageTimer *timer);

}  // namespace lrcapi

