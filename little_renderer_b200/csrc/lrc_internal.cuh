// lrc_internal.cuh - shared device/host definitions of the CUDA backend (sm_100a).
#pragma once
#include <cstdint>
#include <cstddef>
#include <cuda_runtime.h>
#include "../../include/lrc.h"
#include "pt_math.cuh"

namespace lrc {

// A BVH node as the reference's path tracer reads it (engine/gpu/shaders/trace/trace.wgsl:2
// `Node`, written by put_nodes, engine/gpu/trace_gpu.c:883-896): box, and children (absolute
// node indices) or, for a leaf, b = 0x80000000 | count and a = its first entry of aux.
struct __align__(16) Node {
    float lo[3];
    uint32_t a;
    float hi[3];
    uint32_t b;
};
static_assert(sizeof(Node) == 32, "Node is 32 bytes");

constexpr uint32_t LEAF_BIT = 0x80000000u;

// Device status word bits (ctx->d_status): a bounded wait that ran out, a traversal stack that
// would have overflowed. The host reads them after a call; nothing traps.
constexpr uint32_t ST_TIMEOUT_SORT = 1u;
constexpr uint32_t ST_TIMEOUT_PLOC = 2u;
constexpr uint32_t ST_STACK_OVERFLOW = 4u;
constexpr uint32_t ST_TIMEOUT_BARRIER = 8u;
constexpr uint32_t ST_BAD_TREE = 16u;
constexpr uint32_t ST_MEDIUM = 64u;        // a medium's tracking took more steps than its bound (stopped)
constexpr uint32_t ST_LOOP = 32u;          // the wavefront's loop ran past its bound (stopped)

// spins before a bounded wait gives up (each ~ a few hundred ns with the back-off): ~1 s
constexpr uint32_t SPIN_LIMIT = 1u << 22;

// ---- IEEE single-precision arithmetic in the reference's order, never contracted ----------
__device__ __forceinline__ float fadd(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float fsub(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ float fmul(float a, float b) { return __fmul_rn(a, b); }
// WGSL min / max (the shaders' builders): e2 if e2 < e1 (> for max), else e1
__device__ __forceinline__ float wmin(float a, float b) { return b < a ? b : a; }
__device__ __forceinline__ float wmax(float a, float b) { return b > a ? b : a; }
// r_fmin / r_fmax (engine/base/lrmath.h): the other number when b is a NaN
__device__ __forceinline__ float rfmin(float a, float b) { return b != b ? a : (a < b ? a : b); }
__device__ __forceinline__ float rfmax(float a, float b) { return b != b ? a : (a > b ? a : b); }

// ---- scratch arena: one cudaMalloc'd block per context, carved per call ----------------------
struct Carve {
    char *base;
    size_t off, cap;
    template <class T>
    T *take(size_t count, size_t align = 256) {
        off = (off + align - 1) / align * align;
        T *p = reinterpret_cast<T *>(base + off);
        off += count * sizeof(T);
        return p;
    }
};

// GPU time by stage: CUDA events around each stage when on (lrc_set_timing)
struct StageTimer {
    bool on = false;
    int open = -1;
    cudaEvent_t open_ev = nullptr;
    struct Rec { int stage; cudaEvent_t a, b; };
    Rec recs[256];
    int nrec = 0;
    double ms[LRC_NUM_STAGES] = {};
    int launches[LRC_NUM_STAGES] = {};
    void begin(int stage, cudaStream_t st) {
        if (!on) return;
        end(st);
        cudaEventCreate(&open_ev);
        cudaEventRecord(open_ev, st);
        open = stage;
    }
    void end(cudaStream_t st) {
        if (!on || open < 0) return;
        cudaEvent_t b;
        cudaEventCreate(&b);
        cudaEventRecord(b, st);
        if (nrec == 256) collect();
        recs[nrec++] = {open, open_ev, b};
        open = -1;
    }
    void collect() {
        for (int i = 0; i < nrec; i++) {
            float t = 0;
            cudaEventSynchronize(recs[i].b);
            cudaEventElapsedTime(&t, recs[i].a, recs[i].b);
            ms[recs[i].stage] += t;
            launches[recs[i].stage]++;
            cudaEventDestroy(recs[i].a);
            cudaEventDestroy(recs[i].b);
        }
        nrec = 0;
    }
};

// builder internals (build.cu)
size_t build_scratch_bytes(uint32_t n, int key_bits, int builder);
// boxes (n x 8 floats, device) -> the tree: d_nodes points at the tree's node node0 and d_aux at
// aux[ref0] (the values written are absolute: node0 + ..., ref0 + ...). d_lo_ext (6 floats on the
// device: lo, ext) overrides p.lo / p.ext when given. Scratch: at least build_scratch_bytes.
cudaError_t build_device(const lrc_build_params &p, const float *d_boxes, Node *d_nodes, uint32_t *d_aux,
                         void *d_scratch, size_t scratch_bytes, uint32_t *d_status, int num_sms, cudaStream_t st,
                         uint32_t *d_sorted_codes_out = nullptr);
cudaError_t build_device_ext(const lrc_build_params &p, const float *d_boxes, const float *d_lo_ext, Node *d_nodes,
                             uint32_t *d_aux, void *d_scratch, size_t scratch_bytes, uint32_t *d_status, int num_sms,
                             cudaStream_t st, uint32_t *d_sorted_codes_out, StageTimer *timer = nullptr);
// triangle_bounds of n triangles (12 words each) into boxes (8 floats each), and the mesh box's
// order keys into d_bkeys (6 words); bounds_params turns the keys into bounds6 and lo_ext
cudaError_t triangle_boxes(const uint32_t *d_tris, uint32_t n, float *d_boxes, uint32_t *d_bkeys, cudaStream_t st,
                           int num_sms);
cudaError_t bounds_params(const uint32_t *d_bkeys, float *d_bounds6, float *d_lo_ext, cudaStream_t st);

// a stable radix sort of 32-bit keys (4 passes of 8 bits) for other kernels' use: carve the
// scratch, clear the histograms, let a key kernel write S.keys[0..n) and add each key's 4 digits
// into S.hist[pass][256], then run: the permutation (sorted position -> original index) comes out
struct SortU32 {
    uint32_t *keys;
    uint32_t *hist;
    char *base;
    uint32_t n;
};
size_t sort_u32_scratch_bytes(uint64_t n);
SortU32 sort_u32_carve(void *scratch, uint64_t n);
cudaError_t sort_u32_clear(const SortU32 &S, cudaStream_t st);
cudaError_t sort_u32_run(const SortU32 &S, uint32_t *d_status, cudaStream_t st, const uint32_t **perm_out);

// refit (refit.cu): the boxes of a built tree (root at node 0, leaves' aux = item + ref_add) made
// again from the items' boxes up - item k's lo at boxes float4 [k * stride4 + lo_at], hi at the
// next - and the tree's SAH cost (nodes' areas over the root's, in double, in a fixed order)
size_t refit_scratch_bytes(uint32_t n);
cudaError_t refit_device(Node *d_nodes, const uint32_t *d_aux, uint32_t n, uint32_t ref_add, const float *d_boxes,
                         uint32_t stride4, uint32_t lo_at, void *scratch, size_t scratch_bytes, uint32_t *d_status,
                         cudaStream_t st);
cudaError_t tree_cost_device(const Node *d_nodes, uint32_t n, double *d_out, cudaStream_t st);
// the ray queries' walk over 8-wide nodes (wide.cu): 80-byte nodes (5 float4), triangle entries
struct WideTables {
    const float4 *nodes;
    const uint32_t *refs;
    const float4 *tris;      // 3 float4 per triangle
    uint32_t nnodes, nrefs, ntris;
};
// capacity of wide nodes and triangle entries for a binary tree with naux leaf entries
size_t wide_node_cap(uint32_t naux);
size_t wide_scratch_bytes(uint32_t naux);
// the wide tree of the binary tree d_bin (nn nodes, root 0, leaves' aux = triangle ids) into
// d_wnodes (wcap nodes) and d_wrefs (rcap entries); *nwide: the wide nodes made. Waits for the stream
// (one launch a level). A leaf that does not fit a node's slots: ST_BAD_TREE.
cudaError_t wide_build(const Node *d_bin, uint32_t nn, const uint32_t *d_aux, uint32_t naux, const float *d_tris,
                       uint32_t ntris, float4 *d_wnodes, uint32_t wcap, uint32_t *d_wrefs, uint32_t rcap, void *scratch,
                       size_t scratch_bytes, uint32_t *d_status, cudaStream_t st, uint32_t *nwide);
cudaError_t wide_intersect(const WideTables &wt, const float *d_orig, const float *d_dir, uint64_t nrays, float tmin,
                           float tmax, int32_t *d_prim, float *d_t, uint32_t *d_status, cudaStream_t st);
cudaError_t wide_occluded(const WideTables &wt, const float *d_orig, const float *d_dir, const float *d_tmax, uint64_t nrays,
                          float tmin, uint8_t *d_out, uint32_t *d_status, cudaStream_t st);
// totals: [0] wide nodes fetched (80 bytes each), [1] triangle tests
cudaError_t wide_count(const WideTables &wt, const float *d_orig, const float *d_dir, uint64_t nrays, float tmin, float tmax,
                       unsigned long long *d_stats, uint32_t *d_status, cudaStream_t st);
// the walk's tree of a triangle tree (nn nodes, root at 0, leaves' aux = triangle ids): the same
// nodes with each leaf's box the bounds of its triangles' corners widened by 2^-17 of the largest
// coordinate of the source root box (at most the 1e-3 the builders pad with), inner boxes the unions
size_t walk_tree_scratch_bytes(uint32_t nn);
cudaError_t walk_tree_device(const Node *d_src, uint32_t nn, const uint32_t *d_aux, uint32_t naux, const float *d_tris,
                             uint32_t ntris, Node *d_dst, void *scratch, size_t scratch_bytes, uint32_t *d_status,
                             cudaStream_t st);

// traversal internals (traverse.cu)
struct TraceTables {
    const Node *nodes;
    const uint32_t *aux;
    const float4 *tris;      // 3 float4 per triangle (q, u, v; .w holds normals / material bits)
    uint32_t root;           // absolute node index of the root
    uint32_t nnodes, naux, ntris;   // sizes: an index out of them is reported (ST_BAD_TREE), not followed
};
// closest hits; batches of 2^18 rays and more are reordered first when scratch (at least
// intersect_scratch_bytes) is given
size_t intersect_scratch_bytes(uint64_t nrays);
cudaError_t intersect_device(const TraceTables &tt, const float *d_orig, const float *d_dir, uint64_t nrays,
                             float tmin, float tmax, int32_t *d_prim, float *d_t, uint32_t *d_status,
                             cudaStream_t st, int num_sms, void *scratch, size_t scratch_bytes);
cudaError_t count_device(const TraceTables &tt, const float *d_orig, const float *d_dir, uint64_t nrays, float tmin,
                         float tmax, unsigned long long *d_stats, uint32_t *d_status, cudaStream_t st);
cudaError_t occluded_device(const TraceTables &tt, const float *d_orig, const float *d_dir, const float *d_tmax,
                            uint64_t nrays, float tmin, uint8_t *d_out, uint32_t *d_status, cudaStream_t st);

// A participating medium as the device reads it: the reference's Volume (engine/scene/volume.h:21-46)
// with its derived majorants (volume_update)
struct VolDev {
    float lo[3], hi[3];          // the box the grid fills
    float alo[3], ahi[3];        // the smallest box around the voxels with density (+ one voxel)
    float sigma_t, g, max_density;
    float albedo[3];
    int nx, ny, nz, bnx, bny, bnz;
    const float *density;        // nx * ny * nz, x fastest
    const float *brick_max;      // bnx * bny * bnz: each brick's largest reachable density
};
constexpr int kMaxVolumes = 8;   // MAX_VOLUMES (engine/scene/scene.h:12)

// the path tracer's view of a scene (pathtrace.cu)
struct PtScene {
    const float4 *nodes;        // the world's BVH (shape ids in aux: primitives, then triangles)
    const uint32_t *aux;
    uint32_t root, nnodes, naux;
    const float4 *prims;        // 6 float4 per primitive (upload_world's layout)
    uint32_t nprims;
    const float4 *tris;         // 3 float4 per triangle
    uint32_t ntris;
    const float *normals;       // vertex normals (3 floats each), or null
    const float4 *mats;         // 4 float4 per material
    uint32_t nmats;
    int32_t light;              // Scene.light: a quad primitive, or -1
    const uint16_t *mask;       // 64 x 64 blue-noise ranks
    const float *tab;           // the BSDF's 2112 table floats
    // instances: records (8 float4 each), the top level over their boxes, the meshes' triangles,
    // BVHs (one nodes / aux array, each mesh's root at mesh_info.x) and mesh_info (root, first
    // triangle, triangles, 0)
    const float4 *inst;
    uint32_t ninst;
    const float4 *tlas_nodes;
    const uint32_t *tlas_aux;
    uint32_t tlas_nnodes;
    const float4 *mtris;
    uint32_t nmtris;
    const float4 *mnodes;
    const uint32_t *maux;
    uint32_t mnnodes, mnaux;
    const uint4 *mesh_info;
    uint32_t nmeshes;
    // the sky: radiance + pixel probability (w x h), each row's distribution, the rows'
    const float4 *env_rgbp;
    const float *env_cond, *env_marg;
    int env_w, env_h, has_env, env_weighted;
    float env_scale;
    // participating media (none: nvol 0)
    const VolDev *vols;
    uint32_t nvol;
    // the materials' textures: each texmap's (w, h, srgb | wrap_u << 1 | wrap_v << 3, its first
    // texel), the RGBA8 texels (level 0), the sRGB decoding table (256); the world triangles'
    // texture coordinates: 3 indices each (-1: none), the uvs and their tangents (none: ntex 0,
    // tri_uv null)
    const uint4 *texs;
    const uint32_t *texels;
    const float *srgb;
    uint32_t ntex;
    const int32_t *tri_uv;
    const float2 *uvs;
    const float4 *tangents;
    uint32_t nuv;
};
struct PtParams {
    int W, H, y0, rows, spp0, spp, max_depth, mis, sampler_on, exact, group;
    uint64_t seed;
    float clamp;
    pt::V3 origin, upper_left, horizontal, vertical;   // the Camera (camera.h)
    int skip_caustics;                                 // TraceParams.skip_caustics
    float indirect_clamp;                              // TraceParams.indirect_clamp (0: off)
    // the denoiser's planes (lrc_trace with LRC_TRACE_GUIDED; null: none): each sample's luminance
    // over the guide's albedo (plane 3) added to the moments (plane 1) as (l, l^2), and the last
    // sample's l and number in its z and w
    float4 *moments;
    const float4 *guide;
};
// temporal gradients (trace_reproject.wgsl gmatch / gfilter, trace.wgsl main's gradient branch):
// one gradient sample per tile of GRAD_TILE x GRAD_TILE new pixels, row-major tiles
constexpr int GRAD_TILE = 4;
struct GradTile {
    int32_t k, o;      // the new pixel the sample is for; the old pixel it was taken in (-1: no sample)
    float dx, dy;      // the old pixel's offset from where the new pixel's centre was in the old image
    float l;           // the old sample's luminance over the albedo
    uint32_t kk;       // its sample number
    float lam[4];      // lambda = |new - old| / max(new, old): the sample's, then after each of the
                       // filter's 3 passes (-1: none)
};
// each tile's gradient sample traced in the scene of P (P.seed: the old image's), lam[0] set
cudaError_t pt_gradients(const PtScene &S, const PtParams &P, GradTile *d_tiles, uint32_t ntiles, const float4 *d_guide,
                         unsigned long long *d_rays, uint32_t *d_status, cudaStream_t st);
cudaError_t pt_prim_boxes(const float *d_prims, uint32_t n, float *d_boxes, cudaStream_t st);
cudaError_t pt_trace(const PtScene &S, const PtParams &P, float *d_accum, unsigned long long *d_rays, uint32_t *d_status,
                     cudaStream_t st);
cudaError_t pt_intersect(const PtScene &S, const float *d_orig, const float *d_dir, uint64_t n, float tmin, float tmax,
                         int32_t *d_prim, int32_t *d_inst, float *d_t, uint32_t *d_status, cudaStream_t st);
// light tracing (caustics.cu): `photons` light paths (P's camera, image size, max_depth and exact
// mode) whose 32.32 contributions are added into d_sums (W x H x 3); and image += sums / 2^32
// (d_next: 8 bytes of scratch for the stream counter; variant: the launch's register cap, -1 the
// default, lt_variants() of them)
cudaError_t lt_trace(const PtScene &S, const PtParams &P, unsigned long long photons, uint64_t seed,
                     unsigned long long *d_sums, unsigned long long *d_next, unsigned long long *d_rays,
                     uint32_t *d_status, int num_sms, int variant, cudaStream_t st);
int lt_variants();
cudaError_t lt_resolve(const unsigned long long *d_sums, float *d_image, size_t n, int num_sms, cudaStream_t st);
// the denoiser (denoise.cu): the guide planes 2 and 3 of an image (W x H: P's whole image), and
// the denoised image from planes 0-3 (passes a-trous passes; scratch of dn_scratch_bytes)
cudaError_t dn_guide(const PtScene &S, const PtParams &P, float4 *d_planes, uint32_t *d_status, cudaStream_t st);
size_t dn_scratch_bytes(int W, int H);
cudaError_t dn_denoise(const float4 *d_planes, int W, int H, int passes, float4 *d_out, void *scratch,
                       cudaStream_t st);
cudaError_t pt_inst_boxes(const float *d_rec, uint32_t n, float *d_boxes, cudaStream_t st);

// One job of a batch: a band of one image of one scene. Its tasks are (pixel, lane slot) pairs,
// task0 + p * group + s for pixel p of the band (row-major) and slot s < group; slot s traces
// samples spp0 + s, spp0 + s + group, ... as lane s of the plain fast kernel does, and leaves
// its sum and sample count in partial[] and its ray count in prays[]. The resolve pass then adds
// each pixel's slots in the fast kernel's fixed tree order into accum, so a batched image is the
// plain one to the bit. Exact jobs have group 1 and the per-pixel stream of trace_image.
struct BatchJob {
    PtScene S;
    PtParams P;
    unsigned long long task0, ntasks;   // the job's first task in the batch, its tasks (pixels x group)
    unsigned long long pix0;            // its first pixel among all the batch's bands (resolve pass)
    float4 *partial;                    // ntasks (sum rgb, samples)
    uint32_t *prays;                    // ntasks ray counts
    float4 *pmom;                       // ntasks (sum l, sum l^2, the last sample's l, 0) (a guided job), or null
    float4 *accum;                      // the image (W x H)
    unsigned long long *rays;           // the job's ray count (added to)
};
// the persistent trace kernel over the batch's tasks [0, ntasks) in job order (launch shape
// `variant`, grid blocks), then the resolve pass over its npix pixels
cudaError_t batch_trace(const BatchJob *d_jobs, uint32_t njobs, unsigned long long ntasks, unsigned long long *d_next,
                        uint32_t *d_status, int variant, int grid, bool media, cudaStream_t st);
cudaError_t batch_resolve(const BatchJob *d_jobs, uint32_t njobs, unsigned long long npix, cudaStream_t st);
// the same with the job and pixel counts read from a run block in device memory (run[1], run[3])
cudaError_t batch_resolve_run(const BatchJob *d_jobs, const unsigned long long *d_run, int num_sms, cudaStream_t st);
// the launch shapes: how many; a shape's threads per block, the blocks per SM its registers are
// capped for, and the blocks of it that fit on one SM (-1: no such shape)
int batch_variants();
int batch_variant_shape(int variant, int *block, int *minb);

// The wavefront batch's paths in flight: M slots, each holding one task and the path of its current
// sample between the kernels of a bounce (advance, closest hit, shade, shadow rays). Arrays of M
// (vis: 2M) in structure-of-arrays order, so that a warp's slots are read in whole sectors.
struct WfState {
    uint32_t M;
    unsigned long long *task;   // the slot's task (~0: none)
    uint32_t *job;              // its job (queue order)
    uint32_t *kk;               // the sample it traces (the Sampler's index)
    uint32_t *trays;            // rays traced for the task so far
    uint32_t *flags;            // F_PATH, F_ENDED and the Nee flags of the bounce just shaded
    uint2 *xy;                  // the task's pixel
    float4 *sum;                // the task's sum so far (rgb, samples)
    float4 *mom;                // its luminance moments so far and its last sample's (guided jobs)
    float4 *ro;                 // the path's ray origin, bounce_pdf
    float4 *rd;                 // its direction, depth | emit << 16 | caus << 24 (int bits)
    float4 *thr;                // its throughput
    float4 *rad;                // its radiance so far
    ulonglong2 *rng;            // its Rng (state, inc)
    float4 *hit;                // the closest hit: t, world shape, instance, instance triangle (int bits)
    float4 *nthr, *nvl, *nve;   // the bounce's next event estimation: throughput, lamp and sky values
    uint8_t *vis;               // 2 per slot: the lamp's / the sky's shadow ray unoccluded
    uint32_t *rq;               // the ray queue: slots with a path (M)
    float4 *sq_o, *sq_d;        // the shadow queue (2M): origin + (slot << 1 | kind) bits, direction + tmax
    uint32_t *ctl;              // [0] rays queued, [1] shadow rays queued, [2] [3] their fetch counters, [4] passes
    unsigned long long *next;   // the task queue's next task; next[1]: how many tasks this run takes
    unsigned long long *run;    // the run: [0] its tasks, [1] jobs, [2] largest pass count, [3] pixels
                                // (written before each run, so that one captured graph serves every run)
};
// the device bytes of a wavefront of M slots, and its arrays carved from them (256-byte aligned base)
size_t wf_bytes(uint32_t M);
WfState wf_carve(void *base, uint32_t M);
// the wavefront's trace shapes (closest-hit and shadow kernels: threads per block, register-cap
// blocks per SM, blocks per SM that fit): how many; -1 for none
int wf_variants();
int wf_variant_shape(int variant, int *block, int *minb);
// Captures the wavefront's loop into the graph stream st is capturing: the slots cleared and the
// task queue set to the run block's tasks (W.run[0]), then a while node whose body (captured on
// body_st) runs the advance, closest-hit, shade and shadow kernels until no slot holds a path.
// instances: some job's scene has instances (else the traversal kernels without the two-level
// walk run). The loop stops after W.run[2] passes whatever is left (ST_LOOP in the status word): a
// bound well above what the tasks need (a pass per bounce of each slot's tasks). Nothing of the
// run (its jobs, tasks, bounds) is in the graph: one capture serves every run of the same buffers.
// The run block's four words (tasks, jobs, largest pass count, pixels) from host memory, on st.
cudaError_t wf_set_run(const WfState &W, const unsigned long long *h_run4, cudaStream_t st);
cudaError_t wf_capture_loop(const BatchJob *d_jobs, const WfState &W, uint32_t *d_status, int variant, bool instances,
                            int num_sms, cudaStream_t st, cudaStream_t body_st);
// The same loop with each pass's kernels launched from the host (no graph; the host reads the
// queued count after every pass): for profilers that cannot see into a graph's loop.
// a stepped run's measurements (stats given): the closest-hit kernel's time (CUDA events around each
// launch), the rays it traced, its launches, all kernels launched, and (count, with variant 0's
// shape, whose counting build it then runs) the box and triangle tests of its walks
struct WfStepStats {
    double isect_ms;
    unsigned long long isect_rays, isect_launches, launches, box_tests, tri_tests;
};
cudaError_t wf_run_stepped(const BatchJob *d_jobs, uint32_t njobs, unsigned long long ntasks, const WfState &W,
                           uint32_t *d_status, int variant, bool instances, int num_sms, uint32_t max_passes,
                           cudaStream_t st, WfStepStats *stats = nullptr, bool count = false);
// the sky's sampling tables as env_prepare makes them (host_tables.cu): marg h + 1, cond h x (w + 1),
// prob w x h; returns false when no pixel weighs anything (sum 0)
bool env_tables(const float *rgb, int w, int h, float *marg, float *cond, float *prob);
// min / max over n boxes (8 floats each) into the bound keys (6 words; as triangle_boxes's)
cudaError_t boxes_bounds(const float *d_boxes, uint32_t n, uint32_t *d_bkeys, cudaStream_t st, int num_sms, bool init);

// the defaults of what the caller may give (host_tables.cu)
void default_blue_noise(uint16_t *out);
void default_bsdf_tables(float *out);

}  // namespace lrc
