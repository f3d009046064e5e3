// batch.cu - many render jobs (scene, image band, samples) built and traced together.
//
// The reference renders one scene at a time: its band scheduler (engine/gpu/view_gpu.c:1081-1190,
// gpu_view_trace_more) sizes each submit from the measured time of a pass, and every submit is a
// dispatch of the megakernel over one image. A batch instead holds any number of jobs over any
// number of resident scenes, and runs them as one queue of (pixel, lane slot) tasks drained by one
// persistent kernel (pathtrace.cu batch_kernel): the jobs are ordered by the samples a task
// carries, most first, so the cheap tasks fill the end (longest-processing-time order), and the
// resolve pass adds every pixel into its image in the plain kernel's order, so a batched image is
// the plain one to the bit.
//
// A run may first rebuild the jobs' scenes (LBVH or PLOC), and may be replayed as one CUDA graph:
// builds, the counters' reset, the trace kernel and the resolve pass, captured once after a run
// that sized every buffer. The graph is captured again when a scene's buffers or sizes changed.
//
// The project's autotuner (lrc_batch_tune) picks the trace kernel's launch shape - threads per
// block, the register cap and so the paths each SM keeps in flight - by timing each shape on the
// same prefix of the queue: the measured ms per task, as the band scheduler uses its measured ms
// per pass.
#include "api_internal.cuh"
#include <algorithm>
#include <cstddef>
#include <cstring>
#include <new>
#include <numeric>
#include <vector>

using namespace lrcapi;

struct lrc_batch {
    struct Job {
        lrc_scene *s;
        lrc_trace_params p;
        int32_t y0, rows;
        uint32_t spp0, spp;
        float *accum;
        int32_t builder, key_bits;
        InstView view;                    // the job's own instances (moved), or none: the scene's
        bool guided = false;              // accum holds the denoiser's 4 planes (moments added)
    };
    lrc_ctx *ctx = nullptr;
    std::vector<Job> jobs;
    // the device side of the last prepared run
    lrc::BatchJob *d_jobs = nullptr;
    size_t jobs_cap = 0;
    void *d_part = nullptr;               // partial sums, then ray counts, of every task
    size_t part_cap = 0;
    unsigned long long *d_ctr = nullptr;  // [0] the queue's next task, [1 + j] job j's rays
    size_t ctr_cap = 0;
    void *scratch = nullptr;              // the builds' scratch arena
    size_t scratch_cap = 0;
    std::vector<lrc::BatchJob> table;     // in queue order
    std::vector<uint32_t> order;          // queue position -> job index
    unsigned long long ntasks = 0, npix = 0;
    bool prepared = false;
    // the engine: 0 the persistent megakernel (launch shape variant, grid blocks), 1 the wavefront
    // (wf_slots paths in flight, closest-hit / shadow kernels' shape wf_variant); tuned or set
    int engine = 1;
    int variant = 0, grid = 0;
    int wf_variant = LRC_WAVEFRONT_DEFAULT_VARIANT;
    uint32_t wf_slots = 1u << 20;
    void *d_wf = nullptr;
    size_t wf_cap = 0;
    cudaStream_t body = nullptr;          // the stream the wavefront loop's body is captured on
    // the graph of the last GRAPH run and what it was captured for
    lrc::WfStepStats step_stats{};        // the last STEPPED run's measurements
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    unsigned graph_flags = 0;
    std::vector<unsigned char> graph_sig;
    // the wavefront's graph captured before the current one, kept: runs that alternate between two
    // keys (a server's waves with and without instanced jobs) replay both, capturing neither again
    cudaGraph_t alt_graph = nullptr;
    cudaGraphExec_t alt_exec = nullptr;
    unsigned alt_flags = 0;
    std::vector<unsigned char> alt_sig;
    int graph_used = 0;
    cudaEvent_t ev_launch = nullptr;      // recorded right before a run's trace is launched (the server's wave timing)
    lrc::BatchJob *h_table = nullptr;     // pinned staging of the job table's upload (and the run block after it)
    size_t h_table_cap = 0;
    cudaEvent_t ev_table = nullptr;       // the last upload from it done (it may be written again)
};

namespace {

constexpr unsigned kBatchFlags = LRC_BATCH_BUILD | LRC_BATCH_GRAPH | LRC_BATCH_ZERO | LRC_BATCH_STEPPED | LRC_BATCH_COUNT;

int group_for(const lrc_trace_params &p, uint32_t spp) {
    if (p.exact) return 1;
    int g = 1;
    while (g * 2 <= (int)spp && g < 16) g *= 2;   // as lrc_trace: lanes per pixel, a power of 2 <= spp, <= 16
    return g;
}

lrc::PtParams params_of(const lrc_batch::Job &J) {
    lrc::PtParams P{};
    const lrc_trace_params *p = &J.p;
    P.W = p->width; P.H = p->height; P.y0 = J.y0; P.rows = J.rows; P.spp0 = (int)J.spp0; P.spp = (int)J.spp;
    P.max_depth = p->max_depth; P.mis = p->mis; P.sampler_on = p->sampler; P.exact = p->exact;
    P.group = group_for(*p, J.spp);
    P.seed = p->seed;
    P.clamp = p->clamp;
    P.skip_caustics = p->skip_caustics != 0;
    P.indirect_clamp = p->indirect_clamp;
    if (J.guided) {
        const size_t N = (size_t)p->width * p->height;
        P.moments = reinterpret_cast<float4 *>(J.accum) + N;
        P.guide = reinterpret_cast<const float4 *>(J.accum) + 3 * N;
    }
    P.origin = {p->origin[0], p->origin[1], p->origin[2]};
    P.upper_left = {p->upper_left[0], p->upper_left[1], p->upper_left[2]};
    P.horizontal = {p->horizontal[0], p->horizontal[1], p->horizontal[2]};
    P.vertical = {p->vertical[0], p->vertical[1], p->vertical[2]};
    return P;
}

// the current graph dropped (the kept one stays)
void drop_graph(lrc_batch *b) {
    if (b->exec) cudaGraphExecDestroy(b->exec);
    if (b->graph) cudaGraphDestroy(b->graph);
    b->exec = nullptr;
    b->graph = nullptr;
    b->graph_sig.clear();
}

// both graphs dropped (their buffers may move)
void destroy_graph(lrc_batch *b) {
    drop_graph(b);
    if (b->alt_exec) cudaGraphExecDestroy(b->alt_exec);
    if (b->alt_graph) cudaGraphDestroy(b->alt_graph);
    b->alt_exec = nullptr;
    b->alt_graph = nullptr;
    b->alt_sig.clear();
}

// the current graph and the kept one trade places
void swap_graphs(lrc_batch *b) {
    std::swap(b->graph, b->alt_graph);
    std::swap(b->exec, b->alt_exec);
    std::swap(b->graph_flags, b->alt_flags);
    b->graph_sig.swap(b->alt_sig);
}

// the path tracer's view of a job's scene once the run's builds are done (a build makes the tree
// over all its shapes)
lrc::PtScene view_of(const lrc_batch::Job &J, bool building) {
    lrc::PtScene S = pt_scene(J.s);
    if (J.view.inst) {
        S.inst = reinterpret_cast<const float4 *>(J.view.inst);
        S.tlas_nodes = reinterpret_cast<const float4 *>(J.view.tlas_nodes);
        S.tlas_aux = J.view.tlas_aux;
    }
    if (building && J.builder >= 0) {
        const uint32_t n = J.s->ntris + J.s->nprims;
        S.nnodes = n ? 2 * n - 1 : 0;
        S.naux = n;
    }
    return S;
}

// what a captured run depends on: every job's scene view and build buffers, its band and image
std::vector<unsigned char> signature(const lrc_batch *b, unsigned flags) {
    std::vector<unsigned char> sig;
    auto put = [&](const void *p, size_t n) {
        const unsigned char *c = static_cast<const unsigned char *>(p);
        sig.insert(sig.end(), c, c + n);
    };
    put(&flags, sizeof flags);
    for (const lrc_batch::Job &J : b->jobs) {
        lrc::PtScene S = view_of(J, (flags & LRC_BATCH_BUILD) != 0);
        put(&S, sizeof S);
        const void *bufs[4] = {J.s->d_boxes, J.s->d_small, J.s->d_nodes, J.s->d_aux};
        put(bufs, sizeof bufs);
        const void *ptrs[2] = {J.s, J.accum};
        put(ptrs, sizeof ptrs);
        put(&J.p, offsetof(lrc_trace_params, skip_caustics) + sizeof(int32_t));
        put(&J.guided, sizeof J.guided);
        const int32_t w[6] = {J.y0, J.rows, (int32_t)J.spp0, (int32_t)J.spp, J.builder, J.key_bits};
        put(w, sizeof w);
    }
    const void *own[5] = {b->scratch, b->d_jobs, b->d_part, b->d_ctr, b->d_wf};
    put(own, sizeof own);
    const int shape[5] = {b->engine, b->variant, b->grid, b->wf_variant, (int)b->wf_slots};
    put(shape, sizeof shape);
    return sig;
}

int check_job(lrc_ctx *c, const lrc_batch::Job &J, bool will_build) {
    lrc_scene *s = J.s;
    if (!will_build || J.builder < 0) {
        if (!s->built_n && !s->tlas_n) return fail(c, LRC_E_INVALID, "a job's scene has nothing built");
    } else if (!s->ntris && !s->nprims) {
        return fail(c, LRC_E_INVALID, "a job's scene has nothing to build");
    }
    if (s->ninst && s->tlas_n != s->ninst) return fail(c, LRC_E_INVALID, "a job's instances changed: lrc_scene_build_instances");
    if (!s->d_mats || !s->nmats) return fail(c, LRC_E_INVALID, "a job's scene has no materials");
    if (s->light >= (int32_t)s->nprims) return fail(c, LRC_E_INVALID, "a job's light is not one of its primitives");
    return LRC_OK;
}

// the distinct scenes the run builds, each with its first job's builder and key bits
std::vector<const lrc_batch::Job *> builds_of(const lrc_batch *b) {
    std::vector<const lrc_batch::Job *> out;
    for (const lrc_batch::Job &J : b->jobs) {
        if (J.builder < 0) continue;
        bool seen = false;
        for (const lrc_batch::Job *o : out) seen = seen || o->s == J.s;
        if (!seen) out.push_back(&J);
    }
    return out;
}

// the job's scene built: builder 0 LBVH, 1 PLOC, 2 LBVH and then PLOC (the PLOC tree is kept)
int build_job(lrc_batch *b, const lrc_batch::Job *J, cudaStream_t st, bool capturing) {
    const int first = J->builder == 2 ? 0 : J->builder;
    int rc = scene_build_on(J->s, first, J->key_bits, &b->scratch, &b->scratch_cap, st, nullptr, capturing);
    if (!rc && J->builder == 2) rc = scene_build_on(J->s, 1, J->key_bits, &b->scratch, &b->scratch_cap, st, nullptr, capturing);
    return rc;
}

uint32_t max_passes(const lrc_batch *b, unsigned long long limit);

// the job table in queue order, the partial buffers and counters sized, the table uploaded; with
// building, each job's scene as the run's builds leave it (its triangles may have been set again
// since the last build, and builds inside a replayed graph are recorded only after the launch)
int prepare(lrc_batch *b, bool building) {
    lrc_ctx *c = b->ctx;
    const size_t nj = b->jobs.size();
    b->order.resize(nj);
    std::iota(b->order.begin(), b->order.end(), 0u);
    // longest-processing-time order: samples per task, then pixels, most first
    std::stable_sort(b->order.begin(), b->order.end(), [&](uint32_t x, uint32_t y) {
        const lrc_batch::Job &A = b->jobs[x], &B = b->jobs[y];
        const double sa = (double)A.spp / group_for(A.p, A.spp), sb = (double)B.spp / group_for(B.p, B.spp);
        if (sa != sb) return sa > sb;
        return (uint64_t)A.p.width * A.rows > (uint64_t)B.p.width * B.rows;
    });
    b->table.assign(nj, lrc::BatchJob{});
    unsigned long long task = 0, pix = 0;
    for (size_t q = 0; q < nj; q++) {
        const lrc_batch::Job &J = b->jobs[b->order[q]];
        lrc::BatchJob &T = b->table[q];
        T.S = view_of(J, building);
        T.P = params_of(J);
        T.task0 = task;
        T.pix0 = pix;
        const unsigned long long np = (unsigned long long)J.p.width * J.rows;
        T.ntasks = np * T.P.group;
        task += T.ntasks;
        pix += np;
        T.accum = reinterpret_cast<float4 *>(J.accum);
    }
    b->ntasks = task;
    b->npix = pix;
    cudaError_t e = reserve(&b->d_part, &b->part_cap, al(task * 16) + al(task * 4) + al(task * 16) + 256);
    if (!e) e = reserve(reinterpret_cast<void **>(&b->d_ctr), &b->ctr_cap, (nj + 1) * 8 + 256);
    if (!e) e = reserve(reinterpret_cast<void **>(&b->d_jobs), &b->jobs_cap, nj * sizeof(lrc::BatchJob) + 256);
    if (!e && b->engine == 1) e = reserve(&b->d_wf, &b->wf_cap, lrc::wf_bytes(b->wf_slots));
    if (!e && b->engine == 1 && !b->body) e = cudaStreamCreateWithFlags(&b->body, cudaStreamNonBlocking);
    if (e) return cuda_status(c, e, "batch memory");
    char *part = static_cast<char *>(b->d_part);
    float4 *partial = reinterpret_cast<float4 *>(part);
    uint32_t *prays = reinterpret_cast<uint32_t *>(part + al(task * 16));
    float4 *pmom = reinterpret_cast<float4 *>(part + al(task * 16) + al(task * 4));
    for (size_t q = 0; q < nj; q++) {
        lrc::BatchJob &T = b->table[q];
        T.partial = partial + T.task0;
        T.prays = prays + T.task0;
        T.pmom = T.P.moments ? pmom + T.task0 : nullptr;
        T.rays = b->d_ctr + 1 + b->order[q];
    }
    // the table uploaded from pinned staging, without waiting for the stream: work queued before
    // (another run still on the device) goes on; the staging is written again only once the copy
    // from it is done
    if (b->ev_table) e = cudaEventSynchronize(b->ev_table);
    else e = cudaEventCreateWithFlags(&b->ev_table, cudaEventDisableTiming);
    if (!e && b->h_table_cap < nj + 1) {                // (+1: the wavefront's run block)
        if (b->h_table) cudaFreeHost(b->h_table);
        b->h_table = nullptr;
        b->h_table_cap = 0;
        e = cudaMallocHost(reinterpret_cast<void **>(&b->h_table), (nj + nj / 4 + 16) * sizeof(lrc::BatchJob));
        if (!e) b->h_table_cap = nj + nj / 4 + 16;
    }
    if (!e) {
        std::copy(b->table.begin(), b->table.end(), b->h_table);
        e = cudaMemcpyAsync(b->d_jobs, b->h_table, nj * sizeof(lrc::BatchJob), cudaMemcpyHostToDevice, c->st);
    }
    if (!e && b->engine == 1) {                         // the run block: tasks, jobs, pass bound, pixels
        unsigned long long *run = reinterpret_cast<unsigned long long *>(b->h_table + nj);
        run[0] = b->ntasks;
        run[1] = nj;
        run[2] = max_passes(b, b->ntasks);
        run[3] = b->npix;
        e = lrc::wf_set_run(lrc::wf_carve(b->d_wf, b->wf_slots), run, c->st);
    }
    if (!e) e = cudaEventRecord(b->ev_table, c->st);
    if (e) return cuda_status(c, e, "batch table");
    if (b->grid <= 0) {
        int block = 0, minb = 0;
        int per_sm = lrc::batch_variant_shape(b->variant, &block, &minb);
        b->grid = std::max(per_sm, 1) * c->num_sms;
    }
    b->prepared = true;
    return LRC_OK;
}

// whether some job's scene has participating media (the megakernel with their tracking then runs)
bool any_media(const lrc_batch *b) {
    for (const lrc::BatchJob &T : b->table)
        if (T.S.nvol) return true;
    return false;
}

// whether some job's scene has instances (the traversal kernels then walk two levels)
bool any_instances(const lrc_batch *b) {
    for (const lrc::BatchJob &T : b->table)
        if (T.S.ninst) return true;
    return false;
}

// a bound on the wavefront's passes for the first `limit` tasks: each slot runs at most
// ceil(limit / slots) tasks one after another, each of at most (samples a task holds) paths of at
// most max_depth + 1 bounces, plus one pass to start and one to end each task
uint32_t max_passes(const lrc_batch *b, unsigned long long limit) {
    unsigned long long per_task = 1, depth = 1;
    for (const lrc_batch::Job &J : b->jobs) {
        const int g = group_for(J.p, J.spp);
        per_task = std::max<unsigned long long>(per_task, (J.spp + g - 1) / g);
        depth = std::max<unsigned long long>(depth, (unsigned long long)J.p.max_depth + 1);
    }
    const unsigned long long rounds = (limit + b->wf_slots - 1) / b->wf_slots + 1;
    const unsigned long long bound = rounds * (per_task * (depth + 1) + 2) + 16;
    return (uint32_t)std::min<unsigned long long>(bound, 0xffffffffull);
}

// the run's device work on stream st: builds (with_builds), resets, trace, resolve (with_resolve;
// without it nothing but the per-task sums is written: the autotuner's runs). The wavefront's loop
// can only be captured (st capturing).
int enqueue(lrc_batch *b, unsigned flags, cudaStream_t st, bool capturing, bool with_builds, bool with_resolve,
            unsigned long long limit) {
    lrc_ctx *c = b->ctx;
    if (with_builds && (flags & LRC_BATCH_BUILD)) {
        for (const lrc_batch::Job *J : builds_of(b)) {
            int rc = build_job(b, J, st, capturing);
            if (rc) return rc;
        }
    }
    const size_t nj = b->jobs.size();
    // (a captured wavefront run depends on the buffers alone: the counters cleared whole, the bands
    // zeroed before its launch, its counts in the run block)
    const bool wf_graph = b->engine == 1 && capturing;
    cudaError_t e = with_resolve ? cudaMemsetAsync(b->d_ctr, 0, wf_graph ? b->ctr_cap : (nj + 1) * 8, st) : cudaSuccess;
    if (!e && with_resolve && (flags & LRC_BATCH_ZERO) && !wf_graph) {
        for (size_t i = 0; i < nj && !e; i++) {
            const lrc_batch::Job &J = b->jobs[i];
            e = cudaMemsetAsync(J.accum + (size_t)J.y0 * J.p.width * 4, 0, (size_t)J.rows * J.p.width * 16, st);
            if (!e && J.guided)                      // the band's moments (plane 1) too
                e = cudaMemsetAsync(J.accum + ((size_t)J.p.width * J.p.height + (size_t)J.y0 * J.p.width) * 4, 0,
                                    (size_t)J.rows * J.p.width * 16, st);
        }
    }
    if (!e && b->engine == 0)
        e = lrc::batch_trace(b->d_jobs, (uint32_t)nj, limit, b->d_ctr, c->d_status, b->variant, b->grid, any_media(b), st);
    if (!e && b->engine == 1 && !capturing && (flags & LRC_BATCH_STEPPED)) {
        const lrc::WfState W = lrc::wf_carve(b->d_wf, b->wf_slots);
        e = lrc::wf_run_stepped(b->d_jobs, (uint32_t)nj, limit, W, c->d_status, b->wf_variant, any_instances(b),
                                c->num_sms, max_passes(b, limit), st, &b->step_stats, (flags & LRC_BATCH_COUNT) != 0);
    } else if (!e && b->engine == 1) {
        if (!capturing) return fail(c, LRC_E_INVALID, "the wavefront runs as a captured graph");
        const lrc::WfState W = lrc::wf_carve(b->d_wf, b->wf_slots);
        e = lrc::wf_capture_loop(b->d_jobs, W, c->d_status, b->wf_variant, any_instances(b), c->num_sms, st, b->body);
    }
    if (!e && with_resolve)
        e = wf_graph ? lrc::batch_resolve_run(b->d_jobs, lrc::wf_carve(b->d_wf, b->wf_slots).run, c->num_sms, st)
                     : lrc::batch_resolve(b->d_jobs, (uint32_t)nj, b->npix, st);
    if (e) return cuda_status(c, e, "batch run");
    return LRC_OK;
}

// captures enqueue(...) into a new executable graph
int capture_exec(lrc_batch *b, unsigned flags, bool with_builds, bool with_resolve, unsigned long long limit,
                 cudaGraph_t *g_out, cudaGraphExec_t *x_out) {
    lrc_ctx *c = b->ctx;
    *g_out = nullptr;
    *x_out = nullptr;
    cudaError_t e = cudaStreamBeginCapture(c->st, cudaStreamCaptureModeThreadLocal);
    if (e) return cuda_status(c, e, "batch graph capture");
    int rc = enqueue(b, flags, c->st, true, with_builds, with_resolve, limit);
    cudaGraph_t g = nullptr;
    e = cudaStreamEndCapture(c->st, &g);
    if (rc || e) {
        if (g) cudaGraphDestroy(g);
        cudaGetLastError();
        return rc ? rc : cuda_status(c, e, "batch graph capture");
    }
    e = cudaGraphInstantiate(x_out, g, 0);
    if (e) {
        cudaGraphDestroy(g);
        return cuda_status(c, e, "batch graph instantiate");
    }
    *g_out = g;
    return LRC_OK;
}

// the run's graph, kept for replays: builds inside when GRAPH (the megakernel engine captures only
// GRAPH runs; the wavefront's trace is always a graph, its builds plain launches without GRAPH)
int capture(lrc_batch *b, unsigned flags, const std::vector<unsigned char> &key) {
    drop_graph(b);
    int rc = capture_exec(b, flags, (flags & LRC_BATCH_GRAPH) != 0, true, b->ntasks, &b->graph, &b->exec);
    if (rc) return rc;
    b->graph_flags = flags;
    b->graph_sig = key;
    return LRC_OK;
}

// what a captured wavefront run without builds depends on: its buffers and shape (the jobs, tasks
// and bounds travel in the table and the run block); with builds, every job (signature)
std::vector<unsigned char> graph_key(const lrc_batch *b, unsigned flags) {
    if (b->engine != 1 || ((flags & LRC_BATCH_BUILD) && (flags & LRC_BATCH_GRAPH))) return signature(b, flags);
    std::vector<unsigned char> k;
    auto put = [&](const void *p, size_t n) {
        const unsigned char *c = static_cast<const unsigned char *>(p);
        k.insert(k.end(), c, c + n);
    };
    const unsigned f = flags & ~LRC_BATCH_ZERO;
    const void *bufs[5] = {b->d_jobs, b->d_ctr, b->d_wf, b->body, b->ctx->d_status};
    const unsigned long long sizes[2] = {b->ctr_cap, b->wf_slots};
    const int shape[3] = {b->wf_variant, any_instances(b) ? 1 : 0, b->ctx->num_sms};
    put(&f, sizeof f);
    put(bufs, sizeof bufs);
    put(sizes, sizeof sizes);
    put(shape, sizeof shape);
    return k;
}

// the wavefront's autotuner: the time of the first n tasks at each wavefront size (paths in
// flight), then at each closest-hit / shadow launch shape at the best size; keeps the fastest
int tune_wavefront(lrc_batch *b, unsigned long long n, int32_t *variant, int32_t *slots, double *ns_per_task) {
    lrc_ctx *c = b->ctx;
    const uint32_t sizes[] = {1u << 18, 1u << 19, 1u << 20, 1u << 21, 1u << 22, 1u << 23};
    uint32_t top = 1u << 18;
    for (uint32_t m : sizes)
        if ((unsigned long long)m / 2 < n) top = m;   // (no larger than the tasks need)
    cudaError_t e = reserve(&b->d_wf, &b->wf_cap, lrc::wf_bytes(top));
    if (!e && !b->body) e = cudaStreamCreateWithFlags(&b->body, cudaStreamNonBlocking);
    if (e) return cuda_status(c, e, "batch tune memory");
    destroy_graph(b);                                // (its buffers may move)
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    const int keep_v = b->wf_variant;
    const uint32_t keep_m = b->wf_slots;
    auto time_one = [&](uint32_t m, int v, float &ms) -> int {
        b->wf_slots = m;
        b->wf_variant = v;
        // (the run block at this size's place: the first n tasks)
        const unsigned long long run[4] = {n, b->jobs.size(), max_passes(b, n), b->npix};
        cudaError_t er = lrc::wf_set_run(lrc::wf_carve(b->d_wf, m), run, c->st);
        if (er) return cuda_status(c, er, "batch tune");
        cudaGraph_t g;
        cudaGraphExec_t x;
        int rc = capture_exec(b, 0, false, false, n, &g, &x);
        if (rc) return rc;
        cudaError_t err = cudaSuccess;
        for (int rep = 0; rep < 2 && !err; rep++) {   // (the first run pays the kernels' module load)
            err = cudaEventRecord(e0, c->st);
            if (!err) err = cudaGraphLaunch(x, c->st);
            if (!err) err = cudaEventRecord(e1, c->st);
            if (!err) err = cudaEventSynchronize(e1);
            if (!err) err = cudaEventElapsedTime(&ms, e0, e1);
        }
        cudaGraphExecDestroy(x);
        cudaGraphDestroy(g);
        return err ? cuda_status(c, err, "batch tune") : LRC_OK;
    };
    float best = 3e38f;
    uint32_t best_m = keep_m;
    int best_v = keep_v, rc = LRC_OK;
    for (uint32_t m : sizes) {
        if (m > top || rc) continue;
        float ms = 0;
        rc = time_one(m, keep_v, ms);
        if (!rc && ms < best) {
            best = ms;
            best_m = m;
        }
    }
    for (int v = 0; v < lrc::wf_variants() && !rc; v++) {
        if (v == keep_v) continue;
        float ms = 0;
        rc = time_one(best_m, v, ms);
        if (!rc && ms < best) {
            best = ms;
            best_v = v;
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    b->wf_slots = rc ? keep_m : best_m;
    b->wf_variant = rc ? keep_v : best_v;
    if (rc) return rc;
    rc = check_status(c);
    if (rc) return rc;
    if (variant) *variant = best_v;
    if (slots) *slots = (int32_t)best_m;
    if (ns_per_task) *ns_per_task = best * 1e6 / (double)n;
    return LRC_OK;
}

void note_built(lrc_batch *b) {   // (what captured builds' host side records)
    for (const lrc_batch::Job *J : builds_of(b)) J->s->built_n = J->s->ntris + J->s->nprims;
}

}  // namespace

namespace lrcapi {
void batch_set_launch_event(lrc_batch *b, cudaEvent_t e) { b->ev_launch = e; }

int batch_reserve(lrc_batch *b, unsigned long long tasks, size_t jobs) {
    lrc_ctx *c = b->ctx;
    DeviceGuard g(c->device);
    cudaError_t e = reserve(&b->d_part, &b->part_cap, al(tasks * 16) + al(tasks * 4) + al(tasks * 16) + 256);
    if (!e) e = reserve(reinterpret_cast<void **>(&b->d_ctr), &b->ctr_cap, (jobs + 1) * 8 + 256);
    if (!e) e = reserve(reinterpret_cast<void **>(&b->d_jobs), &b->jobs_cap, jobs * sizeof(lrc::BatchJob) + 256);
    if (!e && b->engine == 1) e = reserve(&b->d_wf, &b->wf_cap, lrc::wf_bytes(b->wf_slots));
    if (!e && b->h_table_cap < jobs + 1) {
        if (b->h_table) cudaFreeHost(b->h_table);
        b->h_table = nullptr;
        b->h_table_cap = 0;
        e = cudaMallocHost(reinterpret_cast<void **>(&b->h_table), (jobs + 16) * sizeof(lrc::BatchJob));
        if (!e) b->h_table_cap = jobs + 16;
    }
    return e ? cuda_status(c, e, "batch reserve") : LRC_OK;
}

cudaError_t batch_counts_async(lrc_batch *b, unsigned long long *h_rays, uint32_t *h_passes) {
    lrc_ctx *c = b->ctx;
    const size_t nj = b->jobs.size();
    cudaError_t e = cudaSuccess;
    if (nj && b->prepared) e = cudaMemcpyAsync(h_rays, b->d_ctr + 1, nj * 8, cudaMemcpyDeviceToHost, c->st);
    *h_passes = 0;
    if (!e && b->prepared && b->engine == 1 && b->d_wf) {
        const lrc::WfState W = lrc::wf_carve(b->d_wf, b->wf_slots);
        e = cudaMemcpyAsync(h_passes, W.ctl + 4, 4, cudaMemcpyDeviceToHost, c->st);
    }
    return e;
}

int batch_add_view(lrc_batch *b, lrc_scene *s, const lrc_trace_params *p, int32_t y0, int32_t rows, uint32_t spp0,
                   uint32_t spp, float *d_accum, const InstView &view, bool guided) {
    int rc = lrc_batch_add(b, s, p, y0, rows, spp0, spp, d_accum, -1, 30);
    if (rc) return rc;
    if (view.inst && !s->tlas_n) {
        b->jobs.pop_back();
        return fail(b->ctx, LRC_E_INVALID, "own instances for a scene without instances");
    }
    b->jobs.back().view = view;
    b->jobs.back().guided = guided;
    return LRC_OK;
}
}  // namespace lrcapi

extern "C" {

int lrc_batch_create(lrc_ctx *c, lrc_batch **out) {
    if (!c || !out) return LRC_E_INVALID;
    *out = nullptr;
    lrc_batch *b = new (std::nothrow) lrc_batch;
    if (!b) return LRC_RETRY;
    b->ctx = c;
    *out = b;
    return LRC_OK;
}

void lrc_batch_destroy(lrc_batch *b) {
    if (!b) return;
    DeviceGuard g(b->ctx->device);
    cudaStreamSynchronize(b->ctx->st);
    destroy_graph(b);
    cudaFree(b->d_jobs);
    cudaFree(b->d_part);
    cudaFree(b->d_ctr);
    cudaFree(b->scratch);
    cudaFree(b->d_wf);
    if (b->h_table) cudaFreeHost(b->h_table);
    if (b->ev_table) cudaEventDestroy(b->ev_table);
    if (b->body) cudaStreamDestroy(b->body);
    delete b;
}

int lrc_batch_add(lrc_batch *b, lrc_scene *s, const lrc_trace_params *p, int32_t y0, int32_t rows, uint32_t spp0,
                  uint32_t spp, float *d_accum, int32_t builder, int32_t key_bits) {
    if (!b || !s || !p || !d_accum || s->ctx != b->ctx) return LRC_E_INVALID;
    lrc_ctx *c = b->ctx;
    if (p->width <= 0 || p->height <= 0 || y0 < 0 || rows <= 0 || y0 + rows > p->height || spp == 0)
        return fail(c, LRC_E_INVALID, "a batch job needs a band of rows in the image and spp >= 1");
    if (p->exact && spp0 != 0) return fail(c, LRC_E_INVALID, "exact mode starts at each pixel's first sample (spp0 = 0)");
    if ((uint64_t)spp0 + spp >= (1ull << 31)) return fail(c, LRC_E_INVALID, "spp0 + spp must stay below 2^31");
    if (p->max_depth < 0 || p->max_depth > 0xffff) return fail(c, LRC_E_INVALID, "max_depth must be in [0, 65535]");
    if (builder < -1 || builder > 2) return fail(c, LRC_E_INVALID, "builder: -1 (none), 0 (LBVH), 1 (PLOC) or 2 (both)");
    if (builder >= 0 && key_bits != 30 && key_bits != 63) return fail(c, LRC_E_INVALID, "key_bits must be 30 or 63");
    if (s->ninst && builder >= 0) return fail(c, LRC_E_INVALID, "instanced scenes are built by lrc_scene_build_instances");
    b->jobs.push_back({s, *p, y0, rows, spp0, spp, d_accum, builder, key_bits, InstView{}});
    b->prepared = false;
    return LRC_OK;
}

int lrc_batch_add_guided(lrc_batch *b, lrc_scene *s, const lrc_trace_params *p, int32_t y0, int32_t rows,
                         uint32_t spp0, uint32_t spp, float *d_planes, int32_t builder, int32_t key_bits) {
    int rc = lrc_batch_add(b, s, p, y0, rows, spp0, spp, d_planes, builder, key_bits);
    if (rc) return rc;
    b->jobs.back().guided = true;
    return LRC_OK;
}

int lrc_batch_clear(lrc_batch *b) {
    if (!b) return LRC_E_INVALID;
    b->jobs.clear();
    b->prepared = false;
    return LRC_OK;
}

int lrc_batch_jobs(const lrc_batch *b) { return b ? (int)b->jobs.size() : 0; }

int lrc_batch_run(lrc_batch *b, unsigned flags) {
    if (!b || (flags & ~kBatchFlags)) return LRC_E_INVALID;
    if ((flags & LRC_BATCH_STEPPED) && (flags & LRC_BATCH_GRAPH)) return fail(b->ctx, LRC_E_INVALID, "STEPPED is not GRAPH");
    lrc_ctx *c = b->ctx;
    if (b->jobs.empty()) return LRC_OK;
    for (const lrc_batch::Job &J : b->jobs) {
        int rc = check_job(c, J, (flags & LRC_BATCH_BUILD) != 0);
        if (rc) return rc;
        // (the wavefront defers shadow rays, which a medium's transmittance cannot wait for: it
        // draws the path's random numbers only when the ray gets through)
        if (J.s->nvol && b->engine == 1)
            return fail(c, LRC_E_INVALID, "a scene with media runs on the batch's engine 0 (lrc_batch_set_engine)");
    }
    DeviceGuard g(c->device);
    for (lrc_batch::Job &J : b->jobs) {
        if (!J.s->tables) {
            int rc = lrc_scene_set_tables(J.s, nullptr, nullptr);
            if (rc) return rc;
        }
    }
    b->graph_used = 0;
    if (b->engine == 1 && (flags & LRC_BATCH_STEPPED)) {   // (plain launches, pass by pass)
        if (flags & LRC_BATCH_BUILD)
            for (const lrc_batch::Job *J : builds_of(b)) {
                int rc = build_job(b, J, c->st, false);
                if (rc) return rc;
            }
        int rc = prepare(b, (flags & LRC_BATCH_BUILD) != 0);
        if (!rc) rc = enqueue(b, flags, c->st, false, false, true, b->ntasks);
        return rc;
    }
    const bool cached = b->exec && b->prepared && b->graph_flags == flags && signature(b, flags) == b->graph_sig;
    if (b->engine == 1) {
        // The wavefront: the table and the run block uploaded every run (behind the work queued
        // before, not waiting for it); the graph captured again only when its buffers or shape
        // changed (or, with builds inside, any job), so that consecutive runs of different jobs
        // replay one graph and a run can be queued while the one before still runs.
        const bool graph_builds = (flags & LRC_BATCH_BUILD) && (flags & LRC_BATCH_GRAPH);
        if ((flags & LRC_BATCH_BUILD) && (!graph_builds || !cached)) {
            // builds as plain launches (with GRAPH: a first run sizes the buffers a captured build needs)
            for (const lrc_batch::Job *J : builds_of(b)) {
                int rc = build_job(b, J, c->st, false);
                if (rc) return rc;
            }
        }
        int rc = prepare(b, (flags & LRC_BATCH_BUILD) != 0);
        if (rc) return rc;
        const std::vector<unsigned char> key = graph_key(b, flags);
        bool reuse = b->exec && b->graph_flags == flags && key == b->graph_sig;
        if (!reuse && b->alt_exec && b->alt_flags == flags && key == b->alt_sig) {
            swap_graphs(b);
            reuse = true;
        }
        if (!reuse) {
            swap_graphs(b);                             // (the current graph kept, the one kept before it dropped)
            rc = capture(b, flags, key);
            if (rc) return rc;
        }
        cudaError_t e = cudaSuccess;
        if (flags & LRC_BATCH_ZERO) {                       // (the bands zeroed outside the graph)
            for (size_t i = 0; i < b->jobs.size() && !e; i++) {
                const lrc_batch::Job &J = b->jobs[i];
                e = cudaMemsetAsync(J.accum + (size_t)J.y0 * J.p.width * 4, 0, (size_t)J.rows * J.p.width * 16, c->st);
                if (!e && J.guided)                         // the band's moments (plane 1) too
                    e = cudaMemsetAsync(J.accum + ((size_t)J.p.width * J.p.height + (size_t)J.y0 * J.p.width) * 4, 0,
                                        (size_t)J.rows * J.p.width * 16, c->st);
            }
        }
        if (!e && b->ev_launch) e = cudaEventRecord(b->ev_launch, c->st);
        if (!e) e = cudaGraphLaunch(b->exec, c->st);
        if (e) return cuda_status(c, e, "batch graph launch");
        b->graph_used = reuse ? 1 : 0;
        if (graph_builds) note_built(b);
        return LRC_OK;
    }
    if ((flags & LRC_BATCH_GRAPH) && cached) {
        cudaError_t e = cudaGraphLaunch(b->exec, c->st);
        if (e) return cuda_status(c, e, "batch graph launch");
        b->graph_used = 1;
        if (flags & LRC_BATCH_BUILD) note_built(b);
        return LRC_OK;
    }
    if (flags & LRC_BATCH_BUILD) {
        // builds first: they size the trees the table points at
        for (const lrc_batch::Job *J : builds_of(b)) {
            int rc = build_job(b, J, c->st, false);
            if (rc) return rc;
        }
    }
    int rc = prepare(b, (flags & LRC_BATCH_BUILD) != 0);
    if (rc) return rc;
    rc = enqueue(b, flags, c->st, false, false, true, b->ntasks);
    if (rc) return rc;
    if (flags & LRC_BATCH_GRAPH) {
        // the next run replays this one: captured now, with every buffer sized
        cudaError_t e = cudaStreamSynchronize(c->st);
        if (e) return cuda_status(c, e, "batch run");
        rc = capture(b, flags, signature(b, flags));
        if (rc) return rc;
    }
    return LRC_OK;
}

int lrc_batch_rays(lrc_batch *b, uint64_t *per_job, uint64_t *total) {
    if (!b) return LRC_E_INVALID;
    lrc_ctx *c = b->ctx;
    DeviceGuard g(c->device);
    int rc = check_status(c);
    if (rc) return rc;
    const size_t nj = b->jobs.size();
    std::vector<unsigned long long> r(nj, 0);
    if (nj && b->prepared) {
        cudaError_t e = cudaMemcpy(r.data(), b->d_ctr + 1, nj * 8, cudaMemcpyDeviceToHost);
        if (e) return cuda_status(c, e, "batch rays");
    }
    uint64_t t = 0;
    for (size_t i = 0; i < nj; i++) {
        if (per_job) per_job[i] = r[i];
        t += r[i];
    }
    if (total) *total = t;
    return LRC_OK;
}

int lrc_batch_passes(lrc_batch *b, uint32_t *passes, uint64_t *kernels) {
    if (!b) return LRC_E_INVALID;
    lrc_ctx *c = b->ctx;
    uint32_t n = 0;
    uint64_t k = 0;
    if (b->prepared && b->engine == 1 && b->d_wf) {
        DeviceGuard g(c->device);
        int rc = check_status(c);
        if (rc) return rc;
        const lrc::WfState W = lrc::wf_carve(b->d_wf, b->wf_slots);
        cudaError_t e = cudaMemcpy(&n, W.ctl + 4, 4, cudaMemcpyDeviceToHost);
        if (e) return cuda_status(c, e, "batch passes");
        k = 2 + 4 * (uint64_t)n;                         // clear, then advance / closest hit / shade / shadow a pass, resolve
    } else if (b->prepared) {
        k = 2;                                           // the persistent trace kernel and the resolve pass
    }
    if (passes) *passes = n;
    if (kernels) *kernels = k;
    return LRC_OK;
}

int lrc_batch_step_stats(const lrc_batch *b, double *intersect_ms, uint64_t *intersect_rays, uint64_t *box_tests,
                         uint64_t *tri_tests, uint64_t *kernels) {
    if (!b) return LRC_E_INVALID;
    const lrc::WfStepStats &S = b->step_stats;
    if (intersect_ms) *intersect_ms = S.isect_ms;
    if (intersect_rays) *intersect_rays = S.isect_rays;
    if (box_tests) *box_tests = S.box_tests;
    if (tri_tests) *tri_tests = S.tri_tests;
    if (kernels) *kernels = S.launches;
    return LRC_OK;
}

int lrc_batch_shape(int32_t variant, int32_t *block, int32_t *minb, int32_t *per_sm) {
    int bl = 0, mb = 0;
    int n = lrc::batch_variant_shape(variant, &bl, &mb);
    if (n < 0) return -1;
    if (block) *block = bl;
    if (minb) *minb = mb;
    if (per_sm) *per_sm = n;
    return lrc::batch_variants();
}

int lrc_batch_set_shape(lrc_batch *b, int32_t variant, int32_t grid) {
    if (!b || variant < 0 || variant >= lrc::batch_variants() || grid < 0) return LRC_E_INVALID;
    b->variant = variant;
    b->grid = grid;
    if (!grid) {
        int block = 0, minb = 0;
        DeviceGuard g(b->ctx->device);
        b->grid = std::max(lrc::batch_variant_shape(variant, &block, &minb), 1) * b->ctx->num_sms;
    }
    return LRC_OK;
}

int lrc_batch_tune(lrc_batch *b, uint64_t sample_tasks, int32_t *variant, int32_t *grid, double *ns_per_task) {
    if (!b) return LRC_E_INVALID;
    lrc_ctx *c = b->ctx;
    if (b->jobs.empty()) return fail(c, LRC_E_INVALID, "an empty batch has nothing to tune on");
    for (const lrc_batch::Job &J : b->jobs) {
        int rc = check_job(c, J, false);
        if (rc) return rc;
    }
    DeviceGuard g(c->device);
    for (lrc_batch::Job &J : b->jobs) {
        if (!J.s->tables) {
            int rc = lrc_scene_set_tables(J.s, nullptr, nullptr);
            if (rc) return rc;
        }
    }
    int rc = b->prepared ? LRC_OK : prepare(b, false);
    if (rc) return rc;
    // the queue's head: the most expensive tasks (the trace kernels write only per-task sums, which
    // the next run overwrites, so tuning changes no image)
    // (the wavefront's sizes are timed on at least 2^24 tasks, or all: a sixteenth of a small queue
    // cannot fill its larger sizes, and a size is timed only where the sample fills it)
    const unsigned long long dflt = b->engine == 1 ? std::max<unsigned long long>(b->ntasks / 16 + 1, 1ull << 24)
                                                   : b->ntasks / 16 + 1;
    const unsigned long long n = std::min<unsigned long long>(b->ntasks, sample_tasks ? sample_tasks : dflt);
    if (b->engine == 1) return tune_wavefront(b, n, variant, grid, ns_per_task);
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    double best = 1e300;
    int best_v = 0, best_grid = 0;
    cudaError_t e = cudaSuccess;
    for (int v = 0; v < lrc::batch_variants() && !e; v++) {
        int block = 0, minb = 0;
        const int per_sm = lrc::batch_variant_shape(v, &block, &minb);
        if (per_sm < 1) continue;
        const int grid_v = per_sm * c->num_sms;
        float ms = 0;
        for (int rep = 0; rep < 2 && !e; rep++) {   // the first launch of a shape pays its module load
            e = cudaMemsetAsync(b->d_ctr, 0, 8, c->st);
            if (!e) e = cudaEventRecord(e0, c->st);
            if (!e) e = lrc::batch_trace(b->d_jobs, (uint32_t)b->jobs.size(), rep ? n : std::min<unsigned long long>(n, 4096),
                                         b->d_ctr, c->d_status, v, grid_v, any_media(b), c->st);
            if (!e) e = cudaEventRecord(e1, c->st);
            if (!e) e = cudaEventSynchronize(e1);
            if (!e) e = cudaEventElapsedTime(&ms, e0, e1);
        }
        if (!e && ms < best) {
            best = ms;
            best_v = v;
            best_grid = grid_v;
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (e) return cuda_status(c, e, "batch tune");
    rc = check_status(c);
    if (rc) return rc;
    b->variant = best_v;
    b->grid = best_grid;
    if (variant) *variant = best_v;
    if (grid) *grid = best_grid;
    if (ns_per_task) *ns_per_task = best * 1e6 / (double)n;
    return LRC_OK;
}

int lrc_batch_set_engine(lrc_batch *b, int32_t engine) {
    if (!b || (engine != 0 && engine != 1)) return LRC_E_INVALID;
    b->engine = engine;
    return LRC_OK;
}

int lrc_batch_set_wavefront(lrc_batch *b, uint32_t slots, int32_t variant) {
    if (!b || variant < 0 || variant >= lrc::wf_variants() || slots < 256 || slots % 256 || slots > (1u << 26))
        return LRC_E_INVALID;
    b->wf_slots = slots;
    b->wf_variant = variant;
    return LRC_OK;
}

int lrc_batch_wavefront_shape(int32_t variant, int32_t *block, int32_t *minb, int32_t *per_sm) {
    int bl = 0, mb = 0;
    int n = lrc::wf_variant_shape(variant, &bl, &mb);
    if (n < 0) return -1;
    if (block) *block = bl;
    if (minb) *minb = mb;
    if (per_sm) *per_sm = n;
    return lrc::wf_variants();
}

int lrc_batch_engine(const lrc_batch *b, int32_t *engine, uint32_t *slots, int32_t *wf_variant) {
    if (!b) return LRC_E_INVALID;
    if (engine) *engine = b->engine;
    if (slots) *slots = b->wf_slots;
    if (wf_variant) *wf_variant = b->wf_variant;
    return LRC_OK;
}

int lrc_batch_info(const lrc_batch *b, uint64_t *tasks, uint64_t *pixels, int32_t *variant, int32_t *grid,
                   int32_t *graph_used) {
    if (!b) return LRC_E_INVALID;
    if (tasks) *tasks = b->ntasks;
    if (pixels) *pixels = b->npix;
    if (variant) *variant = b->variant;
    if (grid) *grid = b->grid;
    if (graph_used) *graph_used = b->graph_used;
    return LRC_OK;
}

}  // extern "C"
