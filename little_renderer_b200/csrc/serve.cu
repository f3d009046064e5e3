// serve.cu - a render server: jobs (scene, image, spp, optionally moved instances) admitted as
// they arrive, by an HBM byte budget, and traced together in waves through the batch's wavefront.
//
// No counterpart in the reference, whose GPU view traces one scene at a time and paces its submits
// by the band scheduler (gpu_view_trace_more, engine/gpu/view_gpu.c:1081-1190: rows x repeats per
// submit from the measured ms per pass). Here every wave takes bands of rows of the admitted jobs
// and runs them as one batch: jobs that arrive while others are on the GPU join at the next wave
// (continuous batching) and the device's paths in flight are always full. By default (policy 2)
// the jobs with the fewest paths left go first, each band as large as the wave's paths left
// allow: a small job is done within a wave of its admission, and a wave holds few scenes (a wave
// spread evenly over dozens of scenes' trees measured 0.72x the throughput of one packed this way:
// their trees and triangles no longer fit L2 together). Policy 0 shares each wave evenly among all
// admitted jobs, policy 1 serves the oldest first. A band traces all of its pixels' samples, so a
// job's image is the one lrc_trace makes of it alone, to the bit, whatever else shares its waves.
//
// Waves are pipelined on two batches: a step plans the next wave (rows are handed out as waves are
// planned, so its bands are known before the wave ahead of it ends), captures and launches it, and
// only then waits for the wave ahead and reads its ray counts (copied to pinned memory behind it on
// the stream): the device goes from one wave to the next while the host builds the one after. A
// job admitted in a step is planned into that step's wave.
//
// Admission holds a job's bytes - its image, and for moved instances its own records and top level -
// against the budget, in arrival order; a job larger than the whole budget is refused at submit.
// A moved-instance job gets its own copy of the scene's instance layer (records and top level, the
// meshes' trees shared), its top level refit (bvh_refit_boxes's bottom-up refit) or built again on
// the device when admitted, so jobs of the same scene at different frames run side by side. A
// denoised job (the step after the path tracer for low-spp jobs) holds the denoiser's 4 planes
// while it is traced: the guide made at admission, the moments added by its waves, the a-trous
// passes run when its last band is done and the planes freed.
#include "api_internal.cuh"
#include <algorithm>
#include <chrono>
#include <deque>
#include <new>
#include <unordered_map>
#include <vector>

using namespace lrcapi;

struct lrc_server {
    struct Job {
        uint64_t id = 0;
        lrc_scene *s = nullptr;
        lrc_trace_params p{};
        uint32_t spp = 0;
        std::vector<float> records;     // moved instances (32 floats each), or none
        int tlas_mode = 0;
        bool denoise = false;           // traced with the denoiser's planes, denoised when done
        float *d_img = nullptr;         // W x H float4 (sum, count); denoised: (rgb, 1)
        float *d_planes = nullptr;      // a denoised job's 4 planes while it is traced
        float *d_inst = nullptr;        // the job's instance records
        Node *d_tlas = nullptr;         // and their top level
        uint32_t *d_tlas_aux = nullptr;
        size_t bytes = 0;
        int32_t next_row = 0;           // rows handed to waves so far
        uint64_t rays = 0;
        double t_submit = 0, t_admit = 0, t_done = 0;
        int state = 0;                  // 0 queued, 1 admitted, 2 finished
        cudaEvent_t ev_done = nullptr;  // on the side stream: its image complete (finished jobs)
    };
    // a wave on one of the two batches: its jobs (in the batch's job order), whether its band ends
    // each, the ray counts and passes copied back behind it, its events (launch, end)
    struct Wave {
        lrc_batch *batch = nullptr;
        std::vector<Job *> jobs;
        std::vector<char> last;
        unsigned long long *h_rays = nullptr;   // pinned
        size_t rays_cap = 0;
        uint32_t *h_passes = nullptr;           // pinned
        cudaEvent_t ev0 = nullptr, ev1 = nullptr;
        bool pending = false;
    };
    lrc_ctx *ctx = nullptr;
    lrc_batch *batch = nullptr;         // (wave[0]'s: lrc_server_batch)
    Wave wave[2];
    int next = 0;                       // the slot the next wave is planned into
    unsigned long long reserved_tasks = 0;   // both batches' run buffers hold waves this large
    size_t reserved_jobs = 0;
    cudaStream_t side = nullptr;        // finished jobs' denoising and reads, behind their last wave only
    uint64_t budget = 0, wave_paths = 0, in_use = 0;
    uint64_t next_id = 1;
    std::deque<Job *> queued;
    std::vector<Job *> active;
    std::unordered_map<uint64_t, Job *> jobs;
    int32_t finished = 0;
    // scratch for the jobs' top levels (build / refit)
    void *scratch = nullptr;
    size_t scratch_cap = 0;
    float *d_boxes = nullptr;
    size_t boxes_cap = 0;
    uint32_t *d_small = nullptr;
    void *dn = nullptr;                 // the denoiser's scratch
    size_t dn_cap = 0;
    uint64_t waves = 0, kernels = 0;    // waves run and the trace kernels they launched
    double gpu_ms = 0;                  // the waves' device time (CUDA events from each launch to its end)
    int policy = 2;                     // how a wave is made (lrc_server_set_policy)
};

namespace {

double now_ms() {
    using namespace std::chrono;
    return duration<double, std::milli>(steady_clock::now().time_since_epoch()).count();
}

size_t job_bytes(const lrc_server::Job &J) {
    size_t b = (size_t)J.p.width * J.p.height * (J.denoise ? 80 : 16);   // (denoised: planes + image)
    const size_t n = J.records.size() / 32;
    if (n) b += n * 128 + (2 * n - 1) * 32 + n * 4;
    return b;
}

void free_job(lrc_server *sv, lrc_server::Job *J) {
    lrc_ctx *c = sv->ctx;
    if (J->ev_done) {                                   // (its denoising on the side stream done first)
        cudaStreamWaitEvent(c->st, J->ev_done, 0);
        cudaEventDestroy(J->ev_done);
        J->ev_done = nullptr;
    }
    if (J->d_img) cudaFreeAsync(J->d_img, c->st);
    if (J->d_planes) cudaFreeAsync(J->d_planes, c->st);
    if (J->d_inst) cudaFreeAsync(J->d_inst, c->st);
    if (J->d_tlas) cudaFreeAsync(J->d_tlas, c->st);
    if (J->d_tlas_aux) cudaFreeAsync(J->d_tlas_aux, c->st);
    J->d_img = nullptr;
    J->d_planes = nullptr;
    J->d_inst = nullptr;
    J->d_tlas = nullptr;
    J->d_tlas_aux = nullptr;
}

// the path tracer's view of a job's scene: its own instance layer, if it has one
lrc::PtScene job_view(const lrc_server::Job *J) {
    lrc::PtScene S = pt_scene(J->s);
    if (J->d_inst) {
        S.inst = reinterpret_cast<const float4 *>(J->d_inst);
        S.tlas_nodes = reinterpret_cast<const float4 *>(J->d_tlas);
        S.tlas_aux = J->d_tlas_aux;
    }
    return S;
}

// the job's device memory: its image (cleared) and, for moved instances, its records and top level
int admit(lrc_server *sv, lrc_server::Job *J) {
    lrc_ctx *c = sv->ctx;
    const size_t img = (size_t)J->p.width * J->p.height * 16;
    cudaError_t e = cudaMallocAsync(reinterpret_cast<void **>(&J->d_img), img, c->st);
    if (!e && !J->denoise) e = cudaMemsetAsync(J->d_img, 0, img, c->st);
    const uint32_t n = (uint32_t)(J->records.size() / 32);
    if (!e && n) {
        lrc_scene *s = J->s;
        e = cudaMallocAsync(reinterpret_cast<void **>(&J->d_inst), (size_t)n * 128, c->st);
        if (!e) e = cudaMallocAsync(reinterpret_cast<void **>(&J->d_tlas), (2 * (size_t)n - 1) * 32, c->st);
        if (!e) e = cudaMallocAsync(reinterpret_cast<void **>(&J->d_tlas_aux), (size_t)n * 4, c->st);
        if (!e) e = cudaMemcpyAsync(J->d_inst, J->records.data(), (size_t)n * 128, cudaMemcpyHostToDevice, c->st);
        if (!e && J->tlas_mode == LRC_TLAS_REBUILD) {
            e = reserve(reinterpret_cast<void **>(&sv->d_boxes), &sv->boxes_cap, (size_t)n * 32);
            if (!e) e = reserve(&sv->scratch, &sv->scratch_cap, lrc::build_scratch_bytes(n, 30, 0));
            if (!e) e = build_tlas_on(c, J->d_inst, n, J->d_tlas, J->d_tlas_aux, sv->d_boxes, sv->d_small, sv->scratch,
                                      sv->scratch_cap, c->st, nullptr);
        } else if (!e) {
            // the scene's top level, refit for the job's boxes (its topology as built)
            e = cudaMemcpyAsync(J->d_tlas, s->d_tlas_nodes, (2 * (size_t)n - 1) * 32, cudaMemcpyDeviceToDevice, c->st);
            if (!e) e = cudaMemcpyAsync(J->d_tlas_aux, s->d_tlas_aux, (size_t)n * 4, cudaMemcpyDeviceToDevice, c->st);
            if (!e) e = reserve(&sv->scratch, &sv->scratch_cap, lrc::refit_scratch_bytes(n));
            if (!e) e = lrc::refit_device(J->d_tlas, J->d_tlas_aux, n, 0, J->d_inst, 8, 6, sv->scratch, sv->scratch_cap,
                                          c->d_status, c->st);
        }
    }
    if (!e && J->denoise) {                          // the planes: samples and moments cleared, the guide
        const size_t N = (size_t)J->p.width * J->p.height;
        e = cudaMallocAsync(reinterpret_cast<void **>(&J->d_planes), N * 64, c->st);
        if (!e) e = cudaMemsetAsync(J->d_planes, 0, N * 32, c->st);
        if (!e) {
            lrc::PtParams P{};
            P.W = J->p.width; P.H = J->p.height; P.rows = J->p.height;
            P.origin = {J->p.origin[0], J->p.origin[1], J->p.origin[2]};
            P.upper_left = {J->p.upper_left[0], J->p.upper_left[1], J->p.upper_left[2]};
            P.horizontal = {J->p.horizontal[0], J->p.horizontal[1], J->p.horizontal[2]};
            P.vertical = {J->p.vertical[0], J->p.vertical[1], J->p.vertical[2]};
            e = lrc::dn_guide(job_view(J), P, reinterpret_cast<float4 *>(J->d_planes), c->d_status, c->st);
        }
    }
    if (e) {
        free_job(sv, J);
        return cuda_status(c, e, "server admission");
    }
    J->state = 1;
    J->t_admit = now_ms();
    sv->in_use += J->bytes;
    return LRC_OK;
}

// a launched wave waited for: its device time and passes, each job's rays; the jobs whose last
// band it held finished (a denoised one's planes filtered into its image, on the side stream after
// the wave, not after the wave launched behind it), their instance layers freed
int finish_wave(lrc_server *sv, lrc_server::Wave &W, int32_t *finished) {
    lrc_ctx *c = sv->ctx;
    cudaError_t e = cudaEventSynchronize(W.ev1);
    if (e) return cuda_status(c, e, "server wave");
    W.pending = false;
    if (W.h_passes[1]) {                                // (an error the wave's kernels reported)
        int rc = check_status(c);
        if (rc) return rc;
    }
    float ms = 0;
    if (cudaEventElapsedTime(&ms, W.ev0, W.ev1) == cudaSuccess) sv->gpu_ms += ms;
    sv->waves++;
    sv->kernels += 2 + 4 * (uint64_t)W.h_passes[0];   // clear, then advance / closest hit / shade / shadow a pass, resolve
    const double t = now_ms();
    bool any = false;
    for (size_t q = 0; q < W.jobs.size(); q++) {
        lrc_server::Job *J = W.jobs[q];
        J->rays += W.h_rays[q];
        if (!W.last[q]) continue;
        any = true;
        if (!J->ev_done && (e = cudaEventCreateWithFlags(&J->ev_done, cudaEventDisableTiming)))
            return cuda_status(c, e, "server job event");
        e = cudaStreamWaitEvent(sv->side, W.ev1, 0);
        if (!e && J->denoise) {                         // the image denoised, the planes freed
            e = reserve(&sv->dn, &sv->dn_cap, lrc::dn_scratch_bytes(J->p.width, J->p.height));
            if (!e) e = lrc::dn_denoise(reinterpret_cast<const float4 *>(J->d_planes), J->p.width, J->p.height, 5,
                                        reinterpret_cast<float4 *>(J->d_img), sv->dn, sv->side);
            if (!e) e = cudaFreeAsync(J->d_planes, sv->side);
            if (!e) {
                J->d_planes = nullptr;
                sv->in_use -= (size_t)J->p.width * J->p.height * 64;
                J->bytes -= (size_t)J->p.width * J->p.height * 64;
            }
        }
        if (!e) e = cudaEventRecord(J->ev_done, sv->side);
        // (work queued on the context's stream from now on - a read of lrc_server_result's image
        // there - comes after the job's completion on the side stream)
        if (!e) e = cudaStreamWaitEvent(c->st, J->ev_done, 0);
        if (e) return cuda_status(c, e, "server finish");
        J->state = 2;
        J->t_done = t;
        sv->finished++;
        if (finished) (*finished)++;
        if (J->d_inst) {                                // (its instances are done with; its image stays)
            cudaFreeAsync(J->d_inst, c->st);
            cudaFreeAsync(J->d_tlas, c->st);
            cudaFreeAsync(J->d_tlas_aux, c->st);
            J->d_inst = nullptr;
            J->d_tlas = nullptr;
            J->d_tlas_aux = nullptr;
            sv->in_use -= J->bytes - (size_t)J->p.width * J->p.height * 16;
            J->bytes = (size_t)J->p.width * J->p.height * 16;
        }
    }
    if (any) {
        std::vector<lrc_server::Job *> still;
        for (lrc_server::Job *J : sv->active)
            if (J->state != 2) still.push_back(J);
        sv->active.swap(still);
    }
    return LRC_OK;
}

}  // namespace

extern "C" {

double lrc_server_clock(void) { return now_ms(); }

int lrc_server_create(lrc_ctx *c, uint64_t hbm_budget_bytes, uint64_t wave_paths, lrc_server **out) {
    if (!c || !out || !hbm_budget_bytes || !wave_paths) return LRC_E_INVALID;
    *out = nullptr;
    lrc_server *sv = new (std::nothrow) lrc_server;
    if (!sv) return LRC_RETRY;
    sv->ctx = c;
    sv->budget = hbm_budget_bytes;
    sv->wave_paths = wave_paths;
    DeviceGuard g(c->device);
    int rc = LRC_OK;
    cudaError_t e = cudaSuccess;
    for (lrc_server::Wave &W : sv->wave) {
        if (!rc) rc = lrc_batch_create(c, &W.batch);
        if (!rc) rc = lrc_batch_set_wavefront(W.batch, 1u << 22, LRC_WAVEFRONT_DEFAULT_VARIANT);   // (4M paths in flight: a wave's tail stays short)
        if (!rc && !e) e = cudaEventCreate(&W.ev0);
        if (!rc && !e) e = cudaEventCreate(&W.ev1);
        if (!rc && !e) e = cudaMallocHost(reinterpret_cast<void **>(&W.h_passes), 16);
        if (!rc && !e) batch_set_launch_event(W.batch, W.ev0);
    }
    sv->batch = sv->wave[0].batch;
    if (!rc && !e) e = cudaStreamCreateWithFlags(&sv->side, cudaStreamNonBlocking);
    if (!rc && !e) e = cudaMalloc(&sv->d_small, 256);
    if (rc || e) {
        lrc_server_destroy(sv);
        return rc ? rc : cuda_status(c, e, "server");
    }
    *out = sv;
    return LRC_OK;
}

void lrc_server_destroy(lrc_server *sv) {
    if (!sv) return;
    DeviceGuard g(sv->ctx->device);
    cudaStreamSynchronize(sv->ctx->st);
    for (lrc_server::Wave &W : sv->wave) {
        if (W.batch) lrc_batch_destroy(W.batch);
        if (W.ev0) cudaEventDestroy(W.ev0);
        if (W.ev1) cudaEventDestroy(W.ev1);
        if (W.h_rays) cudaFreeHost(W.h_rays);
        if (W.h_passes) cudaFreeHost(W.h_passes);
    }
    for (auto &kv : sv->jobs) {
        free_job(sv, kv.second);
        delete kv.second;
    }
    cudaStreamSynchronize(sv->ctx->st);
    if (sv->side) {
        cudaStreamSynchronize(sv->side);
        cudaStreamDestroy(sv->side);
    }
    cudaFree(sv->scratch);
    cudaFree(sv->d_boxes);
    cudaFree(sv->d_small);
    cudaFree(sv->dn);
    delete sv;
}

int lrc_server_submit(lrc_server *sv, lrc_scene *s, const lrc_trace_params *p, uint32_t spp, const float *records,
                      uint32_t n, int tlas_mode, uint64_t *id) {
    if (!sv || !s || !p || s->ctx != sv->ctx || (n && !records)) return LRC_E_INVALID;
    lrc_ctx *c = sv->ctx;
    if (p->width <= 0 || p->height <= 0 || spp == 0 || spp >= (1u << 31))
        return fail(c, LRC_E_INVALID, "a job is a whole image with spp >= 1");
    if (p->exact) return fail(c, LRC_E_INVALID, "served jobs trace in fast mode");
    if (s->nvol) return fail(c, LRC_E_INVALID, "the server's wavefront does not trace media (lrc_trace does)");
    const bool denoise = (tlas_mode & LRC_SERVE_DENOISE) != 0;
    tlas_mode &= ~LRC_SERVE_DENOISE;
    if (denoise && (uint64_t)p->width * p->height >= (1ull << 31)) return fail(c, LRC_E_INVALID, "image too large to denoise");
    if (n && (n != s->ninst || !s->tlas_n)) return fail(c, LRC_E_INVALID, "moved instances: the scene's instances, built");
    if (n && (tlas_mode < LRC_TLAS_REFIT || tlas_mode > LRC_TLAS_REBUILD))
        return fail(c, LRC_E_INVALID, "a job's top level is refit or rebuilt");
    lrc_server::Job *J = new (std::nothrow) lrc_server::Job;
    if (!J) return LRC_RETRY;
    J->id = sv->next_id++;
    J->s = s;
    J->p = *p;
    J->spp = spp;
    if (n) J->records.assign(records, records + (size_t)n * 32);
    J->tlas_mode = tlas_mode;
    J->denoise = denoise;
    J->bytes = job_bytes(*J);
    if (J->bytes > sv->budget) {
        delete J;
        return fail(c, LRC_E_TOO_BIG, "the job needs more device memory than the whole budget");
    }
    J->t_submit = now_ms();
    sv->queued.push_back(J);
    sv->jobs[J->id] = J;
    if (id) *id = J->id;
    return LRC_OK;
}

int lrc_server_step(lrc_server *sv, int32_t *finished) {
    if (!sv) return LRC_E_INVALID;
    lrc_ctx *c = sv->ctx;
    DeviceGuard g(c->device);
    if (finished) *finished = 0;
    // admission, in arrival order, while the budget holds
    while (!sv->queued.empty() && sv->in_use + sv->queued.front()->bytes <= sv->budget) {
        lrc_server::Job *J = sv->queued.front();
        int rc = admit(sv, J);
        if (rc) return rc;
        sv->queued.pop_front();
        sv->active.push_back(J);
    }
    // the next wave, into the free slot: bands of the admitted jobs with rows left. Policy 0: the
    // next band of every job, the wave's paths shared evenly; 1: the oldest jobs first, each band
    // as large as the wave's paths left allow (few scenes a wave, each wave's jobs ending sooner);
    // 2: as 1, the jobs with the fewest paths left first. Rows are handed out here, so the wave
    // after can be planned before this one ends.
    lrc_server::Wave &N = sv->wave[sv->next];
    int rc = N.pending ? finish_wave(sv, N, finished) : LRC_OK;   // (never: a slot is freed before it is planned again)
    if (rc) return rc;
    std::vector<lrc_server::Job *> order;
    for (lrc_server::Job *J : sv->active)
        if (J->next_row < J->p.height) order.push_back(J);
    if (sv->policy == 2)
        std::stable_sort(order.begin(), order.end(), [](const lrc_server::Job *a, const lrc_server::Job *b) {
            return (uint64_t)a->p.width * (a->p.height - a->next_row) * a->spp <
                   (uint64_t)b->p.width * (b->p.height - b->next_row) * b->spp;
        });
    bool launched = false;
    if (!order.empty()) {
        const uint64_t share = sv->wave_paths / order.size() + 1;
        uint64_t used = 0;
        rc = lrc_batch_clear(N.batch);
        N.jobs.clear();
        N.last.clear();
        for (lrc_server::Job *J : order) {
            const uint64_t row_paths = (uint64_t)J->p.width * J->spp;
            int32_t rows;
            if (sv->policy == 0) {
                rows = (int32_t)std::max<uint64_t>(1, share / row_paths);
            } else {
                if (used >= sv->wave_paths) break;
                rows = (int32_t)std::max<uint64_t>(1, (sv->wave_paths - used + row_paths - 1) / row_paths);
            }
            rows = std::min(rows, J->p.height - J->next_row);
            used += (uint64_t)rows * row_paths;
            InstView v{J->d_inst, J->d_tlas, J->d_tlas_aux};
            if (!rc) rc = batch_add_view(N.batch, J->s, &J->p, J->next_row, rows, 0, J->spp,
                                         J->denoise ? J->d_planes : J->d_img, v, J->denoise);
            if (rc) break;
            J->next_row += rows;
            N.jobs.push_back(J);
            N.last.push_back(J->next_row >= J->p.height);
        }
        // both batches' buffers sized for a wave (its paths bound its tasks) before any wave runs,
        // and again should a wave outgrow them: a run that must allocate waits for the device
        cudaError_t e = cudaSuccess;
        const unsigned long long want = std::max<unsigned long long>(used, sv->wave_paths + (2ull << 20));
        const size_t want_jobs = std::max<size_t>(N.jobs.size(), 256);
        if (!rc && (want > sv->reserved_tasks || want_jobs > sv->reserved_jobs)) {
            for (lrc_server::Wave &W : sv->wave)
                if (!rc) rc = batch_reserve(W.batch, want, want_jobs);
            sv->reserved_tasks = want;
            sv->reserved_jobs = want_jobs;
        }
        if (!rc && N.rays_cap < N.jobs.size()) {
            if (N.h_rays) cudaFreeHost(N.h_rays);
            N.h_rays = nullptr;
            N.rays_cap = 0;
            e = cudaMallocHost(reinterpret_cast<void **>(&N.h_rays), (N.jobs.size() + 64) * 8);
            if (!e) N.rays_cap = N.jobs.size() + 64;
        }
        if (!rc && !e) rc = lrc_batch_run(N.batch, 0);
        // behind it on the stream: its counts, the status word, its end
        if (!rc && !e) e = batch_counts_async(N.batch, N.h_rays, N.h_passes);
        if (!rc && !e) e = cudaMemcpyAsync(N.h_passes + 1, c->d_status, 4, cudaMemcpyDeviceToHost, c->st);
        if (!rc && !e) e = cudaEventRecord(N.ev1, c->st);
        if (e) return cuda_status(c, e, "server wave");
        if (rc) return rc;
        N.pending = true;
        launched = true;
    }
    // the wave ahead: waited for, its counts read, the jobs it ends finished
    lrc_server::Wave &P = sv->wave[1 - sv->next];
    if (P.pending) rc = finish_wave(sv, P, finished);
    if (launched) sv->next = 1 - sv->next;
    return rc;
}

int lrc_server_result(lrc_server *sv, uint64_t id, const float **d_image, uint64_t *rays, double *t_submit,
                      double *t_admit, double *t_done) {
    if (!sv) return LRC_E_INVALID;
    auto it = sv->jobs.find(id);
    if (it == sv->jobs.end()) return fail(sv->ctx, LRC_E_INVALID, "no such job");
    const lrc_server::Job *J = it->second;
    if (J->state != 2) return LRC_RETRY;
    if (d_image) *d_image = J->d_img;
    if (rays) *rays = J->rays;
    if (t_submit) *t_submit = J->t_submit;
    if (t_admit) *t_admit = J->t_admit;
    if (t_done) *t_done = J->t_done;
    return LRC_OK;
}

int lrc_server_read(lrc_server *sv, uint64_t id, float *out) {
    if (!sv || !out) return LRC_E_INVALID;
    auto it = sv->jobs.find(id);
    if (it == sv->jobs.end()) return fail(sv->ctx, LRC_E_INVALID, "no such job");
    const lrc_server::Job *J = it->second;
    if (J->state != 2) return LRC_RETRY;
    DeviceGuard g(sv->ctx->device);
    // on the side stream, behind the job's own completion only (not the wave launched since)
    cudaError_t e = J->ev_done ? cudaStreamWaitEvent(sv->side, J->ev_done, 0) : cudaSuccess;
    if (!e) e = cudaMemcpyAsync(out, J->d_img, (size_t)J->p.width * J->p.height * 16, cudaMemcpyDeviceToHost, sv->side);
    if (!e) e = cudaStreamSynchronize(sv->side);
    if (e) return cuda_status(sv->ctx, e, "server read");
    return LRC_OK;
}

int lrc_server_release(lrc_server *sv, uint64_t id) {
    if (!sv) return LRC_E_INVALID;
    auto it = sv->jobs.find(id);
    if (it == sv->jobs.end()) return fail(sv->ctx, LRC_E_INVALID, "no such job");
    lrc_server::Job *J = it->second;
    if (J->state != 2) return fail(sv->ctx, LRC_E_INVALID, "the job is not finished");
    DeviceGuard g(sv->ctx->device);
    free_job(sv, J);
    sv->in_use -= J->bytes;
    sv->finished--;
    sv->jobs.erase(it);
    delete J;
    return LRC_OK;
}

lrc_batch *lrc_server_batch(lrc_server *sv) { return sv ? sv->batch : nullptr; }

int lrc_server_set_wavefront(lrc_server *sv, uint32_t slots, int32_t variant) {
    if (!sv) return LRC_E_INVALID;
    for (lrc_server::Wave &W : sv->wave) {
        int rc = lrc_batch_set_wavefront(W.batch, slots, variant);
        if (rc) return rc;
    }
    sv->reserved_tasks = 0;                            // (the next wave sizes the buffers again)
    return LRC_OK;
}

int lrc_server_stats(const lrc_server *sv, uint64_t *waves, uint64_t *kernels, double *gpu_ms) {
    if (!sv) return LRC_E_INVALID;
    if (waves) *waves = sv->waves;
    if (kernels) *kernels = sv->kernels;
    if (gpu_ms) *gpu_ms = sv->gpu_ms;
    return LRC_OK;
}

int lrc_server_set_policy(lrc_server *sv, int32_t policy) {
    if (!sv || policy < 0 || policy > 2) return LRC_E_INVALID;
    sv->policy = policy;
    return LRC_OK;
}

int lrc_server_state(const lrc_server *sv, int32_t *queued, int32_t *active, int32_t *finished, uint64_t *bytes) {
    if (!sv) return LRC_E_INVALID;
    if (queued) *queued = (int32_t)sv->queued.size();
    if (active) *active = (int32_t)sv->active.size();
    if (finished) *finished = sv->finished;
    if (bytes) *bytes = sv->in_use;
    return LRC_OK;
}

}  // extern "C"
