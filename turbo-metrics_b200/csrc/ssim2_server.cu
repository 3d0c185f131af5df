// ssim2_server.cu -- continuous-batching SSIMULACRA2 server (C ABI s2_server_*).
//
// Workload: jobs of one reference image and k distorted candidates (an
// encoder's CRF / quality search scores many candidates against one source),
// arriving at any time, of any size.  The reference's own cached-reference
// path (crates/ssimulacra2-cuda/src/lib.rs:440-860, ssim2-gpu Ssim2Batch
// pipeline_batch.rs:247-382) scores one size at a time on a caller's thread;
// here a worker thread keeps the GPU fed:
//
//   admission   jobs enter in arrival order while the device bytes they need
//               (inputs + the reference's XYB pyramid) fit the HBM budget; the
//               head of the queue is never overtaken (no starvation);
//   upload      an uploader thread admits jobs and sends their host images up
//               on a copy stream, into a stream-ordered memory pool grown to
//               the budget at creation (no mapping on the serving path), so
//               the round loop never waits for admission or upload issue;
//   batching    each round takes, in arrival order, every admitted job's
//               pending work -- the reference pyramid build (once per job) and
//               candidates -- up to a pair / pixel cap, and runs it as one
//               submission (prep + persistent fused + finalize launches);
//               candidates read the job's resident reference pyramid
//               (built once per job, by the prep launch of the round that
//               converts the reference, ahead of the candidates' tiles);
//   overlap     two submission workspaces alternate: the worker plans and
//               enqueues round i+1 while round i runs, then harvests round i;
//   completion  a job completes when all its candidates are harvested; its
//               latency (arrival -> completion) is recorded and its memory
//               returned to the pool.
//
// Results do not depend on what else is in a round: every candidate is scored
// with the same tile geometry (fixed strip height), and the per-pair sums are
// reduced in a fixed order, so a job scores bit-identically alone and mixed.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <vector>

#include "ssim2_engine_internal.h"

namespace {

using Clock = std::chrono::steady_clock;

struct Job {
    uint64_t id = 0;
    uint32_t w = 0, h = 0;
    const uint8_t *ref_host = nullptr;
    size_t ref_pitch = 0;
    std::vector<const uint8_t *> cand_host;
    size_t cand_pitch = 0;
    Clock::time_point arrival, done_at;
    // device side
    unsigned char *dev = nullptr;  // inputs (ref then candidates, packed rows) + reference pyramid
    size_t bytes = 0;
    size_t ref_levels_off = 0;
    size_t lvl_off[s2::kScales] = {0, 0, 0, 0, 0, 0};
    int ns = 0;
    cudaEvent_t uploaded = nullptr, up_start = nullptr;  // the job's uploads on the copy stream
    bool admitted = false, uploading = false, ref_scheduled = false, cancelled = false, finished = false;
    int next_cand = 0, inflight = 0, harvested = 0;
    std::vector<double> scores;
    std::vector<int32_t> status;
    s2_status job_status = S2_OK;
};

struct RoundEntry {
    Job *job;
    int cand;  // -1 = reference pyramid build
};

}  // namespace

struct s2_server {
    s2_server_config cfg{};
    Engine eng[2];
    cudaStream_t compute = nullptr, copy = nullptr;
    cudaMemPool_t pool = nullptr;
    std::thread worker, uploader;
    std::mutex mu;
    std::condition_variable cv_work, cv_done, cv_up;
    bool uploader_done = false;
    std::deque<Job *> queue;  // arrival order: not yet admitted, then admitted
    std::unordered_map<uint64_t, Job *> jobs;
    uint64_t next_id = 1;
    size_t bytes_in_use = 0;
    bool stop = false;
    s2_status fatal = S2_OK;
    // statistics
    std::vector<double> latencies_ms;
    uint64_t pairs_done = 0, jobs_done = 0, rounds = 0;
    double gpu_ms = 0.0;  // device time of the rounds' kernels (CUDA events)
    double t_wait = 0.0, t_upload = 0.0, t_submit = 0.0;  // worker time: GPU waits, upload issue, plan+enqueue
    double copy_ms = 0.0;                                  // copy-stream time of finished jobs' uploads
    uint64_t bytes_uploaded = 0;
    Clock::time_point t0;

    std::vector<RoundEntry> round[2];
    bool inflight[2] = {false, false};

    size_t workspace_bytes() const { return eng[0].allocated + eng[1].allocated; }

    // Device bytes a job needs while admitted.
    // Layout: the images (reference, then candidates, packed rows), the
    // reference's XYB pyramid.
    static size_t job_bytes(Job &j, size_t esize) {
        const size_t img = (size_t)j.w * 3 * j.h;
        size_t off = s2_align_up(img * (1 + j.cand_host.size()), 256);
        j.ref_levels_off = off;
        j.ns = s2_num_scales(j.w, j.h, S2_SCALES_CPU);
        off += s2_align_up(s2_image_levels_layout(j.w, j.h, j.ns, esize, j.lvl_off), 256);
        return off;
    }

    // Admit from the head of the queue while the budget allows (caller holds
    // mu); the uploads are issued by upload() after the lock is released.
    void admit_locked(std::vector<Job *> &fresh) {
        for (Job *j : queue) {
            if (j->admitted || j->cancelled) continue;
            if (cfg.hbm_budget && bytes_in_use + j->bytes + workspace_bytes() > cfg.hbm_budget) break;
            if (cudaMallocFromPoolAsync((void **)&j->dev, j->bytes, pool, copy) != cudaSuccess) break;
            j->admitted = true;
            j->uploading = true;
            bytes_in_use += j->bytes;
            fresh.push_back(j);
        }
    }

    // Copy admitted jobs' host images up on the copy stream (worker thread,
    // no lock held: a copy from pageable memory blocks until staged).
    // One image host -> device: a single linear copy when the rows are packed
    // (a 2-D copy of short rows moves a fraction of the link bandwidth).
    cudaError_t copy_image(unsigned char *dst, const uint8_t *src, size_t pitch, size_t row, uint32_t rows) {
        if (pitch == row) return cudaMemcpyAsync(dst, src, row * rows, cudaMemcpyHostToDevice, copy);
        return cudaMemcpy2DAsync(dst, row, src, pitch, row, rows, cudaMemcpyHostToDevice, copy);
    }

    // Uploader thread: admit in arrival order while the budget allows, send
    // the admitted jobs' images up, hand them to the round loop.
    void upload_loop() {
        std::vector<Job *> fresh;
        for (;;) {
            fresh.clear();
            {
                std::unique_lock<std::mutex> lock(mu);
                if (stop) break;
                admit_locked(fresh);
                if (fresh.empty()) {
                    cv_up.wait_for(lock, std::chrono::milliseconds(1));
                    continue;
                }
            }
            const auto ta = Clock::now();
            const s2_status up = upload(fresh);
            {
                std::lock_guard<std::mutex> lock(mu);
                t_upload += std::chrono::duration<double>(Clock::now() - ta).count();
                if (up != S2_OK) {
                    fatal = S2_ERR_CUDA;
                    stop = true;
                }
            }
            cv_work.notify_all();
            if (up != S2_OK) {
                cv_done.notify_all();
                break;
            }
        }
        {
            std::lock_guard<std::mutex> lock(mu);
            uploader_done = true;
        }
        cv_work.notify_all();
    }

    s2_status upload(const std::vector<Job *> &fresh) {
        for (Job *j : fresh) {
            const size_t img = (size_t)j->w * 3 * j->h, row = (size_t)j->w * 3;
            if (cudaEventCreate(&j->up_start) != cudaSuccess || cudaEventRecord(j->up_start, copy) != cudaSuccess)
                return S2_ERR_CUDA;
            if (copy_image(j->dev, j->ref_host, j->ref_pitch, row, j->h) != cudaSuccess) return S2_ERR_CUDA;
            for (size_t c = 0; c < j->cand_host.size(); c++)
                if (copy_image(j->dev + img * (1 + c), j->cand_host[c], j->cand_pitch, row, j->h) != cudaSuccess)
                    return S2_ERR_CUDA;
            if (cudaEventCreate(&j->uploaded) != cudaSuccess || cudaEventRecord(j->uploaded, copy) != cudaSuccess)
                return S2_ERR_CUDA;
        }
        std::lock_guard<std::mutex> lock(mu);
        for (Job *j : fresh) j->uploading = false;
        return S2_OK;
    }

    // Build the next round from admitted jobs, in arrival order (caller holds mu).
    void build_round_locked(std::vector<RoundEntry> &r) {
        r.clear();
        uint64_t pixels = 0;
        for (Job *j : queue) {
            if (!j->admitted || j->uploading) break;  // FIFO: later jobs wait too
            if (j->cancelled) continue;
            const uint64_t px = (uint64_t)j->w * j->h;
            if (!j->ref_scheduled) {
                if (!r.empty() && (r.size() >= cfg.max_batch_pairs || pixels + px > cfg.max_batch_pixels)) return;
                r.push_back({j, -1});
                j->ref_scheduled = true;
                pixels += px;
            }
            while (j->next_cand < (int)j->cand_host.size()) {
                if (!r.empty() && (r.size() >= cfg.max_batch_pairs || pixels + px > cfg.max_batch_pixels)) return;
                r.push_back({j, j->next_cand++});
                j->inflight++;
                pixels += px;
            }
        }
    }

    // Enqueue a round on the compute stream (no lock needed: only the worker
    // touches admitted jobs' device fields and the engines).
    s2_status submit_round(int k) {
        std::vector<RoundEntry> &r = round[k];
        std::vector<s2_pair_desc> d(r.size());
        std::vector<PairExtra> ex(r.size());
        std::vector<cudaEvent_t> waits;
        for (size_t i = 0; i < r.size(); i++) {
            Job *j = r[i].job;
            const size_t img = (size_t)j->w * 3 * j->h, row = (size_t)j->w * 3;
            memset(&d[i], 0, sizeof d[i]);
            d[i].width = j->w;
            d[i].height = j->h;
            d[i].format = S2_FMT_SRGB8;
            for (int s = 0; s < s2::kScales; s++)
                ex[i].ref_levels[s] = s < j->ns ? j->dev + j->ref_levels_off + j->lvl_off[s] : nullptr;
            if (r[i].cand < 0) {
                d[i].ref = j->dev;
                d[i].ref_pitch = row;
                ex[i].prep_mask = 1;
                ex[i].score = false;
            } else {
                d[i].dis = j->dev + img * (1 + r[i].cand);
                d[i].dis_pitch = row;
                ex[i].prep_mask = 2;
                ex[i].score = true;
            }
            if (std::find(waits.begin(), waits.end(), j->uploaded) == waits.end()) waits.push_back(j->uploaded);
        }
        for (cudaEvent_t e : waits)
            if (cudaStreamWaitEvent(compute, e, 0) != cudaSuccess) return S2_ERR_CUDA;
        Plan &p = eng[k].plan_storage;
        s2_status st = eng[k].plan(d.data(), (int)d.size(), p, ex.data());
        if (st == S2_OK) st = eng[k].enqueue(p, compute);
        return st;
    }

    // Wait for round k and hand its results to the jobs (caller holds no lock).
    void harvest_round(int k) {
        eng[k].wait();
        float ms[3] = {0.f, 0.f, 0.f};
        const bool timed = eng[k].timings(ms) == S2_OK;
        std::vector<Job *> completed;
        {
            std::lock_guard<std::mutex> lock(mu);
            if (timed) gpu_ms += (double)ms[0] + ms[1] + ms[2];
            const s2::DevResult *res = eng[k].results_h;
            for (size_t i = 0; i < round[k].size(); i++) {
                const RoundEntry &e = round[k][i];
                if (e.cand < 0) continue;
                Job *j = e.job;
                j->scores[e.cand] = res[i].score;
                j->status[e.cand] = res[i].status;
                j->inflight--;
                j->harvested++;
                pairs_done++;
            }
            for (auto it = queue.begin(); it != queue.end();) {
                Job *j = *it;
                const bool all = j->harvested == (int)j->cand_host.size();
                if (j->admitted && j->inflight == 0 && (all || (j->cancelled && j->ref_scheduled))) {
                    j->done_at = Clock::now();
                    j->finished = true;
                    if (j->cancelled && !all) j->job_status = S2_ERR_CANCELLED;
                    latencies_ms.push_back(std::chrono::duration<double, std::milli>(j->done_at - j->arrival).count());
                    jobs_done++;
                    completed.push_back(j);
                    it = queue.erase(it);
                } else {
                    ++it;
                }
            }
            for (Job *j : completed) {
                bytes_in_use -= j->bytes;
                // freed on the copy stream, where later jobs' memory is
                // allocated: the rounds that read it are complete (this
                // harvest waited for them), so reuse needs no wait on the
                // compute stream, whose queue already holds the next round
                cudaFreeAsync(j->dev, copy);
                j->dev = nullptr;
                float ms = 0.0f;
                if (cudaEventElapsedTime(&ms, j->up_start, j->uploaded) == cudaSuccess) copy_ms += ms;
                bytes_uploaded += (uint64_t)j->w * 3 * j->h * (1 + j->cand_host.size());
                cudaEventDestroy(j->uploaded);
                cudaEventDestroy(j->up_start);
                j->uploaded = j->up_start = nullptr;
            }
        }
        round[k].clear();
        inflight[k] = false;
        if (!completed.empty()) {
            cv_done.notify_all();
            cv_up.notify_one();  // budget freed
        }
    }

    // Round loop (worker thread): build a round from uploaded jobs, enqueue
    // it, harvest the previous one.
    void run() {
        int cur = 0;
        for (;;) {
            {
                std::unique_lock<std::mutex> lock(mu);
                build_round_locked(round[cur]);
                if (round[cur].empty() && !inflight[cur ^ 1]) {
                    if (stop && uploader_done) break;
                    cv_work.wait_for(lock, std::chrono::milliseconds(2));
                    continue;
                }
            }
            if (!round[cur].empty()) {
                const auto tb = Clock::now();
                s2_status st = submit_round(cur);
                t_submit += std::chrono::duration<double>(Clock::now() - tb).count();
                if (st != S2_OK) {
                    {
                        std::lock_guard<std::mutex> lock(mu);
                        fatal = st;
                        for (Job *j : queue) j->job_status = st;
                        stop = true;
                    }
                    cv_done.notify_all();
                    cv_up.notify_all();
                    break;
                }
                inflight[cur] = true;
                rounds++;
            }
            if (inflight[cur ^ 1]) {
                const auto tc = Clock::now();
                harvest_round(cur ^ 1);
                t_wait += std::chrono::duration<double>(Clock::now() - tc).count();
            }
            cur ^= 1;
        }
        for (int k = 0; k < 2; k++)
            if (inflight[k]) harvest_round(k);
    }
};

extern "C" {

void s2_server_config_default(s2_server_config *c) {
    if (!c) return;
    memset(c, 0, sizeof *c);
    c->struct_size = sizeof *c;
    c->device = 0;
    c->max_batch_pairs = 256;
    c->max_batch_pixels = 32ull << 20;
    c->hbm_budget = 40ull << 30;
    c->max_queued_jobs = 128;  // bounds the latency of an overloaded server
}

s2_status s2_server_create(const s2_server_config *cfg_in, s2_server **out) {
    if (!out) return S2_ERR_INVALID_ARG;
    *out = nullptr;
    s2_server_config cfg;
    if (cfg_in) cfg = *cfg_in;
    else s2_server_config_default(&cfg);
    if (cfg.struct_size != sizeof cfg || cfg.max_batch_pairs == 0 || cfg.max_batch_pixels == 0)
        return S2_ERR_INVALID_ARG;
    s2_server *sv = new (std::nothrow) s2_server();
    if (!sv) return S2_ERR_OOM;
    sv->cfg = cfg;
    s2_config ec;
    s2_config_default(&ec);
    ec.device = cfg.device;
    ec.strip_rows = kStripMid;  // fixed tile geometry: a job scores the same alone and mixed
    s2_status st = S2_OK;
    for (int k = 0; k < 2 && st == S2_OK; k++) st = sv->eng[k].init(&ec);
    for (int k = 0; k < 2 && st == S2_OK; k++) st = sv->eng[k].set_profiling(true);
    for (int k = 0; k < 2; k++) sv->eng[k].desc_kernel = true;
    for (int k = 0; k < 2 && st == S2_OK; k++) st = sv->eng[k].reserve(cfg.max_batch_pairs, cfg.max_batch_pixels, true);
    cudaMemPoolProps props;
    memset(&props, 0, sizeof props);
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = cfg.device;
    if (st == S2_OK && (cudaStreamCreateWithFlags(&sv->compute, cudaStreamNonBlocking) != cudaSuccess ||
                        cudaStreamCreateWithFlags(&sv->copy, cudaStreamNonBlocking) != cudaSuccess ||
                        cudaMemPoolCreate(&sv->pool, &props) != cudaSuccess))
        st = S2_ERR_CUDA;
    if (st == S2_OK) {
        uint64_t keep = cfg.hbm_budget ? cfg.hbm_budget : ~0ull;
        cudaMemPoolSetAttribute(sv->pool, cudaMemPoolAttrReleaseThreshold, &keep);
        // Job memory is allocated and freed on the copy stream; a block is
        // never reused through a wait on another stream (which would queue
        // new uploads behind a round of kernels)
        int no = 0;
        cudaMemPoolSetAttribute(sv->pool, cudaMemPoolReuseAllowInternalDependencies, &no);
        // Grow the pool to the budget once, here: growing it while serving
        // maps memory on the admission path (measured: 0.6 s of stalls while
        // a burst of jobs was admitted).  Without a budget, or when the
        // device cannot hold it, the pool grows on demand instead.
        if (cfg.hbm_budget > sv->workspace_bytes()) {
            void *p = nullptr;
            if (cudaMallocFromPoolAsync(&p, cfg.hbm_budget - sv->workspace_bytes(), sv->pool, sv->copy) == cudaSuccess) {
                cudaFreeAsync(p, sv->copy);
                cudaStreamSynchronize(sv->copy);
            }
            cudaGetLastError();
        }
    }
    if (st != S2_OK) {
        for (int k = 0; k < 2; k++) sv->eng[k].release();
        delete sv;
        return st;
    }
    sv->t0 = Clock::now();
    sv->worker = std::thread([sv] {
        cudaSetDevice(sv->cfg.device);
        sv->run();
    });
    sv->uploader = std::thread([sv] {
        cudaSetDevice(sv->cfg.device);
        sv->upload_loop();
    });
    *out = sv;
    return S2_OK;
}

void s2_server_destroy(s2_server *sv) {
    if (!sv) return;
    {
        std::lock_guard<std::mutex> lock(sv->mu);
        sv->stop = true;
        for (Job *j : sv->queue)
            if (!j->admitted) j->cancelled = true;
    }
    sv->cv_work.notify_all();
    sv->cv_up.notify_all();
    if (sv->uploader.joinable()) sv->uploader.join();
    if (sv->worker.joinable()) sv->worker.join();
    cudaSetDevice(sv->cfg.device);
    cudaStreamSynchronize(sv->compute);
    cudaStreamSynchronize(sv->copy);
    for (auto &kv : sv->jobs) {
        Job *j = kv.second;
        if (j->dev) cudaFree(j->dev);
        if (j->uploaded) cudaEventDestroy(j->uploaded);
        delete j;
    }
    for (int k = 0; k < 2; k++) sv->eng[k].release();
    if (sv->pool) cudaMemPoolDestroy(sv->pool);
    cudaStreamDestroy(sv->compute);
    cudaStreamDestroy(sv->copy);
    delete sv;
}

s2_status s2_server_submit(s2_server *sv, const s2_job_desc *jd, uint64_t *job_id) {
    if (!sv || !jd || !job_id || !jd->ref || (jd->n_candidates && !jd->candidates)) return S2_ERR_INVALID_ARG;
    if (jd->format != S2_FMT_SRGB8) return S2_ERR_INVALID_ARG;
    if (s2_num_scales(jd->width, jd->height, S2_SCALES_CPU) == 0 || jd->width > 65536 || jd->height > 65536)
        return S2_ERR_INVALID_SIZE;
    if (jd->ref_pitch < (size_t)jd->width * 3 || jd->cand_pitch < (size_t)jd->width * 3) return S2_ERR_DIM_MISMATCH;
    Job *j = new (std::nothrow) Job();
    if (!j) return S2_ERR_OOM;
    j->w = jd->width;
    j->h = jd->height;
    j->ref_host = (const uint8_t *)jd->ref;
    j->ref_pitch = jd->ref_pitch;
    j->cand_host.assign((const uint8_t *const *)jd->candidates, (const uint8_t *const *)jd->candidates + jd->n_candidates);
    j->cand_pitch = jd->cand_pitch;
    j->scores.assign(jd->n_candidates, 0.0);
    j->status.assign(jd->n_candidates, S2_ERR_NOT_READY);
    j->bytes = s2_server::job_bytes(*j, 4);
    std::lock_guard<std::mutex> lock(sv->mu);
    if (sv->fatal != S2_OK) {
        delete j;
        return sv->fatal;
    }
    if (sv->cfg.hbm_budget && j->bytes + sv->workspace_bytes() > sv->cfg.hbm_budget) {
        delete j;
        return S2_ERR_OOM;  // could never be admitted
    }
    if (sv->queue.size() >= sv->cfg.max_queued_jobs) {
        delete j;
        return S2_ERR_BUSY;
    }
    j->id = sv->next_id++;
    j->arrival = Clock::now();
    sv->queue.push_back(j);
    sv->jobs[j->id] = j;
    *job_id = j->id;
    sv->cv_up.notify_one();
    return S2_OK;
}

s2_status s2_server_wait(s2_server *sv, uint64_t job_id, uint32_t timeout_ms, double *scores, int32_t *statuses,
                         double *latency_ms) {
    if (!sv) return S2_ERR_INVALID_ARG;
    std::unique_lock<std::mutex> lock(sv->mu);
    auto it = sv->jobs.find(job_id);
    if (it == sv->jobs.end()) return S2_ERR_INVALID_ARG;
    Job *j = it->second;
    const bool ok = sv->cv_done.wait_for(lock, std::chrono::milliseconds(timeout_ms),
                                         [&] { return j->finished || sv->fatal != S2_OK; });
    if (!ok) return S2_ERR_TIMEOUT;
    if (!j->finished) return sv->fatal;
    const size_t k = j->cand_host.size();
    if (scores) memcpy(scores, j->scores.data(), k * sizeof(double));
    if (statuses) memcpy(statuses, j->status.data(), k * sizeof(int32_t));
    if (latency_ms) *latency_ms = std::chrono::duration<double, std::milli>(j->done_at - j->arrival).count();
    const s2_status st = j->job_status;
    sv->jobs.erase(it);
    delete j;
    return st;
}

s2_status s2_server_cancel(s2_server *sv, uint64_t job_id) {
    if (!sv) return S2_ERR_INVALID_ARG;
    std::lock_guard<std::mutex> lock(sv->mu);
    auto it = sv->jobs.find(job_id);
    if (it == sv->jobs.end()) return S2_ERR_INVALID_ARG;
    Job *j = it->second;
    if (j->finished) return S2_OK;
    j->cancelled = true;
    if (!j->admitted) {  // never reached the device: complete it now
        j->finished = true;
        j->job_status = S2_ERR_CANCELLED;
        j->done_at = Clock::now();
        sv->queue.erase(std::find(sv->queue.begin(), sv->queue.end(), j));
        sv->cv_done.notify_all();
    } else if (!j->ref_scheduled) {
        j->ref_scheduled = true;  // nothing in flight: the next harvest completes it
    }
    sv->cv_work.notify_all();
    return S2_OK;
}

s2_status s2_server_stats(s2_server *sv, s2_server_report *out) {
    if (!sv || !out) return S2_ERR_INVALID_ARG;
    std::lock_guard<std::mutex> lock(sv->mu);
    memset(out, 0, sizeof *out);
    out->jobs_done = sv->jobs_done;
    out->pairs_done = sv->pairs_done;
    out->rounds = sv->rounds;
    out->queued_jobs = sv->queue.size();
    out->hbm_in_use = sv->bytes_in_use + sv->workspace_bytes();
    std::vector<double> l = sv->latencies_ms;
    if (!l.empty()) {
        std::sort(l.begin(), l.end());
        out->p50_ms = l[(size_t)(0.50 * (l.size() - 1))];
        out->p99_ms = l[(size_t)(0.99 * (l.size() - 1))];
        out->max_ms = l.back();
    }
    out->uptime_s = std::chrono::duration<double>(Clock::now() - sv->t0).count();
    out->gpu_busy_s = sv->gpu_ms / 1e3;
    out->worker_wait_s = sv->t_wait;
    out->worker_upload_s = sv->t_upload;
    out->worker_submit_s = sv->t_submit;
    out->copy_busy_s = sv->copy_ms / 1e3;
    out->bytes_uploaded = sv->bytes_uploaded;
    return S2_OK;
}

s2_status s2_server_reset_stats(s2_server *sv) {
    if (!sv) return S2_ERR_INVALID_ARG;
    std::lock_guard<std::mutex> lock(sv->mu);
    sv->latencies_ms.clear();
    sv->pairs_done = sv->jobs_done = sv->rounds = 0;
    sv->gpu_ms = 0.0;
    sv->t_wait = sv->t_upload = sv->t_submit = 0.0;
    sv->copy_ms = 0.0;
    sv->bytes_uploaded = 0;
    sv->t0 = Clock::now();
    return S2_OK;
}

}  // extern "C"
