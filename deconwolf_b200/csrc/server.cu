// server.cu -- a deconvolution request server on one GPU (continuous batching).
//
// Requests (an image, a PSF, options: the arguments of one dw_function call)
// are queued by dwcu_server_submit from any thread.  One worker thread per
// server admits them in arrival order while their device memory fits the HBM
// budget (and at most max_active run at once), keeps every admitted job's
// state (image, OTF, weights, x_k, x_{k-1}) resident, gives each job its own
// stream, and interleaves their iterations: every turn it tops up each job
// that has fewer than two chunks of iterations in flight with one more chunk.
// Jobs of different sizes therefore overlap on the device; a request that
// arrives while others run is admitted as soon as memory frees up.  The
// result is copied to the caller's buffer and the request's latency (submit
// to result on the host) recorded.
//
// A job's arithmetic does not depend on what runs beside it, so a result is
// the same as that of dwcu_deconvolve on the same inputs.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstdarg>
#include <cstdio>
#include <cstdint>
#include <cstring>
#include <deque>
#include <map>
#include <mutex>
#include <thread>
#include <vector>

#include "../../include/dwcu.h"

namespace dwcu {
void record_error(const char *msg);
}

namespace {

using clk = std::chrono::steady_clock;

int sfail(int code, const char *fmt, ...)
{
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    dwcu::record_error(buf);
    return code;
}

struct Request {
    int64_t id = 0;
    const float *im = nullptr, *psf = nullptr;
    int64_t M = 0, N = 0, P = 0, pM = 0, pN = 0, pP = 0;
    dwcu_opts opts{};
    float *out = nullptr;
    int64_t need = 0;  // device bytes of the job
    clk::time_point t_submit;
    // state
    int status = DWCU_ERROR_NOT_READY;
    bool cancel = false;
    dwcu_opts result{};
    double latency_s = 0;
    // while active
    dwcu_job *job = nullptr;
    cudaStream_t stream = nullptr;
    std::deque<cudaEvent_t> inflight;  // one event per chunk not yet known complete
    int remaining = 0;
    // faults a pageable result buffer in while the request waits and runs
    std::thread prefault;
    void join_prefault()
    {
        if (prefault.joinable()) prefault.join();
    }
    ~Request() { join_prefault(); }
};

}  // namespace

struct dwcu_server {
    int device = 0;
    double budget = 0;
    int max_active = 8;
    int chunk = 5;
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::map<int64_t, Request *> all;
    std::deque<Request *> queue;
    std::vector<Request *> active;
    double used = 0;
    int64_t next_id = 1;
    bool stop = false;
    std::thread worker;
    // statistics
    int64_t submitted = 0, completed = 0, failed = 0, cancelled = 0;
    std::vector<double> latencies;
    double vox_iters = 0;
    clk::time_point t_first, t_last;
    bool have_first = false;
    std::vector<cudaEvent_t> event_pool;

    cudaEvent_t get_event()
    {
        if (!event_pool.empty()) {
            cudaEvent_t e = event_pool.back();
            event_pool.pop_back();
            return e;
        }
        cudaEvent_t e = nullptr;
        cudaEventCreateWithFlags(&e, cudaEventDisableTiming);
        return e;
    }
    void put_event(cudaEvent_t e) { event_pool.push_back(e); }

    void finish(Request *r, int status)
    {
        // called by the worker without the lock held; the job's stream is idle
        r->join_prefault();
        if (r->job) {
            dwcu_job_destroy(r->job);
            r->job = nullptr;
        }
        for (cudaEvent_t e : r->inflight) put_event(e);
        r->inflight.clear();
        if (r->stream) {
            cudaStreamDestroy(r->stream);
            r->stream = nullptr;
        }
        std::lock_guard<std::mutex> lk(mu);
        used -= (double) r->need;
        active.erase(std::remove(active.begin(), active.end(), r), active.end());
        r->status = status;
        const auto now = clk::now();
        r->latency_s = std::chrono::duration<double>(now - r->t_submit).count();
        if (status == DWCU_SUCCESS) {
            ++completed;
            latencies.push_back(r->latency_s);
            vox_iters += (double) (r->M * r->N * r->P) * (double) r->result.iterations_done;
            t_last = now;
        } else if (status == DWCU_ERROR_CANCELLED) {
            ++cancelled;
        } else {
            ++failed;
        }
        cv_done.notify_all();
    }

    // start a request: job, stream, upload and setup (blocks on this job's stream)
    int start(Request *r)
    {
        int rc = dwcu_job_create(r->M, r->N, r->P, r->pM, r->pN, r->pP, &r->opts, &r->job);
        if (rc) return rc;
        if (cudaStreamCreateWithFlags(&r->stream, cudaStreamNonBlocking) != cudaSuccess)
            return sfail(DWCU_ERROR_CUDA, "stream creation failed");
        dwcu_job_set_stream(r->job, r->stream);
        rc = dwcu_job_setup(r->job, r->im, r->psf, 0);
        if (rc) return rc;
        r->remaining = std::max(r->opts.n_iter, r->opts.maxiter);
        return DWCU_SUCCESS;
    }

    // one more chunk of iterations on the job's stream
    int step(Request *r)
    {
        int32_t rem = 0;
        int rc = dwcu_job_step(r->job, chunk, &rem);
        if (rc) return rc;
        r->remaining = rem;
        cudaEvent_t e = get_event();
        if (cudaEventRecord(e, r->stream) != cudaSuccess) {
            put_event(e);
            return sfail(DWCU_ERROR_CUDA, "event record failed");
        }
        r->inflight.push_back(e);
        return DWCU_SUCCESS;
    }

    void run()
    {
        cudaSetDevice(device);
        for (;;) {
            // admit in arrival order while memory and slots allow
            std::vector<Request *> to_start;
            {
                std::unique_lock<std::mutex> lk(mu);
                if (stop && queue.empty() && active.empty()) return;
                while (!queue.empty() && (int) active.size() + (int) to_start.size() < max_active) {
                    Request *r = queue.front();
                    if (r->cancel) {
                        r->join_prefault();  // the caller may free the buffer once it sees the status
                        queue.pop_front();
                        r->status = DWCU_ERROR_CANCELLED;
                        ++cancelled;
                        cv_done.notify_all();
                        continue;
                    }
                    const bool idle = active.empty() && to_start.empty();
                    if (!idle && used + (double) r->need > budget) break;
                    queue.pop_front();
                    used += (double) r->need;
                    active.push_back(r);
                    to_start.push_back(r);
                }
                if (active.empty() && queue.empty()) {
                    cv_work.wait_for(lk, std::chrono::milliseconds(50));
                    continue;
                }
            }
            bool progressed = false;
            // keep the running jobs fed before any blocking setup
            std::vector<Request *> act;
            {
                std::lock_guard<std::mutex> lk(mu);
                act = active;
            }
            for (Request *r : act) {
                if (!r->job) continue;
                while (!r->inflight.empty() && cudaEventQuery(r->inflight.front()) == cudaSuccess) {
                    put_event(r->inflight.front());
                    r->inflight.pop_front();
                    progressed = true;
                }
                bool cancel;
                {
                    std::lock_guard<std::mutex> lk(mu);
                    cancel = r->cancel;
                }
                if (cancel) {
                    cudaStreamSynchronize(r->stream);
                    finish(r, DWCU_ERROR_CANCELLED);
                    progressed = true;
                    continue;
                }
                if (dwcu_job_done(r->job)) {
                    if (!r->inflight.empty()) continue;  // its last chunk is still running
                    r->result = r->opts;
                    r->result.error_trace = r->opts.error_trace;
                    r->result.trace_capacity = r->opts.trace_capacity;
                    r->join_prefault();
                    const int rc = dwcu_job_result(r->job, r->out, 0, &r->result);
                    finish(r, rc);
                    progressed = true;
                    continue;
                }
                if (r->inflight.size() < 2) {
                    const int rc = step(r);
                    if (rc) {
                        cudaStreamSynchronize(r->stream);
                        finish(r, rc);
                    }
                    progressed = true;
                }
            }
            for (Request *r : to_start) {
                const int rc = start(r);
                if (rc) {
                    if (r->stream) cudaStreamSynchronize(r->stream);
                    finish(r, rc);
                } else {
                    const int rc2 = step(r);
                    if (rc2) {
                        cudaStreamSynchronize(r->stream);
                        finish(r, rc2);
                    }
                }
                progressed = true;
            }
            if (!progressed) std::this_thread::sleep_for(std::chrono::microseconds(200));
        }
    }
};

extern "C" {

int dwcu_server_create(int32_t device, double hbm_budget, int32_t max_active, int32_t iters_per_turn,
                       dwcu_server **out)
{
    if (!out) return sfail(DWCU_ERROR_INVALID_VALUE, "out is NULL");
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) {
        cudaGetLastError();
        return sfail(DWCU_ERROR_CUDA, "no CUDA device available (the engine has no CPU path)");
    }
    if (device < 0 || device >= n) return sfail(DWCU_ERROR_INVALID_VALUE, "device %d out of range", device);
    auto *sv = new dwcu_server();
    sv->device = device;
    if (hbm_budget <= 0) {
        size_t fr = 0, tot = 0;
        cudaSetDevice(device);
        cudaMemGetInfo(&fr, &tot);
        hbm_budget = 0.85 * (double) fr;
    }
    sv->budget = hbm_budget;
    sv->max_active = max_active > 0 ? max_active : 8;
    sv->chunk = iters_per_turn > 0 ? iters_per_turn : 5;
    sv->worker = std::thread([sv] { sv->run(); });
    *out = sv;
    return DWCU_SUCCESS;
}

int dwcu_server_submit(dwcu_server *sv, const float *im, int64_t M, int64_t N, int64_t P, const float *psf,
                       int64_t pM, int64_t pN, int64_t pP, const dwcu_opts *s, float *out, int64_t *id)
{
    if (!sv || !im || !psf || !s || !out || !id) return sfail(DWCU_ERROR_INVALID_VALUE, "NULL argument");
    if (s->device != sv->device) return sfail(DWCU_ERROR_INVALID_VALUE, "request device differs from the server's");
    int64_t work[3], need = 0;
    int rc = dwcu_plan_size(M, N, P, pM, pN, pP, s->border_quality, s->method, work, &need);
    if (rc) return rc;
    auto *r = new Request();
    r->im = im; r->psf = psf; r->out = out;
    r->M = M; r->N = N; r->P = P; r->pM = pM; r->pN = pN; r->pP = pP;
    r->opts = *s;
    r->need = need;
    r->t_submit = clk::now();
    {
        // (asked on the server's device; the caller's current device is restored)
        int cur = 0;
        const bool had = cudaGetDevice(&cur) == cudaSuccess;
        cudaSetDevice(sv->device);
        cudaPointerAttributes pa;
        const bool locked = cudaPointerGetAttributes(&pa, out) == cudaSuccess && pa.type == cudaMemoryTypeHost;
        cudaGetLastError();
        if (had) cudaSetDevice(cur);
        // (not when the result overwrites the image, which is uploaded later)
        const size_t n = (size_t) (M * N * P);
        const uintptr_t o0 = (uintptr_t) out, i0 = (uintptr_t) im, nb = sizeof(float) * n;
        const bool overlap = o0 < i0 + nb && i0 < o0 + nb;
        if (!locked && !overlap) {
            r->prefault = std::thread([out, n]() {
                const size_t chunk = (size_t) 1 << 22;
                for (size_t i = 0; i < n; i += chunk) memset(out + i, 0, sizeof(float) * std::min(chunk, n - i));
            });
        }
    }
    std::lock_guard<std::mutex> lk(sv->mu);
    if (sv->stop) {
        delete r;
        return sfail(DWCU_ERROR_INVALID_VALUE, "the server is shutting down");
    }
    r->id = sv->next_id++;
    sv->all[r->id] = r;
    sv->queue.push_back(r);
    ++sv->submitted;
    if (!sv->have_first) {
        sv->have_first = true;
        sv->t_first = r->t_submit;
    }
    *id = r->id;
    sv->cv_work.notify_all();
    return DWCU_SUCCESS;
}

int dwcu_server_wait(dwcu_server *sv, int64_t id, double timeout_s, dwcu_opts *s_out)
{
    if (!sv) return sfail(DWCU_ERROR_INVALID_VALUE, "server is NULL");
    std::unique_lock<std::mutex> lk(sv->mu);
    auto it = sv->all.find(id);
    if (it == sv->all.end()) return sfail(DWCU_ERROR_INVALID_VALUE, "unknown request %lld", (long long) id);
    Request *r = it->second;
    auto pred = [r] { return r->status != DWCU_ERROR_NOT_READY; };
    if (timeout_s < 0)
        sv->cv_done.wait(lk, pred);
    else if (!sv->cv_done.wait_for(lk, std::chrono::duration<double>(timeout_s), pred))
        return DWCU_ERROR_NOT_READY;
    if (s_out) {
        float *tr = s_out->error_trace;
        const int32_t cap = s_out->trace_capacity;
        *s_out = r->result;
        s_out->error_trace = tr;
        s_out->trace_capacity = cap;
    }
    if (r->status != DWCU_SUCCESS && r->status != DWCU_ERROR_CANCELLED)
        return sfail(r->status, "request %lld failed (status %d)", (long long) id, r->status);
    return r->status;
}

int dwcu_server_cancel(dwcu_server *sv, int64_t id)
{
    if (!sv) return sfail(DWCU_ERROR_INVALID_VALUE, "server is NULL");
    std::lock_guard<std::mutex> lk(sv->mu);
    auto it = sv->all.find(id);
    if (it == sv->all.end()) return sfail(DWCU_ERROR_INVALID_VALUE, "unknown request %lld", (long long) id);
    it->second->cancel = true;
    sv->cv_work.notify_all();
    return DWCU_SUCCESS;
}

int dwcu_server_get_stats(dwcu_server *sv, dwcu_server_stats *st)
{
    if (!sv || !st) return sfail(DWCU_ERROR_INVALID_VALUE, "NULL argument");
    std::lock_guard<std::mutex> lk(sv->mu);
    st->submitted = sv->submitted;
    st->completed = sv->completed;
    st->failed = sv->failed;
    st->cancelled = sv->cancelled;
    st->active = (int64_t) sv->active.size();
    st->queued = (int64_t) sv->queue.size();
    st->device_bytes_in_use = sv->used;
    std::vector<double> l = sv->latencies;
    std::sort(l.begin(), l.end());
    auto pct = [&](double p) {
        if (l.empty()) return 0.0;
        const size_t k = (size_t) std::min<double>((double) l.size() - 1, std::ceil(p * (double) l.size()) - 1);
        return l[k];
    };
    st->latency_p50_s = pct(0.50);
    st->latency_p99_s = pct(0.99);
    double sum = 0;
    for (double v : l) sum += v;
    st->latency_mean_s = l.empty() ? 0 : sum / (double) l.size();
    st->voxel_iterations = sv->vox_iters;
    st->wall_s = sv->have_first && sv->completed ? std::chrono::duration<double>(sv->t_last - sv->t_first).count() : 0;
    return DWCU_SUCCESS;
}

void dwcu_server_destroy(dwcu_server *sv)
{
    if (!sv) return;
    {
        std::lock_guard<std::mutex> lk(sv->mu);
        for (Request *r : sv->queue) r->cancel = true;
        sv->stop = true;
        sv->cv_work.notify_all();
    }
    if (sv->worker.joinable()) sv->worker.join();
    for (auto &kv : sv->all) delete kv.second;
    cudaSetDevice(sv->device);
    for (cudaEvent_t e : sv->event_pool) cudaEventDestroy(e);
    delete sv;
}

}  // extern "C"
