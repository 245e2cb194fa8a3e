// fvm_serve.cu -- request loop over a batch (C ABI fvm_server_*): continuous
// batching of independent solves.  No reference counterpart.
//
// Client threads submit requests into an arrival-ordered queue.  One worker
// thread owns the batch and repeats:
//   1. admit queued requests in order while an instance slot is free and the
//      admitted solves' memory estimate stays inside the budget (a request
//      that can never fit is rejected; the queue head that does not fit yet
//      blocks the ones behind it, so admission stays first come first served);
//   2. advance every admitted solve by k batched steps, k = the fewest steps
//      any admitted solve still needs, capped by the chunk size -- so at least
//      one solve finishes at every chunk end and new arrivals wait at most one
//      chunk.  The chunk is queued asynchronously; requests that arrive while
//      it runs are admitted (their set-up runs on the batch's admission
//      stream, overlapping the chunk) and join at the next chunk;
//   3. retire the solves that reached their step count: final state to the
//      caller's arrays, diagnostics into the result, instance parked for reuse.
// Retired instances keep their device memory and are reset in place when a
// request of the same grid size arrives; parked memory is freed (oldest
// first) whenever an admission needs it to stay inside the budget.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <deque>
#include <map>
#include <mutex>
#include <thread>
#include <vector>

#include "fvm_handle.h"

namespace {

struct Request {
    long long ticket = 0;
    fvm_sim_params p{};
    int steps = 0;
    float *out[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};
    double submit_s = 0, admit_s = 0;
    int id = -1;       // batch instance id once admitted
    int done = 0;      // steps taken
    size_t bytes = 0;  // admission estimate
};

using Clock = std::chrono::steady_clock;

}  // namespace

struct fvm_server {
    fvm_batch *b = nullptr;
    int device = 0;
    size_t budget = 0;
    int max_active = 0;
    int chunk = 64;
    Clock::time_point t0;
    std::thread worker;
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::deque<Request> pending;
    std::vector<Request> active;
    std::deque<fvm_result> ready;  // finished, not yet collected (completion order)
    long long next_ticket = 1;
    long long submitted = 0, completed = 0, rejected = 0, batched_steps = 0;
    size_t active_bytes = 0, parked_bytes = 0;
    double cell_updates = 0, busy_s = 0;
    std::vector<float> step_ms;  // device time of each batched step
    bool stop = false;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    cudaStream_t stream = nullptr;

    double now() const { return std::chrono::duration<double>(Clock::now() - t0).count(); }
};

static int serr(int code, const char *msg) { return fvm_internal_set_error(code, msg); }

// Result record of a request that ends without running (rejected or cancelled).
static fvm_result unrun(const Request &r, int status, double t) {
    fvm_result x;
    memset(&x, 0, sizeof x);
    x.ticket = r.ticket;
    x.status = status;
    x.nx = r.p.nx;
    x.ny = r.p.ny;
    x.submit_s = r.submit_s;
    x.admit_s = -1.0;
    x.done_s = t;
    return x;
}

// Worker side: admit from the queue head.  Called with the lock held; drops
// it around the batch calls.
static void admit(fvm_server *s, std::unique_lock<std::mutex> &lk) {
    while (!s->pending.empty() && (s->max_active <= 0 || (int)s->active.size() < s->max_active)) {
        Request &head = s->pending.front();
        const size_t need = fvm_batch_instance_bytes(head.p.nx, head.p.ny);
        if (need > s->budget) {
            s->ready.push_back(unrun(head, FVM_ERR_BUDGET, s->now()));
            s->rejected++;
            s->pending.pop_front();
            s->cv_done.notify_all();
            continue;
        }
        if (s->active_bytes + need > s->budget) break;  // wait for retirements
        Request r = head;
        s->pending.pop_front();
        lk.unlock();
        // keep admitted + parked memory inside the budget: free parked
        // instances unless one of this size will be reused
        size_t parked = 0;
        if (!fvm_internal_batch_has_parked(s->b, r.p.nx, r.p.ny))
            fvm_batch_trim(s->b, s->budget - s->active_bytes - need, &parked);
        int id = -1;
        const int rc = fvm_batch_add(s->b, &r.p, &id);
        fvm_batch_trim(s->b, (size_t)-1, &parked);
        lk.lock();
        s->parked_bytes = parked;
        if (rc != FVM_OK) {
            s->ready.push_back(unrun(r, rc, s->now()));
            s->completed++;
            s->cv_done.notify_all();
            continue;
        }
        r.id = id;
        r.bytes = need;
        r.admit_s = s->now();
        s->active_bytes += need;
        s->active.push_back(r);
    }
}

// Worker side: collect the final state of a finished request and park its instance.
static fvm_result retire(fvm_server *s, const Request &r, int status) {
    fvm_result x;
    memset(&x, 0, sizeof x);
    x.ticket = r.ticket;
    x.nx = r.p.nx;
    x.ny = r.p.ny;
    x.steps = r.done;
    x.submit_s = r.submit_s;
    x.admit_s = r.admit_s;
    int rc = status;
    if (rc == FVM_OK && (r.out[0] || r.out[1] || r.out[2] || r.out[3] || r.out[4]))
        rc = fvm_batch_read_fields(s->b, r.id, r.out[0], r.out[1], r.out[2], r.out[3], r.out[4]);
    if (rc == FVM_OK) rc = fvm_batch_diagnostics(s->b, r.id, &x.diag);
    fvm_sim_params q;
    if (rc == FVM_OK && (rc = fvm_batch_instance(s->b, r.id, &q)) == FVM_OK) {
        x.t_final = q.t_current;
        x.dt_last = q.dt;
    }
    unsigned long long nonfinite = 0;
    if (rc == FVM_OK) rc = fvm_batch_nonfinite_count(s->b, r.id, &nonfinite);
    if (rc == FVM_OK && (nonfinite > 0 || !(std::isfinite(x.diag.mass) && std::isfinite(x.diag.energy) &&
                                            std::isfinite(x.diag.cd))))
        rc = FVM_ERR_NONFINITE;
    fvm_batch_retire(s->b, r.id);
    x.status = rc;
    x.done_s = s->now();
    return x;
}

static void worker_main(fvm_server *s) {
    cudaSetDevice(s->device);
    std::unique_lock<std::mutex> lk(s->mu);
    for (;;) {
        s->cv_work.wait(lk, [&] { return s->stop || !s->pending.empty() || !s->active.empty(); });
        if (s->stop) break;
        admit(s, lk);
        if (s->active.empty()) continue;
        int k = s->chunk;
        double cells = 0;
        for (const Request &r : s->active) {
            k = std::min(k, r.steps - r.done);
            cells += (double)r.p.nx * r.p.ny;
        }
        const size_t stepping = s->active.size();  // solves in this chunk
        lk.unlock();
        int rc = FVM_OK;
        float ms = 0.0f;
        if (k > 0) {
            cudaEventRecord(s->ev0, s->stream);
            rc = fvm_batch_step(s->b, k);
            cudaEventRecord(s->ev1, s->stream);
        }
        lk.lock();
        // admit arrivals while the chunk runs; they join at the next chunk
        if (rc == FVM_OK) admit(s, lk);
        lk.unlock();
        if (k > 0) {
            if (rc == FVM_OK) rc = fvm_batch_synchronize(s->b);
            if (rc == FVM_OK && cudaEventElapsedTime(&ms, s->ev0, s->ev1) != cudaSuccess) ms = 0.0f;
        }
        lk.lock();
        if (rc == FVM_OK && k > 0) {
            s->batched_steps += k;
            s->busy_s += ms * 1e-3;
            s->cell_updates += cells * k;
            s->step_ms.insert(s->step_ms.end(), (size_t)k, ms / k);
        }
        // retire finished solves (all of them if the chunk failed); solves
        // admitted during the chunk (index >= stepping) did not step
        std::vector<Request> keep;
        for (size_t idx = 0; idx < s->active.size(); idx++) {
            Request &r = s->active[idx];
            if (idx >= stepping && rc == FVM_OK) {
                keep.push_back(r);
                continue;
            }
            if (rc == FVM_OK) r.done += k;
            if (rc != FVM_OK || r.done >= r.steps) {
                lk.unlock();
                fvm_result x = retire(s, r, rc);
                size_t parked = 0;
                fvm_batch_trim(s->b, (size_t)-1, &parked);
                lk.lock();
                s->parked_bytes = parked;
                s->active_bytes -= r.bytes;
                s->ready.push_back(x);
                s->completed++;
            } else {
                keep.push_back(r);
            }
        }
        s->active.swap(keep);
        s->cv_done.notify_all();
    }
    // cancelled: everything not finished
    const double t = s->now();
    for (const Request &r : s->pending) s->ready.push_back(unrun(r, FVM_ERR_STATE, t));
    for (const Request &r : s->active) s->ready.push_back(unrun(r, FVM_ERR_STATE, t));
    s->pending.clear();
    s->active.clear();
    s->cv_done.notify_all();
}

extern "C" int fvm_server_create(fvm_server **out, const fvm_ext *ext, size_t hbm_budget_bytes, int max_active,
                                 int max_chunk_steps) {
    if (!out) return serr(FVM_ERR_INVALID, "null out");
    *out = nullptr;
    if (hbm_budget_bytes == 0) return serr(FVM_ERR_INVALID, "fvm_server_create: zero memory budget");
    if (max_chunk_steps < 0 || max_active < 0) return serr(FVM_ERR_INVALID, "fvm_server_create: negative limit");
    fvm_server *s = new fvm_server();
    if (int r = fvm_batch_create(&s->b, ext)) {
        delete s;
        return r;
    }
    cudaGetDevice(&s->device);
    s->budget = hbm_budget_bytes;
    s->max_active = max_active;
    s->chunk = max_chunk_steps > 0 ? max_chunk_steps : 64;
    if (cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreate(&s->ev0) != cudaSuccess || cudaEventCreate(&s->ev1) != cudaSuccess) {
        fvm_batch_destroy(s->b);
        delete s;
        return serr(FVM_ERR_CUDA, "fvm_server_create: stream/event creation failed");
    }
    fvm_batch_set_stream(s->b, s->stream);
    s->t0 = Clock::now();
    s->worker = std::thread(worker_main, s);
    *out = s;
    return FVM_OK;
}

extern "C" int fvm_server_submit(fvm_server *s, const fvm_sim_params *p, int steps, float *rho, float *rho_u,
                                 float *rho_v, float *E, float *rho_e, long long *ticket_out) {
    if (!s || !p || !ticket_out) return serr(FVM_ERR_INVALID, "null argument");
    if (steps <= 0) return serr(FVM_ERR_INVALID, "fvm_server_submit: steps must be positive");
    if (p->nx <= 0 || p->ny <= 0) return serr(FVM_ERR_INVALID, "fvm_server_submit: nx, ny must be positive");
    Request r;
    r.p = *p;
    r.steps = steps;
    float *o[5] = {rho, rho_u, rho_v, E, rho_e};
    for (int k = 0; k < 5; k++) r.out[k] = o[k];
    {
        std::lock_guard<std::mutex> g(s->mu);
        if (s->stop) return serr(FVM_ERR_STATE, "fvm_server_submit: server is stopping");
        r.ticket = s->next_ticket++;
        r.submit_s = s->now();
        s->pending.push_back(r);
        s->submitted++;
    }
    s->cv_work.notify_one();
    *ticket_out = r.ticket;
    return FVM_OK;
}

extern "C" int fvm_server_poll(fvm_server *s, fvm_result *out, int cap, int *n_out) {
    if (!s || !n_out || (cap > 0 && !out)) return serr(FVM_ERR_INVALID, "null argument");
    std::lock_guard<std::mutex> g(s->mu);
    int n = 0;
    while (n < cap && !s->ready.empty()) {
        out[n++] = s->ready.front();
        s->ready.pop_front();
    }
    *n_out = n;
    return FVM_OK;
}

extern "C" int fvm_server_wait(fvm_server *s, long long ticket, double timeout_s, fvm_result *out) {
    if (!s || !out) return serr(FVM_ERR_INVALID, "null argument");
    std::unique_lock<std::mutex> lk(s->mu);
    if (ticket <= 0 || ticket >= s->next_ticket) return serr(FVM_ERR_INVALID, "fvm_server_wait: unknown ticket");
    auto found = [&] {
        for (auto it = s->ready.begin(); it != s->ready.end(); ++it)
            if (it->ticket == ticket) {
                *out = *it;
                s->ready.erase(it);
                return true;
            }
        return false;
    };
    if (timeout_s < 0) {
        s->cv_done.wait(lk, found);
        return FVM_OK;
    }
    if (s->cv_done.wait_for(lk, std::chrono::duration<double>(timeout_s), found)) return FVM_OK;
    return serr(FVM_ERR_TIMEOUT, "fvm_server_wait: request not finished in time");
}

extern "C" int fvm_server_drain(fvm_server *s, double timeout_s) {
    if (!s) return serr(FVM_ERR_INVALID, "null server");
    std::unique_lock<std::mutex> lk(s->mu);
    auto idle = [&] { return s->pending.empty() && s->active.empty(); };
    if (timeout_s < 0) {
        s->cv_done.wait(lk, idle);
        return FVM_OK;
    }
    if (s->cv_done.wait_for(lk, std::chrono::duration<double>(timeout_s), idle)) return FVM_OK;
    return serr(FVM_ERR_TIMEOUT, "fvm_server_drain: requests still running");
}

static double percentile(std::vector<float> v, double q) {
    if (v.empty()) return 0.0;
    const size_t k = std::min(v.size() - 1, (size_t)std::floor(q * (double)(v.size() - 1) + 0.5));
    std::nth_element(v.begin(), v.begin() + (long)k, v.end());
    return v[k];
}

extern "C" int fvm_server_get_stats(fvm_server *s, fvm_server_stats *out) {
    if (!s || !out) return serr(FVM_ERR_INVALID, "null argument");
    std::vector<float> ms;
    {
        std::lock_guard<std::mutex> g(s->mu);
        memset(out, 0, sizeof *out);
        out->submitted = s->submitted;
        out->completed = s->completed;
        out->rejected = s->rejected;
        out->batched_steps = s->batched_steps;
        out->active = (int)s->active.size();
        out->pending = (int)s->pending.size();
        out->budget_bytes = s->budget;
        out->active_bytes = s->active_bytes;
        out->parked_bytes = s->parked_bytes;
        out->cell_updates = s->cell_updates;
        out->busy_s = s->busy_s;
        ms = s->step_ms;
    }
    double sum = 0;
    for (float x : ms) sum += x;
    out->step_ms_mean = ms.empty() ? 0.0 : sum / (double)ms.size();
    out->step_ms_p50 = percentile(ms, 0.50);
    out->step_ms_p99 = percentile(ms, 0.99);
    return FVM_OK;
}

extern "C" int fvm_server_destroy(fvm_server *s) {
    if (!s) return FVM_OK;
    {
        std::lock_guard<std::mutex> g(s->mu);
        s->stop = true;
    }
    s->cv_work.notify_all();
    if (s->worker.joinable()) s->worker.join();
    fvm_batch_destroy(s->b);
    if (s->ev0) cudaEventDestroy(s->ev0);
    if (s->ev1) cudaEventDestroy(s->ev1);
    if (s->stream) cudaStreamDestroy(s->stream);
    delete s;
    return FVM_OK;
}
