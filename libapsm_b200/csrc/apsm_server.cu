// Request server over a detector pool (the apsm_server_* entry points of
// include/apsm_b200.h): continuous batching of per-TTI train / detect
// requests.
//
// A worker thread owns the pool's lanes.  It completes the batches whose GPU
// work finished (estimates handed to the callers) and, for every idle lane,
// admits the oldest waiting requests into a new batch:
//   * a detector with a batch in flight is not admitted again until that
//     batch finished (its resident state is in use), and its later requests
//     keep their order: once one of a detector's requests waits, all of its
//     later ones wait too;
//   * a detection request is not put before a training request of the same
//     detector that arrived earlier (a batch runs its training jobs first);
//   * the batch is bounded by a request count and by the device scratch the
//     pool's HBM budget leaves per lane (apsm_pool_job_bytes);
//   * a batch holds one kind of request, that of its oldest admitted request,
//     so detections never wait behind a training sweep in the same batch
//     (a detector whose next request is of the other kind waits for a later
//     batch, keeping its order).
// Batches on different lanes overlap on the device.  Request times are taken
// with a monotonic host clock: submission, admission and completion.
//
// Failure model (the reference's is CUDA_CHECK: print and exit, cpp/lib/cuda/
// cuda_errorhandling.cuh:98-134).  Every ticket ends with a status:
//   * a request that is not admitted into a batch by its deadline is dropped
//     (APSM_ERR_DEADLINE); one admitted in time runs to completion, and its
//     completion time tells whether it finished late;
//   * apsm_server_cancel ends a request that is not admitted yet
//     (APSM_ERR_CANCELLED);
//   * a malformed request (unknown detector or kind, missing buffer) or one
//     whose scratch alone exceeds the pool's HBM budget is rejected at
//     submission: no ticket, so it can never fail the batch it would join;
//   * a batch whose launch fails (e.g. its lane's scratch cannot grow) ends
//     its requests with that status; the pool and the server stay usable.
// Fault injection for tests of these paths is host-side only: the pool can
// fail its next lane-scratch growths (apsm_pool_inject_fault) and the server
// can lose its next submitted requests (apsm_server_inject_fault), which then
// end only by their deadline or a cancel.
#include "apsm_b200.h"

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <mutex>
#include <string>
#include <thread>
#include <unordered_map>
#include <unordered_set>
#include <vector>

namespace {

double now_s()
{
    using namespace std::chrono;
    return duration<double>(steady_clock::now().time_since_epoch()).count();
}

struct ServerReq {
    apsm_job job;
    double t_submit = 0, t_start = 0, t_done = 0;
    double deadline = 0; // server clock, 0: none
    apsm_status st = APSM_OK;
    int state = 0; // 0 waiting, 1 running, 2 done
    bool lost = false; // dropped on the way in (fault injection): never queued
};

} // namespace

struct apsm_server {
    apsm_pool* pool = nullptr;
    uint32_t max_batch = 64;
    uint32_t n_lanes = 1;
    std::thread worker;
    std::mutex mu;
    std::condition_variable cv_submit, cv_done;
    bool stop = false;
    std::deque<uint64_t> queue;
    std::unordered_map<uint64_t, ServerReq> reqs;
    std::vector<std::vector<uint64_t>> lane_reqs;
    std::vector<char> lane_busy;
    std::unordered_set<uint32_t> busy_dets;
    uint64_t next_ticket = 1;
    uint64_t batches = 0, batched = 0;
    uint64_t dropped = 0, cancelled = 0, rejected = 0;
    double default_deadline = 0; // seconds after submission, 0: none
    uint32_t fault_drop = 0;     // requests still to lose on submission (fault injection)
    std::unordered_set<uint64_t> lost;

    void run();
    void complete(uint32_t lane, apsm_status st);
    void finish_one(uint64_t tk, apsm_status st, double t);
    void expire(double t);
    double next_deadline() const;
    bool admit(uint32_t lane);
};

void apsm_server::finish_one(uint64_t tk, apsm_status st, double t)
{
    auto it = reqs.find(tk);
    if (it == reqs.end()) return;
    it->second.state = 2;
    it->second.st = st;
    it->second.t_done = t;
    cv_done.notify_all();
}

// Drops the waiting (and lost) requests whose deadline passed; called with mu held.
void apsm_server::expire(double t)
{
    for (auto it = queue.begin(); it != queue.end();) {
        const ServerReq& r = reqs[*it];
        if (r.deadline > 0 && t > r.deadline) {
            finish_one(*it, APSM_ERR_DEADLINE, t);
            ++dropped;
            it = queue.erase(it);
        } else {
            ++it;
        }
    }
    for (auto it = lost.begin(); it != lost.end();) {
        const ServerReq& r = reqs[*it];
        if (r.deadline > 0 && t > r.deadline) {
            finish_one(*it, APSM_ERR_DEADLINE, t);
            ++dropped;
            it = lost.erase(it);
        } else {
            ++it;
        }
    }
}

double apsm_server::next_deadline() const
{
    double d = 0;
    auto take = [&](uint64_t tk) {
        auto it = reqs.find(tk);
        if (it != reqs.end() && it->second.deadline > 0 && (d == 0 || it->second.deadline < d)) d = it->second.deadline;
    };
    for (uint64_t tk : queue) take(tk);
    for (uint64_t tk : lost) take(tk);
    return d;
}

void apsm_server::complete(uint32_t lane, apsm_status st)
{
    const double t = now_s();
    for (uint64_t tk : lane_reqs[lane]) {
        auto it = reqs.find(tk);
        if (it == reqs.end()) continue;
        it->second.state = 2;
        it->second.st = st;
        it->second.t_done = t;
        busy_dets.erase(it->second.job.detector);
    }
    lane_reqs[lane].clear();
    lane_busy[lane] = 0;
    cv_done.notify_all();
}

// Builds and launches a batch on an idle lane; called with mu held.
bool apsm_server::admit(uint32_t lane)
{
    expire(now_s());
    if (queue.empty()) return false;
    const uint64_t budget = apsm_pool_budget(pool);
    uint64_t cap = ~0ull;
    if (budget) {
        const uint64_t used = apsm_pool_bytes_in_use(pool);
        cap = budget > used ? (budget - used) / n_lanes : 0;
        cap = std::max<uint64_t>(cap, 1);
    }
    std::vector<uint64_t> take;
    std::vector<apsm_job> jobs;
    std::unordered_set<uint32_t> blocked, trained, detected;
    uint64_t bytes = 0;
    int batch_kind = -1;
    for (auto it = queue.begin(); it != queue.end() && jobs.size() < max_batch;) {
        const uint64_t tk = *it;
        const apsm_job& j = reqs[tk].job;
        const uint32_t d = j.detector;
        bool ok = !busy_dets.count(d) && !blocked.count(d);
        if (ok && batch_kind >= 0 && int(j.kind) != batch_kind) ok = false;
        if (ok && j.kind == APSM_JOB_TRAIN && (trained.count(d) || detected.count(d))) ok = false;
        const uint64_t b = apsm_pool_job_bytes(pool, &j);
        if (ok && !jobs.empty() && bytes + b > cap) ok = false;
        if (!ok) {
            blocked.insert(d);
            ++it;
            continue;
        }
        bytes += b;
        batch_kind = int(j.kind);
        (j.kind == APSM_JOB_TRAIN ? trained : detected).insert(d);
        jobs.push_back(j);
        take.push_back(tk);
        it = queue.erase(it);
    }
    if (jobs.empty()) return false;
    const double t = now_s();
    for (uint64_t tk : take) {
        reqs[tk].state = 1;
        reqs[tk].t_start = t;
        busy_dets.insert(reqs[tk].job.detector);
    }
    lane_reqs[lane] = take;
    lane_busy[lane] = 1;
    ++batches;
    batched += jobs.size();
    mu.unlock();
    const apsm_status st = apsm_pool_run(pool, lane, jobs.data(), uint32_t(jobs.size()), APSM_RUN_HOST_ASYNC);
    mu.lock();
    if (st != APSM_OK) complete(lane, st);
    return true;
}

void apsm_server::run()
{
    std::unique_lock<std::mutex> lk(mu);
    for (;;) {
        expire(now_s());
        bool any_busy = false, progress = false;
        for (uint32_t l = 0; l < n_lanes; ++l) {
            if (!lane_busy[l]) continue;
            lk.unlock();
            const int q = apsm_pool_query(pool, l);
            apsm_status st = APSM_OK;
            if (q != 0) st = q < 0 ? apsm_status(-q) : apsm_pool_wait(pool, l);
            lk.lock();
            if (q != 0) {
                complete(l, st);
                progress = true;
            } else {
                any_busy = true;
            }
        }
        for (uint32_t l = 0; l < n_lanes; ++l)
            if (!lane_busy[l] && admit(l)) {
                progress = true;
                any_busy = true;
            }
        if (stop && queue.empty() && !any_busy) break;
        if (progress) continue;
        if (any_busy) {
            lk.unlock();
            std::this_thread::yield(); // poll the lanes again
            lk.lock();
        } else {
            // idle: wake for a submission, the next deadline, or after 1 ms
            double wait_s = 1e-3;
            const double nd = next_deadline();
            if (nd > 0) wait_s = std::max(0.0, std::min(wait_s, nd - now_s()));
            cv_submit.wait_for(lk, std::chrono::duration<double>(wait_s));
        }
    }
}

extern "C" apsm_status apsm_server_create(apsm_pool* pool, uint32_t lanes, uint32_t max_batch, apsm_server** out)
{
    if (!pool || !out || lanes == 0 || max_batch == 0) return APSM_ERR_INVALID_ARGUMENT;
    // lanes must exist on the pool: a stream per lane
    for (uint32_t l = 0; l < lanes; ++l)
        if (!apsm_pool_stream(pool, l)) return APSM_ERR_INVALID_ARGUMENT;
    auto* s = new apsm_server();
    apsm_pool_set_timing(pool, 0); // per-stage events cost latency; the server reports request times
    s->pool = pool;
    s->n_lanes = lanes;
    s->max_batch = max_batch;
    s->lane_reqs.resize(lanes);
    s->lane_busy.assign(lanes, 0);
    s->worker = std::thread([s] { s->run(); });
    *out = s;
    return APSM_OK;
}

extern "C" void apsm_server_destroy(apsm_server* s)
{
    if (!s) return;
    {
        std::lock_guard<std::mutex> g(s->mu);
        s->stop = true;
    }
    s->cv_submit.notify_all();
    if (s->worker.joinable()) s->worker.join();
    delete s;
}

extern "C" apsm_status apsm_server_submit_deadline(apsm_server* s, const apsm_job* job, double deadline_s,
                                                   uint64_t* ticket)
{
    if (!s || !job || !ticket) return APSM_ERR_INVALID_ARGUMENT;
    // malformed or oversized requests are rejected here, so they never join (and fail) a batch
    apsm_status chk = apsm_pool_check_job(s->pool, job);
    if (chk == APSM_OK) {
        const uint64_t budget = apsm_pool_budget(s->pool);
        if (budget && apsm_pool_job_bytes(s->pool, job) > budget) chk = APSM_ERR_OUT_OF_MEMORY;
    }
    {
        std::lock_guard<std::mutex> g(s->mu);
        if (chk != APSM_OK) {
            ++s->rejected;
            return chk;
        }
        if (s->stop) return APSM_ERR_INVALID_ARGUMENT;
        const uint64_t tk = s->next_ticket++;
        ServerReq r;
        r.job = *job;
        r.t_submit = now_s();
        const double rel = deadline_s < 0 ? s->default_deadline : deadline_s;
        r.deadline = rel > 0 ? r.t_submit + rel : 0;
        if (s->fault_drop > 0) { // injected: the request is lost on its way into the queue
            --s->fault_drop;
            r.lost = true;
            s->lost.insert(tk);
        } else {
            s->queue.push_back(tk);
        }
        s->reqs.emplace(tk, r);
        *ticket = tk;
    }
    s->cv_submit.notify_one();
    return APSM_OK;
}

extern "C" apsm_status apsm_server_submit(apsm_server* s, const apsm_job* job, uint64_t* ticket)
{
    return apsm_server_submit_deadline(s, job, -1.0, ticket);
}

extern "C" apsm_status apsm_server_set_deadline(apsm_server* s, double seconds)
{
    if (!s || !(seconds >= 0)) return APSM_ERR_INVALID_ARGUMENT;
    std::lock_guard<std::mutex> g(s->mu);
    s->default_deadline = seconds;
    return APSM_OK;
}

extern "C" apsm_status apsm_server_cancel(apsm_server* s, uint64_t ticket)
{
    if (!s) return APSM_ERR_INVALID_ARGUMENT;
    {
        std::lock_guard<std::mutex> g(s->mu);
        auto it = s->reqs.find(ticket);
        if (it == s->reqs.end()) return APSM_ERR_INVALID_ARGUMENT;
        ServerReq& r = it->second;
        if (r.state == 1) return APSM_ERR_UNSUPPORTED; // on the GPU already: runs to completion
        if (r.state == 2) return APSM_ERR_INVALID_ARGUMENT;
        if (r.lost) {
            s->lost.erase(ticket);
        } else {
            auto q = std::find(s->queue.begin(), s->queue.end(), ticket);
            if (q != s->queue.end()) s->queue.erase(q);
        }
        s->finish_one(ticket, APSM_ERR_CANCELLED, now_s());
        ++s->cancelled;
    }
    s->cv_submit.notify_one();
    return APSM_OK;
}

extern "C" apsm_status apsm_server_counts(apsm_server* s, uint64_t* dropped, uint64_t* cancelled, uint64_t* rejected)
{
    if (!s) return APSM_ERR_INVALID_ARGUMENT;
    std::lock_guard<std::mutex> g(s->mu);
    if (dropped) *dropped = s->dropped;
    if (cancelled) *cancelled = s->cancelled;
    if (rejected) *rejected = s->rejected;
    return APSM_OK;
}

extern "C" apsm_status apsm_server_inject_fault(apsm_server* s, int fault, uint32_t count)
{
    if (!s || fault != APSM_FAULT_DROP_REQUEST) return APSM_ERR_INVALID_ARGUMENT;
    std::lock_guard<std::mutex> g(s->mu);
    s->fault_drop = count;
    return APSM_OK;
}

extern "C" int apsm_server_poll(apsm_server* s, uint64_t ticket, apsm_status* status)
{
    if (!s) return -1;
    std::lock_guard<std::mutex> g(s->mu);
    auto it = s->reqs.find(ticket);
    if (it == s->reqs.end()) return -1;
    if (it->second.state != 2) return 0;
    if (status) *status = it->second.st;
    return 1;
}

extern "C" apsm_status apsm_server_wait(apsm_server* s, uint64_t ticket, double timeout_s)
{
    if (!s) return APSM_ERR_INVALID_ARGUMENT;
    std::unique_lock<std::mutex> lk(s->mu);
    auto done = [&] {
        auto it = s->reqs.find(ticket);
        return it == s->reqs.end() || it->second.state == 2;
    };
    if (!s->cv_done.wait_for(lk, std::chrono::duration<double>(timeout_s), done)) return APSM_ERR_TIMEOUT;
    auto it = s->reqs.find(ticket);
    if (it == s->reqs.end()) return APSM_ERR_INVALID_ARGUMENT;
    return it->second.st;
}

extern "C" apsm_status apsm_server_times(apsm_server* s, uint64_t ticket, double* submit_s, double* start_s,
                                         double* done_s)
{
    if (!s) return APSM_ERR_INVALID_ARGUMENT;
    std::lock_guard<std::mutex> g(s->mu);
    auto it = s->reqs.find(ticket);
    if (it == s->reqs.end()) return APSM_ERR_INVALID_ARGUMENT;
    if (submit_s) *submit_s = it->second.t_submit;
    if (start_s) *start_s = it->second.t_start;
    if (done_s) *done_s = it->second.t_done;
    return APSM_OK;
}

extern "C" apsm_status apsm_server_release(apsm_server* s, uint64_t ticket)
{
    if (!s) return APSM_ERR_INVALID_ARGUMENT;
    std::lock_guard<std::mutex> g(s->mu);
    auto it = s->reqs.find(ticket);
    if (it == s->reqs.end() || it->second.state != 2) return APSM_ERR_INVALID_ARGUMENT;
    s->reqs.erase(it);
    return APSM_OK;
}

extern "C" apsm_status apsm_server_stats(apsm_server* s, uint64_t* batches, uint64_t* jobs)
{
    if (!s) return APSM_ERR_INVALID_ARGUMENT;
    std::lock_guard<std::mutex> g(s->mu);
    if (batches) *batches = s->batches;
    if (jobs) *jobs = s->batched;
    return APSM_OK;
}

extern "C" double apsm_server_clock(void) { return now_s(); }
