// Continuous-batching server for split finite-volume solves.
//
// Clients submit solves (configuration, initial grid, step count) at any
// time from any thread.  A worker thread owns the GPU: between rounds of
// `ticks_per_round` batched steps it admits queued requests in arrival order
// as device memory (the budget) frees up, keeps every admitted solve's state
// resident on the device, advances all of them together, and returns each
// finished solve's grid to its client, recording queue, run and completion
// times.  Requests that arrive while others run join the next round, so
// their work overlaps on the device with the work already there.
//
// The mixed and fast FP64 forms serve through cfd_batch (one persistent
// launch per sweep for all members); the bit-identical FP64 form serves each
// member with its own cfd_solver on its own stream.  No counterpart in the reference (one problem per
// process, euler_equations/euler_simulation_code/sourcecode/main.cpp:17-49).
#include <algorithm>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <thread>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/cfdgpu.h"
#include "../../include/cfdgpu_host.h"
#include "../csrc/cfd_error.h"

namespace {

using Clock = std::chrono::steady_clock;

double secs(Clock::time_point a, Clock::time_point b) {
    return std::chrono::duration<double>(b - a).count();
}

// Pinned host memory for request grids, carved first-fit out of one
// allocation made when the server starts (pinning is slow; reuse is free).
// Callers hold the server lock.
class PinnedArena {
    char* base_ = nullptr;
    std::map<size_t, size_t> free_;  // offset -> bytes, coalesced
 public:
    bool init(size_t bytes) {
        if (!bytes || cudaHostAlloc(reinterpret_cast<void**>(&base_), bytes,
                                    cudaHostAllocDefault) != cudaSuccess) {
            base_ = nullptr;
            return false;
        }
        free_[0] = bytes;
        return true;
    }
    ~PinnedArena() {
        if (base_) cudaFreeHost(base_);
    }
    static size_t round(size_t bytes) { return (bytes + 255) / 256 * 256; }
    double* alloc(size_t bytes) {
        if (!base_) return nullptr;
        bytes = round(bytes);
        for (auto it = free_.begin(); it != free_.end(); ++it) {
            if (it->second < bytes) continue;
            const size_t off = it->first, left = it->second - bytes;
            free_.erase(it);
            if (left) free_[off + bytes] = left;
            return reinterpret_cast<double*>(base_ + off);
        }
        return nullptr;
    }
    void release(double* p, size_t bytes) {
        size_t off = reinterpret_cast<char*>(p) - base_;
        bytes = round(bytes);
        auto next = free_.lower_bound(off);
        if (next != free_.end() && off + bytes == next->first) {
            bytes += next->second;
            next = free_.erase(next);
        }
        if (next != free_.begin()) {
            auto prev = std::prev(next);
            if (prev->first + prev->second == off) {
                prev->second += bytes;
                return;
            }
        }
        free_[off] = bytes;
    }
};

struct Request {
    int64_t id;
    cfd_config cfg;
    // ghosted AoS initial grid, reused for the result: in the server's pinned
    // arena when it had room, else in `own`
    double* grid = nullptr;
    size_t elems = 0;
    std::vector<double> own;
    PinnedArena* arena = nullptr;  // owner of `grid` when pinned
    ~Request() {
        if (arena && grid) arena->release(grid, elems * sizeof(double));
    }
    // room for `n` doubles (pinned when the arena has it)
    void place(PinnedArena* a, size_t n) {
        elems = n;
        grid = a ? a->alloc(n * sizeof(double)) : nullptr;
        if (grid) {
            arena = a;
        } else {
            own.resize(n);
            grid = own.data();
        }
    }
    int recipe = 0;           // > 0: initial condition built on the device at admission
    uint64_t seed = 0;
    int nbubbles = 0;
    int steps;
    int state = CFD_REQ_QUEUED;
    int error = 0;
    Clock::time_point t_submit, t_admit, t_done;
    int member = -1;          // batch member id (mixed and fast FP64 forms)
    cfd_solver* solver = nullptr;  // FP64
    cudaStream_t stream = nullptr; // FP64: the solve's own stream
    cudaEvent_t ev = nullptr;      // FP64: end of its part of a round
    int issued = 0;                // FP64: steps enqueued so far
    size_t bytes = 0;
    cfd_status final_status{};
};

}  // namespace

struct cfd_server {
    cfd_server_options opt{};
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::deque<int64_t> queue;
    PinnedArena arena;  // request grids (under mu); declared first, destroyed after reqs
    std::map<int64_t, std::unique_ptr<Request>> reqs;
    std::vector<int64_t> running;
    int64_t next_id = 1;
    bool stop = false;
    std::thread worker;
    cfd_batch* batch = nullptr;
    cudaStream_t stream = nullptr;
    size_t budget = 0, used = 0;
    Clock::time_point t0;
    // statistics
    double cell_updates = 0.0;
    double busy_s = 0.0;
    double device_s = 0.0;   // CUDA-event time of the step rounds
    cudaEvent_t ev0[2] = {nullptr, nullptr}, ev1[2] = {nullptr, nullptr};  // round timing, two in flight
    int64_t completed = 0, rounds = 0, admitted = 0;
    int max_running = 0;
    int worker_error = 0;
    int device = 0;
};

namespace {

// The mixed and fast FP64 forms run as members of one batch.
bool batched(const cfd_server* s) {
    return s->opt.precision == CFD_PREC_MIXED || s->opt.precision == CFD_PREC_FP64_FAST;
}

size_t fp64_bytes(const cfd_config& c) {
    size_t b = 0;
    cfd_device_bytes(&c, &b);
    return b;
}

// Admission under the lock: FIFO, but a request that does not fit does not
// block smaller ones behind it (it keeps its place at the head).
void admit(cfd_server* s, std::vector<Request*>& to_start) {
    size_t free_b = s->budget > s->used ? s->budget - s->used : 0;
    for (auto it = s->queue.begin(); it != s->queue.end();) {
        Request* r = s->reqs[*it].get();
        size_t need = 0;
        if (batched(s)) cfd_batch_member_bytes(&r->cfg, &need);
        else need = fp64_bytes(r->cfg);
        if (need <= free_b) {
            free_b -= need;
            s->used += need;
            r->bytes = need;
            r->state = CFD_REQ_RUNNING;
            r->t_admit = Clock::now();
            to_start.push_back(r);
            it = s->queue.erase(it);
        } else {
            ++it;
        }
    }
}

void finish(cfd_server* s, Request* r, int err) {
    r->t_done = Clock::now();
    r->error = err;
    r->state = err ? CFD_REQ_FAILED : CFD_REQ_DONE;
    s->used -= r->bytes;
    if (!err) {
        s->completed++;
        s->cell_updates += (double)r->cfg.nx * r->cfg.ny * r->final_status.n;
    }
}

// Returns a finished request's grid to it and releases its device state.
int collect(cfd_server* s, Request* r) {
    if (!r->grid) {  // device-built initial condition: room for the result
        size_t elems = 0;
        cfd_ic_grid_elems(&r->cfg, &elems);
        std::lock_guard<std::mutex> lk(s->mu);
        r->place(&s->arena, elems);
    }
    int rc;
    if (batched(s)) {
        rc = cfd_batch_download(s->batch, r->member, r->grid, CFD_LAYOUT_GHOSTED_AOS);
        cfd_batch_remove(s->batch, r->member);
    } else {
        rc = cfd_download(r->solver, r->grid, CFD_LAYOUT_GHOSTED_AOS);
        cfd_destroy(r->solver);
        r->solver = nullptr;
        cudaStreamDestroy(r->stream);
        r->stream = nullptr;
        cudaEventDestroy(r->ev);
        r->ev = nullptr;
    }
    return rc;
}

// The worker: one round of steps for every running solve, then completion.
// Host work overlaps the round in flight: requests admitted before the round
// are started (allocation and upload, on the batch's copy stream or on each
// FP64 solve's stream) while it runs and join the next round, and the grids
// of finished solves are copied back meanwhile.  Mixed precision pipelines
// the rounds: the status read queued after round r is collected while round
// r+1 runs, so the GPU always has the next round queued (a solve found done
// one round late has idled in that round; its result is unchanged).
void worker_main(cfd_server* s) {
    cudaSetDevice(s->device);
    const int K = std::max(1, s->opt.ticks_per_round);
    const bool use_batch = batched(s);  // the mixed or fast FP64 form
    std::vector<Request*> finished;  // found done, grids not yet collected
    bool gather_pending = false;     // batch: status read queued after the last round
    std::vector<Request*> gathered;  // the solves that read covers
    int slot = 0;                    // event pair of the round being launched
    bool timed[2] = {false, false};
    // device time of the round in event pair `sl` (waits for it)
    auto account = [&](int sl) {
        if (!timed[sl]) return;
        float dev_ms = 0.f;
        cudaEventSynchronize(s->ev1[sl]);
        cudaEventElapsedTime(&dev_ms, s->ev0[sl], s->ev1[sl]);
        timed[sl] = false;
        std::lock_guard<std::mutex> lk(s->mu);
        s->device_s += 1e-3 * dev_ms;
        s->rounds++;
    };
    while (true) {
        std::vector<Request*> start;
        {
            std::unique_lock<std::mutex> lk(s->mu);
            s->cv_work.wait(lk, [&] {
                return s->stop || !s->queue.empty() || !s->running.empty() || !finished.empty() ||
                       gather_pending;
            });
            if (s->stop) break;
            admit(s, start);
        }
        std::vector<Request*> run;
        {
            std::lock_guard<std::mutex> lk(s->mu);
            for (int64_t id : s->running) {
                Request* r = s->reqs[id].get();
                if (std::find(finished.begin(), finished.end(), r) == finished.end())
                    run.push_back(r);
            }
            s->max_running = std::max<int>(s->max_running, (int)run.size());
        }
        const auto t_iter = Clock::now();
        // one round of steps (asynchronous)
        if (!run.empty()) {
            cudaEventRecord(s->ev0[slot], s->stream);
            if (use_batch) {
                if (cfd_batch_step(s->batch, K)) s->worker_error = CFD_ERR_CUDA;
            } else {
                for (Request* r : run) {
                    cudaStreamWaitEvent(r->stream, s->ev0[slot], 0);
                    int k = std::min(K, r->steps - r->issued);
                    if (k > 0 && cfd_advance(r->solver, k) == CFD_OK) r->issued += k;
                    cudaEventRecord(r->ev, r->stream);
                    cudaStreamWaitEvent(s->stream, r->ev, 0);
                }
            }
            cudaEventRecord(s->ev1[slot], s->stream);
            timed[slot] = true;
        }
        // start admitted requests (device allocation + upload, asynchronous)
        // while the round runs; they join the next round
        for (Request* r : start) {
            int rc;
            if (use_batch) {
                rc = r->recipe ? cfd_batch_add_recipe(s->batch, &r->cfg, r->recipe, r->seed,
                                                      r->nbubbles, r->steps, &r->member)
                               : cfd_batch_add(s->batch, &r->cfg, r->grid, r->steps,
                                               &r->member);
            } else {
                cfd_config c = r->cfg;
                rc = cudaStreamCreateWithFlags(&r->stream, cudaStreamNonBlocking) == cudaSuccess &&
                             cudaEventCreateWithFlags(&r->ev, cudaEventDisableTiming) == cudaSuccess
                         ? CFD_OK
                         : CFD_ERR_CUDA;
                c.stream = r->stream;
                if (!rc) rc = cfd_create(&c, &r->solver);
                if (!rc)
                    rc = r->recipe ? cfd_upload_recipe(r->solver, r->recipe, r->seed, r->nbubbles,
                                                       0, 0.0)
                                   : cfd_upload(r->solver, r->grid, CFD_LAYOUT_GHOSTED_AOS,
                                                0, 0.0);
                if (rc) {
                    // a failed start gives back everything it took: finish() returns
                    // the request's bytes to the budget, so its device state must go too
                    if (r->solver) cfd_destroy(r->solver);
                    r->solver = nullptr;
                    if (r->stream) cudaStreamDestroy(r->stream);
                    r->stream = nullptr;
                    if (r->ev) cudaEventDestroy(r->ev);
                    r->ev = nullptr;
                }
            }
            std::lock_guard<std::mutex> lk(s->mu);
            if (rc) {
                finish(s, r, rc);
                s->cv_done.notify_all();
            } else {
                s->running.push_back(r->id);
                s->admitted++;
            }
        }
        // batch: the status read queued after the previous round (it waits
        // for that round only; this round keeps the GPU busy meanwhile)
        if (use_batch && gather_pending) {
            int n = 0;
            const int cap = (int)gathered.size() + 64;
            std::vector<int> ids(cap), steps(cap), fin(cap);
            std::vector<double> tt(cap);
            int rc = cfd_batch_poll_collect(s->batch, cap, ids.data(), steps.data(), fin.data(),
                                            tt.data(), &n);
            gather_pending = false;
            std::map<int, int> pos;
            for (int i = 0; i < n && i < cap; ++i) pos[ids[i]] = i;
            for (Request* r : gathered) {
                auto it = pos.find(r->member);
                if (rc || it == pos.end()) {
                    finished.push_back(r);
                    continue;
                }
                int i = it->second;
                if (fin[i] || steps[i] >= r->steps) {
                    memset(&r->final_status, 0, sizeof r->final_status);
                    r->final_status.n = steps[i];
                    r->final_status.t = tt[i];
                    r->final_status.done = fin[i];
                    finished.push_back(r);
                }
            }
            account(slot ^ 1);  // the previous round has completed
        }
        // grids of the finished solves, while the round runs
        for (Request* r : finished) {
            int rc = collect(s, r);
            std::lock_guard<std::mutex> lk(s->mu);
            s->running.erase(std::find(s->running.begin(), s->running.end(), r->id));
            finish(s, r, rc);
        }
        const bool collected = !finished.empty();
        if (collected) s->cv_done.notify_all();
        if (run.empty()) {
            finished.clear();
            account(slot ^ 1);
            account(slot);
            continue;
        }
        if (use_batch) {
            // the status after this round, collected during the next one
            gathered.clear();
            for (Request* r : run)
                if (std::find(finished.begin(), finished.end(), r) == finished.end())
                    gathered.push_back(r);
            finished.clear();
            if (!gathered.empty()) {
                if (cfd_batch_poll_issue(s->batch)) {
                    finished = gathered;  // the read failed: report them with their error
                    gathered.clear();
                } else {
                    gather_pending = true;
                }
            }
        } else {
            // completion check: a status read only for solves that may have
            // finished (all steps issued, or a finite end time)
            finished.clear();
            for (Request* r : run) {
                if (r->issued < r->steps && std::isinf(r->cfg.T)) continue;
                cfd_status st;
                int rc = cfd_get_status(r->solver, &st);
                if (rc || st.done || st.n >= r->steps) {
                    r->final_status = st;
                    finished.push_back(r);
                }
            }
            account(slot);
        }
        {
            std::lock_guard<std::mutex> lk(s->mu);
            s->busy_s += secs(t_iter, Clock::now());
        }
        slot ^= 1;
    }
    account(0);
    account(1);
}

}  // namespace

namespace {

int enqueue(cfd_server* s, std::unique_ptr<Request> r, int64_t* id_out) {
    r->t_submit = Clock::now();
    const cfd_config* cfg = &r->cfg;
    size_t need = 0;
    if (batched(s)) {
        r->cfg.precision = s->opt.precision;  // the member's form
        cfd_batch_member_bytes(cfg, &need);
    } else {
        need = fp64_bytes(*cfg);
    }
    std::lock_guard<std::mutex> lk(s->mu);
    if (need > s->budget) {
        if (r->arena) {  // give the grid back while holding the lock
            r->arena->release(r->grid, r->elems * sizeof(double));
            r->arena = nullptr;
        }
        return cfd_fail(CFD_ERR_BUDGET, "request needs %zu bytes, the budget is %zu", need, s->budget);
    }
    r->id = s->next_id++;
    *id_out = r->id;
    s->queue.push_back(r->id);
    s->reqs[r->id] = std::move(r);
    s->cv_work.notify_one();
    return CFD_OK;
}

}  // namespace

extern "C" {

int cfd_server_create(const cfd_server_options* opt, cfd_server** out) {
    if (!opt || !out) return cfd_fail(CFD_ERR_INVALID, "null argument");
    if (opt->precision != CFD_PREC_MIXED && opt->precision != CFD_PREC_FP64 &&
        opt->precision != CFD_PREC_FP64_FAST)
        return cfd_fail(CFD_ERR_INVALID, "bad precision");
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
        return cfd_fail(CFD_ERR_CUDA, "no CUDA device available");
    auto* s = new cfd_server();
    s->opt = *opt;
    if (s->opt.ticks_per_round <= 0) s->opt.ticks_per_round = 16;
    cudaGetDevice(&s->device);
    s->stream = (cudaStream_t)opt->stream;
    if (!s->stream) cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking);
    size_t fr = 0, tot = 0;
    cudaMemGetInfo(&fr, &tot);
    s->budget = opt->budget_bytes ? opt->budget_bytes
                                  : (size_t)((opt->budget_fraction > 0 ? opt->budget_fraction : 0.8) *
                                             (double)fr);
    if (batched(s)) {
        int rc = cfd_batch_create(s->stream, (size_t)-1 / 2, &s->batch);
        if (rc) {
            delete s;
            return rc;
        }
    }
    for (int i = 0; i < 2; ++i) {
        cudaEventCreate(&s->ev0[i]);
        cudaEventCreate(&s->ev1[i]);
    }
    if (opt->host_pinned_bytes) s->arena.init(opt->host_pinned_bytes);  // pageable if it fails
    s->t0 = Clock::now();
    s->worker = std::thread(worker_main, s);
    *out = s;
    return CFD_OK;
}

int cfd_server_submit(cfd_server* s, const cfd_config* cfg, const double* ic, int steps,
                      int64_t* id_out) {
    if (!s || !cfg || !ic || !id_out || steps <= 0) return cfd_fail(CFD_ERR_INVALID, "bad argument");
    size_t elems = 0;
    cfd_ic_grid_elems(cfg, &elems);
    auto r = std::make_unique<Request>();
    r->cfg = *cfg;
    r->cfg.stream = nullptr;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        r->place(&s->arena, elems);
    }
    memcpy(r->grid, ic, elems * sizeof(double));  // outside the lock
    r->steps = steps;
    return enqueue(s, std::move(r), id_out);
}

int cfd_server_submit_recipe(cfd_server* s, const cfd_config* cfg, int recipe, uint64_t seed,
                             int nbubbles, int steps, int64_t* id_out) {
    if (!s || !cfg || !id_out || steps <= 0 || recipe <= 0)
        return cfd_fail(CFD_ERR_INVALID, "bad argument");
    auto r = std::make_unique<Request>();
    r->cfg = *cfg;
    r->cfg.stream = nullptr;
    r->recipe = recipe;
    r->seed = seed;
    r->nbubbles = nbubbles;
    r->steps = steps;
    return enqueue(s, std::move(r), id_out);
}

int cfd_server_wait(cfd_server* s, int64_t id, double timeout_s, cfd_request_info* info,
                    double* result) {
    if (!s) return cfd_fail(CFD_ERR_INVALID, "null server");
    std::unique_lock<std::mutex> lk(s->mu);
    auto it = s->reqs.find(id);
    if (it == s->reqs.end()) return cfd_fail(CFD_ERR_INVALID, "no request %lld", (long long)id);
    Request* r = it->second.get();
    auto pred = [&] { return r->state == CFD_REQ_DONE || r->state == CFD_REQ_FAILED; };
    if (timeout_s < 0) s->cv_done.wait(lk, pred);
    else if (!s->cv_done.wait_for(lk, std::chrono::duration<double>(timeout_s), pred)) {
        if (info) {
            memset(info, 0, sizeof *info);
            info->state = r->state;
        }
        return CFD_OK;
    }
    if (info) {
        memset(info, 0, sizeof *info);
        info->state = r->state;
        info->error = r->error;
        info->steps = r->final_status.n;
        info->t = r->final_status.t;
        info->queue_s = secs(r->t_submit, r->t_admit);
        info->run_s = secs(r->t_admit, r->t_done);
        info->latency_s = secs(r->t_submit, r->t_done);
        info->submit_s = secs(s->t0, r->t_submit);
    }
    if (result && r->state == CFD_REQ_DONE) memcpy(result, r->grid, r->elems * sizeof(double));
    return r->state == CFD_REQ_FAILED ? cfd_fail(r->error, "request %lld failed", (long long)id)
                                      : CFD_OK;
}

int cfd_server_release(cfd_server* s, int64_t id) {
    if (!s) return cfd_fail(CFD_ERR_INVALID, "null server");
    std::lock_guard<std::mutex> lk(s->mu);
    auto it = s->reqs.find(id);
    if (it == s->reqs.end()) return cfd_fail(CFD_ERR_INVALID, "no request");
    if (it->second->state != CFD_REQ_DONE && it->second->state != CFD_REQ_FAILED)
        return cfd_fail(CFD_ERR_STATE, "request still in flight");
    s->reqs.erase(it);
    return CFD_OK;
}

int cfd_server_get_stats(cfd_server* s, cfd_server_stats* st) {
    if (!s || !st) return cfd_fail(CFD_ERR_INVALID, "null argument");
    std::lock_guard<std::mutex> lk(s->mu);
    memset(st, 0, sizeof *st);
    st->completed = s->completed;
    st->admitted = s->admitted;
    st->queued = (int64_t)s->queue.size();
    st->running = (int64_t)s->running.size();
    st->max_running = s->max_running;
    st->rounds = s->rounds;
    st->cell_updates = s->cell_updates;
    st->busy_s = s->busy_s;
    st->device_s = s->device_s;
    st->wall_s = secs(s->t0, Clock::now());
    st->used_bytes = s->used;
    st->budget_bytes = s->budget;
    return CFD_OK;
}

int cfd_server_destroy(cfd_server* s) {
    if (!s) return CFD_OK;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stop = true;
    }
    s->cv_work.notify_all();
    if (s->worker.joinable()) s->worker.join();
    for (auto& kv : s->reqs) {
        Request* r = kv.second.get();
        if (r->solver) cfd_destroy(r->solver);
        if (r->stream) cudaStreamDestroy(r->stream);
        if (r->ev) cudaEventDestroy(r->ev);
    }
    if (s->batch) cfd_batch_destroy(s->batch);
    for (int i = 0; i < 2; ++i) {
        if (s->ev0[i]) cudaEventDestroy(s->ev0[i]);
        if (s->ev1[i]) cudaEventDestroy(s->ev1[i]);
    }
    if (!s->opt.stream && s->stream) cudaStreamDestroy(s->stream);
    delete s;
    return CFD_OK;
}

}  // extern "C"
