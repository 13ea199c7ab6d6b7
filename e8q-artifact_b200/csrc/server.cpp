// Serving loop: continuous batching of search requests over one index.
//
// At start the server sizes its batches: max_admit = the largest batch (up
// to max_batch_queries) whose device scratch at (max_k, max_nprobe) fits the
// memory budget; every slot then holds a captured plan for 64, 128, ...
// max_admit queries (own workspace, autotuned settings). submit() copies a
// request's queries to the host and queues it. The dispatcher thread waits
// for a free slot and pending requests, admits requests in FIFO order while
// the batch stays within max_admit queries, packs their queries and per-query
// k / nprobe into the slot's pinned staging, and enqueues the batch on the
// slot's stream: H2D copies, one graph launch (rotate + route + grouped scan,
// batched or precision mode), D2H copies, an event. It never waits for the
// GPU, so a second slot's batch is queued while the first runs. The completion thread waits on slots in dispatch order,
// checks the slot's device error word, copies each request's rows out of the
// staging and wakes its pollers; latencies are submit -> results ready.
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <functional>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "e8qc.h"
#include "internal.h"
#include "serve_target.h"
#include "workspace.h"

namespace e8qc {
void set_last_error(const std::string& s);
void plan_enqueue(e8qc_plan* P, const float* queries, size_t nq, const uint32_t* k, const uint32_t* nprobe,
                  uint32_t* out_ids, float* out_dists, cudaStream_t s);
void plan_check(e8qc_plan* P, cudaStream_t s);
}  // namespace e8qc

using namespace e8qc;
using Clock = std::chrono::steady_clock;

namespace {

struct Request {
    uint64_t id = 0;
    size_t nq = 0, k = 0, nprobe = 0;
    std::vector<float> q;
    std::vector<uint32_t> ids;
    std::vector<float> d;
    int status = 1;  // 1 pending / running, 0 done, < 0 failed (E8QC_ECANCELED, E8QC_ETIMEOUT, ...)
    bool canceled = false;  // canceled while its batch ran: its rows are discarded
    Clock::time_point t_submit, t_done, deadline;
};

template <class T>
struct PinnedBuf {
    T* p = nullptr;
    ~PinnedBuf() {
        if (p) cudaFreeHost(p);
    }
    void alloc(size_t count) {
        E8QC_CUDA(cudaMallocHost(reinterpret_cast<void**>(&p), std::max<size_t>(count, 1) * sizeof(T)));
    }
};

struct Slot {
    cudaStream_t stream = nullptr;
    cudaEvent_t done = nullptr;
    e8qc_plan* plan = nullptr;  // captured graphs of this slot's batch sizes, own workspace
    PinnedBuf<float> hq, hd;
    PinnedBuf<uint32_t> hk, hnp, hids;
    std::vector<std::shared_ptr<Request>> reqs;
    size_t nq = 0, bytes = 0;
    int error = 0;
    std::string error_msg;
    ~Slot() {
        if (plan) e8qc_plan_destroy(plan);
        if (done) cudaEventDestroy(done);
        if (stream) cudaStreamDestroy(stream);
    }
};

}  // namespace

struct e8qc_server {
    std::shared_ptr<SearchTarget> target;
    e8qc_server_config cfg{};
    size_t dim = 0, nlist = 0;
    size_t max_admit = 0;  // largest batch the budget admits at (max_k, max_nprobe); the plans' size
    int device = 0;
    std::mutex mu;
    std::condition_variable cv_dispatch, cv_complete, cv_done;
    std::deque<std::shared_ptr<Request>> pending;
    std::unordered_map<uint64_t, std::shared_ptr<Request>> live;
    std::vector<std::unique_ptr<Slot>> slots;
    std::deque<int> free_slots, inflight;
    uint64_t next_id = 1;
    bool stopping = false, dispatcher_done = false;
    std::thread dispatcher, completer;
    // stats
    uint64_t submitted = 0, rejected = 0, completed = 0, failed = 0, queries_done = 0, batches = 0,
             batch_queries = 0, peak_bytes = 0, canceled = 0, expired = 0;
    std::vector<double> lat_ms;
    Clock::time_point first_submit{}, last_done{};
    bool any_submit = false;
};

namespace {

int fail_status(std::string& msg, const std::exception& e) {
    msg = e.what();
    if (auto* er = dynamic_cast<const Error*>(&e)) return er->code;
    return E8QC_ECUDA;
}

// Pack one admitted batch into its slot's pinned staging and enqueue it as
// one captured graph launch (dispatcher thread, no lock).
void launch_batch(e8qc_server* S, Slot& sl) {
    size_t row = 0;
    for (auto& r : sl.reqs) {
        std::memcpy(sl.hq.p + row * S->dim, r->q.data(), r->nq * S->dim * sizeof(float));
        for (size_t i = 0; i < r->nq; ++i) {
            sl.hk.p[row + i] = static_cast<uint32_t>(r->k);
            sl.hnp.p[row + i] = static_cast<uint32_t>(r->nprobe);
        }
        row += r->nq;
    }
    plan_enqueue(sl.plan, sl.hq.p, sl.nq, sl.hk.p, sl.hnp.p, sl.hids.p, sl.hd.p, sl.stream);
    E8QC_CUDA(cudaEventRecord(sl.done, sl.stream));
}

void dispatcher_main(e8qc_server* S) {
    cudaSetDevice(S->device);
    std::unique_lock<std::mutex> lk(S->mu);
    for (;;) {
        auto ready = [&] { return S->stopping || (!S->free_slots.empty() && !S->pending.empty()); };
        if (S->cfg.request_timeout_ms > 0 && !S->pending.empty()) {
            // wake for the earliest deadline too (the queue is in submit
            // order, so the front's is the earliest)
            S->cv_dispatch.wait_until(lk, S->pending.front()->deadline, ready);
        } else {
            S->cv_dispatch.wait(lk, ready);
        }
        if (S->cfg.request_timeout_ms > 0) {
            const Clock::time_point now = Clock::now();
            bool any = false;
            while (!S->pending.empty() && S->pending.front()->deadline <= now) {
                auto r = S->pending.front();
                S->pending.pop_front();
                r->status = E8QC_ETIMEOUT;
                r->t_done = now;
                ++S->expired;
                ++S->failed;
                any = true;
            }
            if (any) S->cv_done.notify_all();
        }
        if (!S->stopping && (S->free_slots.empty() || S->pending.empty())) continue;
        if (S->stopping) {
            S->dispatcher_done = true;
            S->cv_complete.notify_all();
            return;
        }
        const int si = S->free_slots.front();
        Slot& sl = *S->slots[si];
        // admission: FIFO while the batch fits both limits
        sl.reqs.clear();
        // (the slot's plan reserved the scratch of max_admit queries at
        // (max_k, max_nprobe), the largest batch within the memory budget)
        size_t nq = 0;
        while (!S->pending.empty() && nq + S->pending.front()->nq <= S->max_admit) {
            nq += S->pending.front()->nq;
            sl.reqs.push_back(S->pending.front());
            S->pending.pop_front();
        }
        S->free_slots.pop_front();
        sl.nq = nq;
        sl.bytes = S->target->bytes(S->cfg.mode, nq, S->cfg.max_k, S->cfg.max_nprobe);
        sl.error = 0;
        sl.error_msg.clear();
        S->peak_bytes = std::max<uint64_t>(S->peak_bytes, sl.bytes);
        lk.unlock();
        try {
            launch_batch(S, sl);
        } catch (const std::exception& e) {
            sl.error = fail_status(sl.error_msg, e);
        }
        lk.lock();
        S->inflight.push_back(si);
        S->cv_complete.notify_one();
    }
}

void completer_main(e8qc_server* S) {
    cudaSetDevice(S->device);
    std::unique_lock<std::mutex> lk(S->mu);
    for (;;) {
        S->cv_complete.wait(lk, [&] { return !S->inflight.empty() || S->dispatcher_done; });
        if (S->inflight.empty()) return;  // the dispatcher has exited and nothing is in flight
        const int si = S->inflight.front();
        Slot& sl = *S->slots[si];
        lk.unlock();
        int st = sl.error;
        if (st != 0) cudaStreamSynchronize(sl.stream);  // whatever was enqueued before the failure drains
        if (st == 0) {
            try {
                E8QC_CUDA(cudaEventSynchronize(sl.done));
                plan_check(sl.plan, sl.stream);
            } catch (const std::exception& e) {
                st = fail_status(sl.error_msg, e);
            }
        }
        const Clock::time_point now = Clock::now();
        size_t row = 0;
        for (auto& r : sl.reqs) {
            if (st == 0) {
                r->ids.resize(r->nq * r->k);
                r->d.resize(r->nq * r->k);
                for (size_t i = 0; i < r->nq; ++i) {
                    std::memcpy(&r->ids[i * r->k], sl.hids.p + (row + i) * S->cfg.max_k, r->k * 4);
                    std::memcpy(&r->d[i * r->k], sl.hd.p + (row + i) * S->cfg.max_k, r->k * 4);
                }
            }
            row += r->nq;
        }
        lk.lock();
        for (auto& r : sl.reqs) {
            r->t_done = now;
            r->status = (st == 0 && r->canceled) ? E8QC_ECANCELED : st;
            if (r->status == E8QC_ECANCELED) {
                ++S->canceled;
            } else if (st == 0) {
                ++S->completed;
                S->queries_done += r->nq;
                S->lat_ms.push_back(std::chrono::duration<double, std::milli>(now - r->t_submit).count());
            } else {
                ++S->failed;
            }
        }
        S->last_done = now;
        ++S->batches;
        S->batch_queries += sl.nq;
        sl.reqs.clear();
        S->inflight.pop_front();
        S->free_slots.push_back(si);
        S->cv_dispatch.notify_one();
        S->cv_done.notify_all();
    }
}

int guard(const std::function<void()>& f) {
    try {
        f();
        return E8QC_OK;
    } catch (const Error& e) {
        set_last_error(e.msg);
        return e.code;
    } catch (const std::bad_alloc&) {
        set_last_error("host allocation failed");
        return E8QC_ENOMEM;
    } catch (const std::exception& e) {
        set_last_error(e.what());
        return E8QC_EINVAL;
    }
}

e8qc_server* server_make(std::shared_ptr<SearchTarget> t, const e8qc_server_config* cfg) {
    auto S = std::make_unique<e8qc_server>();
    S->target = t;
    if (cfg) S->cfg = *cfg;
    t->check_mode(S->cfg.mode);
    S->dim = t->dim;
    S->nlist = t->nlist;
    S->device = t->device;
    if (S->cfg.max_batch_queries == 0) S->cfg.max_batch_queries = 4096;
    if (S->cfg.max_k == 0) S->cfg.max_k = kMaxK;
    if (S->cfg.max_k > static_cast<size_t>(kMaxK)) fail(E8QC_EINVAL, "max_k must be <= 128");
    if (S->cfg.max_nprobe == 0 || S->cfg.max_nprobe > S->nlist) S->cfg.max_nprobe = S->nlist;
    if (S->cfg.memory_budget == 0) S->cfg.memory_budget = size_t(4) << 30;
    if (S->cfg.slots <= 0) S->cfg.slots = 2;
    if (S->cfg.slots > 16) fail(E8QC_EINVAL, "at most 16 slots");
    if (S->cfg.request_timeout_ms < 0) fail(E8QC_EINVAL, "request_timeout_ms must be >= 0");
    int prev = 0;
    E8QC_CUDA(cudaGetDevice(&prev));
    E8QC_CUDA(cudaSetDevice(S->device));
    struct Restore {
        int d;
        ~Restore() { cudaSetDevice(d); }
    } restore{prev};
    t->prepare(S->cfg.mode);
    const size_t B = S->cfg.max_batch_queries, K = S->cfg.max_k;
    // the largest batch whose scratch at (max_k, max_nprobe) fits the budget
    size_t nw = 1;
    for (size_t step = B; step > 0; step >>= 1)
        while (nw + step <= B &&
               t->bytes(S->cfg.mode, nw + step, K, S->cfg.max_nprobe) <= S->cfg.memory_budget)
            nw += step;
    S->max_admit = nw;
    for (int i = 0; i < S->cfg.slots; ++i) {
        auto sl = std::make_unique<Slot>();
        E8QC_CUDA(cudaStreamCreateWithFlags(&sl->stream, cudaStreamNonBlocking));
        E8QC_CUDA(cudaEventCreateWithFlags(&sl->done, cudaEventDisableTiming));
        sl->hq.alloc(nw * S->dim);
        sl->hk.alloc(nw);
        sl->hnp.alloc(nw);
        sl->hids.alloc(nw * K);
        sl->hd.alloc(nw * K);
        // captured graphs for batches of 64, 128, ... nw queries; the first
        // slot autotunes each size, the others take the stored settings
        sl->plan = plan_make(t, S->cfg.mode, nw, K, S->cfg.max_nprobe, i == 0);
        S->free_slots.push_back(i);
        S->slots.push_back(std::move(sl));
    }
    e8qc_server* raw = S.release();
    raw->dispatcher = std::thread(dispatcher_main, raw);
    raw->completer = std::thread(completer_main, raw);
    return raw;
}

}  // namespace

extern "C" int e8qc_server_start(e8qc_index* idx, const e8qc_server_config* cfg, e8qc_server** out) {
    return guard([&] {
        if (!idx || !out) fail(E8QC_EINVAL, "null argument");
        *out = server_make(e8q_target(idx), cfg);
    });
}

extern "C" int e8qc_server_start_me8q(e8qc_me8q* idx, const e8qc_server_config* cfg, e8qc_server** out) {
    return guard([&] {
        if (!idx || !out) fail(E8QC_EINVAL, "null argument");
        *out = server_make(me8q_target(idx), cfg);
    });
}

extern "C" int e8qc_server_submit(e8qc_server* S, const float* queries, size_t nq, size_t k, size_t nprobe,
                                  uint64_t* request_id) {
    return guard([&] {
        if (!S || !request_id) fail(E8QC_EINVAL, "null argument");
        if (nq == 0 || !queries) fail(E8QC_EINVAL, "a request needs at least one query");
        if (k == 0 || k > S->cfg.max_k) fail(E8QC_EINVAL, "k must be in [1, max_k]");
        if (nprobe == 0 || nprobe > S->cfg.max_nprobe) fail(E8QC_EINVAL, "nprobe must be in [1, max_nprobe]");
        const bool too_big = nq > S->max_admit;
        {
            std::lock_guard<std::mutex> lk(S->mu);
            if (S->stopping) fail(E8QC_ESTATE, "server is stopping");
            if (too_big) {
                ++S->rejected;
                fail(E8QC_ENOMEM, "request exceeds the server's batch size or memory budget");
            }
        }
        host_alloc_point();
        auto r = std::make_shared<Request>();
        r->nq = nq;
        r->k = k;
        r->nprobe = nprobe;
        r->q.assign(queries, queries + nq * S->dim);
        r->t_submit = Clock::now();
        r->deadline = r->t_submit + std::chrono::milliseconds(S->cfg.request_timeout_ms);
        std::lock_guard<std::mutex> lk(S->mu);
        if (S->stopping) fail(E8QC_ESTATE, "server is stopping");
        r->id = S->next_id++;
        if (!S->any_submit) {
            S->first_submit = r->t_submit;
            S->any_submit = true;
        }
        ++S->submitted;
        S->live[r->id] = r;
        S->pending.push_back(r);
        *request_id = r->id;
        S->cv_dispatch.notify_one();
    });
}

extern "C" int e8qc_server_poll(e8qc_server* S, uint64_t id, int timeout_ms, uint32_t* out_ids, float* out_dists,
                                int* done) {
    int req_status = E8QC_OK;
    const int rc = guard([&] {
        if (!S || !done) fail(E8QC_EINVAL, "null argument");
        *done = 0;
        std::unique_lock<std::mutex> lk(S->mu);
        auto it = S->live.find(id);
        if (it == S->live.end()) fail(E8QC_ERANGE, "unknown or already collected request id");
        std::shared_ptr<Request> r = it->second;
        auto ready = [&] { return r->status != 1; };
        if (timeout_ms < 0) S->cv_done.wait(lk, ready);
        else S->cv_done.wait_for(lk, std::chrono::milliseconds(timeout_ms), ready);
        if (!ready()) return;
        S->live.erase(id);
        lk.unlock();
        *done = 1;
        req_status = r->status;
        if (r->status == 0) {
            if (out_ids) std::memcpy(out_ids, r->ids.data(), r->ids.size() * 4);
            if (out_dists) std::memcpy(out_dists, r->d.data(), r->d.size() * 4);
        }
    });
    if (rc != E8QC_OK) return rc;
    if (req_status == E8QC_ECANCELED) set_last_error("the request was canceled");
    else if (req_status == E8QC_ETIMEOUT) set_last_error("the request expired before a batch slot took it (request_timeout_ms)");
    else if (req_status == E8QC_ESTATE) set_last_error("the server stopped before the request ran");
    else if (req_status != E8QC_OK) set_last_error("the batch that carried this request failed");
    return req_status;
}

extern "C" int e8qc_server_cancel(e8qc_server* S, uint64_t id) {
    return guard([&] {
        if (!S) fail(E8QC_EINVAL, "null argument");
        std::lock_guard<std::mutex> lk(S->mu);
        auto it = S->live.find(id);
        if (it == S->live.end()) fail(E8QC_ERANGE, "unknown or already collected request id");
        const std::shared_ptr<Request>& r = it->second;
        if (r->status != 1) return;  // complete: it keeps its results
        auto pit = std::find(S->pending.begin(), S->pending.end(), r);
        if (pit != S->pending.end()) {
            S->pending.erase(pit);
            r->status = E8QC_ECANCELED;
            r->t_done = Clock::now();
            ++S->canceled;
            S->cv_done.notify_all();
        } else {
            r->canceled = true;  // in a batch on the device: resolved when it ends
        }
    });
}

extern "C" int e8qc_server_get_stats(e8qc_server* S, int reset, e8qc_server_stats* out) {
    return guard([&] {
        if (!S || !out) fail(E8QC_EINVAL, "null argument");
        std::lock_guard<std::mutex> lk(S->mu);
        e8qc_server_stats st{};
        st.submitted = S->submitted;
        st.rejected = S->rejected;
        st.completed = S->completed;
        st.failed = S->failed;
        st.queries_completed = S->queries_done;
        st.batches = S->batches;
        st.peak_batch_bytes = S->peak_bytes;
        st.canceled = S->canceled;
        st.expired = S->expired;
        st.mean_batch_queries = S->batches ? static_cast<double>(S->batch_queries) / S->batches : 0.0;
        if (!S->lat_ms.empty()) {
            std::vector<double> v = S->lat_ms;
            std::sort(v.begin(), v.end());
            auto pct = [&](double p) {
                const double pos = p * static_cast<double>(v.size() - 1);
                return v[static_cast<size_t>(pos + 0.5)];
            };
            st.p50_ms = pct(0.50);
            st.p99_ms = pct(0.99);
            double s = 0;
            for (double x : v) s += x;
            st.mean_ms = s / static_cast<double>(v.size());
            st.max_ms = v.back();
        }
        if (S->any_submit && S->queries_done > 0) {
            const double sec = std::chrono::duration<double>(S->last_done - S->first_submit).count();
            st.qps = sec > 0 ? static_cast<double>(S->queries_done) / sec : 0.0;
        }
        *out = st;
        if (reset) {
            S->submitted = S->rejected = S->completed = S->failed = S->queries_done = S->batches = 0;
            S->batch_queries = S->peak_bytes = 0;
            S->canceled = S->expired = 0;
            S->lat_ms.clear();
            S->any_submit = false;
        }
    });
}

extern "C" int e8qc_server_stop(e8qc_server* S) {
    return guard([&] {
        if (!S) fail(E8QC_EINVAL, "null argument");
        {
            std::lock_guard<std::mutex> lk(S->mu);
            S->stopping = true;
            for (auto& r : S->pending) r->status = E8QC_ESTATE;  // never dispatched
            S->pending.clear();
        }
        S->cv_dispatch.notify_all();
        S->cv_done.notify_all();
        if (S->dispatcher.joinable()) S->dispatcher.join();
        S->cv_complete.notify_all();
        if (S->completer.joinable()) S->completer.join();
        cudaSetDevice(S->device);
        delete S;
    });
}
