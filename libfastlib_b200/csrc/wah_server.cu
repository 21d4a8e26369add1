// Serving loop over resident indexes (no counterpart in the reference, whose
// queries run one per caller thread under a global lock, src/iapi.cpp:33):
// continuous batching of conjunctive range queries.
//
// Requests enter a FIFO.  A worker thread owns `nslots` execution slots, each
// a context of its own (stream, look-back scratch, memory pool).  Whenever a
// slot is idle it takes the pending requests in arrival order, as many as
// fit both the batch size and the scratch budget (the device memory their
// evaluation needs: tile records, counts, row-id buffers), builds one batch
// and launches it; requests that arrive meanwhile wait for the next idle
// slot, so batches of consecutive arrivals run concurrently on the device.
// A slot's batch is finished when its CUDA event has completed; its requests
// are then answered and their scratch returns to the budget.
#include "../../include/wahgpu.h"
#include "wah_api_internal.h"
#define WAH_RANGE_TYPES_ONLY
#include "wah_index_internal.h"

#include <cuda_runtime.h>
#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <vector>

namespace {

using Clock = std::chrono::steady_clock;

struct Request {
    int64_t id = 0;
    std::vector<wahgpu_term> terms;
    uint64_t rid_cap = 0;
    size_t scratch = 0;
    Clock::time_point t_arrive;
    double latency = 0.0;
    uint64_t count = 0;
    std::vector<uint32_t> rids;
    int status = 0;
    bool done = false;
};

struct Slot {
    wahgpu_ctx* ctx = nullptr;
    wahgpu_batch* batch = nullptr;
    cudaEvent_t ev = nullptr;
    std::vector<Request*> reqs;
    size_t scratch = 0;
    bool busy = false;
};

}  // namespace

struct wahgpu_server {
    wahgpu_ctx* owner = nullptr;
    std::vector<Slot> slots;
    uint32_t max_batch = 0;
    size_t budget = 0, in_use = 0;
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::deque<Request*> pending;
    std::unordered_map<int64_t, Request*> reqs;
    int64_t next_id = 1;
    bool stop = false;
    std::thread worker;
    uint64_t batches = 0, served = 0;
};

namespace {

// Device memory one request needs while it is evaluated.
size_t request_scratch(const wahgpu_term* terms, uint64_t rid_cap) {
    const wahgpu_index* x = terms[0].idx;
    const size_t ntiles = x ? x->ntiles : 1;
    return ntiles * sizeof(wah::TileRec) + 16 + (size_t)rid_cap * 4;
}

void finish_slot(wahgpu_server* S, Slot& sl) {
    wahgpu_batch* B = sl.batch;
    // counts and every request's row-id region in one round trip, through
    // pinned staging of the slot's context
    uint32_t* ids = B->rid_cap ? static_cast<uint32_t*>(wg_host_alloc(sl.ctx, B->rid_cap * 4)) : nullptr;
    int rc = (B->rid_cap && !ids) ? WAHGPU_ENOMEM : wg_batch_fetch_all(B, ids);
    const auto now = Clock::now();
    for (size_t i = 0; i < sl.reqs.size(); ++i) {
        Request* r = sl.reqs[i];
        r->status = rc;
        if (!rc) {
            r->count = B->h_counts[i];
            if (r->rid_cap) {
                // the first rid_cap row ids of the query (its own region)
                const uint64_t n = std::min<uint64_t>(B->h_counts[i], B->h_lim[i]);
                r->rids.assign(ids + B->h_base[i], ids + B->h_base[i] + n);
            }
        }
        r->latency = std::chrono::duration<double>(now - r->t_arrive).count();
    }
    wg_host_free(sl.ctx, ids);
    wahgpu_batch_free(B);
    sl.batch = nullptr;
    std::lock_guard<std::mutex> g(S->mu);
    for (Request* r : sl.reqs) r->done = true;
    S->in_use -= sl.scratch;
    S->served += sl.reqs.size();
    sl.reqs.clear();
    sl.scratch = 0;
    sl.busy = false;
    S->cv_done.notify_all();
}

// Builds and launches one batch on an idle slot from the head of the queue.
void launch_slot(wahgpu_server* S, Slot& sl, std::vector<Request*>&& take, size_t scratch) {
    std::vector<wahgpu_term> terms;
    std::vector<uint32_t> qoff{0};
    std::vector<uint64_t> caps;
    uint64_t rid_cap = 0;
    for (Request* r : take) {
        terms.insert(terms.end(), r->terms.begin(), r->terms.end());
        qoff.push_back((uint32_t)terms.size());
        caps.push_back(r->rid_cap);
        rid_cap += r->rid_cap;
    }
    // tile by tile, so a batch's queries share each tile's bitmap words in
    // L2: count-only batches in one pass; batches with row ids count first,
    // then revisit only the items holding ids under each query's limit
    wahgpu_ctx_set_tuning(sl.ctx, WAHGPU_TUNE_RANGE_ORDER, rid_cap ? 2 : 1);
    wahgpu_batch* B = nullptr;
    // row ids: each request its own region of rid_cap ids (a LIMIT), so a
    // query with many hits cannot crowd out the others of its batch
    int rc = rid_cap ? wahgpu_batch_create_capped(sl.ctx, terms.data(), qoff.data(), (uint32_t)take.size(),
                                                  caps.data(), &B)
                     : wahgpu_batch_create(sl.ctx, terms.data(), qoff.data(), (uint32_t)take.size(), 0, 0, &B);
    if (!rc) rc = wahgpu_batch_run(B);
    if (!rc && cudaEventRecord(sl.ev, sl.ctx->stream) != cudaSuccess) rc = WAHGPU_ECUDA;
    if (rc) {
        if (B) wahgpu_batch_free(B);
        std::lock_guard<std::mutex> g(S->mu);
        const auto now = Clock::now();
        for (Request* r : take) {
            r->status = rc;
            r->latency = std::chrono::duration<double>(now - r->t_arrive).count();
            r->done = true;
        }
        S->in_use -= scratch;
        S->cv_done.notify_all();
        return;
    }
    sl.batch = B;
    sl.reqs = std::move(take);
    sl.scratch = scratch;
    sl.busy = true;
    ++S->batches;
}

void worker_loop(wahgpu_server* S) {
    cudaSetDevice(S->owner->device);
    while (true) {
        bool progress = false;
        // answer finished batches
        for (Slot& sl : S->slots) {
            if (sl.busy && cudaEventQuery(sl.ev) == cudaSuccess) {
                finish_slot(S, sl);
                progress = true;
            }
        }
        // admit waiting requests into idle slots
        for (Slot& sl : S->slots) {
            if (sl.busy) continue;
            std::vector<Request*> take;
            size_t scr = 0;
            {
                std::lock_guard<std::mutex> g(S->mu);
                while (!S->pending.empty() && take.size() < S->max_batch) {
                    Request* r = S->pending.front();
                    if (S->in_use + scr + r->scratch > S->budget) break;
                    scr += r->scratch;
                    take.push_back(r);
                    S->pending.pop_front();
                }
                S->in_use += scr;
            }
            if (!take.empty()) {
                launch_slot(S, sl, std::move(take), scr);
                progress = true;
            }
        }
        std::unique_lock<std::mutex> lk(S->mu);
        bool any_busy = false;
        for (Slot& sl : S->slots) any_busy |= sl.busy;
        if (S->stop && S->pending.empty() && !any_busy) break;
        if (!progress) {
            if (any_busy) {
                lk.unlock();
                std::this_thread::sleep_for(std::chrono::microseconds(20));
            } else {
                S->cv_work.wait_for(lk, std::chrono::milliseconds(1));
            }
        }
    }
}

}  // namespace

extern "C" int wahgpu_server_create(wahgpu_ctx* ctx, uint32_t nslots, uint32_t max_batch, uint64_t scratch_budget,
                                    wahgpu_server** out) {
    if (!ctx || !out || nslots == 0 || nslots > 16 || max_batch == 0 || scratch_budget == 0)
        return wg_fail(ctx, WAHGPU_EINVAL, "wahgpu_server_create: bad argument");
    *out = nullptr;
    wahgpu_server* S = new wahgpu_server();
    S->owner = ctx;
    S->max_batch = max_batch;
    S->budget = scratch_budget;
    S->slots.resize(nslots);
    for (Slot& sl : S->slots) {
        int rc = wahgpu_ctx_create(ctx->device, &sl.ctx);
        if (!rc && cudaEventCreateWithFlags(&sl.ev, cudaEventDisableTiming) != cudaSuccess) rc = WAHGPU_ECUDA;
        if (rc) {
            for (Slot& s2 : S->slots) {
                if (s2.ev) cudaEventDestroy(s2.ev);
                if (s2.ctx) wahgpu_ctx_destroy(s2.ctx);
            }
            delete S;
            return wg_fail(ctx, rc, "wahgpu_server_create: slot context creation failed");
        }
    }
    S->worker = std::thread(worker_loop, S);
    *out = S;
    return WAHGPU_OK;
}

// Queues one conjunctive query; returns its request id (> 0).  rid_cap > 0
// asks for its row ids (at most rid_cap).  A request whose scratch alone
// exceeds the server's budget is refused with WAHGPU_EBUSY.
extern "C" int64_t wahgpu_server_submit(wahgpu_server* S, const wahgpu_term* terms, uint32_t nterms, uint64_t rid_cap) {
    if (!S || !terms || nterms == 0 || !terms[0].idx) return WAHGPU_EINVAL;
    Request* r = new Request();
    r->terms.assign(terms, terms + nterms);
    r->rid_cap = rid_cap;
    r->scratch = request_scratch(terms, rid_cap);
    r->t_arrive = Clock::now();
    if (r->scratch > S->budget) {
        delete r;
        return wg_fail(S->owner, WAHGPU_EBUSY, "request needs %zu bytes of scratch, budget %zu",
                       request_scratch(terms, rid_cap), S->budget);
    }
    int64_t id;
    {
        std::lock_guard<std::mutex> g(S->mu);
        id = r->id = S->next_id++;
        S->reqs[id] = r;
        S->pending.push_back(r);
    }
    S->cv_work.notify_one();
    return id;
}

// Waits for request `id`; fills its count, row ids (when asked for at
// submit and out != NULL) and latency (seconds from submit to answer), then
// forgets the request.  Returns the number of row ids written, or an error.
extern "C" int64_t wahgpu_server_wait(wahgpu_server* S, int64_t id, uint64_t* count, uint32_t* rids, uint64_t cap,
                                      double* latency_s) {
    if (!S) return WAHGPU_EINVAL;
    Request* r = nullptr;
    {
        std::unique_lock<std::mutex> lk(S->mu);
        auto it = S->reqs.find(id);
        if (it == S->reqs.end()) return WAHGPU_EINVAL;
        r = it->second;
        S->cv_done.wait(lk, [&] { return r->done; });
        S->reqs.erase(it);
    }
    int64_t rc = r->status;
    if (!rc) {
        if (count) *count = r->count;
        if (latency_s) *latency_s = r->latency;
        rc = 0;
        if (rids && r->rid_cap) {
            if (cap < r->rids.size()) rc = wg_fail(S->owner, WAHGPU_ESIZE, "need room for %zu row ids", r->rids.size());
            else { std::copy(r->rids.begin(), r->rids.end(), rids); rc = (int64_t)r->rids.size(); }
        }
    }
    delete r;
    return rc;
}

// Open-loop replay: query q (terms[qoff[q], qoff[q+1])) is submitted at
// arrival_s[q] seconds after the call starts, by a feeder thread, while the
// worker batches; waits for all and writes counts and latencies (arrival to
// answer).  Returns the wall time of the whole replay in microseconds.
extern "C" int64_t wahgpu_server_replay(wahgpu_server* S, const wahgpu_term* terms, const uint32_t* qoff, uint32_t nq,
                                        const double* arrival_s, uint64_t rid_cap, uint64_t* counts, double* latency_s,
                                        uint32_t* rids, uint64_t* nrids) {
    if (!S || !terms || !qoff || !arrival_s || nq == 0) return WAHGPU_EINVAL;
    std::vector<int64_t> ids(nq, 0);
    std::atomic<int> err{0};
    const auto t0 = Clock::now();
    std::thread feeder([&] {
        for (uint32_t q = 0; q < nq; ++q) {
            const auto due = t0 + std::chrono::duration_cast<Clock::duration>(std::chrono::duration<double>(arrival_s[q]));
            while (Clock::now() < due) {
                const auto left = due - Clock::now();
                if (left > std::chrono::microseconds(200)) std::this_thread::sleep_for(left - std::chrono::microseconds(100));
            }
            Request* r = new Request();
            r->terms.assign(terms + qoff[q], terms + qoff[q + 1]);
            r->rid_cap = rid_cap;
            r->scratch = request_scratch(terms + qoff[q], rid_cap);
            r->t_arrive = due;  // latency counts from the scheduled arrival
            {
                std::lock_guard<std::mutex> g(S->mu);
                ids[q] = r->id = S->next_id++;
                S->reqs[r->id] = r;
                S->pending.push_back(r);
            }
            S->cv_work.notify_one();
        }
    });
    feeder.join();
    for (uint32_t q = 0; q < nq; ++q) {
        uint64_t c = 0;
        double l = 0;
        const int64_t rc = wahgpu_server_wait(S, ids[q], &c, rids ? rids + (size_t)q * rid_cap : nullptr,
                                              rids ? rid_cap : 0, &l);
        if (rc < 0) err = (int)rc;
        if (counts) counts[q] = c;
        if (latency_s) latency_s[q] = l;
        if (nrids) nrids[q] = rc > 0 ? (uint64_t)rc : 0;
    }
    if (err) return err;
    return std::chrono::duration_cast<std::chrono::microseconds>(Clock::now() - t0).count();
}

// Batches launched and requests answered so far.
extern "C" int wahgpu_server_stats(wahgpu_server* S, uint64_t* batches, uint64_t* served) {
    if (!S) return WAHGPU_EINVAL;
    std::lock_guard<std::mutex> g(S->mu);
    if (batches) *batches = S->batches;
    if (served) *served = S->served;
    return WAHGPU_OK;
}

extern "C" int wahgpu_server_free(wahgpu_server* S) {
    if (!S) return WAHGPU_EINVAL;
    {
        std::lock_guard<std::mutex> g(S->mu);
        S->stop = true;
    }
    S->cv_work.notify_all();
    S->worker.join();
    for (auto& kv : S->reqs) delete kv.second;
    for (Slot& sl : S->slots) {
        if (sl.ev) cudaEventDestroy(sl.ev);
        if (sl.ctx) wahgpu_ctx_destroy(sl.ctx);
    }
    delete S;
    return WAHGPU_OK;
}
