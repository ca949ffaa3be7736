// xw_server.cpp -- the continuous-batching request loop (xw_server_* and
// xw_submit/xw_poll/xw_wait/xw_cancel in include/xw.h).
//
// The reference serves one search per process (xweigh_cuda_main.cpp:281-285
// -> run_annealer, xweigh_cuda.cu:1419-2436): allocate a population, anneal,
// free.  Here one device's population stays resident and requests flow
// through it:
//
//   submitter threads --xw_submit--> prep queue
//   worker threads: Sylvester short-circuit, or start states + temperature
//                   calibration + replica records (prepare_job)  --> ready
//   engine thread, one round at a time:
//     admit ready requests (first come, first served) while their replicas
//       fit the resident cap and their records fit the device arena;
//     one persistent anneal launch per lanes-per-row class over every
//       resident replica, `quantum` iterations each;
//     an exchange launch for tempering requests (at their own interval
//       boundaries, XwJob::exchange_iters);
//     one collection launch: per request, the first solver (least solve
//       iteration, then index), summed counters, and the chosen W;
//     read those few bytes per request; retire finished requests and free
//       their slot, replica ids and arena range.
//
// Replicas run in stop mode 2 (each stops at its own solve), every request
// advances by exactly `quantum` iterations per round from its own start,
// and the Philox streams depend only on the request's seed and replica
// index, so a request's results do not depend on which requests shared its
// rounds.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <stdexcept>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "../../include/xw.h"
#include "xw_host_internal.h"
#include "xw_kernels.h"

namespace xw {
namespace {

// Launch classes of a round: 0 holds the orders up to 16 (at most 16
// candidates per move), which may run two replicas per warp; 1..4 the other
// orders by rows per lane 1, 2, 4, 8.
constexpr int kClasses = 5;
constexpr size_t kBestStride = (size_t)XW_MAX_N * XW_MAX_N;

int class_of(int n, int candidate_samples) {
    if (n <= 16 && candidate_samples <= 16) return 0;
    return n <= 32 ? 1 : n <= 64 ? 2 : n <= 128 ? 3 : 4;
}
int opl_of_class(int c) { return c == 0 ? 1 : 1 << (c - 1); }
int kind_of_class(int c) { return c == 0 ? kTunePairKind : opl_of_class(c); }

// First-fit allocator of [0, capacity) ranges with coalescing on release.
struct RangeAlloc {
    std::map<uint64_t, uint64_t> free_;   // offset -> size
    uint64_t capacity = 0, used = 0;

    void init(uint64_t cap) {
        free_.clear();
        if (cap) free_[0] = cap;
        capacity = cap;
        used = 0;
    }
    bool alloc(uint64_t size, uint64_t* off) {
        for (auto it = free_.begin(); it != free_.end(); ++it) {
            if (it->second < size) continue;
            *off = it->first;
            const uint64_t rest = it->second - size, at = it->first + size;
            free_.erase(it);
            if (rest) free_[at] = rest;
            used += size;
            return true;
        }
        return false;
    }
    void release(uint64_t off, uint64_t size) {
        used -= size;
        auto next = free_.lower_bound(off);
        if (next != free_.begin()) {
            auto prev = std::prev(next);
            if (prev->first + prev->second == off) {
                off = prev->first;
                size += prev->second;
                free_.erase(prev);
            }
        }
        if (next != free_.end() && off + size == next->first) {
            size += next->second;
            free_.erase(next);
        }
        free_[off] = size;
    }
};

bool sylvester_applies(int n, int w) { return w > 0 && (w & (w - 1)) == 0 && n % w == 0; }

struct Request {
    uint64_t id = 0;
    xw_job_spec spec{};
    xw_params params{};
    std::vector<int8_t> starts;
    int state = XW_REQ_QUEUED;
    int32_t status = XW_OK;
    std::string error;
    bool cancel = false;
    double t_submit = 0.0, t_admit = -1.0, t_finish = -1.0, t_solve = -1.0;
    uint64_t attained = 0;                      // iterations per replica so far
    // built by a worker
    XwJob job{};
    std::vector<uint8_t> records;
    std::vector<double> temps;
    double t_init = 0.0;
    // placement, engine thread only
    int slot = -1;
    uint64_t arena_off = 0, rep_begin = 0, ladder_off = 0;
    bool has_ladder = false;
    // result
    xw_request_result res{};
    std::vector<int8_t> best;
    // checkpoints and snapshots, taken by the engine at the end of a round
    bool ckpt_want = false;
    uint64_t ckpt_seq = 0;                      // checkpoints taken so far
    xw_request_result ckpt_res{};
    std::vector<int8_t> ckpt_best;
    std::deque<std::pair<uint64_t, std::string>> saves;   // (ticket, path) pending
    uint64_t save_tickets = 0, saves_done = 0;
    std::map<uint64_t, std::pair<int32_t, std::string>> save_results;
};

using ReqPtr = std::shared_ptr<Request>;

}  // namespace

struct Server {
    xw_server_config cfg{};
    int sms = 0;
    int optin_smem = 0;   // opt-in shared memory per CTA
    std::chrono::steady_clock::time_point t0 = std::chrono::steady_clock::now();

    std::mutex mu;
    std::condition_variable cv_engine, cv_prep, cv_done;
    std::unordered_map<uint64_t, ReqPtr> table;
    std::deque<ReqPtr> prep_queue;
    std::map<uint64_t, ReqPtr> ready;          // built, waiting for admission, by id
    uint64_t next_id = 1;
    bool stopping = false;
    std::string fatal;                         // engine failure: no more requests
    xw_server_stats stats{};
    std::thread engine;
    std::vector<std::thread> workers;

    // device state (engine thread after creation)
    cudaStream_t stream = nullptr;
    cudaStream_t side[kClasses] = {};                // per-class anneal launches
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    cudaEvent_t fork = nullptr, join[kClasses] = {};
    XwJob* d_jobs = nullptr;
    uint8_t* d_arena = nullptr;
    uint64_t* d_rec_off = nullptr;
    uint32_t* d_items = nullptr;               // kClasses x max_replica_ids
    uint32_t* d_counters = nullptr;            // kClasses
    uint32_t* d_chunk_done = nullptr;          // max_replica_ids: chunks finished per replica
    double* d_ladder = nullptr;
    JobOut* d_out = nullptr;
    uint64_t* d_best_off = nullptr;
    int8_t* d_best = nullptr;
    uint64_t* d_stamp = nullptr;
    JobOut* h_out = nullptr;                   // pinned
    uint64_t* h_stamp = nullptr;               // pinned
    RangeAlloc arena_alloc, rep_alloc, ladder_alloc;
    std::vector<int> free_slots;
    std::vector<ReqPtr> slot_req;
    std::vector<int> active;                   // slots with a resident request
    std::vector<int> selected;                 // slots the current round advances
    uint64_t resident = 0;
    bool items_dirty = true;
    std::vector<uint32_t> items_host[kClasses];
    uint32_t class_slot[kClasses] = {};
    bool class_general[kClasses] = {};
    bool class_one_zero[kClasses] = {};       // every request of the class is W(n, n-1)
    std::map<std::pair<int, uint32_t>, int> per_sm_cache;
    int last_njobs = 0;

    double now() const {
        return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    }

    void start();
    void stop();
    void worker_loop();
    void engine_loop();
    void admit_locked(std::vector<ReqPtr>& admitted);
    void place(const ReqPtr& q);
    void select_round();
    void rebuild_items();
    int blocks_for(int cls, bool general, uint32_t slot_bytes, int wpb, int rpw, size_t items);
    void round(bool& any_tempering);
    void retire(const ReqPtr& q, const JobOut& o, double t_host, uint64_t stamp, int state, const VerifyStats& vs);
    DeviceVerifier verifier;   // retiring requests' W, checked on the tensor cores
    void checkpoint(const ReqPtr& q, const JobOut& o, bool want_best, size_t nsaves);
    void finish_locked(const ReqPtr& q, int state);
    void fail_all(const std::string& msg);
};

namespace {

void fill_result_header(Request& q) {
    xw_request_result& r = q.res;
    r.n = q.spec.n;
    r.w = q.spec.w;
    r.replicas = q.spec.replicas;
    r.submit_seconds = q.t_submit;
    r.admit_seconds = q.t_admit;
    r.finish_seconds = q.t_finish;
    r.state = q.state;
    r.status = q.status;
    std::snprintf(r.error, sizeof r.error, "%s", q.error.c_str());
}

}  // namespace

void Server::finish_locked(const ReqPtr& q, int state) {
    for (const auto& sv : q->saves)
        q->save_results[sv.first] = {XW_ERR_INVALID, "request finished before its snapshot was taken"};
    q->saves.clear();
    q->saves_done = q->save_tickets;
    q->state = state;
    q->t_finish = now();
    q->records.clear();
    q->records.shrink_to_fit();
    q->starts.clear();
    q->starts.shrink_to_fit();
    fill_result_header(*q);
    ++stats.finished;
    if (state == XW_REQ_CANCELLED) ++stats.cancelled;
    if (state == XW_REQ_FAILED) ++stats.failed;
    if (q->res.solved) ++stats.solved;
    if (q->res.sylvester) ++stats.sylvester;
    stats.moves += q->res.moves;
    cv_done.notify_all();
}

void Server::worker_loop() {
    for (;;) {
        ReqPtr q;
        {
            std::unique_lock<std::mutex> lk(mu);
            cv_prep.wait(lk, [&] { return stopping || !prep_queue.empty(); });
            if (stopping) return;
            q = prep_queue.front();
            prep_queue.pop_front();
            if (q->state != XW_REQ_QUEUED) continue;   // cancelled while queued
        }
        const int n = q->spec.n, w = q->spec.w;
        try {
            if (cfg.sylvester_shortcut && sylvester_applies(n, w) && q->starts.empty()) {
                std::vector<int8_t> W((size_t)n * n);
                if (xw_sylvester(n, w, W.data()) != XW_OK) throw std::runtime_error(xw_last_error());
                const bool ok = xw_verify(n, w, W.data()) == 3;
                std::lock_guard<std::mutex> lk(mu);
                q->best = std::move(W);
                q->res.solved = 1;
                q->res.verified = ok;
                q->res.sylvester = 1;
                q->res.best_replica = -1;
                q->res.time_to_solution_seconds = now() - q->t_submit;
                if (q->state == XW_REQ_QUEUED) finish_locked(q, XW_REQ_DONE);
                continue;
            }
            prepare_job(q->spec, q->params, q->starts.empty() ? nullptr : q->starts.data(), 0, false, q->job,
                        q->records, q->temps, q->t_init);
            q->job.exchange_iters = q->params.tempering ? (uint64_t)q->params.exchange_interval : 0;
            std::lock_guard<std::mutex> lk(mu);
            if (q->state != XW_REQ_QUEUED) continue;
            ready[q->id] = q;
            cv_engine.notify_one();
        } catch (const std::exception& e) {
            std::lock_guard<std::mutex> lk(mu);
            q->status = XW_ERR_INVALID;
            q->error = e.what();
            if (q->state == XW_REQ_QUEUED) finish_locked(q, XW_REQ_FAILED);
        }
    }
}

// Engine thread, with mu held: move ready requests into the resident set
// while they fit.  First come, first served: the first request that does
// not fit stops admission.
void Server::admit_locked(std::vector<ReqPtr>& admitted) {
    while (!ready.empty()) {
        ReqPtr q = ready.begin()->second;
        if (q->state != XW_REQ_QUEUED) {
            ready.erase(ready.begin());
            continue;
        }
        const uint64_t R = (uint64_t)q->spec.replicas;
        const uint64_t bytes = R * q->job.record_bytes;
        if (resident > 0 && resident + R > (uint64_t)cfg.max_resident_replicas) break;
        if (free_slots.empty()) break;
        uint64_t rb = 0, ao = 0, lo = 0;
        if (!rep_alloc.alloc(R, &rb)) break;
        if (!arena_alloc.alloc((bytes + 255) / 256, &ao)) {
            rep_alloc.release(rb, R);
            break;
        }
        const bool lad = q->params.tempering != 0;
        if (lad && !ladder_alloc.alloc(R, &lo)) {
            rep_alloc.release(rb, R);
            arena_alloc.release(ao, (bytes + 255) / 256);
            break;
        }
        q->slot = free_slots.back();
        free_slots.pop_back();
        q->rep_begin = rb;
        q->arena_off = ao * 256;
        q->ladder_off = lo;
        q->has_ladder = lad;
        q->state = XW_REQ_RUNNING;
        q->t_admit = now();
        resident += R;
        ++stats.admitted;
        ready.erase(ready.begin());
        admitted.push_back(q);
    }
}

// Engine thread: upload an admitted request's job entry, records, record
// offsets and ladder.
void Server::place(const ReqPtr& q) {
    XwJob J = q->job;
    const int R = q->spec.replicas;
    J.rep_begin = (uint32_t)q->rep_begin;
    J.ladder_off = q->ladder_off;
    for (int r = 0; r < R; ++r) {
        RepHeader* H = reinterpret_cast<RepHeader*>(q->records.data() + (size_t)r * J.record_bytes);
        H->job = (uint32_t)q->slot;
    }
    std::vector<uint64_t> offs(R);
    for (int r = 0; r < R; ++r) offs[r] = q->arena_off + (uint64_t)r * J.record_bytes;
    check_cuda(cudaMemcpyAsync(d_arena + q->arena_off, q->records.data(), q->records.size(), cudaMemcpyHostToDevice,
                               stream),
               "upload request records");
    check_cuda(cudaMemcpyAsync(d_rec_off + q->rep_begin, offs.data(), sizeof(uint64_t) * R, cudaMemcpyHostToDevice,
                               stream),
               "upload record offsets");
    if (q->has_ladder)
        check_cuda(cudaMemcpyAsync(d_ladder + q->ladder_off, q->temps.data(), sizeof(double) * R,
                                   cudaMemcpyHostToDevice, stream),
                   "upload ladder");
    check_cuda(cudaMemcpyAsync(d_jobs + q->slot, &J, sizeof J, cudaMemcpyHostToDevice, stream), "upload job");
    // pageable sources: the copies above are staged before they return,
    // but keep the buffers until the stream has consumed them
    check_cuda(cudaStreamSynchronize(stream), "cudaStreamSynchronize upload");
    q->job = J;
    q->records.clear();
    q->records.shrink_to_fit();
    slot_req[q->slot] = q;
    active.push_back(q->slot);
    items_dirty = true;
}

// The requests this round advances.  Least attained service: fewest
// iterations first, then oldest, up to max_active_replicas -- a request
// that solves in its first rounds is not queued behind long searches, and
// each request still advances by whole rounds from its own start.
void Server::select_round() {
    std::vector<int> sel;
    if (cfg.schedule == XW_SCHED_ALL) {
        sel = active;
    } else {
        std::vector<int> order(active);
        std::sort(order.begin(), order.end(), [&](int a, int b) {
            const Request& x = *slot_req[a];
            const Request& y = *slot_req[b];
            return x.attained != y.attained ? x.attained < y.attained : x.id < y.id;
        });
        uint64_t total = 0;
        for (int s : order) {
            const uint64_t R = (uint64_t)slot_req[s]->spec.replicas;
            if (!sel.empty() && total + R > (uint64_t)cfg.max_active_replicas) break;
            sel.push_back(s);
            total += R;
        }
    }
    if (sel != selected) {
        selected.swap(sel);
        items_dirty = true;
    }
}

// Work items per class: replicas of larger orders first (cost grows with n).
void Server::rebuild_items() {
    std::vector<int> order(selected);
    std::stable_sort(order.begin(), order.end(),
                     [&](int a, int b) { return slot_req[a]->spec.n > slot_req[b]->spec.n; });
    for (int c = 0; c < kClasses; ++c) {
        items_host[c].clear();
        class_slot[c] = 0;
        class_general[c] = false;
        class_one_zero[c] = true;
    }
    for (int s : order) {
        const ReqPtr& q = slot_req[s];
        const int c = class_of(q->spec.n, q->job.candidate_samples);
        for (int r = 0; r < q->spec.replicas; ++r) items_host[c].push_back((uint32_t)(q->rep_begin + r));
        class_slot[c] = std::max(class_slot[c], anneal_slot_bytes(q->spec.n, q->job.m, opl_of_class(c)));
        class_general[c] = class_general[c] || q->job.general != 0;
        class_one_zero[c] = class_one_zero[c] && q->job.m == 1 && !q->job.sparse;
    }
    for (int c = 0; c < kClasses; ++c)
        if (!items_host[c].empty())
            check_cuda(cudaMemcpyAsync(d_items + (size_t)c * cfg.max_replica_ids, items_host[c].data(),
                                       sizeof(uint32_t) * items_host[c].size(), cudaMemcpyHostToDevice, stream),
                       "upload work items");
    items_dirty = false;
}

int Server::blocks_for(int cls, bool general, uint32_t slot_bytes, int wpb, int rpw, size_t items) {
    const auto key = std::make_pair(((cls * 64 + wpb) * 2 + (general ? 1 : 0)) * 4 + rpw, slot_bytes);
    auto it = per_sm_cache.find(key);
    int per_sm = 0;
    if (it == per_sm_cache.end()) {
        check_cuda(cudaOccupancyMaxActiveBlocksPerMultiprocessor(
                       &per_sm, anneal_kernel_fn(opl_of_class(cls), general, rpw), 32 * wpb,
                       (size_t)wpb * rpw * slot_bytes),
                   "cudaOccupancyMaxActiveBlocksPerMultiprocessor");
        per_sm_cache[key] = per_sm;
    } else {
        per_sm = it->second;
    }
    if (per_sm < 1) throw std::length_error("CUDA anneal kernel has zero occupancy for this request mix");
    const int groups = wpb * rpw;
    const int want = (int)((items + groups - 1) / groups);
    return std::max(1, std::min(want, per_sm * sms));
}

void Server::round(bool& any_tempering) {
    if (items_dirty) rebuild_items();
    int njobs = 0;   // slots in use lie below the high-water mark
    for (int s : active) njobs = std::max(njobs, s + 1);
    last_njobs = njobs;
    check_cuda(cudaEventRecord(ev0, stream), "cudaEventRecord");
    check_cuda(cudaMemsetAsync(d_counters, 0, sizeof(uint32_t) * kClasses, stream), "reset work counters");
    // per class: warps per block, CTAs, and chunks per replica (a class with
    // more replicas than its resident warps runs chunked, as batches do)
    int cls_wpb[kClasses] = {}, cls_blocks[kClasses] = {}, cls_rpw[kClasses] = {};
    uint32_t cls_chunks[kClasses] = {};
    bool any_chunked = false;
    for (int c = 0; c < kClasses; ++c) {
        if (items_host[c].empty()) continue;
        TunedShape t = tuned_shape(kind_of_class(c), class_slot[c], cfg.device);
        if (cfg.warps_per_block > 0) t.wpb = cfg.warps_per_block;
        if (cfg.replicas_per_warp > 0) t.rpw = cfg.replicas_per_warp;
        if (c != 0) t.rpw = 1;
        // a CTA's slots must fit the opt-in shared memory (large orders)
        const int fit = std::max(1, optin_smem / (int)std::max<uint32_t>(1, class_slot[c] * (uint32_t)t.rpw));
        const int wpb = std::max(1, std::min({16, t.wpb, fit}));
        cls_wpb[c] = wpb;
        cls_rpw[c] = t.rpw;
        cls_blocks[c] = blocks_for(c, class_general[c], class_slot[c], wpb, t.rpw, items_host[c].size());
        cls_chunks[c] = choose_chunks((uint32_t)items_host[c].size(), (uint32_t)(cls_blocks[c] * wpb * t.rpw));
        if (cls_chunks[c] > (uint32_t)cfg.quantum_iters) cls_chunks[c] = 1;
        any_chunked = any_chunked || cls_chunks[c] > 1;
    }
    if (any_chunked)
        check_cuda(cudaMemsetAsync(d_chunk_done, 0, sizeof(uint32_t) * cfg.max_replica_ids, stream),
                   "reset chunk counters");
    // the classes' persistent launches run side by side on their own
    // streams, so that one launch's tail overlaps the other's work
    int nclass = 0;
    for (int c = 0; c < kClasses; ++c) nclass += !items_host[c].empty();
    if (nclass > 1) check_cuda(cudaEventRecord(fork, stream), "cudaEventRecord");
    for (int c = 0; c < kClasses; ++c) {
        if (items_host[c].empty()) continue;
        cudaStream_t st = stream;
        if (nclass > 1) {
            st = side[c];
            check_cuda(cudaStreamWaitEvent(st, fork, 0), "cudaStreamWaitEvent");
        }
        const int wpb = cls_wpb[c];
        AnnealArgs a;
        a.jobs = d_jobs;
        a.arena = d_arena;
        a.rec_off = d_rec_off;
        a.items = d_items + (size_t)c * cfg.max_replica_ids;
        a.n_items = (uint32_t)items_host[c].size();
        a.slot_bytes = class_slot[c];
        a.counter = d_counters + c;
        a.iters = (uint64_t)cfg.quantum_iters;
        a.stop_on_solve = 2;
        a.one_zero = class_one_zero[c] && cls_rpw[c] == 1 ? 1 : 0;
        a.chunks = cls_chunks[c];
        if (a.chunks > 1) a.chunk_done = d_chunk_done;
        a.chunk_wait_ns = chunk_wait_limit_ns();
        check_cuda(launch_anneal(a, opl_of_class(c), class_general[c], wpb, cls_blocks[c], st, cls_rpw[c]),
                   "launch anneal_kernel");
        if (nclass > 1) {
            check_cuda(cudaEventRecord(join[c], st), "cudaEventRecord");
            check_cuda(cudaStreamWaitEvent(stream, join[c], 0), "cudaStreamWaitEvent");
        }
    }
    any_tempering = false;
    for (int s : selected) any_tempering |= slot_req[s]->params.tempering != 0;
    if (any_tempering)
        check_cuda(launch_exchange(d_jobs, njobs, d_arena, d_rec_off, d_ladder, 2, stream), "launch exchange_kernel");
    check_cuda(launch_collect(d_jobs, njobs, d_arena, d_rec_off, d_best_off, d_out, d_best, stream, 1),
               "launch collect_kernel");
    check_cuda(launch_stamp(d_stamp, stream), "launch stamp");
    check_cuda(cudaEventRecord(ev1, stream), "cudaEventRecord");
    check_cuda(cudaMemcpyAsync(h_out, d_out, sizeof(JobOut) * njobs, cudaMemcpyDeviceToHost, stream),
               "read request results");
    check_cuda(cudaMemcpyAsync(h_stamp, d_stamp, sizeof(uint64_t), cudaMemcpyDeviceToHost, stream), "read clock");
    check_cuda(cudaStreamSynchronize(stream), "cudaStreamSynchronize round");
    float ms = 0.0f;
    check_cuda(cudaEventElapsedTime(&ms, ev0, ev1), "cudaEventElapsedTime");
    std::lock_guard<std::mutex> lk(mu);
    stats.device_seconds += ms * 1e-3;
    ++stats.rounds;
}

// Engine thread: read back the chosen W, take its score and exact check
// from the round's device verification (vs), free the request's device
// resources.
void Server::retire(const ReqPtr& q, const JobOut& o, double t_host, uint64_t stamp, int state,
                    const VerifyStats& vs) {
    const int n = q->spec.n;
    std::vector<int8_t> W((size_t)n * n);
    check_cuda(cudaMemcpy(W.data(), d_best + (size_t)q->slot * kBestStride, W.size(), cudaMemcpyDeviceToHost),
               "read request best state");
    const int64_t st[2] = {vs.score, vs.conflicts};
    const bool solved = o.first_solver >= 0;
    const bool verified = solved && vs.exact == 1;
    XwJob zero;
    std::memset(&zero, 0, sizeof zero);
    zero.done = 1;
    check_cuda(cudaMemcpyAsync(d_jobs + q->slot, &zero, sizeof zero, cudaMemcpyHostToDevice, stream),
               "clear job slot");
    check_cuda(cudaStreamSynchronize(stream), "cudaStreamSynchronize retire");
    const int R = q->spec.replicas;
    std::lock_guard<std::mutex> lk(mu);
    rep_alloc.release(q->rep_begin, (uint64_t)R);
    arena_alloc.release(q->arena_off / 256, ((uint64_t)R * q->job.record_bytes + 255) / 256);
    if (q->has_ladder) ladder_alloc.release(q->ladder_off, (uint64_t)R);
    free_slots.push_back(q->slot);
    slot_req[q->slot].reset();
    resident -= (uint64_t)R;
    items_dirty = true;

    xw_request_result& r = q->res;
    r.solved = solved;
    r.verified = verified;
    r.sylvester = 0;
    r.best_replica = o.best_replica;
    r.score = st[0];
    r.conflicts = st[1];
    r.moves = o.moves;
    r.candidate_evaluations = o.cand_evals;
    r.iterations = o.iters;
    r.solved_iteration = solved ? o.solved_it : 0;
    r.t_init = q->t_init;
    if (solved) {
        // device clock -> server clock through this round's stamp
        const double lag = stamp >= o.solve_ns ? (double)(stamp - o.solve_ns) * 1e-9 : 0.0;
        q->t_solve = std::max(q->t_admit, t_host - lag);
        r.time_to_solution_seconds = q->t_solve - q->t_submit;
    } else {
        r.time_to_solution_seconds = -1.0;
    }
    if (o.err) {
        q->status = XW_ERR_INTERNAL;
        q->error = "CUDA replica failed its device self-check";
        state = XW_REQ_FAILED;
    } else if (solved && !verified) {
        q->status = XW_ERR_INTERNAL;
        q->error = "score reached zero but exact verification failed";
        state = XW_REQ_FAILED;
    }
    q->best = std::move(W);
    finish_locked(q, state);
}

// Engine thread, after a round: the request's best W so far and its
// progress (want_best), and its first `nsaves` pending snapshots: the job
// entry and every replica record as this round left them, as a one-job
// population snapshot.
void Server::checkpoint(const ReqPtr& q, const JobOut& o, bool want_best, size_t nsaves) {
    const int n = q->spec.n, w = q->spec.w, R = q->spec.replicas;
    if (want_best) {
        std::vector<int8_t> W((size_t)n * n);
        check_cuda(cudaMemcpy(W.data(), d_best + (size_t)q->slot * kBestStride, W.size(), cudaMemcpyDeviceToHost),
                   "read request best state");
        int64_t st[4] = {0, 0, 0, 0};
        xw_score(n, w, W.data(), st);
        std::lock_guard<std::mutex> lk(mu);
        xw_request_result r = q->res;
        r.solved = o.first_solver >= 0;
        r.best_replica = o.best_replica;
        r.score = st[0];
        r.conflicts = st[1];
        r.moves = o.moves;
        r.candidate_evaluations = o.cand_evals;
        r.iterations = o.iters;
        r.solved_iteration = o.first_solver >= 0 ? o.solved_it : 0;
        r.t_init = q->t_init;
        q->ckpt_res = r;
        q->ckpt_best = std::move(W);
        q->ckpt_want = false;
        ++q->ckpt_seq;
        cv_done.notify_all();
    }
    if (nsaves == 0) return;
    xw::Snapshot sn;
    std::string err;
    try {
        sn.jobs.resize(1);
        sn.arena.resize((size_t)R * q->job.record_bytes);
        check_cuda(cudaMemcpy(sn.jobs.data(), d_jobs + q->slot, sizeof(XwJob), cudaMemcpyDeviceToHost),
                   "read request job");
        check_cuda(cudaMemcpy(sn.arena.data(), d_arena + q->arena_off, sn.arena.size(), cudaMemcpyDeviceToHost),
                   "read request records");
        XwJob& J = sn.jobs[0];
        J.rep_begin = 0;
        J.ladder_off = 0;
        sn.rec_off.resize(R);
        for (int r = 0; r < R; ++r) {
            sn.rec_off[r] = (uint64_t)r * J.record_bytes;
            reinterpret_cast<RepHeader*>(sn.arena.data() + sn.rec_off[r])->job = 0;
        }
        sn.ladder = q->has_ladder ? q->temps : std::vector<double>(1, 0.0);
        sn.t_init.assign(1, q->t_init);
        sn.params = q->params;
    } catch (const std::exception& e) {
        err = e.what();
    }
    for (size_t k = 0; k < nsaves; ++k) {
        std::pair<uint64_t, std::string> sv;
        {
            std::lock_guard<std::mutex> lk(mu);
            if (q->saves.empty()) break;
            sv = q->saves.front();
            q->saves.pop_front();
        }
        int32_t code = XW_OK;
        std::string msg = err;
        if (!err.empty()) {
            code = XW_ERR_CUDA;
        } else {
            try {
                xw::write_snapshot(sv.second, sn);
            } catch (const std::exception& e) {
                code = XW_ERR_IO;
                msg = e.what();
            }
        }
        std::lock_guard<std::mutex> lk(mu);
        q->save_results[sv.first] = {code, msg};
        q->saves_done = std::max(q->saves_done, sv.first);
        cv_done.notify_all();
    }
    if (!err.empty()) throw std::runtime_error(err);
}

void Server::fail_all(const std::string& msg) {
    std::lock_guard<std::mutex> lk(mu);
    fatal = msg;
    for (auto& kv : table) {
        const ReqPtr& q = kv.second;
        if (q->state == XW_REQ_QUEUED || q->state == XW_REQ_RUNNING) {
            q->status = XW_ERR_CUDA;
            q->error = msg;
            finish_locked(q, XW_REQ_FAILED);
        }
    }
    ready.clear();
    prep_queue.clear();
}

void Server::engine_loop() {
    try {
        check_cuda(cudaSetDevice(cfg.device), "cudaSetDevice");
        for (;;) {
            std::vector<ReqPtr> admitted;
            std::vector<char> cancel_flag;
            {
                std::unique_lock<std::mutex> lk(mu);
                for (;;) {
                    if (stopping) return;
                    admit_locked(admitted);
                    if (!active.empty() || !admitted.empty()) break;
                    cv_engine.wait(lk);
                }
            }
            for (const ReqPtr& q : admitted) place(q);
            select_round();
            const double t_round0 = now();
            bool any_tempering = false;
            round(any_tempering);
            const double t_host = now();
            const uint64_t stamp = *h_stamp;
            for (int s : selected) slot_req[s]->attained = h_out[s].iters;
            std::vector<std::pair<ReqPtr, std::pair<bool, size_t>>> wanted;
            {
                std::lock_guard<std::mutex> lk(mu);
                stats.busy_seconds += t_host - t_round0;
                cancel_flag.resize(slot_req.size(), 0);
                for (int s : active) {
                    const ReqPtr& q = slot_req[s];
                    cancel_flag[s] = q->cancel;
                    if (q->ckpt_want || !q->saves.empty())
                        wanted.push_back({q, {q->ckpt_want, q->saves.size()}});
                }
            }
            // checkpoints and snapshots asked for since the last round, of
            // the state this round left (before any request retires)
            for (const auto& wv : wanted) checkpoint(wv.first, h_out[wv.first->slot], wv.second.first, wv.second.second);
            std::vector<int> keep;
            keep.reserve(active.size());
            const std::vector<int> current(active);
            std::vector<std::pair<int, int>> leaving;   // slot, final state
            for (int s : current) {
                const ReqPtr& q = slot_req[s];
                const JobOut& o = h_out[s];
                const uint64_t budget = q->job.budget_iters;
                const bool out_of_budget = budget && o.iters >= budget;
                const bool out_of_time = q->params.max_seconds > 0.0 && t_host - q->t_admit >= q->params.max_seconds;
                if (o.first_solver >= 0 || o.err) {
                    leaving.push_back({s, XW_REQ_DONE});
                } else if (cancel_flag[s]) {
                    leaving.push_back({s, XW_REQ_CANCELLED});
                } else if (out_of_budget || out_of_time) {
                    leaving.push_back({s, XW_REQ_DONE});
                } else {
                    keep.push_back(s);
                }
            }
            if (!leaving.empty()) {
                // the round's retiring W, rescored and checked in one batch
                std::vector<VerifyItem> items;
                for (const auto& lv : leaving) {
                    const ReqPtr& q = slot_req[lv.first];
                    items.push_back({d_best + (size_t)q->slot * kBestStride, q->spec.n, q->spec.w});
                }
                std::vector<VerifyStats> vs;
                verifier.run(items, stream, vs);
                for (size_t k = 0; k < leaving.size(); ++k) {
                    const ReqPtr q = slot_req[leaving[k].first];
                    retire(q, h_out[leaving[k].first], t_host, stamp, leaving[k].second, vs[k]);
                }
            }
            active.swap(keep);
        }
    } catch (const std::exception& e) {
        fail_all(e.what());
    }
}

void Server::start() {
    check_cuda(cudaSetDevice(cfg.device), "cudaSetDevice");
    cudaDeviceProp props{};
    props = device_properties(cfg.device);
    sms = props.multiProcessorCount;
    check_cuda(cudaDeviceGetAttribute(&optin_smem, cudaDevAttrMaxSharedMemoryPerBlockOptin, cfg.device),
               "cudaDeviceGetAttribute max opt-in shared memory");
    for (int c = 0; c < kClasses; ++c)
        for (bool general : {false, true})
            for (int rpw = 1; rpw <= (c == 0 ? 2 : 1); ++rpw)
                raise_smem_limit(anneal_kernel_fn(opl_of_class(c), general, rpw), cfg.device);
    raise_smem_limit(anneal_kernel_fn(1, false, 1, true), cfg.device);
    if (cfg.max_active_replicas <= 0) {
        // eight waves of the resident warps at the order-32 slot: enough work
        // per round to keep every SM busy through the round's tails (the C5
        // stream, 400 requests: 0.567 G moves/s at four waves and 1000
        // iterations per round, 0.612 G at eight and 2000, with p50/p99
        // time-to-exact 1.16 s / 23.3 s against 1.44 s / 25.2 s; a stream the
        // device keeps up with: p50 0.096 s against 0.099 s)
        int per_sm = 0;
        const int wpb = cfg.warps_per_block > 0 ? cfg.warps_per_block : 4;
        const uint32_t slot = anneal_slot_bytes(32, 16, 1);
        check_cuda(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, anneal_kernel_fn(1, false), 32 * wpb,
                                                                 (size_t)wpb * slot),
                   "cudaOccupancyMaxActiveBlocksPerMultiprocessor");
        cfg.max_active_replicas = std::max(256, 8 * per_sm * wpb * sms);
    }
    if (cfg.max_resident_replicas <= 0) cfg.max_resident_replicas = cfg.max_replica_ids;
    cfg.max_resident_replicas = std::min(cfg.max_resident_replicas, cfg.max_replica_ids);
    const size_t J = (size_t)cfg.max_requests, RI = (size_t)cfg.max_replica_ids;
    auto dmalloc = [&](void** p, size_t bytes, const char* what) {
        check_cuda(cudaMalloc(p, std::max<size_t>(bytes, 16)), what);
    };
    check_cuda(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking), "cudaStreamCreate");
    check_cuda(cudaEventCreate(&ev0), "cudaEventCreate");
    check_cuda(cudaEventCreate(&ev1), "cudaEventCreate");
    check_cuda(cudaEventCreateWithFlags(&fork, cudaEventDisableTiming), "cudaEventCreate");
    for (int c = 0; c < kClasses; ++c) {
        check_cuda(cudaStreamCreateWithFlags(&side[c], cudaStreamNonBlocking), "cudaStreamCreate");
        check_cuda(cudaEventCreateWithFlags(&join[c], cudaEventDisableTiming), "cudaEventCreate");
    }
    dmalloc((void**)&d_jobs, sizeof(XwJob) * J, "cudaMalloc job table");
    dmalloc((void**)&d_arena, cfg.arena_bytes, "cudaMalloc replica arena");
    dmalloc((void**)&d_rec_off, sizeof(uint64_t) * RI, "cudaMalloc record offsets");
    dmalloc((void**)&d_items, sizeof(uint32_t) * RI * kClasses, "cudaMalloc work items");
    dmalloc((void**)&d_counters, sizeof(uint32_t) * kClasses, "cudaMalloc work counters");
    dmalloc((void**)&d_chunk_done, sizeof(uint32_t) * cfg.max_replica_ids, "cudaMalloc chunk counters");
    dmalloc((void**)&d_ladder, sizeof(double) * RI, "cudaMalloc ladders");
    dmalloc((void**)&d_out, sizeof(JobOut) * J, "cudaMalloc results");
    dmalloc((void**)&d_best_off, sizeof(uint64_t) * J, "cudaMalloc result offsets");
    dmalloc((void**)&d_best, kBestStride * J, "cudaMalloc result states");
    dmalloc((void**)&d_stamp, sizeof(uint64_t), "cudaMalloc clock");
    check_cuda(cudaMallocHost((void**)&h_out, sizeof(JobOut) * J), "cudaMallocHost results");
    check_cuda(cudaMallocHost((void**)&h_stamp, sizeof(uint64_t)), "cudaMallocHost clock");
    check_cuda(cudaMemsetAsync(d_jobs, 0, sizeof(XwJob) * J, stream), "clear job table");
    std::vector<uint64_t> best_off(J);
    for (size_t j = 0; j < J; ++j) best_off[j] = j * kBestStride;
    check_cuda(cudaMemcpyAsync(d_best_off, best_off.data(), sizeof(uint64_t) * J, cudaMemcpyHostToDevice, stream),
               "upload result offsets");
    check_cuda(cudaStreamSynchronize(stream), "cudaStreamSynchronize");
    arena_alloc.init(cfg.arena_bytes / 256);
    rep_alloc.init(RI);
    ladder_alloc.init(RI);
    slot_req.assign(J, nullptr);
    for (int s = (int)J - 1; s >= 0; --s) free_slots.push_back(s);
    stats.arena_bytes = cfg.arena_bytes;
    stats.quantum_iters = cfg.quantum_iters;
    stats.max_resident_replicas = cfg.max_resident_replicas;
    stats.schedule = cfg.schedule;
    stats.max_active_replicas = cfg.max_active_replicas;
    int threads = cfg.prep_threads;
    if (threads <= 0) threads = std::max(1, (int)std::thread::hardware_concurrency() / 2);
    for (int t = 0; t < threads; ++t) workers.emplace_back([this] { worker_loop(); });
    engine = std::thread([this] { engine_loop(); });
}

void Server::stop() {
    {
        std::lock_guard<std::mutex> lk(mu);
        stopping = true;
    }
    cv_engine.notify_all();
    cv_prep.notify_all();
    if (engine.joinable()) engine.join();
    for (auto& t : workers)
        if (t.joinable()) t.join();
    {
        std::lock_guard<std::mutex> lk(mu);
        for (auto& kv : table) {
            const ReqPtr& q = kv.second;
            if (q->state == XW_REQ_QUEUED || q->state == XW_REQ_RUNNING) finish_locked(q, XW_REQ_CANCELLED);
        }
    }
    if (stream) cudaStreamSynchronize(stream);
    for (void* p : {(void*)d_jobs, (void*)d_arena, (void*)d_rec_off, (void*)d_items, (void*)d_counters, (void*)d_chunk_done,
                    (void*)d_ladder, (void*)d_out, (void*)d_best_off, (void*)d_best, (void*)d_stamp})
        if (p) cudaFree(p);
    if (h_out) cudaFreeHost(h_out);
    if (h_stamp) cudaFreeHost(h_stamp);
    if (ev0) cudaEventDestroy(ev0);
    if (ev1) cudaEventDestroy(ev1);
    if (fork) cudaEventDestroy(fork);
    for (int c = 0; c < kClasses; ++c) {
        if (side[c]) cudaStreamSynchronize(side[c]);
        if (side[c]) cudaStreamDestroy(side[c]);
        if (join[c]) cudaEventDestroy(join[c]);
    }
    if (stream) cudaStreamDestroy(stream);
    stream = nullptr;
}

}  // namespace xw

using xw::ReqPtr;
using xw::Server;

struct xw_server {
    Server s;
};

namespace {

int32_t fail_with(int32_t code, const std::string& msg) {
    xw::set_last_error(msg);
    return code;
}

void copy_out(const xw::Request& q, xw_request_result* res, int8_t* best) {
    if (res) {
        *res = q.res;
        res->state = q.state;
        res->status = q.status;
        res->n = q.spec.n;
        res->w = q.spec.w;
        res->replicas = q.spec.replicas;
        res->submit_seconds = q.t_submit;
        res->admit_seconds = q.t_admit;
        res->finish_seconds = q.t_finish;
        std::snprintf(res->error, sizeof res->error, "%s", q.error.c_str());
    }
    if (best && q.state >= XW_REQ_DONE && !q.best.empty()) std::memcpy(best, q.best.data(), q.best.size());
}

}  // namespace

extern "C" {

void xw_server_config_default(xw_server_config* c) {
    if (!c) return;
    std::memset(c, 0, sizeof *c);
    c->device = 0;
    c->quantum_iters = 2000;
    c->max_requests = 1024;
    c->max_resident_replicas = 0;
    c->max_replica_ids = 262144;
    c->warps_per_block = 0;
    c->prep_threads = 0;
    c->sylvester_shortcut = 1;
    c->arena_bytes = 1ull << 30;
    c->schedule = XW_SCHED_LEAST_ATTAINED;
    c->max_active_replicas = 0;
}

int32_t xw_server_create(const xw_server_config* c, xw_server** out) {
    if (!out) return fail_with(XW_ERR_INVALID, "server output pointer is null");
    *out = nullptr;
    xw_server_config cfg;
    xw_server_config_default(&cfg);
    if (c) cfg = *c;
    if (cfg.quantum_iters < 1) return fail_with(XW_ERR_INVALID, "server quantum must be positive");
    if (cfg.max_requests < 1 || cfg.max_requests > (1 << 20))
        return fail_with(XW_ERR_INVALID, "server request slots must be in [1, 1048576]");
    if (cfg.max_replica_ids < 1) return fail_with(XW_ERR_INVALID, "server replica ids must be positive");
    if (cfg.warps_per_block < 0 || cfg.warps_per_block > 16)
        return fail_with(XW_ERR_INVALID, "CUDA warps per block must be in [0, 16]");
    if (cfg.replicas_per_warp < 0 || cfg.replicas_per_warp > 2)
        return fail_with(XW_ERR_INVALID, "replicas per warp must be 0, 1 or 2");
    if (cfg.arena_bytes < 4096) return fail_with(XW_ERR_INVALID, "server arena must be at least 4 KiB");
    if (cfg.schedule != XW_SCHED_ALL && cfg.schedule != XW_SCHED_LEAST_ATTAINED)
        return fail_with(XW_ERR_INVALID, "server schedule must be XW_SCHED_ALL or XW_SCHED_LEAST_ATTAINED");
    auto* h = new (std::nothrow) xw_server;
    if (!h) return fail_with(XW_ERR_CAPACITY, "out of host memory");
    h->s.cfg = cfg;
    try {
        h->s.start();
    } catch (const std::exception& e) {
        h->s.stop();
        delete h;
        return fail_with(XW_ERR_CUDA, e.what());
    }
    *out = h;
    return XW_OK;
}

int32_t xw_submit(xw_server* h, const xw_request* r, uint64_t* id) {
    if (!h || !r || !id) return fail_with(XW_ERR_INVALID, "server, request and id must be non-null");
    Server& s = h->s;
    xw_params p;
    if (r->params) p = *r->params;
    else xw_params_default(&p);
    p.device = s.cfg.device;
    p.stop_on_solve = 2;
    p.replicas = r->replicas;
    const std::string err = xw::validate(r->n, r->w, p);
    if (!err.empty()) return fail_with(XW_ERR_INVALID, err);
    const char* why = xw_impossibility_reason(r->n, r->w);
    if (why && *why) return fail_with(XW_ERR_INVALID, why);
    if (r->n > XW_MAX_ORDER_SHARED)
        return fail_with(XW_ERR_CAPACITY, xw::strfmt("order %d is beyond the served orders' maximum of %d", r->n,
                                                     XW_MAX_ORDER_SHARED));
    if (r->replicas < 1) return fail_with(XW_ERR_INVALID, "CUDA replica count must be positive");
    if (r->replicas > s.cfg.max_replica_ids || r->replicas > s.cfg.max_resident_replicas)
        return fail_with(XW_ERR_CAPACITY, "request has more replicas than the server can hold");
    if (p.tempering) {
        if (r->replicas > XW_MAX_RUNGS)
            return fail_with(XW_ERR_INVALID, xw::strfmt("a tempering ladder has at most %d rungs", XW_MAX_RUNGS));
        if (p.exchange_interval % s.cfg.quantum_iters != 0)
            return fail_with(XW_ERR_INVALID, xw::strfmt("exchange interval %d is not a multiple of the server "
                                                        "quantum %d", p.exchange_interval, s.cfg.quantum_iters));
    }
    const int m = std::min(r->w, r->n - r->w);
    const uint64_t rec = ((128 + 2 * (uint64_t)xw_pad16((uint32_t)(r->n * r->n)) +
                           xw_pad16((uint32_t)(r->n * m))) + 127) & ~uint64_t(127);
    if (rec * (uint64_t)r->replicas > s.cfg.arena_bytes)
        return fail_with(XW_ERR_CAPACITY, "request records exceed the server arena");
    auto q = std::make_shared<xw::Request>();
    q->spec.n = r->n;
    q->spec.w = r->w;
    q->spec.seed = r->seed;
    q->spec.replicas = r->replicas;
    q->spec.max_moves = r->max_moves;
    q->params = p;
    if (r->starts) q->starts.assign(r->starts, r->starts + (size_t)r->replicas * r->n * r->n);
    std::lock_guard<std::mutex> lk(s.mu);
    if (!s.fatal.empty()) return fail_with(XW_ERR_CUDA, s.fatal);
    if (s.stopping) return fail_with(XW_ERR_INVALID, "server is stopping");
    q->id = s.next_id++;
    q->t_submit = s.now();
    q->res.admit_seconds = -1.0;
    q->res.finish_seconds = -1.0;
    q->res.time_to_solution_seconds = -1.0;
    s.table[q->id] = q;
    s.prep_queue.push_back(q);
    ++s.stats.submitted;
    s.cv_prep.notify_one();
    *id = q->id;
    return XW_OK;
}

int32_t xw_poll(xw_server* h, uint64_t id, xw_request_result* res, int8_t* best) {
    if (!h) return fail_with(XW_ERR_INVALID, "server is null");
    std::lock_guard<std::mutex> lk(h->s.mu);
    auto it = h->s.table.find(id);
    if (it == h->s.table.end()) return fail_with(XW_ERR_NOT_FOUND, xw::strfmt("unknown request %llu",
                                                                              (unsigned long long)id));
    copy_out(*it->second, res, best);
    return XW_OK;
}

int32_t xw_wait(xw_server* h, uint64_t id, double timeout_seconds, xw_request_result* res, int8_t* best) {
    if (!h) return fail_with(XW_ERR_INVALID, "server is null");
    Server& s = h->s;
    std::unique_lock<std::mutex> lk(s.mu);
    auto it = s.table.find(id);
    if (it == s.table.end()) return fail_with(XW_ERR_NOT_FOUND, xw::strfmt("unknown request %llu",
                                                                           (unsigned long long)id));
    ReqPtr q = it->second;
    auto finished = [&] { return q->state >= XW_REQ_DONE; };
    if (timeout_seconds < 0.0) {
        s.cv_done.wait(lk, finished);
    } else if (!s.cv_done.wait_for(lk, std::chrono::duration<double>(timeout_seconds), finished)) {
        copy_out(*q, res, nullptr);
        return fail_with(XW_ERR_TIMEOUT, "request is still running");
    }
    copy_out(*q, res, best);
    return XW_OK;
}

int32_t xw_checkpoint(xw_server* h, uint64_t id, double timeout_seconds, xw_request_result* res, int8_t* best) {
    if (!h) return fail_with(XW_ERR_INVALID, "server is null");
    Server& s = h->s;
    std::unique_lock<std::mutex> lk(s.mu);
    auto it = s.table.find(id);
    if (it == s.table.end()) return fail_with(XW_ERR_NOT_FOUND, xw::strfmt("unknown request %llu",
                                                                           (unsigned long long)id));
    ReqPtr q = it->second;
    if (q->state >= XW_REQ_DONE) {
        copy_out(*q, res, best);
        return XW_OK;
    }
    const uint64_t seq0 = q->ckpt_seq;
    q->ckpt_want = true;
    s.cv_engine.notify_one();
    auto ready = [&] { return q->ckpt_seq > seq0 || q->state >= XW_REQ_DONE; };
    if (timeout_seconds < 0.0) {
        s.cv_done.wait(lk, ready);
    } else if (!s.cv_done.wait_for(lk, std::chrono::duration<double>(timeout_seconds), ready)) {
        copy_out(*q, res, nullptr);
        return fail_with(XW_ERR_TIMEOUT, "no engine round has ended for the request yet");
    }
    if (q->state >= XW_REQ_DONE) {
        copy_out(*q, res, best);
        return XW_OK;
    }
    if (res) {
        copy_out(*q, res, nullptr);
        const int32_t state = res->state, status = res->status;
        const double ts = res->submit_seconds, ta = res->admit_seconds, tf = res->finish_seconds;
        char error[sizeof res->error];
        std::memcpy(error, res->error, sizeof error);
        *res = q->ckpt_res;
        res->state = state;
        res->status = status;
        res->n = q->spec.n;
        res->w = q->spec.w;
        res->replicas = q->spec.replicas;
        res->submit_seconds = ts;
        res->admit_seconds = ta;
        res->finish_seconds = tf;
        std::memcpy(res->error, error, sizeof error);
    }
    if (best && !q->ckpt_best.empty()) std::memcpy(best, q->ckpt_best.data(), q->ckpt_best.size());
    return XW_OK;
}

int32_t xw_request_save(xw_server* h, uint64_t id, const char* path, double timeout_seconds) {
    if (!h || !path || !*path) return fail_with(XW_ERR_INVALID, "server and path must be non-null");
    Server& s = h->s;
    std::unique_lock<std::mutex> lk(s.mu);
    auto it = s.table.find(id);
    if (it == s.table.end()) return fail_with(XW_ERR_NOT_FOUND, xw::strfmt("unknown request %llu",
                                                                           (unsigned long long)id));
    ReqPtr q = it->second;
    if (q->state >= XW_REQ_DONE)
        return fail_with(XW_ERR_INVALID, "request has finished: its population is no longer resident");
    const uint64_t ticket = ++q->save_tickets;
    q->saves.emplace_back(ticket, std::string(path));
    s.cv_engine.notify_one();
    auto done = [&] { return q->saves_done >= ticket; };
    if (timeout_seconds < 0.0) {
        s.cv_done.wait(lk, done);
    } else if (!s.cv_done.wait_for(lk, std::chrono::duration<double>(timeout_seconds), done)) {
        // the snapshot may still be written later; its result is dropped
        return fail_with(XW_ERR_TIMEOUT, "no engine round has ended for the request yet");
    }
    auto r = q->save_results.find(ticket);
    if (r == q->save_results.end()) return fail_with(XW_ERR_INTERNAL, "snapshot result missing");
    const std::pair<int32_t, std::string> out = r->second;
    q->save_results.erase(r);
    if (out.first != XW_OK) return fail_with(out.first, out.second);
    return XW_OK;
}

int32_t xw_submit_snapshot(xw_server* h, const char* path, uint64_t* id) {
    if (!h || !path || !id) return fail_with(XW_ERR_INVALID, "server, path and id must be non-null");
    Server& s = h->s;
    xw::Snapshot sn;
    try {
        sn = xw::read_snapshot(path);
    } catch (const std::exception& e) {
        return fail_with(XW_ERR_INVALID, e.what());
    }
    if (sn.jobs.size() != 1) return fail_with(XW_ERR_INVALID, "a request snapshot holds exactly one job");
    XwJob J = sn.jobs[0];
    const int R = J.replicas;
    if (J.n > XW_MAX_ORDER_SHARED || J.large)
        return fail_with(XW_ERR_CAPACITY, xw::strfmt("order %d is beyond the served orders' maximum of %d", J.n,
                                                     XW_MAX_ORDER_SHARED));
    if (R > s.cfg.max_replica_ids || R > s.cfg.max_resident_replicas)
        return fail_with(XW_ERR_CAPACITY, "request has more replicas than the server can hold");
    if ((uint64_t)R * J.record_bytes > s.cfg.arena_bytes)
        return fail_with(XW_ERR_CAPACITY, "request records exceed the server arena");
    xw_params p = sn.params;
    p.device = s.cfg.device;
    p.stop_on_solve = 2;
    p.replicas = R;
    if (p.tempering) {
        if (R > XW_MAX_RUNGS)
            return fail_with(XW_ERR_INVALID, xw::strfmt("a tempering ladder has at most %d rungs", XW_MAX_RUNGS));
        if (p.exchange_interval % s.cfg.quantum_iters != 0)
            return fail_with(XW_ERR_INVALID, xw::strfmt("exchange interval %d is not a multiple of the server "
                                                        "quantum %d", p.exchange_interval, s.cfg.quantum_iters));
        if ((uint64_t)J.ladder_off + R > sn.ladder.size())
            return fail_with(XW_ERR_INVALID, "corrupt population snapshot: ladder");
    }
    auto q = std::make_shared<xw::Request>();
    q->spec.n = J.n;
    q->spec.w = J.w;
    q->spec.seed = 0;
    q->spec.replicas = R;
    q->spec.max_moves = 0;
    q->params = p;
    // a batch snapshot exchanges after every launch of exchange_interval
    // iterations; the server at the same iteration counts
    J.exchange_iters = p.tempering ? (uint64_t)p.exchange_interval : 0;
    J.done = 0;
    q->records.resize((size_t)R * J.record_bytes);
    for (int r = 0; r < R; ++r) {
        const uint8_t* src = sn.arena.data() + sn.rec_off[J.rep_begin + r];
        std::memcpy(q->records.data() + (size_t)r * J.record_bytes, src, J.record_bytes);
        q->attained = std::max(q->attained, reinterpret_cast<const RepHeader*>(src)->it);
    }
    if (p.tempering) q->temps.assign(sn.ladder.begin() + J.ladder_off, sn.ladder.begin() + J.ladder_off + R);
    q->t_init = sn.t_init[0];
    J.rep_begin = 0;
    J.ladder_off = 0;
    q->job = J;
    std::lock_guard<std::mutex> lk(s.mu);
    if (!s.fatal.empty()) return fail_with(XW_ERR_CUDA, s.fatal);
    if (s.stopping) return fail_with(XW_ERR_INVALID, "server is stopping");
    q->id = s.next_id++;
    q->t_submit = s.now();
    q->res.admit_seconds = -1.0;
    q->res.finish_seconds = -1.0;
    q->res.time_to_solution_seconds = -1.0;
    s.table[q->id] = q;
    s.ready[q->id] = q;   // built already: straight to admission
    ++s.stats.submitted;
    s.cv_engine.notify_one();
    *id = q->id;
    return XW_OK;
}

int32_t xw_cancel(xw_server* h, uint64_t id) {
    if (!h) return fail_with(XW_ERR_INVALID, "server is null");
    Server& s = h->s;
    std::lock_guard<std::mutex> lk(s.mu);
    auto it = s.table.find(id);
    if (it == s.table.end()) return fail_with(XW_ERR_NOT_FOUND, xw::strfmt("unknown request %llu",
                                                                           (unsigned long long)id));
    const ReqPtr& q = it->second;
    if (q->state == XW_REQ_QUEUED) {
        s.ready.erase(q->id);
        q->res.time_to_solution_seconds = -1.0;
        s.finish_locked(q, XW_REQ_CANCELLED);
    } else if (q->state == XW_REQ_RUNNING) {
        q->cancel = true;
    }
    return XW_OK;
}

int32_t xw_release(xw_server* h, uint64_t id) {
    if (!h) return fail_with(XW_ERR_INVALID, "server is null");
    std::lock_guard<std::mutex> lk(h->s.mu);
    auto it = h->s.table.find(id);
    if (it == h->s.table.end()) return fail_with(XW_ERR_NOT_FOUND, xw::strfmt("unknown request %llu",
                                                                              (unsigned long long)id));
    if (it->second->state < XW_REQ_DONE) return fail_with(XW_ERR_INVALID, "request has not finished");
    h->s.table.erase(it);
    return XW_OK;
}

int32_t xw_server_get_stats(xw_server* h, xw_server_stats* out) {
    if (!h || !out) return fail_with(XW_ERR_INVALID, "server and output must be non-null");
    Server& s = h->s;
    std::lock_guard<std::mutex> lk(s.mu);
    *out = s.stats;
    uint64_t queued = 0, running = 0, resident = 0;
    for (auto& kv : s.table) {
        if (kv.second->state == XW_REQ_QUEUED) ++queued;
        if (kv.second->state == XW_REQ_RUNNING) {
            ++running;
            resident += (uint64_t)kv.second->spec.replicas;
        }
    }
    out->queued = queued;
    out->running = running;
    out->resident_replicas = resident;
    out->arena_bytes_used = s.arena_alloc.used * 256;
    return XW_OK;
}

void xw_server_destroy(xw_server* h) {
    if (!h) return;
    h->s.stop();
    delete h;
}

}  // extern "C"
