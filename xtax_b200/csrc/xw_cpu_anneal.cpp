// xw_cpu_anneal.cpp -- the CPU annealer behind the xweigh drop-in.
//
// The reference's CPU tool anneals one W(n,w) with one worker thread per
// core (anneal_worker, run_annealer and the monitor thread,
// src/xweigh_anneal.hpp:909-1291): each worker runs simulated annealing on
// its own state (greedy choice among sampled candidates, Metropolis on the
// L1 score, geometric cooling, reheat and reseed from the global best when
// stuck); with two or more workers they form a parallel-tempering ladder
// whose rungs a monitor thread exchanges every exchange_interval moves per
// worker, and the monitor also writes the best matrix every save_interval.
// This is that engine on the host library's CpuState, with the reference's
// seeds, draw order and log lines, so that a single-thread run retraces the
// reference's run move for move.  It is the fallback for hosts without a
// B200.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <limits>
#include <mutex>
#include <random>
#include <stdexcept>
#include <string>
#include <thread>
#include <vector>

#include "../../include/xw.h"
#include "xw_cpu_anneal.h"
#include "xw_host_internal.h"

namespace xw {

namespace {

bool better_pair(int64_t sa, int64_t ca, int64_t sb, int64_t cb) { return sa < sb || (sa == sb && ca < cb); }

double unit(std::mt19937& rng) { return std::generate_canonical<double, 53>(rng); }

std::string num(double v) {
    char buf[64];
    std::snprintf(buf, sizeof buf, "%g", v);
    return buf;
}

// one worker's best state, replayed from its accepted moves on improvement
struct WorkerBest {
    std::mutex mu;
    std::vector<int8_t> entries;
    int64_t score = 0, conflicts = 0;
};

// one cache line per worker: the monitor reads them while workers write
struct alignas(64) WorkerStatus {
    std::atomic<int> rung{0};
    std::atomic<int64_t> score{0};
};

struct Shared {
    std::atomic<bool> done{false};
    std::atomic<uint64_t> total_moves{0};
    std::mutex best_mu;
    std::atomic<int64_t> best_score{0}, best_conflicts{0};
    int best_owner = 0;
    std::atomic<uint64_t> best_version{1};   // the start state is version 1, written first
    std::vector<WorkerBest> bests;
    std::vector<WorkerStatus> statuses;
    std::vector<double> temperatures;
    std::mutex print_mu;
    double last_log = -1e30;

    Shared(const CpuState& start, int threads) : bests((size_t)threads), statuses((size_t)threads) {
        best_score = start.score();
        best_conflicts = start.conflicts();
        for (WorkerBest& b : bests) {
            b.entries = start.entries();
            b.score = start.score();
            b.conflicts = start.conflicts();
        }
    }
};

// a worker publishes a state that beats the shared best (anneal.hpp:901-907)
bool should_publish(const CpuState& s, const Shared& sh) {
    return better_pair(s.score(), s.conflicts(), sh.best_score.load(std::memory_order_relaxed),
                       sh.best_conflicts.load(std::memory_order_relaxed));
}

void worker(const CpuAnnealParams& p, uint32_t seed, int id, double t_init, const CpuState& start, Shared& sh,
            std::chrono::steady_clock::time_point t0) {
    CpuState cur = start;
    std::mt19937 rng(seed);
    CpuParams cp;
    cp.sign_fraction = p.sign_fraction;
    cp.target_fraction = p.target_fraction;
    cp.target_samples = p.target_samples;
    int64_t lbest_s = cur.score(), lbest_c = cur.conflicts();
    std::vector<CpuMove> path;
    path.reserve((size_t)std::min(p.stuck_threshold, 250000));
    int msi = 0, cool = 0;
    uint64_t local_moves = 0, unreported = 0;
    double T = t_init;
    const int n = cur.order(), w = cur.weight();

    auto save_local_best = [&]() {
        WorkerBest& b = sh.bests[(size_t)id];
        std::lock_guard<std::mutex> lock(b.mu);
        for (const CpuMove& mv : path) CpuState::apply_to_entries(b.entries, n, mv);
        b.score = cur.score();
        b.conflicts = cur.conflicts();
        path.clear();
    };
    auto restore_global_best = [&]() {
        int owner;
        {
            std::lock_guard<std::mutex> lock(sh.best_mu);
            owner = sh.best_owner;
        }
        std::vector<int8_t> e;
        int64_t s, c;
        {
            WorkerBest& b = sh.bests[(size_t)owner];
            std::lock_guard<std::mutex> lock(b.mu);
            e = b.entries;
            s = b.score;
            c = b.conflicts;
        }
        cur = CpuState::from_entries(n, w, std::move(e));
        if (cur.score() != s || cur.conflicts() != c) throw std::runtime_error("xweigh best snapshot score mismatch");
        lbest_s = s;
        lbest_c = c;
        path.clear();
        WorkerBest& mine = sh.bests[(size_t)id];
        std::lock_guard<std::mutex> lock(mine.mu);
        mine.entries = cur.entries();
        mine.score = s;
        mine.conflicts = c;
    };

    while (!sh.done.load(std::memory_order_relaxed)) {
        if (p.tempering) T = sh.temperatures[(size_t)sh.statuses[(size_t)id].rung.load(std::memory_order_relaxed)];
        // the best of `samples` proposals (greedy), or one
        CpuMove sel;
        int64_t sel_ds = 0, sel_dc = 0;
        bool have = false;
        const bool greedy = unit(rng) < p.greedy_fraction;
        const int samples = greedy ? p.candidate_samples : 1;
        for (int k = 0; k < samples; ++k) {
            CpuMove cand;
            const bool targeted = unit(rng) < p.target_fraction;
            if (!cur.propose(rng, cp, targeted, cand)) continue;
            int64_t ds, dc;
            cur.evaluate(cand, ds, dc);
            if (!have || better_pair(ds, dc, sel_ds, sel_dc)) {
                sel = cand;
                sel_ds = ds;
                sel_dc = dc;
                have = true;
            }
        }
        if (!have) continue;
        ++local_moves;
        ++unreported;
        const bool accept = sel_ds <= 0 || unit(rng) < std::exp(-(double)sel_ds / std::max(T, 1e-12));
        if (accept) {
            cur.commit(sel);
            path.push_back(sel);
        }
        if (better_pair(cur.score(), cur.conflicts(), lbest_s, lbest_c)) {
            lbest_s = cur.score();
            lbest_c = cur.conflicts();
            msi = 0;
            save_local_best();
        } else {
            ++msi;
        }
        if (accept && should_publish(cur, sh)) {
            bool published = false;
            {
                std::lock_guard<std::mutex> lock(sh.best_mu);
                if (better_pair(cur.score(), cur.conflicts(), sh.best_score.load(std::memory_order_relaxed),
                                sh.best_conflicts.load(std::memory_order_relaxed))) {
                    sh.best_score.store(cur.score(), std::memory_order_relaxed);
                    sh.best_conflicts.store(cur.conflicts(), std::memory_order_relaxed);
                    sh.best_owner = id;
                    sh.best_version.fetch_add(1, std::memory_order_relaxed);
                    published = true;
                    if (cur.solved()) sh.done.store(true, std::memory_order_relaxed);
                }
            }
            if (published) {
                const double el = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
                std::lock_guard<std::mutex> lock(sh.print_mu);
                if (cur.solved() || el - sh.last_log >= 0.05) {
                    sh.last_log = el;
                    if (p.log)
                        p.log("[t=" + num(el) + "s] new best score=" + std::to_string(cur.score()) +
                              " conflicts=" + std::to_string(cur.conflicts()) + " (thread " + std::to_string(id) +
                              ")");
                }
            }
        }
        if (!p.tempering) {
            if (++cool >= p.moves_per_cool) {
                cool = 0;
                T = std::max(p.t_min, T * p.cooling);
            }
            if (msi >= p.stuck_threshold) {
                msi = 0;
                T = std::max(p.t_min, t_init * p.reheat);
                const int64_t g = sh.best_score.load(std::memory_order_relaxed);
                if ((double)cur.score() > p.reseed_factor * (double)std::max<int64_t>(1, g)) restore_global_best();
            }
        }
        if (path.size() >= 250000) {
            // a long run without improvement: the replay list is dropped and
            // the state reloaded from this worker's best or the global one
            int owner;
            {
                std::lock_guard<std::mutex> lock(sh.best_mu);
                owner = sh.best_owner;
            }
            if (owner == id) {
                std::vector<int8_t> e;
                {
                    WorkerBest& b = sh.bests[(size_t)id];
                    std::lock_guard<std::mutex> lock(b.mu);
                    e = b.entries;
                }
                cur = CpuState::from_entries(n, w, std::move(e));
                path.clear();
                msi = 0;
            } else {
                restore_global_best();
            }
        }
        if ((local_moves & 255u) == 0) sh.statuses[(size_t)id].score.store(cur.score(), std::memory_order_relaxed);
        if (unreported >= 4096) {
            sh.total_moves.fetch_add(unreported, std::memory_order_relaxed);
            unreported = 0;
        }
    }
    sh.total_moves.fetch_add(unreported, std::memory_order_relaxed);
    sh.statuses[(size_t)id].score.store(cur.score(), std::memory_order_relaxed);
}

}  // namespace

double reference_worker_bytes(int n, int w) {
    const int m = std::min(w, n - w);
    return (double)n * n * 4.0 + 8.0 * n + 2.0 * (double)n * m;
}

CpuAnnealResult cpu_anneal(const CpuState& start, CpuAnnealParams p) {
    CpuAnnealResult out;
    if (p.threads < 1) throw std::invalid_argument("threads must be positive");
    if (p.threads < 2) p.tempering = false;
    if (start.solved()) {
        out.best = start;
        return out;
    }
    const uint32_t base = p.seed ? (uint32_t)p.seed : (uint32_t)std::random_device{}();
    CpuParams cp;
    cp.sign_fraction = p.sign_fraction;
    cp.target_fraction = p.target_fraction;
    cp.target_samples = p.target_samples;
    cp.t_init = p.t_init;
    const double t_init = calibrate_temperature(start, cp, base);
    out.t_init = t_init;
    Shared sh(start, p.threads);
    if (p.tempering) {
        // geometric ladder t_min .. t_init, one rung per worker
        sh.temperatures.resize((size_t)p.threads);
        const double bottom = std::min(p.t_min, t_init);
        const double ratio = std::pow(t_init / std::max(bottom, 1e-12), 1.0 / (double)(p.threads - 1));
        double t = bottom;
        for (int k = 0; k < p.threads; ++k) {
            sh.temperatures[(size_t)k] = t;
            sh.statuses[(size_t)k].rung.store(k, std::memory_order_relaxed);
            sh.statuses[(size_t)k].score.store(start.score(), std::memory_order_relaxed);
            t *= ratio;
        }
    }
    const auto t0 = std::chrono::steady_clock::now();
    if (p.log)
        p.log("[t=0s] start score=" + std::to_string(start.score()) + " conflicts=" +
              std::to_string(start.conflicts()) + " n=" + std::to_string(start.order()) + " w=" +
              std::to_string(start.weight()) + " threads=" + std::to_string(p.threads) + " worker_mib=" +
              num(reference_worker_bytes(start.order(), start.weight()) / (1024.0 * 1024.0)) + " t_init=" +
              num(t_init) + (p.tempering ? " (parallel tempering)" : ""));

    std::mt19937 seed_rng(base);
    std::vector<std::thread> workers;
    std::vector<std::exception_ptr> errors((size_t)p.threads);
    for (int k = 0; k < p.threads; ++k) {
        const uint32_t seed = seed_rng() ^ ((uint32_t)k * 0x9e3779b9u);
        workers.emplace_back([&, seed, k]() {
            try {
                worker(p, seed, k, t_init, start, sh, t0);
            } catch (...) {
                errors[(size_t)k] = std::current_exception();
                sh.done.store(true);
            }
        });
    }
    std::thread monitor([&]() {
        std::mt19937 xrng(base ^ 0xc0ffeeu);
        uint64_t last_exchange = 0, saved_version = 0;
        double last_save = -1e30;
        while (!sh.done.load(std::memory_order_relaxed)) {
            const double el = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
            if ((p.stop && p.stop->load(std::memory_order_relaxed)) || (p.max_seconds > 0.0 && el >= p.max_seconds)) {
                sh.done.store(true, std::memory_order_relaxed);
                break;
            }
            const uint64_t moves = sh.total_moves.load(std::memory_order_relaxed);
            const uint64_t stride = (uint64_t)p.exchange_interval * (uint64_t)p.threads;
            if (p.tempering && moves - last_exchange >= stride) {
                // adjacent rungs bottom-up on the workers' last reported
                // scores (anneal.hpp:1187-1221)
                last_exchange = moves;
                std::vector<int> owner((size_t)p.threads);
                for (int k = 0; k < p.threads; ++k)
                    owner[(size_t)sh.statuses[(size_t)k].rung.load(std::memory_order_relaxed)] = k;
                for (int r = 0; r + 1 < p.threads; ++r) {
                    const int a = owner[(size_t)r], b = owner[(size_t)r + 1];
                    const double t1 = sh.temperatures[(size_t)r], t2 = sh.temperatures[(size_t)r + 1];
                    const double s1 = (double)sh.statuses[(size_t)a].score.load(std::memory_order_relaxed);
                    const double s2 = (double)sh.statuses[(size_t)b].score.load(std::memory_order_relaxed);
                    const double x = (1.0 / t1 - 1.0 / t2) * (s1 - s2);
                    if (x >= 0.0 || unit(xrng) < std::exp(x)) {
                        sh.statuses[(size_t)a].rung.store(r + 1, std::memory_order_relaxed);
                        sh.statuses[(size_t)b].rung.store(r, std::memory_order_relaxed);
                        std::swap(owner[(size_t)r], owner[(size_t)r + 1]);
                    }
                }
            }
            const uint64_t version = sh.best_version.load(std::memory_order_relaxed);
            if (version != saved_version && el - last_save >= p.save_interval) {
                std::vector<int8_t> snap;
                uint64_t snap_version;
                int owner;
                {
                    std::lock_guard<std::mutex> lock(sh.best_mu);
                    owner = sh.best_owner;
                    snap_version = sh.best_version.load(std::memory_order_relaxed);
                }
                {
                    WorkerBest& b = sh.bests[(size_t)owner];
                    std::lock_guard<std::mutex> lock(b.mu);
                    snap = b.entries;
                }
                if (p.save) p.save(snap);
                saved_version = snap_version;
                last_save = el;
            }
            std::this_thread::sleep_for(std::chrono::milliseconds(2));
        }
    });
    for (std::thread& t : workers) t.join();
    monitor.join();
    for (const auto& e : errors)
        if (e) std::rethrow_exception(e);

    out.seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    out.moves = sh.total_moves.load(std::memory_order_relaxed);
    if (p.log)
        p.log("done moves=" + std::to_string(out.moves) + " seconds=" + num(out.seconds) + " moves_per_sec=" +
              num(out.seconds > 0.0 ? (double)out.moves / out.seconds : 0.0));
    int owner = 0;
    int64_t bs = std::numeric_limits<int64_t>::max(), bc = std::numeric_limits<int64_t>::max();
    for (int k = 0; k < p.threads; ++k) {
        WorkerBest& b = sh.bests[(size_t)k];
        std::lock_guard<std::mutex> lock(b.mu);
        if (better_pair(b.score, b.conflicts, bs, bc)) {
            owner = k;
            bs = b.score;
            bc = b.conflicts;
        }
    }
    out.best = CpuState::from_entries(start.order(), start.weight(), sh.bests[(size_t)owner].entries);
    if (out.best.score() != bs || out.best.conflicts() != bc)
        throw std::runtime_error("xweigh final best snapshot mismatch");
    return out;
}

}  // namespace xw

// ---- C ABI ----------------------------------------------------------------

using namespace xw;

extern "C" {

void xw_cpu_params_default(xw_cpu_params* p) {
    if (!p) return;
    const CpuAnnealParams d;
    p->threads = (int32_t)std::max(1u, std::thread::hardware_concurrency());
    p->tempering = 1;
    p->seed = d.seed;
    p->max_seconds = d.max_seconds;
    p->save_interval = d.save_interval;
    p->sign_fraction = d.sign_fraction;
    p->greedy_fraction = d.greedy_fraction;
    p->candidate_samples = d.candidate_samples;
    p->target_fraction = d.target_fraction;
    p->target_samples = d.target_samples;
    p->exchange_interval = d.exchange_interval;
    p->t_init = d.t_init;
    p->t_min = d.t_min;
    p->cooling = d.cooling;
    p->moves_per_cool = d.moves_per_cool;
    p->stuck_threshold = d.stuck_threshold;
    p->reheat = d.reheat;
    p->reseed_factor = d.reseed_factor;
}

int32_t xw_cpu_run(int32_t n, int32_t w, const xw_cpu_params* p, const int8_t* start, xw_log_fn log,
                   xw_checkpoint_fn checkpoint, void* user, xw_cpu_result* out, int8_t* best_out) {
    if (!p || !out) {
        set_last_error("null argument");
        return XW_ERR_INVALID;
    }
    std::memset(out, 0, sizeof *out);
    if (n < 1 || n > XW_MAX_ORDER_CUDA || w < 1 || w > n) {
        set_last_error("CPU xweigh order and weight must satisfy 1 <= w <= n <= 1024");
        return XW_ERR_INVALID;
    }
    if (p->threads < 1 || p->candidate_samples < 1 || p->target_samples < 1 || p->exchange_interval < 1 ||
        p->moves_per_cool < 1 || p->stuck_threshold < 1 || !(p->t_min > 0.0) || !(p->cooling > 0.0) ||
        !(p->cooling < 1.0) || !(p->reheat > 0.0) || !(p->reseed_factor >= 1.0)) {
        set_last_error("CPU xweigh parameters out of range");
        return XW_ERR_INVALID;
    }
    try {
        CpuAnnealParams q;
        q.threads = p->threads;
        q.tempering = p->tempering != 0;
        q.seed = p->seed;
        q.max_seconds = p->max_seconds;
        q.save_interval = p->save_interval;
        q.sign_fraction = p->sign_fraction;
        q.greedy_fraction = p->greedy_fraction;
        q.candidate_samples = p->candidate_samples;
        q.target_fraction = p->target_fraction;
        q.target_samples = p->target_samples;
        q.exchange_interval = p->exchange_interval;
        q.t_init = p->t_init;
        q.t_min = p->t_min;
        q.cooling = p->cooling;
        q.moves_per_cool = p->moves_per_cool;
        q.stuck_threshold = p->stuck_threshold;
        q.reheat = p->reheat;
        q.reseed_factor = p->reseed_factor;
        if (log) q.log = [&](const std::string& line) { log(line.c_str(), user); };
        if (checkpoint) q.save = [&](const std::vector<int8_t>& W) { checkpoint(W.data(), n, user); };
        q.stop = &stop_flag();
        const uint32_t seed = p->seed ? (uint32_t)p->seed : (uint32_t)std::random_device{}();
        if (!p->seed) q.seed = seed;
        const CpuState s0 = start ? CpuState::from_entries(n, w, std::vector<int8_t>(start, start + (size_t)n * n))
                                  : CpuState::random_start(n, w, seed);
        const CpuAnnealResult r = cpu_anneal(s0, q);
        out->score = r.best.score();
        out->conflicts = r.best.conflicts();
        out->solved = r.best.solved() ? 1 : 0;
        out->verified = r.best.solved() && r.best.verify_weighing() ? 1 : 0;
        out->moves = r.moves;
        out->seconds = r.seconds;
        out->t_init = r.t_init;
        out->threads = q.threads;
        if (best_out) std::memcpy(best_out, r.best.entries().data(), (size_t)n * n);
        if (out->solved && !out->verified) {
            set_last_error("score reached zero but exact verification failed");
            return XW_ERR_INTERNAL;
        }
        return XW_OK;
    } catch (const std::invalid_argument& e) {
        set_last_error(e.what());
        return XW_ERR_INVALID;
    } catch (const std::bad_alloc&) {
        set_last_error("insufficient host memory");
        return XW_ERR_CAPACITY;
    } catch (const std::exception& e) {
        set_last_error(e.what());
        return XW_ERR_INTERNAL;
    }
}

}  // extern "C"
