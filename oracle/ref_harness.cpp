// ref_harness.cpp -- test-only driver around the reference's header-only
// xweigh engine (src/xweigh_anneal.hpp of flinty-mathematics/xtax).
//
// This file is test infrastructure: it is compiled against the reference
// sources where they lie (see oracle/Makefile) into oracle/_ref/ and prints
// JSON lines that tests/golden/make_golden.py turns into committed fixtures.
// Nothing in the product links or runs it.
//
// Each command exercises one public entry point of the reference engine:
//   start   n w seed            State::random_start            (anneal.hpp:117-131)
//   moves   n w seed count      propose_move / evaluate / commit (anneal.hpp:192-219)
//   compound n w seed count     double flips and sign-changing switches, applied
//                               as sequences of reference sign flips / switches
//                               (the decomposition restart_population uses,
//                               xweigh_cuda.cu:2108-2126)
//   walk    n w seed moves      a single-worker annealing walk that follows
//                               anneal_worker (anneal.hpp:909-1104) with
//                               tempering off, as run_annealer does for one
//                               thread (anneal.hpp:1106-1170)
//   csv     n w path            read_state_csv (anneal.hpp:669-756)
//   verify  n w path            verify_support / verify_weighing (anneal.hpp:221-264)

#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "xweigh_anneal.hpp"

namespace {

void print_entries(const std::vector<int8_t>& entries) {
    std::printf("[");
    for (size_t i = 0; i < entries.size(); ++i)
        std::printf(i ? ",%d" : "%d", (int)entries[i]);
    std::printf("]");
}

uint64_t fnv1a(uint64_t h, uint64_t v) {
    for (int i = 0; i < 8; ++i) {
        h ^= (v >> (8 * i)) & 0xffu;
        h *= 1099511628211ull;
    }
    return h;
}

int cmd_start(int n, int w, uint32_t seed) {
    xweigh::State s = xweigh::State::random_start(n, w, seed);
    std::printf("{\"cmd\":\"start\",\"n\":%d,\"w\":%d,\"seed\":%u,\"score\":%lld,"
                "\"conflicts\":%lld,\"support_ok\":%d,\"entries\":",
                n, w, seed, (long long)s.score(), (long long)s.conflicts(),
                s.verify_support() ? 1 : 0);
    print_entries(s.entries());
    std::printf("}\n");
    return 0;
}

// Random proposals on a random start: each line records the move, the
// reference evaluation and the score after committing it (every move is
// committed, so the state walks).
int cmd_moves(int n, int w, uint32_t seed, int count) {
    xweigh::State s = xweigh::State::random_start(n, w, seed);
    std::mt19937 rng(seed ^ 0x5eedu);
    xweigh::Params params;
    std::printf("{\"cmd\":\"moves\",\"n\":%d,\"w\":%d,\"seed\":%u,\"start\":", n, w, seed);
    print_entries(s.entries());
    std::printf(",\"moves\":[");
    bool first = true;
    for (int i = 0; i < count; ++i) {
        xweigh::Move m;
        const bool targeted = (i & 1) != 0;
        if (!s.propose_move(rng, params, targeted, m)) continue;
        const xweigh::Evaluation e = s.evaluate(m);
        s.commit(m, e);
        std::printf("%s[%d,%d,%d,%d,%d,%d,%d,%lld,%lld,%lld,%lld]", first ? "" : ",",
                    (int)m.kind, m.row1, m.row2, m.col1, m.col2,
                    m.minority_pos1, m.minority_pos2,
                    (long long)e.score_delta, (long long)e.conflict_delta,
                    (long long)s.score(), (long long)s.conflicts());
        first = false;
    }
    std::printf("],\"final\":");
    print_entries(s.entries());
    std::printf("}\n");
    return 0;
}

// Compound moves of the device move set, expressed through reference moves.
// kind 2: double sign flip (r1,c1),(r2,c2) = two reference sign flips.
// kind 1 with signs: a support switch followed by a sign flip of each moved
// entry whose sign is to change.
int cmd_compound(int n, int w, uint32_t seed, int count) {
    xweigh::State s = xweigh::State::random_start(n, w, seed);
    std::mt19937 rng(seed ^ 0xc0de5u);
    xweigh::Params params;
    std::printf("{\"cmd\":\"compound\",\"n\":%d,\"w\":%d,\"seed\":%u,\"start\":", n, w, seed);
    print_entries(s.entries());
    std::printf(",\"moves\":[");
    bool first = true;
    for (int i = 0; i < count; ++i) {
        const auto& E = s.entries();
        const bool dbl = (rng() & 1u) != 0;
        int64_t ds = 0, dc = 0;
        if (dbl) {
            // two distinct nonzero positions (possibly in the same row)
            int r1, c1, r2, c2;
            do { r1 = rng() % n; c1 = rng() % n; } while (E[(size_t)c1 * n + r1] == 0);
            do {
                r2 = (rng() & 1u) ? r1 : (int)(rng() % n);
                c2 = rng() % n;
            } while (E[(size_t)c2 * n + r2] == 0 || (r2 == r1 && c2 == c1));
            xweigh::Move a; a.kind = xweigh::MoveKind::sign_flip; a.row1 = r1; a.col1 = c1;
            xweigh::Evaluation ea = s.evaluate(a); s.commit(a, ea);
            xweigh::Move b; b.kind = xweigh::MoveKind::sign_flip; b.row1 = r2; b.col1 = c2;
            xweigh::Evaluation eb = s.evaluate(b); s.commit(b, eb);
            ds = ea.score_delta + eb.score_delta;
            dc = ea.conflict_delta + eb.conflict_delta;
            std::printf("%s[2,%d,%d,%d,%d,0,0,%lld,%lld,%lld,%lld]", first ? "" : ",",
                        r1, r2, c1, c2, (long long)ds, (long long)dc,
                        (long long)s.score(), (long long)s.conflicts());
            first = false;
        } else {
            xweigh::Move m;
            params.sign_fraction = 0.0;
            if (!s.propose_move(rng, params, false, m)) continue;
            if (m.kind != xweigh::MoveKind::support_switch) continue;
            const int v1 = E[(size_t)m.col1 * n + m.row1];
            const int v2 = E[(size_t)m.col2 * n + m.row2];
            const int f1 = (int)(rng() & 1u), f2 = (int)(rng() & 1u);
            xweigh::Evaluation e = s.evaluate(m); s.commit(m, e);
            ds += e.score_delta; dc += e.conflict_delta;
            if (f1) {
                xweigh::Move f; f.kind = xweigh::MoveKind::sign_flip; f.row1 = m.row1; f.col1 = m.col2;
                xweigh::Evaluation ef = s.evaluate(f); s.commit(f, ef);
                ds += ef.score_delta; dc += ef.conflict_delta;
            }
            if (f2) {
                xweigh::Move f; f.kind = xweigh::MoveKind::sign_flip; f.row1 = m.row2; f.col1 = m.col1;
                xweigh::Evaluation ef = s.evaluate(f); s.commit(f, ef);
                ds += ef.score_delta; dc += ef.conflict_delta;
            }
            // new values after the move: row1 gets (f1 ? -v1 : v1) at col2,
            // row2 gets (f2 ? -v2 : v2) at col1
            std::printf("%s[1,%d,%d,%d,%d,%d,%d,%lld,%lld,%lld,%lld]", first ? "" : ",",
                        m.row1, m.row2, m.col1, m.col2,
                        f1 ? -v1 : v1, f2 ? -v2 : v2,
                        (long long)ds, (long long)dc,
                        (long long)s.score(), (long long)s.conflicts());
            first = false;
        }
    }
    std::printf("],\"final\":");
    print_entries(s.entries());
    std::printf("}\n");
    return 0;
}

// Single-worker walk following anneal_worker with tempering off.  Reports a
// hash of the per-move (score, conflicts, accepted) sequence, the final state
// and the best state.  The walk is bounded by a move count instead of the
// wall clock; everything else (RNG order, candidate selection, Metropolis,
// cooling, reheat, reseed from the best, the 250000-move path reset) follows
// the reference loop.
int cmd_walk(int n, int w, uint32_t seed, long long max_moves,
             double t_init, double t_min, double cooling, int moves_per_cool,
             int stuck_threshold) {
    xweigh::Params params;
    params.threads = 1;
    params.tempering = false;
    params.seed = seed;
    params.t_init = t_init;
    params.t_min = t_min;
    params.cooling = cooling;
    params.moves_per_cool = moves_per_cool;
    params.stuck_threshold = stuck_threshold;

    const uint32_t base_seed = (uint32_t)params.seed;
    xweigh::State start = xweigh::State::random_start(n, w, base_seed);
    const double initial_temperature =
        xweigh::calibrate_temperature(start, params, base_seed);
    std::mt19937 seed_rng(base_seed);
    const uint32_t worker_seed = (uint32_t)seed_rng() ^ (0u * 0x9e3779b9u);

    xweigh::State current = start;
    std::mt19937 rng(worker_seed);
    int64_t best_score = current.score(), best_conflicts = current.conflicts();
    std::vector<int8_t> best_entries = current.entries();
    std::vector<xweigh::Move> accepted_path;
    int moves_since_improvement = 0, cooling_counter = 0;
    long long moves = 0;
    double temperature = initial_temperature;
    uint64_t h = 1469598103934665603ull;
    long long accepted = 0;

    while (moves < max_moves && !current.solved()) {
        xweigh::Move selected;
        xweigh::Evaluation sel;
        bool have = false;
        const bool greedy = xweigh::random_unit(rng) < params.greedy_fraction;
        const int samples = greedy ? params.candidate_samples : 1;
        for (int k = 0; k < samples; ++k) {
            xweigh::Move cand;
            const bool targeted = xweigh::random_unit(rng) < params.target_fraction;
            if (!current.propose_move(rng, params, targeted, cand)) continue;
            const xweigh::Evaluation e = current.evaluate(cand);
            if (!have || xweigh::better_pair(e.score_delta, e.conflict_delta,
                                             sel.score_delta, sel.conflict_delta)) {
                selected = cand; sel = e; have = true;
            }
        }
        if (!have) continue;
        ++moves;
        const bool accept = sel.score_delta <= 0 ||
            xweigh::random_unit(rng) <
                std::exp(-(double)sel.score_delta / std::max(temperature, 1e-12));
        if (accept) {
            current.commit(selected, sel);
            accepted_path.push_back(selected);
            ++accepted;
        }
        if (xweigh::better_pair(current.score(), current.conflicts(),
                                best_score, best_conflicts)) {
            best_score = current.score();
            best_conflicts = current.conflicts();
            moves_since_improvement = 0;
            for (const auto& m : accepted_path)
                xweigh::State::apply_to_entries(best_entries, n, m);
            accepted_path.clear();
        } else {
            ++moves_since_improvement;
        }
        if (++cooling_counter >= params.moves_per_cool) {
            cooling_counter = 0;
            temperature = std::max(params.t_min, temperature * params.cooling);
        }
        if (moves_since_improvement >= params.stuck_threshold) {
            moves_since_improvement = 0;
            temperature = std::max(params.t_min, initial_temperature * params.reheat);
            if ((double)current.score() >
                params.reseed_factor * (double)std::max<int64_t>(1, best_score)) {
                current = xweigh::State::from_entries(n, w, best_entries);
                accepted_path.clear();
            }
        }
        if (accepted_path.size() >= 250000) {
            current = xweigh::State::from_entries(n, w, best_entries);
            accepted_path.clear();
            moves_since_improvement = 0;
        }
        h = fnv1a(h, (uint64_t)current.score());
        h = fnv1a(h, (uint64_t)current.conflicts());
        h = fnv1a(h, accept ? 1u : 0u);
    }
    std::printf("{\"cmd\":\"walk\",\"n\":%d,\"w\":%d,\"seed\":%u,\"t_init_arg\":%.17g,"
                "\"t_min\":%.17g,\"cooling\":%.17g,\"moves_per_cool\":%d,"
                "\"stuck_threshold\":%d,\"max_moves\":%lld,\"initial_temperature\":%.17g,"
                "\"worker_seed\":%u,\"moves\":%lld,\"accepted\":%lld,\"hash\":\"%016llx\","
                "\"score\":%lld,\"conflicts\":%lld,\"best_score\":%lld,\"best_conflicts\":%lld,"
                "\"temperature\":%.17g,\"start\":",
                n, w, seed, t_init, t_min, cooling, moves_per_cool, stuck_threshold,
                max_moves, initial_temperature, worker_seed, moves, accepted,
                (unsigned long long)h, (long long)current.score(),
                (long long)current.conflicts(), (long long)best_score,
                (long long)best_conflicts, temperature);
    print_entries(start.entries());
    std::printf(",\"final\":");
    print_entries(current.entries());
    std::printf(",\"best\":");
    print_entries(best_entries);
    std::printf("}\n");
    return 0;
}

int cmd_csv(int n, int w, const char* path) {
    std::printf("{\"cmd\":\"csv\",\"n\":%d,\"w\":%d,\"path\":\"%s\",", n, w, path);
    try {
        xweigh::State s = xweigh::read_state_csv(path, n, w);
        std::printf("\"ok\":1,\"score\":%lld,\"conflicts\":%lld,\"entries\":",
                    (long long)s.score(), (long long)s.conflicts());
        print_entries(s.entries());
        std::printf("}\n");
    } catch (const std::exception& e) {
        std::string msg = e.what();
        std::string esc;
        for (char ch : msg) { if (ch == '"' || ch == '\\') esc.push_back('\\'); esc.push_back(ch); }
        std::printf("\"ok\":0,\"error\":\"%s\"}\n", esc.c_str());
    }
    return 0;
}

int cmd_sylvester(int n, int w) {
    xweigh::State s = xweigh::State::sylvester_blocks(n, w);
    std::printf("{\"cmd\":\"sylvester\",\"n\":%d,\"w\":%d,\"support_ok\":%d,\"weighing_ok\":%d,\"entries\":",
                n, w, s.verify_support() ? 1 : 0, s.verify_weighing() ? 1 : 0);
    print_entries(s.entries());
    std::printf("}\n");
    return 0;
}

int cmd_calibrate(int n, int w, uint32_t seed) {
    xweigh::Params params;
    xweigh::State s = xweigh::State::random_start(n, w, seed);
    const double t = xweigh::calibrate_temperature(s, params, seed);
    std::printf("{\"cmd\":\"calibrate\",\"n\":%d,\"w\":%d,\"seed\":%u,\"t\":%.17g}\n", n, w, seed, t);
    return 0;
}

// Throughput of the reference's full rescoring + exact verification
// (State::from_entries -> rebuild_gram_and_residual, then verify_weighing)
// over `count` random row-regular ternary matrices on `threads` threads.
int cmd_rescore_bench(int n, int w, int count, int threads) {
    std::vector<std::vector<int8_t>> mats((size_t)count);
    std::mt19937 rng(12345u + (uint32_t)n);
    for (auto& e : mats) {
        e.assign((size_t)n * n, 0);
        std::vector<int> cols((size_t)n);
        for (int r = 0; r < n; ++r) {
            for (int c = 0; c < n; ++c) cols[c] = c;
            std::shuffle(cols.begin(), cols.end(), rng);
            for (int k = 0; k < w; ++k) e[(size_t)cols[k] * n + r] = (rng() & 1u) ? 1 : -1;
        }
    }
    std::atomic<long long> checksum{0};
    const auto t0 = std::chrono::steady_clock::now();
    std::vector<std::thread> pool;
    for (int t = 0; t < threads; ++t)
        pool.emplace_back([&, t]() {
            long long local = 0;
            for (int i = t; i < count; i += threads) {
                xweigh::State s = xweigh::State::from_entries(n, w, mats[(size_t)i]);
                local += s.score() + (s.verify_weighing() ? 1 : 0);
            }
            checksum += local;
        });
    for (auto& th : pool) th.join();
    const double secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    std::printf("{\"cmd\":\"rescore_bench\",\"n\":%d,\"w\":%d,\"count\":%d,\"threads\":%d,\"seconds\":%.6f,"
                "\"matrices_per_sec\":%.3f,\"checksum\":%lld}\n",
                n, w, count, threads, secs, count / secs, (long long)checksum.load());
    return 0;
}

}  // namespace

int main(int argc, char** argv) {
    if (argc < 2) {
        std::fprintf(stderr, "usage: ref_harness cmd args...\n");
        return 2;
    }
    const std::string cmd = argv[1];
    auto I = [&](int k) { return std::atoll(argv[k]); };
    auto D = [&](int k) { return std::atof(argv[k]); };
    if (cmd == "start" && argc == 5) return cmd_start((int)I(2), (int)I(3), (uint32_t)I(4));
    if (cmd == "moves" && argc == 6) return cmd_moves((int)I(2), (int)I(3), (uint32_t)I(4), (int)I(5));
    if (cmd == "compound" && argc == 6) return cmd_compound((int)I(2), (int)I(3), (uint32_t)I(4), (int)I(5));
    if (cmd == "walk" && argc == 11)
        return cmd_walk((int)I(2), (int)I(3), (uint32_t)I(4), I(5), D(6), D(7), D(8), (int)I(9), (int)I(10));
    if (cmd == "csv" && argc == 5) return cmd_csv((int)I(2), (int)I(3), argv[4]);
    if (cmd == "sylvester" && argc == 4) return cmd_sylvester((int)I(2), (int)I(3));
    if (cmd == "calibrate" && argc == 5) return cmd_calibrate((int)I(2), (int)I(3), (uint32_t)I(4));
    if (cmd == "rescore_bench" && argc == 6)
        return cmd_rescore_bench((int)I(2), (int)I(3), (int)I(4), (int)I(5));
    std::fprintf(stderr, "bad command\n");
    return 2;
}
