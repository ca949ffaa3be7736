// xw_cpu_anneal.h -- the CPU annealer (xw_cpu_anneal.cpp): the engine of the
// reference's xweigh tool on the host library's CpuState.
#pragma once

#include <atomic>
#include <cstdint>
#include <functional>
#include <string>
#include <vector>

#include "xw_cpu.h"

namespace xw {

// xweigh::Params (src/xweigh_anneal.hpp:42-67), with the log, checkpoint
// and stop hooks that replace the reference's std::cout, CSV writes and
// global stop flag
struct CpuAnnealParams {
    int threads = 1;
    uint64_t seed = 0;
    double max_seconds = 0.0;
    double save_interval = 2.0;
    double sign_fraction = 0.5;
    double greedy_fraction = 0.5;
    int candidate_samples = 4;
    double target_fraction = 0.7;
    int target_samples = 8;
    bool tempering = true;
    int exchange_interval = 2000;
    double t_init = 0.0;
    double t_min = 0.25;
    double cooling = 0.999;
    int moves_per_cool = 500;
    int stuck_threshold = 50000;
    double reheat = 1.0;
    double reseed_factor = 1.25;
    std::function<void(const std::string&)> log;                 // one line, no newline
    std::function<void(const std::vector<int8_t>&)> save;        // the best W so far
    const std::atomic<int>* stop = nullptr;                      // nonzero: finish now
};

struct CpuAnnealResult {
    CpuState best;
    uint64_t moves = 0;
    double seconds = 0.0;
    double t_init = 0.0;
};

// run_annealer (anneal.hpp:1106-1291): anneal from `start` until solved,
// max_seconds or stop; a single thread runs without tempering.
CpuAnnealResult cpu_anneal(const CpuState& start, CpuAnnealParams p);

// A reference worker's state bytes (State::estimated_bytes plus its W,
// anneal.hpp:185-190: W twice, the int16 Gram, int64 residuals, u16
// minority lists), for the reference's log lines.
double reference_worker_bytes(int n, int w);

}  // namespace xw
