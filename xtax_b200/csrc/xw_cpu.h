// xw_cpu.h -- host-side weighing-matrix state for everything around the GPU
// path that the drop-in keeps on the CPU: random starts, the Sylvester
// construction, temperature calibration, exact verification, CSV I/O.
//
// It follows the reference engine src/xweigh_anneal.hpp (class State,
// :103-667): column-major int8 entries, a dense Gram, int64 row residuals and
// the per-row minority list, with the same mt19937 draw order, so that a
// seed gives the reference's start and calibrated temperature.
#pragma once

#include <cstdint>
#include <random>
#include <string>
#include <vector>

namespace xw {

struct CpuParams {  // the fields of xweigh::Params the moves use
    double sign_fraction = 0.5;
    double target_fraction = 0.7;
    int target_samples = 8;
    double t_init = 0.0;
};

struct CpuMove {
    int kind = 0;  // 0 sign flip, 1 support switch
    int row1 = 0, row2 = 0, col1 = 0, col2 = 0, pos1 = 0, pos2 = 0;
};

class CpuState {
public:
    CpuState() = default;
    CpuState(int n, int w);

    static CpuState random_start(int n, int w, uint32_t seed);   // anneal.hpp:117-131
    static CpuState sylvester_blocks(int n, int w);               // anneal.hpp:133-149
    // throws std::runtime_error on a row whose support is not w
    static CpuState from_entries(int n, int w, std::vector<int8_t> entries);

    int order() const { return n_; }
    int weight() const { return w_; }
    int64_t score() const { return score_; }
    int64_t conflicts() const { return conflicts_; }
    bool solved() const { return score_ == 0; }
    const std::vector<int8_t>& entries() const { return entries_; }

    bool verify_support() const;    // anneal.hpp:221-237
    bool verify_weighing() const;   // anneal.hpp:239-264, exact, int64

    bool propose(std::mt19937& rng, const CpuParams& p, bool targeted, CpuMove& mv) const;
    int64_t evaluate_score(const CpuMove& mv) const;
    // State::evaluate (anneal.hpp:542-596): exact (score delta, conflict delta)
    void evaluate(const CpuMove& mv, int64_t& score_delta, int64_t& conflict_delta) const;
    // State::apply_to_entries: the move on a bare column-major W
    static void apply_to_entries(std::vector<int8_t>& entries, int n, const CpuMove& mv);
    // commit_sign_flip / commit_support_switch (anneal.hpp:598-666): apply
    // the move, update the Gram, residuals, minority list, score, conflicts
    void commit(const CpuMove& mv);

    int minority_count() const { return m_; }
    bool sparse_side() const { return sparse_; }
    const std::vector<uint16_t>& minority() const { return minority_; }
    int gram_at(int a, int b) const { return gram_[(size_t)a * n_ + b]; }

private:
    int n_ = 0, w_ = 0, m_ = 0;
    bool sparse_ = true;
    std::vector<int8_t> entries_;
    std::vector<int32_t> gram_;
    std::vector<int64_t> residual_;
    std::vector<uint16_t> minority_;
    int64_t score_ = 0, conflicts_ = 0;

    int8_t& at(int r, int c) { return entries_[(size_t)c * n_ + r]; }
    int8_t at(int r, int c) const { return entries_[(size_t)c * n_ + r]; }
    uint16_t& mino(int r, int p) { return minority_[(size_t)r * m_ + p]; }
    uint16_t mino(int r, int p) const { return minority_[(size_t)r * m_ + p]; }
    void rebuild_minority();
    void rebuild_gram();
    bool raw_switch(std::mt19937& rng);
    int hot_row(std::mt19937& rng, int samples) const;
    bool propose_flip(std::mt19937& rng, int row, CpuMove& mv) const;
    bool propose_switch(std::mt19937& rng, int row, CpuMove& mv) const;
};

// Elite restart of a stagnant population (xweigh_cuda.cu:1817-2289, the
// host half of run_annealer).  A scanned support switch out of the elite
// (rows r1 < r2, c1 moving from r1 to r2's zero... see xw_restart.cu) with
// its new signs and exact deltas ...
struct ScanResult {
    int row1, row2, col1, col2, new1, new2;
    int64_t score_delta, conflict_delta;
};

// ... as the reference's escape move: the value-preserving switch plus the
// sign flips that give the new signs, with the minority positions of the
// elite's lists
struct EscapeMove {
    CpuMove support;
    bool flip_first = false, flip_second = false;
    int64_t score_delta = 0, conflict_delta = 0;
};
std::vector<EscapeMove> escape_moves_from(const CpuState& elite, const std::vector<ScanResult>& scan);

// ... and the kicked copy of the elite for restarted replica `replica`, the
// `index`-th of `selected` this round: one escape move from the pool, then a
// row kick, a run of random moves, or neither (by (index + round) % 3),
// drawn from mt19937(base_seed ^ round * 0x9e3779b97f4a7c15 ^ replica *
// 0x85ebca6b) as the reference seeds it.
CpuState kick_elite(const CpuState& elite, const std::vector<EscapeMove>& escapes, size_t index, size_t selected,
                    uint64_t restart_round, int replica, uint32_t base_seed, int kick_steps, const CpuParams& p);

// calibrate_temperature (anneal.hpp:881-899)
double calibrate_temperature(const CpuState& s, const CpuParams& p, uint32_t seed);

// read_state_csv / write_entries_csv (anneal.hpp:669-797); throw on error
std::vector<int8_t> read_csv(const std::string& path, int n, int w);
void write_csv(const std::vector<int8_t>& entries, int n, const std::string& path);

// existence pre-checks of xweigh_cuda_main.cpp:32-52 ("" when none applies)
std::string impossibility_reason(int n, int w);

// row-only start: w nonzeros per row at uniform positions, uniform signs,
// from the Philox init stream of (key, stream)
std::vector<int8_t> row_start(int n, int w, uint32_t key0, uint32_t key1, uint32_t stream);

void philox4x32_10_host(const uint32_t ctr[4], uint32_t k0, uint32_t k1, uint32_t out[4]);

}  // namespace xw
