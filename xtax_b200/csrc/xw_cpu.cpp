// xw_cpu.cpp -- host-side weighing-matrix state (see xw_cpu.h).
#include "xw_cpu.h"

#include <algorithm>
#include <bit>
#include <cmath>
#include <cstdio>
#include <filesystem>
#include <fstream>
#include <sstream>
#include <stdexcept>

namespace xw {

namespace {

int uniform(std::mt19937& rng, int count) {
    return std::uniform_int_distribution<int>(0, count - 1)(rng);
}

double unit(std::mt19937& rng) { return std::generate_canonical<double, 53>(rng); }

bool is_square(int v) {
    const int r = (int)std::sqrt((double)v);
    return r * r == v || (r + 1) * (r + 1) == v;
}

}  // namespace

CpuState::CpuState(int n, int w)
    : n_(n), w_(w), m_(std::min(w, n - w)), sparse_(w <= n - w),
      entries_((size_t)n * n, 0), gram_((size_t)n * n, 0), residual_((size_t)n, 0),
      minority_((size_t)n * std::min(w, n - w), 0) {}

void CpuState::rebuild_minority() {
    if (m_ == 0) return;
    for (int r = 0; r < n_; ++r) {
        int pos = 0;
        for (int c = 0; c < n_; ++c) {
            if ((at(r, c) != 0) == sparse_) {
                if (pos >= m_) throw std::runtime_error("invalid regular support");
                mino(r, pos++) = (uint16_t)c;
            }
        }
        if (pos != m_) throw std::runtime_error("invalid regular support");
    }
}

void CpuState::rebuild_gram() {
    std::fill(residual_.begin(), residual_.end(), 0);
    score_ = 0;
    conflicts_ = 0;
    // row sign masks, 64 columns per word: dot = |P&P'|+|N&N'|-|P&N'|-|N&P'|
    const size_t words = ((size_t)n_ + 63) / 64;
    std::vector<uint64_t> pos((size_t)n_ * words, 0), neg((size_t)n_ * words, 0);
    for (int c = 0; c < n_; ++c)
        for (int r = 0; r < n_; ++r) {
            const int8_t v = at(r, c);
            if (v > 0) pos[(size_t)r * words + c / 64] |= 1ull << (c % 64);
            else if (v < 0) neg[(size_t)r * words + c / 64] |= 1ull << (c % 64);
        }
    for (int a = 0; a < n_; ++a) {
        gram_[(size_t)a * n_ + a] = w_;
        for (int b = a + 1; b < n_; ++b) {
            int dot = 0;
            for (size_t k = 0; k < words; ++k) {
                const uint64_t pa = pos[a * words + k], na = neg[a * words + k];
                const uint64_t pb = pos[b * words + k], nb = neg[b * words + k];
                dot += std::popcount(pa & pb) + std::popcount(na & nb) -
                       std::popcount(pa & nb) - std::popcount(na & pb);
            }
            gram_[(size_t)a * n_ + b] = dot;
            gram_[(size_t)b * n_ + a] = dot;
            const int64_t ad = dot < 0 ? -dot : dot;
            score_ += ad;
            residual_[a] += ad;
            residual_[b] += ad;
            conflicts_ += dot != 0;
        }
    }
}

bool CpuState::raw_switch(std::mt19937& rng) {
    if (m_ == 0 || n_ < 2) return false;
    const int r1 = uniform(rng, n_);
    int r2 = uniform(rng, n_ - 1);
    if (r2 >= r1) ++r2;
    const int p1 = uniform(rng, m_);
    const int p2 = uniform(rng, m_);
    const int c1 = sparse_ ? mino(r1, p1) : mino(r2, p2);
    const int c2 = sparse_ ? mino(r2, p2) : mino(r1, p1);
    if (c1 == c2 || at(r1, c2) != 0 || at(r2, c1) != 0) return false;
    const int8_t v1 = at(r1, c1), v2 = at(r2, c2);
    if (v1 == 0 || v2 == 0) return false;
    at(r1, c1) = 0;
    at(r2, c2) = 0;
    at(r1, c2) = v1;
    at(r2, c1) = v2;
    mino(r1, p1) = (uint16_t)(sparse_ ? c2 : c1);
    mino(r2, p2) = (uint16_t)(sparse_ ? c1 : c2);
    return true;
}

CpuState CpuState::random_start(int n, int w, uint32_t seed) {
    CpuState s(n, w);
    std::mt19937 rng(seed);
    for (int r = 0; r < n; ++r)
        for (int k = 0; k < w; ++k) s.at(r, (r + k) % n) = (rng() & 1u) ? 1 : -1;
    s.rebuild_minority();
    if (s.m_ != 0) {
        const uint64_t target = 4ull * (uint64_t)n * (uint64_t)std::min(s.m_, 64);
        uint64_t accepted = 0, attempts = 0;
        while (accepted < target && attempts < target * 12) {
            ++attempts;
            if (s.raw_switch(rng)) ++accepted;
        }
    }
    s.rebuild_gram();
    return s;
}

CpuState CpuState::sylvester_blocks(int n, int w) {
    CpuState s(n, w);
    for (int b = 0; b < n / w; ++b)
        for (int r = 0; r < w; ++r)
            for (int c = 0; c < w; ++c)
                s.at(b * w + r, b * w + c) = (std::popcount((unsigned)(r & c)) & 1) ? -1 : 1;
    s.rebuild_minority();
    s.rebuild_gram();
    return s;
}

CpuState CpuState::from_entries(int n, int w, std::vector<int8_t> entries) {
    if (entries.size() != (size_t)n * n) throw std::runtime_error("invalid xweigh entry buffer size");
    CpuState s(n, w);
    s.entries_ = std::move(entries);
    s.rebuild_minority();
    s.rebuild_gram();
    return s;
}

bool CpuState::verify_support() const {
    std::vector<int> col((size_t)n_, 0);
    for (int r = 0; r < n_; ++r) {
        int rw = 0;
        for (int c = 0; c < n_; ++c) {
            const int v = at(r, c);
            if (v < -1 || v > 1) return false;
            if (v != 0) { ++rw; ++col[c]; }
        }
        if (rw != w_) return false;
    }
    return std::all_of(col.begin(), col.end(), [&](int v) { return v == w_; });
}

bool CpuState::verify_weighing() const {
    if (!verify_support()) return false;
    for (int a = 0; a < n_; ++a)
        for (int b = a + 1; b < n_; ++b) {
            int64_t dot = 0;
            for (int c = 0; c < n_; ++c) dot += (int64_t)at(a, c) * at(b, c);
            if (dot != 0) return false;
        }
    return true;
}

int CpuState::hot_row(std::mt19937& rng, int samples) const {
    int best = uniform(rng, n_);
    for (int k = 1; k < samples; ++k) {
        const int cand = uniform(rng, n_);
        if (residual_[cand] > residual_[best]) best = cand;
    }
    return best;
}

bool CpuState::propose_flip(std::mt19937& rng, int row, CpuMove& mv) const {
    int col;
    if (sparse_ && m_ > 0) {
        col = mino(row, uniform(rng, m_));
    } else {
        const int start = uniform(rng, n_);
        col = start;
        while (at(row, col) == 0) {
            if (++col == n_) col = 0;
            if (col == start) return false;
        }
    }
    mv.kind = 0;
    mv.row1 = row;
    mv.col1 = col;
    return true;
}

bool CpuState::propose_switch(std::mt19937& rng, int r1, CpuMove& mv) const {
    if (m_ == 0 || n_ < 2) return false;
    for (int a = 0; a < 24; ++a) {
        int r2 = uniform(rng, n_ - 1);
        if (r2 >= r1) ++r2;
        const int p1 = uniform(rng, m_);
        const int p2 = uniform(rng, m_);
        const int c1 = sparse_ ? mino(r1, p1) : mino(r2, p2);
        const int c2 = sparse_ ? mino(r2, p2) : mino(r1, p1);
        if (c1 == c2 || at(r1, c2) != 0 || at(r2, c1) != 0) continue;
        if (at(r1, c1) == 0 || at(r2, c2) == 0) continue;
        mv.kind = 1;
        mv.row1 = r1; mv.row2 = r2; mv.col1 = c1; mv.col2 = c2; mv.pos1 = p1; mv.pos2 = p2;
        return true;
    }
    return false;
}

bool CpuState::propose(std::mt19937& rng, const CpuParams& p, bool targeted, CpuMove& mv) const {
    const int row = targeted ? hot_row(rng, p.target_samples) : uniform(rng, n_);
    if (w_ == n_ || unit(rng) < p.sign_fraction) return propose_flip(rng, row, mv);
    if (propose_switch(rng, row, mv)) return true;
    return propose_flip(rng, row, mv);
}

int64_t CpuState::evaluate_score(const CpuMove& mv) const {
    int64_t d = 0;
    auto ab = [](int v) { return (int64_t)(v < 0 ? -v : v); };
    if (mv.kind == 0) {
        const int ch = -2 * at(mv.row1, mv.col1);
        for (int o = 0; o < n_; ++o) {
            if (o == mv.row1) continue;
            const int old = gram_[(size_t)mv.row1 * n_ + o];
            d += ab(old + ch * at(o, mv.col1)) - ab(old);
        }
        return d;
    }
    const int v1 = at(mv.row1, mv.col1), v2 = at(mv.row2, mv.col2);
    for (int o = 0; o < n_; ++o) {
        if (o == mv.row1 || o == mv.row2) continue;
        const int o1 = gram_[(size_t)mv.row1 * n_ + o], o2 = gram_[(size_t)mv.row2 * n_ + o];
        d += ab(o1 + v1 * (at(o, mv.col2) - at(o, mv.col1))) - ab(o1);
        d += ab(o2 + v2 * (at(o, mv.col1) - at(o, mv.col2))) - ab(o2);
    }
    return d;
}

void CpuState::evaluate(const CpuMove& mv, int64_t& score_delta, int64_t& conflict_delta) const {
    int64_t ds = 0, dc = 0;
    auto ab = [](int v) { return (int64_t)(v < 0 ? -v : v); };
    auto cd = [](int o, int nw) { return (int64_t)(nw != 0) - (int64_t)(o != 0); };
    if (mv.kind == 0) {
        const int ch = -2 * at(mv.row1, mv.col1);
        for (int o = 0; o < n_; ++o) {
            if (o == mv.row1) continue;
            const int old = gram_[(size_t)mv.row1 * n_ + o];
            const int nw = old + ch * at(o, mv.col1);
            ds += ab(nw) - ab(old);
            dc += cd(old, nw);
        }
    } else {
        const int v1 = at(mv.row1, mv.col1), v2 = at(mv.row2, mv.col2);
        for (int o = 0; o < n_; ++o) {
            if (o == mv.row1 || o == mv.row2) continue;
            const int o1 = gram_[(size_t)mv.row1 * n_ + o], o2 = gram_[(size_t)mv.row2 * n_ + o];
            const int n1 = o1 + v1 * (at(o, mv.col2) - at(o, mv.col1));
            const int n2 = o2 + v2 * (at(o, mv.col1) - at(o, mv.col2));
            ds += ab(n1) - ab(o1) + ab(n2) - ab(o2);
            dc += cd(o1, n1) + cd(o2, n2);
        }
    }
    score_delta = ds;
    conflict_delta = dc;
}

void CpuState::apply_to_entries(std::vector<int8_t>& e, int n, const CpuMove& mv) {
    auto at = [&](int r, int c) -> int8_t& { return e[(size_t)c * n + r]; };
    if (mv.kind == 0) {
        at(mv.row1, mv.col1) = (int8_t)-at(mv.row1, mv.col1);
        return;
    }
    const int8_t v1 = at(mv.row1, mv.col1), v2 = at(mv.row2, mv.col2);
    at(mv.row1, mv.col1) = 0;
    at(mv.row2, mv.col2) = 0;
    at(mv.row1, mv.col2) = v1;
    at(mv.row2, mv.col1) = v2;
}

void CpuState::commit(const CpuMove& mv) {
    auto ab = [](int v) { return (int64_t)(v < 0 ? -v : v); };
    int64_t ds = 0, dc = 0;
    if (mv.kind == 0) {
        const int r = mv.row1, c = mv.col1;
        const int ch = -2 * at(r, c);
        for (int o = 0; o < n_; ++o) {
            if (o == r) continue;
            const int old = gram_[(size_t)r * n_ + o];
            const int nw = old + ch * at(o, c);
            const int64_t d = ab(nw) - ab(old);
            gram_[(size_t)r * n_ + o] = nw;
            gram_[(size_t)o * n_ + r] = nw;
            residual_[r] += d;
            residual_[o] += d;
            ds += d;
            dc += (int64_t)(nw != 0) - (int64_t)(old != 0);
        }
        at(r, c) = (int8_t)-at(r, c);
    } else {
        const int r1 = mv.row1, r2 = mv.row2, c1 = mv.col1, c2 = mv.col2;
        const int8_t v1 = at(r1, c1), v2 = at(r2, c2);
        for (int o = 0; o < n_; ++o) {
            if (o == r1 || o == r2) continue;
            const int o1 = gram_[(size_t)r1 * n_ + o], o2 = gram_[(size_t)r2 * n_ + o];
            const int n1 = o1 + v1 * (at(o, c2) - at(o, c1));
            const int n2 = o2 + v2 * (at(o, c1) - at(o, c2));
            const int64_t d1 = ab(n1) - ab(o1), d2 = ab(n2) - ab(o2);
            gram_[(size_t)r1 * n_ + o] = n1;
            gram_[(size_t)o * n_ + r1] = n1;
            gram_[(size_t)r2 * n_ + o] = n2;
            gram_[(size_t)o * n_ + r2] = n2;
            residual_[r1] += d1;
            residual_[r2] += d2;
            residual_[o] += d1 + d2;
            ds += d1 + d2;
            dc += (int64_t)(n1 != 0) - (int64_t)(o1 != 0) + (int64_t)(n2 != 0) - (int64_t)(o2 != 0);
        }
        at(r1, c1) = 0;
        at(r2, c2) = 0;
        at(r1, c2) = v1;
        at(r2, c1) = v2;
        mino(r1, mv.pos1) = (uint16_t)(sparse_ ? c2 : c1);
        mino(r2, mv.pos2) = (uint16_t)(sparse_ ? c1 : c2);
    }
    score_ += ds;
    conflicts_ += dc;
}

std::vector<EscapeMove> escape_moves_from(const CpuState& e, const std::vector<ScanResult>& scan) {
    const int n = e.order();
    const bool sparse = e.sparse_side();
    auto at = [&](int r, int c) { return (int)e.entries()[(size_t)c * n + r]; };
    // minority position of (row, column) on the sparse side, in column order
    std::vector<int> mpos((size_t)n * n, -1);
    for (int r = 0; r < n; ++r) {
        int pos = 0;
        for (int c = 0; c < n; ++c)
            if ((at(r, c) != 0) == sparse) mpos[(size_t)r * n + c] = pos++;
    }
    std::vector<EscapeMove> out;
    out.reserve(scan.size());
    for (const ScanResult& x : scan) {
        EscapeMove m;
        m.support.kind = 1;
        m.support.row1 = x.row1;
        m.support.row2 = x.row2;
        m.support.col1 = x.col1;
        m.support.col2 = x.col2;
        m.support.pos1 = mpos[(size_t)x.row1 * n + (sparse ? x.col1 : x.col2)];
        m.support.pos2 = mpos[(size_t)x.row2 * n + (sparse ? x.col2 : x.col1)];
        m.flip_first = x.new1 != at(x.row1, x.col1);
        m.flip_second = x.new2 != at(x.row2, x.col2);
        m.score_delta = x.score_delta;
        m.conflict_delta = x.conflict_delta;
        out.push_back(m);
    }
    return out;
}

CpuState kick_elite(const CpuState& elite, const std::vector<EscapeMove>& escapes, size_t index, size_t selected,
                    uint64_t restart_round, int replica, uint32_t base_seed, int kick_steps, const CpuParams& p) {
    const int n = elite.order(), w = elite.weight();
    CpuState k = elite;
    std::mt19937 rng(base_seed ^ (uint32_t)(restart_round * 0x9e3779b97f4a7c15ull) ^
                     ((uint32_t)replica * 0x85ebca6bu));
    if (!escapes.empty()) {
        const size_t pool = std::min(escapes.size(), std::max<size_t>(selected * 4, 1));
        const EscapeMove& esc = escapes[(index + (size_t)restart_round * selected) % pool];
        k.commit(esc.support);
        if (esc.flip_first) {
            CpuMove f;
            f.kind = 0;
            f.row1 = esc.support.row1;
            f.col1 = esc.support.col2;
            k.commit(f);
        }
        if (esc.flip_second) {
            CpuMove f;
            f.kind = 0;
            f.row1 = esc.support.row2;
            f.col1 = esc.support.col1;
            k.commit(f);
        }
    }
    const int mode = (int)((index + restart_round) % 3);
    int random_steps = kick_steps;
    if (mode == 0) {
        random_steps = 0;
    } else if (mode == 1 && kick_steps > 0 && w >= 3) {
        const int row_kicks = std::clamp(1 + kick_steps / std::max(1, w), 1, 4);
        const int max_flips = std::max(2, w / 2);
        for (int rk = 0; rk < row_kicks; ++rk) {
            const int row = std::uniform_int_distribution<int>(0, n - 1)(rng);
            std::vector<int> cols;
            cols.reserve((size_t)w);
            for (int c = 0; c < n; ++c)
                if (k.entries()[(size_t)c * n + row] != 0) cols.push_back(c);
            std::shuffle(cols.begin(), cols.end(), rng);
            const int flips = std::uniform_int_distribution<int>(2, max_flips)(rng);
            for (int f = 0; f < flips; ++f) {
                CpuMove mv;
                mv.kind = 0;
                mv.row1 = row;
                mv.col1 = cols[(size_t)f];
                k.commit(mv);
            }
        }
        random_steps = kick_steps / 4;
    }
    CpuParams kp = p;
    if (mode == 2) kp.sign_fraction = 0.0;
    int applied = 0;
    for (int a = 0; a < random_steps * 8 && applied < random_steps; ++a) {
        CpuMove mv;
        if (!k.propose(rng, kp, false, mv)) continue;
        k.commit(mv);
        ++applied;
    }
    return k;
}

double calibrate_temperature(const CpuState& s, const CpuParams& p, uint32_t seed) {
    if (p.t_init > 0.0) return p.t_init;
    std::mt19937 rng(seed ^ 0xa511e9b3u);
    long double sum = 0.0L;
    int count = 0;
    for (int k = 0; k < 256; ++k) {
        CpuMove mv;
        if (!s.propose(rng, p, false, mv)) continue;
        const int64_t d = s.evaluate_score(mv);
        if (d > 0) { sum += (long double)d; ++count; }
    }
    if (count == 0) return 1.0;
    const double mean = (double)(sum / count);
    return std::max(1.0, mean / std::log(2.0));
}

std::vector<int8_t> read_csv(const std::string& path, int n, int w) {
    std::ifstream in(path);
    if (!in) throw std::runtime_error("failed to open start matrix: " + path);
    std::vector<int8_t> e((size_t)n * n);
    std::vector<int> colw((size_t)n, 0);
    std::string line;
    int row = 0;
    while (std::getline(in, line)) {
        if (row >= n) throw std::runtime_error("start matrix has more than " + std::to_string(n) + " rows");
        std::stringstream ss(line);
        std::string tok;
        int rw = 0;
        for (int c = 0; c < n; ++c) {
            if (!std::getline(ss, tok, ','))
                throw std::runtime_error("start matrix row " + std::to_string(row + 1) +
                                         " has fewer than " + std::to_string(n) + " entries");
            const size_t a = tok.find_first_not_of(" \t\r\n");
            const size_t b = tok.find_last_not_of(" \t\r\n");
            if (a == std::string::npos) throw std::runtime_error("start matrix contains an empty entry");
            const std::string t = tok.substr(a, b - a + 1);
            size_t used = 0;
            int v = 0;
            try { v = std::stoi(t, &used); } catch (const std::exception&) { used = 0; }
            if (used != t.size() || v < -1 || v > 1)
                throw std::runtime_error("start matrix contains a non-ternary entry");
            e[(size_t)c * n + row] = (int8_t)v;
            if (v != 0) { ++rw; ++colw[c]; }
        }
        if (std::getline(ss, tok, ','))
            throw std::runtime_error("start matrix row " + std::to_string(row + 1) + " has more than " +
                                     std::to_string(n) + " entries");
        if (rw != w)
            throw std::runtime_error("start matrix row " + std::to_string(row + 1) + " has weight " +
                                     std::to_string(rw) + ", expected " + std::to_string(w));
        ++row;
    }
    if (row != n)
        throw std::runtime_error("start matrix has " + std::to_string(row) + " rows, expected " +
                                 std::to_string(n));
    for (int c = 0; c < n; ++c)
        if (colw[c] != w)
            throw std::runtime_error("start matrix column " + std::to_string(c + 1) + " has weight " +
                                     std::to_string(colw[c]) + ", expected " + std::to_string(w));
    CpuState s = CpuState::from_entries(n, w, e);
    if (!s.verify_support()) throw std::runtime_error("start matrix failed fixed-support verification");
    return e;
}

void write_csv(const std::vector<int8_t>& e, int n, const std::string& path) {
    const std::string tmp = path + ".tmp";
    {
        std::ofstream out(tmp, std::ios::binary);
        if (!out) throw std::runtime_error("failed to open output file: " + tmp);
        std::string row;
        for (int r = 0; r < n; ++r) {
            row.clear();
            for (int c = 0; c < n; ++c) {
                const int v = e[(size_t)c * n + r];
                if (v < 0) row += "-1";
                else row.push_back(v == 0 ? '0' : '1');
                row.push_back(c + 1 < n ? ',' : '\n');
            }
            out.write(row.data(), (std::streamsize)row.size());
        }
        out.flush();
        if (!out) throw std::runtime_error("failed while writing: " + tmp);
    }
    std::error_code ec;
    std::filesystem::rename(tmp, path, ec);
    if (ec) throw std::runtime_error("failed to replace " + path + ": " + ec.message());
}

std::string impossibility_reason(int n, int w) {
    if (w == n && n > 2 && n % 4 != 0)
        return "a full weighing matrix is a Hadamard matrix, whose order must be 1, 2, or a multiple of 4";
    if ((n & 1) != 0) {
        if (!is_square(w)) return "odd-order weighing matrices require a square weight";
        if (n > 1) {
            const int root = (int)std::sqrt((double)w);
            if (n < w + root + 1) return "odd-order weighing matrices require n >= w + sqrt(w) + 1";
        }
    }
    if (n % 4 == 2) {
        bool two = false;
        for (int a = 0; (int64_t)a * a <= w && !two; ++a) two = is_square(w - a * a);
        if (!two)
            return "orders congruent to 2 modulo 4 require the weight to be a sum of two integer squares";
    }
    return {};
}

void philox4x32_10_host(const uint32_t ctr[4], uint32_t k0, uint32_t k1, uint32_t out[4]) {
    uint32_t c0 = ctr[0], c1 = ctr[1], c2 = ctr[2], c3 = ctr[3];
    for (int r = 0; r < 10; ++r) {
        const uint64_t p0 = (uint64_t)0xD2511F53u * c0;
        const uint64_t p1 = (uint64_t)0xCD9E8D57u * c2;
        const uint32_t n0 = (uint32_t)(p1 >> 32) ^ c1 ^ k0, n2 = (uint32_t)(p0 >> 32) ^ c3 ^ k1;
        c0 = n0; c1 = (uint32_t)p1; c2 = n2; c3 = (uint32_t)p0;
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
    out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}

std::vector<int8_t> row_start(int n, int w, uint32_t key0, uint32_t key1, uint32_t stream) {
    std::vector<int8_t> e((size_t)n * n, 0);
    std::vector<int> perm((size_t)n);
    auto index = [&](uint32_t b, uint32_t row, int j, uint32_t count) {
        uint32_t out[4];
        for (uint32_t retry = 0;; ++retry) {
            const uint32_t ctr[4] = {(b & 0x00ffffffu) | (retry << 24), row, 0u, 0x40000000u | stream};
            philox4x32_10_host(ctr, key0, key1, out);
            const uint64_t prod = (uint64_t)out[j] * count;
            const uint32_t low = (uint32_t)prod;
            if (low >= count || low >= (0u - count) % count || retry >= 255) return (uint32_t)(prod >> 32);
        }
    };
    for (int r = 0; r < n; ++r) {
        for (int c = 0; c < n; ++c) perm[c] = c;
        for (int i = 0; i < w; ++i) {
            const int j = i + (int)index((uint32_t)(i >> 2), (uint32_t)r, i & 3, (uint32_t)(n - i));
            std::swap(perm[i], perm[j]);
            uint32_t out[4];
            const uint32_t ctr[4] = {32u + (uint32_t)(i >> 2), (uint32_t)r, 0u, 0x40000000u | stream};
            philox4x32_10_host(ctr, key0, key1, out);
            e[(size_t)perm[i] * n + r] = out[i & 3] < 0x80000000u ? 1 : -1;
        }
    }
    return e;
}

}  // namespace xw
