// xw_restart.cu -- the escape-move scan of an elite restart, on the device.
//
// An elite restart (xweigh_cuda.cu:1817-2289) first ranks every support
// switch out of the elite state: rows r1 < r2, a column c1 that is nonzero
// in r1 and zero in r2, a column c2 that is nonzero in r2 and zero in r1,
// and new signs for the two moved entries (xweigh_cuda.cu:1925-2057).  Each
// candidate's exact change of the L1 score and of the conflicts is an O(n)
// pass over the two Gram rows, so the scan is O(n^5) in the worst case: a
// host loop of minutes at n = 200.  Here one CTA per row pair evaluates its
// candidates (one thread per (c1, c2), all four sign choices in one pass
// over the other rows), and the `limit` best are selected without storing
// every candidate:
//   pass 1  a histogram of (score delta, conflict delta) -- both bounded by
//           4n and 2n -- gives the cut-off key below which fewer than
//           `limit` candidates lie;
//   pass 2  collects the candidates below the cut-off and the indices of
//           those on it; the host keeps the first of the latter in scan
//           order.
// The ranking is (score delta, conflict delta, scan order (r1, r2, c1, c2,
// new1, new2)): a total order, so the result does not depend on thread
// timing.  (The reference's streaming nth_element leaves ties among equal
// deltas to its implementation.)
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/xw.h"
#include "xw_cpu.h"
#include "xw_device.cuh"
#include "xw_host_internal.h"

namespace xw {

namespace {

constexpr int kScanThreads = 128;

struct ScanShape {
    int n;
    int ds_off, dc_off, dc_width;   // bin = (ds + ds_off) * dc_width + (dc + dc_off)
    uint32_t bins;
};

ScanShape scan_shape(int n) {
    ScanShape s;
    s.n = n;
    s.ds_off = 4 * n;
    s.dc_off = 2 * n;
    s.dc_width = 4 * n + 1;
    s.bins = (uint32_t)(8 * n + 1) * (uint32_t)s.dc_width;
    return s;
}

struct Found {
    unsigned long long index;   // scan order: ((((r1 n + r2) n + c1) n + c2) 4 + signs)
    uint32_t bin;
    uint32_t pad;
};

// PASS 0 counts keys into `hist`; PASS 1 collects keys below `cut` into
// `below` and scan indices on `cut` into `on` (each with its own counter).
template <int PASS>
__global__ void __launch_bounds__(kScanThreads) escape_scan_kernel(const int8_t* W, const int32_t* G, ScanShape sh,
                                                                   uint32_t* hist, uint32_t cut, Found* below,
                                                                   uint32_t below_cap, unsigned long long* on,
                                                                   uint32_t on_cap, uint32_t* counters) {
    const int n = sh.n;
    const int r1 = blockIdx.y, r2 = blockIdx.x;
    if (r2 <= r1) return;
    __shared__ int32_t g1[XW_MAX_ORDER_LARGE], g2[XW_MAX_ORDER_LARGE];
    __shared__ uint16_t c1s[XW_MAX_ORDER_LARGE], c2s[XW_MAX_ORDER_LARGE];
    __shared__ int k1, k2;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    for (int o = tid; o < n; o += kScanThreads) {
        g1[o] = G[r1 * n + o];
        g2[o] = G[r2 * n + o];
    }
    if (warp == 0) {
        // the movable columns of each row, in column order
        int a = 0, b = 0;
        for (int base = 0; base < n; base += 32) {
            const int c = base + lane;
            const int v1 = c < n ? W[c * n + r1] : 0, v2 = c < n ? W[c * n + r2] : 0;
            const unsigned m1 = __ballot_sync(0xffffffffu, v1 != 0 && v2 == 0);
            const unsigned m2 = __ballot_sync(0xffffffffu, v2 != 0 && v1 == 0);
            const unsigned lower = (1u << lane) - 1u;
            if (v1 != 0 && v2 == 0) c1s[a + __popc(m1 & lower)] = (uint16_t)c;
            if (v2 != 0 && v1 == 0) c2s[b + __popc(m2 & lower)] = (uint16_t)c;
            a += __popc(m1);
            b += __popc(m2);
        }
        if (lane == 0) {
            k1 = a;
            k2 = b;
        }
    }
    __syncthreads();
    const int pairs = k1 * k2;
    for (int j = tid; j < pairs; j += kScanThreads) {
        const int c1 = c1s[j / k2], c2 = c2s[j % k2];
        const int ov1 = W[c1 * n + r1], ov2 = W[c2 * n + r2];
        // deltas of the four sign choices (new1, new2) in {-1,1}^2
        int ds[4] = {0, 0, 0, 0}, dc[4] = {0, 0, 0, 0};
        for (int o = 0; o < n; ++o) {
            if (o == r1 || o == r2) continue;
            const int w1 = W[c1 * n + o], w2 = W[c2 * n + o];
            const int o1 = g1[o], o2 = g2[o];
            const int a1 = abs(o1), a2 = abs(o2);
            const int z1 = o1 != 0, z2 = o2 != 0;
#pragma unroll
            for (int s = 0; s < 4; ++s) {
                const int nv1 = (s & 2) ? 1 : -1, nv2 = (s & 1) ? 1 : -1;
                const int n1 = o1 + nv1 * w2 - ov1 * w1;
                const int n2 = o2 + nv2 * w1 - ov2 * w2;
                ds[s] += abs(n1) - a1 + abs(n2) - a2;
                dc[s] += (n1 != 0) - z1 + (n2 != 0) - z2;
            }
        }
#pragma unroll
        for (int s = 0; s < 4; ++s) {
            const uint32_t bin = (uint32_t)(ds[s] + sh.ds_off) * (uint32_t)sh.dc_width + (uint32_t)(dc[s] + sh.dc_off);
            if (PASS == 0) {
                atomicAdd(&hist[bin], 1u);
            } else if (bin <= cut) {
                const unsigned long long index =
                    ((((unsigned long long)r1 * n + r2) * n + c1) * n + c2) * 4ull + (unsigned long long)s;
                if (bin < cut) {
                    const uint32_t k = atomicAdd(&counters[0], 1u);
                    if (k < below_cap) below[k] = Found{index, bin, 0u};
                } else {
                    const uint32_t k = atomicAdd(&counters[1], 1u);
                    if (k < on_cap) on[k] = index;
                }
            }
        }
    }
}

struct DevBuf {
    void* p = nullptr;
    ~DevBuf() {
        if (p) cudaFree(p);
    }
};

// ---------------------------------------------------------------------------
// Device kicks (restart mode 1).  The reference kicks the elite's copies on
// the host with std::mt19937 (xweigh_cuda.cu:2089-2193) after reading the
// population back; here one CTA per restarted replica rewrites its record
// in place: the elite's best W, the escape move, then by (index + round) % 3
// nothing more, row kicks (2..max(2, w/2) distinct nonzeros of 1..4 random
// rows flip, then kick/4 random moves) or kick random moves that are all
// support switches; a random move is a sign flip of a random nonzero (a
// coin under the job's sign threshold, or no zeros at all) or a
// value-preserving 2x2 support switch, `steps` of them within 8*steps
// attempts.  Draw k is word k%4 of Philox({k/4, round_lo, round_hi,
// 0x20000000 | replica}, job key); an index in [0,count) is Lemire's
// multiply-shift with a rejected word replaced by the next (at most 64
// tries).  Then the record gets the kicked W's scores, minority lists
// (rebuilt in column order), best W, the reheat temperature and cleared
// stagnation counters.

__device__ __forceinline__ uint32_t kick_word(uint32_t& k, uint32_t k0, uint32_t k1, uint32_t r_lo, uint32_t r_hi,
                                              uint32_t tag) {
    const uint4 b = philox4x32_10(make_uint4(k >> 2, r_lo, r_hi, tag), k0, k1);
    const uint32_t v = pick(b, (int)(k & 3u));
    ++k;
    return v;
}

struct KickRng {
    uint32_t k, k0, k1, r_lo, r_hi, tag;
    __device__ uint32_t word() { return kick_word(k, k0, k1, r_lo, r_hi, tag); }
    __device__ uint32_t index(uint32_t count) {
        uint64_t prod = 0;
        for (int t = 0; t < 64; ++t) {
            prod = (uint64_t)word() * count;
            const uint32_t low = (uint32_t)prod;
            if (low >= count || low >= (0u - count) % count) break;
        }
        return (uint32_t)(prod >> 32);
    }
};

__device__ int kick_nonzero(const int8_t* K, int n, int row, int k) {
    for (int c = 0; c < n; ++c)
        if (K[(size_t)c * n + row] != 0 && k-- == 0) return c;
    return -1;
}

constexpr int kKickThreads = 128;

__global__ void __launch_bounds__(kKickThreads) kick_kernel(KickArgs a) {
    const KickJob kj = a.kicks[blockIdx.x];
    const XwJob& J = *a.job;
    const int n = J.n, w = J.w, m = J.m;
    uint8_t* rec = a.arena + a.rec_off[kj.rid];
    RepHeader* H = reinterpret_cast<RepHeader*>(rec);
    int8_t* K = reinterpret_cast<int8_t*>(rec + J.off_w);
    const int tid = threadIdx.x;
    for (int i = tid; i < n * n; i += kKickThreads) K[i] = a.elite[i];
    __syncthreads();
    if (tid == 0) {
        auto at = [&](int r, int c) -> int8_t& { return K[(size_t)c * n + r]; };
        if (kj.esc >= 0) {
            const int* e = a.escapes + 6 * kj.esc;
            at(e[0], e[2]) = 0;
            at(e[1], e[3]) = 0;
            at(e[0], e[3]) = (int8_t)e[4];
            at(e[1], e[2]) = (int8_t)e[5];
        }
        KickRng g{0u, J.key0, J.key1, (uint32_t)a.round, (uint32_t)(a.round >> 32), 0x20000000u | H->stream};
        const int mode = (int)(((uint64_t)kj.index + a.round) % 3ull);
        int steps = kj.kick;
        uint64_t thr = J.thr_sign;
        if (mode == 0) {
            steps = 0;
        } else if (mode == 1 && kj.kick > 0 && w >= 3) {
            int rows = 1 + kj.kick / (w > 1 ? w : 1);
            if (rows > 4) rows = 4;
            const int maxf = w / 2 > 2 ? w / 2 : 2;
            for (int rk = 0; rk < rows; ++rk) {
                const int row = (int)g.index((uint32_t)n);
                int cnt = 0;
                for (int c = 0; c < n; ++c) cnt += at(row, c) != 0;
                const int flips = 2 + (int)g.index((uint32_t)(maxf - 1));
                // a partial Fisher-Yates shuffle of the row's nonzero
                // columns, kept as a permutation of ranks in column order
                // (the k-th nonzero column is found by a scan)
                uint16_t* perm = a.scratch + (size_t)blockIdx.x * XW_MAX_ORDER_LARGE;
                for (int q = 0; q < cnt; ++q) perm[q] = (uint16_t)q;
                for (int f = 0; f < flips && f < cnt; ++f) {
                    const int j = f + (int)g.index((uint32_t)(cnt - f));
                    const uint16_t t = perm[f];
                    perm[f] = perm[j];
                    perm[j] = t;
                }
                for (int f = 0; f < flips && f < cnt; ++f) {
                    const int col = kick_nonzero(K, n, row, perm[f]);
                    at(row, col) = (int8_t)-at(row, col);
                }
            }
            steps = kj.kick / 4;
        } else if (mode == 2) {
            thr = 0;
        }
        int applied = 0;
        for (int t = 0; t < 8 * steps && applied < steps; ++t) {
            const uint32_t u = g.word();
            if (w == n || (uint64_t)u < thr) {
                const int row = (int)g.index((uint32_t)n);
                const int col = kick_nonzero(K, n, row, (int)g.index((uint32_t)w));
                at(row, col) = (int8_t)-at(row, col);
                ++applied;
                continue;
            }
            if (n < 2) continue;
            const int r1 = (int)g.index((uint32_t)n);
            int r2 = (int)g.index((uint32_t)(n - 1));
            if (r2 >= r1) ++r2;
            const int c1 = kick_nonzero(K, n, r1, (int)g.index((uint32_t)w));
            const int c2 = kick_nonzero(K, n, r2, (int)g.index((uint32_t)w));
            if (c1 == c2 || at(r1, c2) != 0 || at(r2, c1) != 0) continue;
            const int8_t v1 = at(r1, c1), v2 = at(r2, c2);
            at(r1, c1) = 0;
            at(r2, c2) = 0;
            at(r1, c2) = v1;
            at(r2, c1) = v2;
            ++applied;
        }
    }
    __syncthreads();
    // scores of the kicked W: thread t takes rows t, t + 128, ...
    __shared__ unsigned long long s_sq;
    __shared__ int s_score, s_conf, s_par;
    if (tid == 0) {
        s_sq = 0;
        s_score = s_conf = s_par = 0;
    }
    __syncthreads();
    int p_score = 0, p_conf = 0, p_par = 0;
    unsigned long long p_sq = 0;
    for (int r = tid; r < n; r += kKickThreads) {
        for (int o = r + 1; o < n; ++o) {
            int dot = 0;
            for (int c = 0; c < n; ++c) dot += K[(size_t)c * n + r] * K[(size_t)c * n + o];
            const int ad = dot < 0 ? -dot : dot;
            p_score += ad;
            p_conf += dot != 0;
            p_sq += (unsigned long long)(dot * dot);
            p_par += ad & 1;
        }
        // the row's minority list, in column order (u16 entries above the
        // shared-memory orders)
        int pos = 0;
        for (int c = 0; c < n && pos < m; ++c)
            if ((K[(size_t)c * n + r] != 0) == (J.sparse != 0)) {
                if (J.large)
                    reinterpret_cast<uint16_t*>(rec + J.off_mino)[(size_t)r * m + pos] = (uint16_t)c;
                else
                    rec[J.off_mino + (size_t)r * m + pos] = (uint8_t)c;
                ++pos;
            }
    }
    atomicAdd(&s_score, p_score);
    atomicAdd(&s_conf, p_conf);
    atomicAdd(&s_par, p_par);
    atomicAdd(&s_sq, p_sq);
    __syncthreads();
    const int score = s_score, conf = s_conf;
    const bool better = score < a.gbest || (score == a.gbest && conf < a.gconf);
    int8_t* B = reinterpret_cast<int8_t*>(rec + J.off_best);
    for (int i = tid; i < n * n; i += kKickThreads) B[i] = better ? K[i] : a.elite[i];
    if (tid == 0) {
        H->score = score;
        H->conflicts = conf;
        H->best_score = better ? score : a.gbest;
        H->best_conflicts = better ? conf : a.gconf;
        H->obj_total = H->obj_kind == 1 ? (int64_t)s_sq : H->obj_kind == 2 ? (int64_t)s_par : (int64_t)score;
        const double t = __dmul_rn(H->reheat_temperature, a.reheat);
        H->temperature = t > a.t_min ? t : a.t_min;
        H->msi = 0;
        H->cool_ctr = 0;
        H->status &= ~XW_STATUS_GRAM;   // the large-order kernel rebuilds G from the new W
    }
}

}  // namespace

void launch_kicks(const KickArgs& a, int count, cudaStream_t stream) {
    if (count <= 0) return;
    kick_kernel<<<count, kKickThreads, 0, stream>>>(a);
    check_cuda(cudaGetLastError(), "launch kick_kernel");
}


std::vector<ScanResult> escape_scan(int n, const int8_t* W, const int32_t* G, size_t limit) {
    std::vector<ScanResult> out;
    if (n < 2 || limit == 0) return out;
    if (n > XW_MAX_ORDER_CUDA) throw std::invalid_argument("escape scan: order above the device path's maximum");
    const ScanShape sh = scan_shape(n);
    DevBuf dW, dG, dHist, dBelow, dOn, dCnt;
    check_cuda(cudaMalloc(&dW.p, (size_t)n * n), "cudaMalloc escape scan");
    check_cuda(cudaMalloc(&dG.p, sizeof(int32_t) * n * n), "cudaMalloc escape scan");
    check_cuda(cudaMalloc(&dHist.p, sizeof(uint32_t) * sh.bins), "cudaMalloc escape scan");
    check_cuda(cudaMalloc(&dCnt.p, sizeof(uint32_t) * 2), "cudaMalloc escape scan");
    check_cuda(cudaMemcpy(dW.p, W, (size_t)n * n, cudaMemcpyHostToDevice), "upload elite");
    check_cuda(cudaMemcpy(dG.p, G, sizeof(int32_t) * n * n, cudaMemcpyHostToDevice), "upload elite Gram");
    check_cuda(cudaMemset(dHist.p, 0, sizeof(uint32_t) * sh.bins), "cudaMemset");
    const dim3 grid(n, n), block(kScanThreads);
    escape_scan_kernel<0><<<grid, block>>>(static_cast<const int8_t*>(dW.p), static_cast<const int32_t*>(dG.p), sh,
                                           static_cast<uint32_t*>(dHist.p), 0u, nullptr, 0u, nullptr, 0u, nullptr);
    check_cuda(cudaGetLastError(), "launch escape scan");
    std::vector<uint32_t> hist(sh.bins);
    check_cuda(cudaMemcpy(hist.data(), dHist.p, sizeof(uint32_t) * sh.bins, cudaMemcpyDeviceToHost),
               "read escape histogram");
    // cut-off: the first key at which the running count reaches `limit`
    uint64_t before = 0;
    uint32_t cut = sh.bins - 1;
    for (uint32_t b = 0; b < sh.bins; ++b) {
        if (before + hist[b] >= limit) {
            cut = b;
            break;
        }
        before += hist[b];
    }
    const uint64_t total_on = hist[cut];
    const uint32_t below_cap = (uint32_t)before;
    check_cuda(cudaMalloc(&dBelow.p, sizeof(Found) * std::max<uint64_t>(below_cap, 1)), "cudaMalloc escape scan");
    check_cuda(cudaMalloc(&dOn.p, sizeof(unsigned long long) * std::max<uint64_t>(total_on, 1)),
               "cudaMalloc escape scan");
    check_cuda(cudaMemset(dCnt.p, 0, sizeof(uint32_t) * 2), "cudaMemset");
    escape_scan_kernel<1><<<grid, block>>>(static_cast<const int8_t*>(dW.p), static_cast<const int32_t*>(dG.p), sh,
                                           nullptr, cut, static_cast<Found*>(dBelow.p), below_cap,
                                           static_cast<unsigned long long*>(dOn.p), (uint32_t)total_on,
                                           static_cast<uint32_t*>(dCnt.p));
    check_cuda(cudaGetLastError(), "launch escape scan");
    std::vector<Found> low(below_cap);
    std::vector<unsigned long long> on(total_on);
    uint32_t cnt[2] = {0, 0};
    check_cuda(cudaMemcpy(cnt, dCnt.p, sizeof cnt, cudaMemcpyDeviceToHost), "read escape counts");
    if (cnt[0] != below_cap || cnt[1] != total_on)
        throw std::runtime_error("escape scan: the two passes counted different candidates");
    if (below_cap)
        check_cuda(cudaMemcpy(low.data(), dBelow.p, sizeof(Found) * below_cap, cudaMemcpyDeviceToHost),
                   "read escape candidates");
    if (total_on)
        check_cuda(cudaMemcpy(on.data(), dOn.p, sizeof(unsigned long long) * total_on, cudaMemcpyDeviceToHost),
                   "read escape candidates");
    std::sort(low.begin(), low.end(), [](const Found& a, const Found& b) {
        return a.bin != b.bin ? a.bin < b.bin : a.index < b.index;
    });
    std::sort(on.begin(), on.end());
    const size_t take_on = std::min<uint64_t>(total_on, limit - std::min<uint64_t>(limit, before));
    auto decode = [&](unsigned long long index, uint32_t bin) {
        ScanResult r;
        const int s = (int)(index & 3ull);
        unsigned long long x = index >> 2;
        r.col2 = (int)(x % n);
        x /= n;
        r.col1 = (int)(x % n);
        x /= n;
        r.row2 = (int)(x % n);
        r.row1 = (int)(x / n);
        r.new1 = (s & 2) ? 1 : -1;
        r.new2 = (s & 1) ? 1 : -1;
        r.score_delta = (int64_t)(bin / (uint32_t)sh.dc_width) - sh.ds_off;
        r.conflict_delta = (int64_t)(bin % (uint32_t)sh.dc_width) - sh.dc_off;
        return r;
    };
    out.reserve(low.size() + take_on);
    for (const Found& f : low) out.push_back(decode(f.index, f.bin));
    for (size_t k = 0; k < take_on; ++k) out.push_back(decode(on[k], cut));
    return out;
}

}  // namespace xw

extern "C" int32_t xw_escape_scan(int32_t n, int32_t w, const int8_t* W, int32_t limit, xw_escape_move* out,
                                  int32_t* count) {
    if (!W || !count || (limit > 0 && !out) || limit < 0 || n < 2 || n > XW_MAX_ORDER_CUDA || w < 1 || w > n) {
        xw::set_last_error("escape scan: invalid arguments");
        return XW_ERR_INVALID;
    }
    xw::CpuState e;
    try {
        e = xw::CpuState::from_entries(n, w, std::vector<int8_t>(W, W + (size_t)n * n));
    } catch (const std::exception& ex) {
        xw::set_last_error(std::string("escape scan: ") + ex.what());
        return XW_ERR_INVALID;
    }
    try {
        std::vector<int32_t> G((size_t)n * n);
        for (int a = 0; a < n; ++a)
            for (int b = 0; b < n; ++b) G[(size_t)a * n + b] = e.gram_at(a, b);
        const std::vector<xw::ScanResult> r = xw::escape_scan(n, W, G.data(), (size_t)limit);
        for (size_t k = 0; k < r.size(); ++k) {
            xw_escape_move& m = out[k];
            m.row1 = r[k].row1;
            m.row2 = r[k].row2;
            m.col1 = r[k].col1;
            m.col2 = r[k].col2;
            m.new1 = r[k].new1;
            m.new2 = r[k].new2;
            m.score_delta = r[k].score_delta;
            m.conflict_delta = r[k].conflict_delta;
        }
        *count = (int32_t)r.size();
        return XW_OK;
    } catch (const std::exception& ex) {
        xw::set_last_error(ex.what());
        return XW_ERR_CUDA;
    }
}
