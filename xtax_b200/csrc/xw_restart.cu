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

}  // namespace

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
