// xw_anneal_large.cu -- the population annealing kernel for orders above the
// shared-memory classes (n up to XW_MAX_ORDER_LARGE).
//
// The reference kernel keeps a replica's W, int16 Gram, residuals and
// minority lists in one CTA's shared memory (make_shared_layout,
// src/xweigh_cuda.cu:72-96) and refuses orders whose state does not fit
// (:1449-1460), about n = 276 on a 227 KiB part.  Here a replica whose
// order is above that of the shared-memory kernel keeps its state in HBM
// and L2 instead:
//   record (arena)   W (int8, column-major), best W, minority lists (u16)
//   gram arena       G (int16, row-major, n x n), row support masks and
//                    sign masks (u64, ceil(n/64) words per row)
//   shared memory    row residuals (int32, the hot-row tournament's random
//                    reads), the iteration's draw words, thresholds
// One warp still owns one replica and lane o still owns rows o, o+32, ...;
// an evaluation reads one or two Gram rows and two or four W columns, all
// coalesced across the warp.  G persists between launches (XW_STATUS_GRAM);
// it is built once from W with popcounts over the sign and support masks,
// and rebuilt whenever the host replaces W (restarts, snapshots).
//
// The iteration is the one of xw_anneal.cu with the same draw layout, the
// same proposal order and the same tie rules, so a replica's trajectory is
// identical in both kernels and the CPU replay checks either.  Two
// differences in bookkeeping only: move descriptors have 10-bit rows and
// columns, and the best W is copied lazily -- when the replica is about to
// leave a best state, or at the end of the launch -- since a copy here is
// n^2 bytes of HBM traffic rather than of shared memory.
#include <cuda_runtime.h>

#include "xw_device.cuh"
#include "xw_kernels.h"

namespace xw {

namespace {

constexpr unsigned FULL = 0xffffffffu;
constexpr uint32_t kThrTable = 64;

// Replica-constant fields the proposal code reads, in the warp's slot.
struct LView {
    const int8_t* W;
    const uint16_t* mino;
    const int32_t* res;
    const uint64_t* mask;
    const uint32_t* dw;
    uint64_t thr_target, thr_dbl, thr_sign, thr_swsign;
    int n, w, m, sparse, ts, bpc, cc, move_set, nw;
    uint32_t stream, k0, k1, pad;
};

struct LSlot {
    uint32_t off_draws, off_view, off_thr, bytes;
};

__host__ __device__ inline LSlot large_slot(int n) {
    LSlot L;
    L.off_draws = xw_pad16((uint32_t)n * 4u);
    L.off_view = L.off_draws + 32u * 16u;
    L.off_thr = L.off_view + xw_pad16((uint32_t)sizeof(LView));
    L.bytes = L.off_thr + kThrTable * 8u;
    return L;
}

struct LGram {
    uint64_t off_mask, off_sign, bytes;
};

__host__ __device__ inline LGram large_gram(int n) {
    const uint64_t nw = (uint64_t)(n + 63) / 64;
    LGram g;
    g.off_mask = ((uint64_t)n * n * 2u + 15u) & ~uint64_t(15);
    g.off_sign = g.off_mask + (uint64_t)n * nw * 8u;
    g.bytes = g.off_sign + (uint64_t)n * nw * 8u;
    return g;
}

__device__ __forceinline__ int iabs(int v) { return v < 0 ? -v : v; }

__device__ __noinline__ uint32_t l_slow_word(uint32_t slot, uint64_t it, uint32_t stream, uint32_t k0, uint32_t k1,
                                             int j) {
    return pick(draw_block(slot, it, stream, k0, k1), j);
}

// word j of block b of candidate c: from the iteration's cached blocks
// when they hold it, else recomputed
__device__ __forceinline__ uint32_t l_word(const LView* v, uint64_t it, int c, int b, int j) {
    if (c < v->cc && b < v->bpc) return v->dw[(1 + c * v->bpc + b) * 4 + j];
    return l_slow_word(cand_slot(c, b), it, v->stream, v->k0, v->k1, j);
}

__device__ __forceinline__ uint32_t l_index(const LView* v, uint64_t it, int c, int b, int j, uint32_t count) {
    return draw_index(l_word(v, it, c, b, j), count, cand_slot(c, b), it, v->stream, v->k0, v->k1, j);
}

__device__ __forceinline__ int l_at(const LView* v, int r, int c) { return v->W[(size_t)c * v->n + r]; }

// word k of a row's support mask, or of its zero set (columns < n)
__device__ __forceinline__ uint64_t mask_word(const uint64_t* row, int k, int nw, int n, bool zeros) {
    uint64_t x = row[k];
    if (zeros) {
        x = ~x;
        if (k == nw - 1 && (n & 63)) x &= (1ull << (n & 63)) - 1ull;
    }
    return x;
}

// first set bit at or after `start`, cyclically
__device__ __noinline__ int l_cyclic_first(const uint64_t* row, int nw, int n, int start, bool zeros) {
    const int ws = start >> 6;
#pragma unroll 1
    for (int k = ws; k < nw; ++k) {
        uint64_t x = mask_word(row, k, nw, n, zeros);
        if (k == ws) x &= ~0ull << (start & 63);
        if (x) return 64 * k + __ffsll((long long)x) - 1;
    }
#pragma unroll 1
    for (int k = 0; k <= ws && k < nw; ++k) {
        const uint64_t x = mask_word(row, k, nw, n, zeros);
        if (x) return 64 * k + __ffsll((long long)x) - 1;
    }
    return -1;
}

// Move descriptor, three words (10-bit rows and columns):
//   x = valid | kind<<1 | r1<<3 | r2<<13 | (W[r1][c1]+1)<<23 | (W[r2][c2]+1)<<25
//   y = c1 | c2<<10 | (v1+1)<<20 | (v2+1)<<22
//   z = p1 | p2<<10
// kinds as in xw_anneal.cu: 0 sign flip, 1 support switch, 2 double flip,
// 3 within-row swap.  The proposer, which runs in parallel across the
// candidates, carries the two current entries, so that decoding a move in
// the serial evaluation and commit needs no dependent load from HBM.
struct LMove {
    uint32_t x, y, z;
};

__device__ __forceinline__ LMove none() { return LMove{0u, 0u, 0u}; }

__device__ __forceinline__ LMove lpack(int kind, int r1, int r2, int c1, int c2, int v1, int v2, int p1, int p2,
                                       int o11, int o22) {
    LMove mv;
    mv.x = 1u | ((uint32_t)kind << 1) | ((uint32_t)r1 << 3) | ((uint32_t)r2 << 13) | ((uint32_t)(o11 + 1) << 23) |
           ((uint32_t)(o22 + 1) << 25);
    mv.y = (uint32_t)c1 | ((uint32_t)c2 << 10) | ((uint32_t)(v1 + 1) << 20) | ((uint32_t)(v2 + 1) << 22);
    mv.z = (uint32_t)p1 | ((uint32_t)p2 << 10);
    return mv;
}

// propose_sign_flip (xweigh_cuda.cu:302-325)
__device__ __noinline__ int l_flip_col(const LView* v, uint64_t it, int c, int b, int j, int row) {
    if (v->sparse && v->m > 0) return v->mino[(size_t)row * v->m + (int)l_index(v, it, c, b, j, (uint32_t)v->m)];
    const int start = (int)l_index(v, it, c, b, j, (uint32_t)v->n);
    return l_cyclic_first(v->mask + (size_t)row * v->nw, v->nw, v->n, start, false);
}

// hot_row (xweigh_cuda.cu:291-300), serial form
__device__ __noinline__ int l_hot_row(const LView* v, uint64_t it, int c) {
    int best = (int)l_index(v, it, c, 4, 0, (uint32_t)v->n);
#pragma unroll 1
    for (int k = 1; k < v->ts; ++k) {
        const int cand = (int)l_index(v, it, c, 4 + k / 4, k % 4, (uint32_t)v->n);
        if (v->res[cand] > v->res[best]) best = cand;
    }
    return best;
}

// propose_double_sign_flip (xweigh_cuda.cu:389-421), attempts 1..15
__device__ __noinline__ LMove l_double_rest(const LView* v, uint64_t it, int c, int row1, int col1) {
#pragma unroll 1
    for (int a = 1; a < 16; ++a) {
        const int b = 20 + (a - 1);
        const int row2 = l_word(v, it, c, b, 0) < 0x80000000u ? row1 : (int)l_index(v, it, c, b, 1, (uint32_t)v->n);
        const int col2 = l_flip_col(v, it, c, b, 2, row2);
        if (col2 < 0 || (row2 == row1 && col2 == col1)) continue;
        return lpack(2, row1, row2, col1, col2, 0, 0, 0, 0, l_at(v, row1, col1), l_at(v, row2, col2));
    }
    return none();
}

// propose_support_switch (xweigh_cuda.cu:327-387), attempts a0..23
__device__ __noinline__ LMove l_switch(const LView* v, uint64_t it, int c, int row1, int a0) {
    const int n = v->n, m = v->m;
    if (m == 0 || n < 2) return none();
#pragma unroll 1
    for (int a = a0; a < 24; ++a) {
        const int B = a == 0 ? 1 : 36 + 2 * (a - 1);
        const int o = a == 0 ? 1 : 0;
        int row2 = (int)l_index(v, it, c, B, o, (uint32_t)(n - 1));
        if (row2 >= row1) ++row2;
        const int p1 = (int)l_index(v, it, c, B, o + 1, (uint32_t)m);
        const int p2 = (int)l_index(v, it, c, B, o + 2, (uint32_t)m);
        const int q1 = v->mino[(size_t)row1 * m + p1], q2 = v->mino[(size_t)row2 * m + p2];
        const int c1 = v->sparse ? q1 : q2, c2 = v->sparse ? q2 : q1;
        if (c1 == c2 || l_at(v, row1, c2) != 0 || l_at(v, row2, c1) != 0) continue;
        const int v1 = l_at(v, row1, c1), v2 = l_at(v, row2, c2);
        if (v1 == 0 || v2 == 0) continue;
        const uint32_t s1 = a == 0 ? l_word(v, it, c, 2, 0) : l_word(v, it, c, B, 3);
        const uint32_t s2 = a == 0 ? l_word(v, it, c, 2, 1) : l_word(v, it, c, B + 1, 0);
        return lpack(1, row1, row2, c1, c2, (uint64_t)s1 < v->thr_swsign ? -v1 : v1,
                     (uint64_t)s2 < v->thr_swsign ? -v2 : v2, p1, p2, v1, v2);
    }
    return none();
}

// within-row swap: a nonzero of the row moves to one of its zeros
__device__ __noinline__ LMove l_row_swap(const LView* v, uint64_t it, int c, int row) {
    if (v->m == 0) return none();
    const uint64_t* nz = v->mask + (size_t)row * v->nw;
    int c1, c2, pos;
    if (v->sparse) {
        pos = (int)l_index(v, it, c, 1, 1, (uint32_t)v->m);
        c1 = v->mino[(size_t)row * v->m + pos];
        c2 = l_cyclic_first(nz, v->nw, v->n, (int)l_index(v, it, c, 1, 2, (uint32_t)v->n), true);
    } else {
        pos = (int)l_index(v, it, c, 1, 2, (uint32_t)v->m);
        c2 = v->mino[(size_t)row * v->m + pos];
        c1 = l_cyclic_first(nz, v->nw, v->n, (int)l_index(v, it, c, 1, 1, (uint32_t)v->n), false);
    }
    if (c1 < 0 || c2 < 0) return none();
    return lpack(3, row, 0, c1, c2, l_word(v, it, c, 1, 3) < 0x80000000u ? 1 : -1, 0, pos, 0, l_at(v, row, c1), 0);
}

// propose_move (xweigh_cuda.cu:423-447) in the draw order of d_propose
// (xw_anneal.cu): every first attempt reads the same draw words, and the
// choice between kinds follows the same tests in the same order.
template <bool GEN>
__device__ __noinline__ LMove l_propose(const LView* v, uint64_t it, int c, bool coop_ok, int coop_row) {
    const int n = v->n, m = v->m;
    const bool targeted = (uint64_t)l_word(v, it, c, 0, 0) < v->thr_target;
    const int row = targeted ? (coop_ok ? coop_row : l_hot_row(v, it, c)) : (int)l_index(v, it, c, 0, 1, (uint32_t)n);
    const bool want_dbl = (!GEN || v->move_set == 0) && (uint64_t)l_word(v, it, c, 0, 2) < v->thr_dbl;
    const bool want_flip = v->w == n || (uint64_t)l_word(v, it, c, 0, 3) < v->thr_sign;
    if (want_dbl) {
        const int dcol1 = l_flip_col(v, it, c, 2, 3, row);
        if (dcol1 >= 0) {
            const int drow2 = l_word(v, it, c, 3, 0) < 0x80000000u ? row : (int)l_index(v, it, c, 3, 1, (uint32_t)n);
            const int dcol2 = l_flip_col(v, it, c, 3, 2, drow2);
            if (dcol2 >= 0 && !(drow2 == row && dcol2 == dcol1))
                return lpack(2, row, drow2, dcol1, dcol2, 0, 0, 0, 0, l_at(v, row, dcol1), l_at(v, drow2, dcol2));
            const LMove mv = l_double_rest(v, it, c, row, dcol1);
            if (mv.x) return mv;
        }
    }
    if (want_flip) {
        const int fcol = l_flip_col(v, it, c, 1, 0, row);
        return fcol < 0 ? none() : lpack(0, row, 0, fcol, 0, 0, 0, 0, 0, l_at(v, row, fcol), 0);
    }
    LMove mv = none();
    if (GEN && v->move_set == 1) {
        mv = l_row_swap(v, it, c, row);
    } else if (m > 0 && n > 1) {
        // support switch, attempt 0 (blocks 1 and 2)
        int row2 = (int)l_index(v, it, c, 1, 1, (uint32_t)(n - 1));
        if (row2 >= row) ++row2;
        const int p1 = (int)l_index(v, it, c, 1, 2, (uint32_t)m);
        const int p2 = (int)l_index(v, it, c, 1, 3, (uint32_t)m);
        const int q1 = v->mino[(size_t)row * m + p1], q2 = v->mino[(size_t)row2 * m + p2];
        const int c1 = v->sparse ? q1 : q2, c2 = v->sparse ? q2 : q1;
        const int v1 = l_at(v, row, c1), v2 = l_at(v, row2, c2);
        if (c1 != c2 && l_at(v, row, c2) == 0 && l_at(v, row2, c1) == 0 && v1 != 0 && v2 != 0) {
            const int nv1 = (uint64_t)l_word(v, it, c, 2, 0) < v->thr_swsign ? -v1 : v1;
            const int nv2 = (uint64_t)l_word(v, it, c, 2, 1) < v->thr_swsign ? -v2 : v2;
            return lpack(1, row, row2, c1, c2, nv1, nv2, p1, p2, v1, v2);
        }
        mv = l_switch(v, it, c, row, 1);
    }
    if (mv.x) return mv;
    const int col = l_flip_col(v, it, c, 2, 2, row);
    return col < 0 ? none() : lpack(0, row, 0, col, 0, 0, 0, 0, 0, l_at(v, row, col), 0);
}

// A decoded move as at most two row updates (see xw_anneal.cu)
struct LUpdate {
    int R1, X1, Y1, A1, B1;
    int R2, X2, Y2, A2, B2;
    int pair;
};

__device__ __forceinline__ LUpdate l_decode(const LMove& mv) {
    const int kind = (mv.x >> 1) & 3, r1 = (mv.x >> 3) & 1023, r2 = (mv.x >> 13) & 1023;
    const int c1 = mv.y & 1023, c2 = (mv.y >> 10) & 1023;
    const int nv1 = (int)((mv.y >> 20) & 3) - 1, nv2 = (int)((mv.y >> 22) & 3) - 1;
    const int w11 = (int)((mv.x >> 23) & 3) - 1, w22 = (int)((mv.x >> 25) & 3) - 1;
    LUpdate u;
    u.R1 = r1;
    u.R2 = -1;
    u.X2 = 0; u.Y2 = 0; u.A2 = 0; u.B2 = 0;
    u.pair = 0;
    if (kind == 0) {
        u.X1 = c1; u.Y1 = c1; u.A1 = -2 * w11; u.B1 = 0;
    } else if (kind == 1) {
        u.X1 = c2; u.Y1 = c1; u.A1 = nv1; u.B1 = -w11;
        u.R2 = r2; u.X2 = c1; u.Y2 = c2; u.A2 = nv2; u.B2 = -w22;
    } else if (kind == 2) {
        if (r1 == r2) {
            u.X1 = c1; u.Y1 = c2; u.A1 = -2 * w11; u.B1 = -2 * w22;
        } else {
            u.X1 = c1; u.Y1 = c1; u.A1 = -2 * w11; u.B1 = 0;
            u.R2 = r2; u.X2 = c2; u.Y2 = c2; u.A2 = -2 * w22; u.B2 = 0;
            u.pair = 1;
        }
    } else {
        u.X1 = c2; u.Y1 = c1; u.A1 = nv1; u.B1 = -w11;
    }
    return u;
}

struct LDeltas {
    int ds, dc, dsq, dpar;
};

template <bool GEN>
__device__ __forceinline__ void lacc(LDeltas& d, int old, int nw) {
    const int ao = iabs(old), an = iabs(nw);
    d.ds += an - ao;
    d.dc += (nw != 0) - (old != 0);
    if (GEN) {
        d.dsq += nw * nw - old * old;
        d.dpar += (an & 1) - (ao & 1);
    }
}

__device__ __forceinline__ int l_pair_new(const LUpdate& u, int op, const int8_t* W, int n) {
    return op + u.A1 * W[(size_t)u.X1 * n + u.R2] + u.A2 * W[(size_t)u.X2 * n + u.R1] +
           (u.X1 == u.X2 ? u.A1 * u.A2 : 0);
}

// evaluate_move_warp (xweigh_cuda.cu:449-599): lane-partial deltas
template <bool GEN>
__device__ __forceinline__ LDeltas l_eval(const LUpdate& u, const int8_t* W, const int16_t* G, int n, int lane) {
    LDeltas d = {0, 0, 0, 0};
    const int16_t* g1 = G + (size_t)u.R1 * n;
    const int8_t* x1 = W + (size_t)u.X1 * n;
    const int8_t* y1 = W + (size_t)u.Y1 * n;
    if (u.R2 < 0) {
#pragma unroll 8
        for (int o = lane; o < n; o += 32) {
            const int o1 = g1[o];
            const int n1 = o1 + u.A1 * x1[o] + u.B1 * y1[o];
            if (o != u.R1) lacc<GEN>(d, o1, n1);
        }
    } else {
        const int16_t* g2 = G + (size_t)u.R2 * n;
        const int8_t* x2 = W + (size_t)u.X2 * n;
        const int8_t* y2 = W + (size_t)u.Y2 * n;
#pragma unroll 4
        for (int o = lane; o < n; o += 32) {
            const int o1 = g1[o], o2 = g2[o];
            const int n1 = o1 + u.A1 * x1[o] + u.B1 * y1[o];
            const int n2 = o2 + u.A2 * x2[o] + u.B2 * y2[o];
            if (o != u.R1 && o != u.R2) {
                lacc<GEN>(d, o1, n1);
                lacc<GEN>(d, o2, n2);
            }
        }
    }
    if (u.pair && lane == 0) {
        const int op = g1[u.R2];
        lacc<GEN>(d, op, l_pair_new(u, op, W, n));
    }
    return d;
}

// commit_* (xweigh_cuda.cu:607-877) and the within-row swap, two-row form
template <bool GEN>
__device__ void l_commit(const LMove& mv, const LUpdate& u, int ds, int8_t* W, int16_t* G, int32_t* res,
                         uint16_t* mino, uint64_t* mask, int n, int m, int nw, int sparse, int lane) {
    // four of the lane's rows per step: their loads are issued together,
    // then their stores, so a step costs one round trip to L2/HBM
    constexpr int kBatch = 4;
    int s1 = 0;
    int16_t* g1 = G + (size_t)u.R1 * n;
    const int8_t* x1 = W + (size_t)u.X1 * n;
    const int8_t* y1 = W + (size_t)u.Y1 * n;
    if (u.R2 < 0) {
#pragma unroll 1
        for (int base = lane; base < n; base += 32 * kBatch) {
            int o1[kBatch], n1[kBatch];
#pragma unroll
            for (int q = 0; q < kBatch; ++q) {
                const int o = base + 32 * q;
                o1[q] = o < n ? g1[o] : 0;
                n1[q] = o < n ? o1[q] + u.A1 * x1[o] + u.B1 * y1[o] : 0;
            }
#pragma unroll
            for (int q = 0; q < kBatch; ++q) {
                const int o = base + 32 * q;
                if (o >= n || o == u.R1) continue;
                g1[o] = (int16_t)n1[q];
                G[(size_t)o * n + u.R1] = (int16_t)n1[q];
                const int e1 = iabs(n1[q]) - iabs(o1[q]);
                res[o] += e1;
                s1 += e1;
            }
        }
    } else {
        int16_t* g2 = G + (size_t)u.R2 * n;
        const int8_t* x2 = W + (size_t)u.X2 * n;
        const int8_t* y2 = W + (size_t)u.Y2 * n;
#pragma unroll 1
        for (int base = lane; base < n; base += 32 * kBatch) {
            int o1[kBatch], n1[kBatch], o2[kBatch], n2[kBatch];
#pragma unroll
            for (int q = 0; q < kBatch; ++q) {
                const int o = base + 32 * q;
                o1[q] = o < n ? g1[o] : 0;
                o2[q] = o < n ? g2[o] : 0;
                n1[q] = o < n ? o1[q] + u.A1 * x1[o] + u.B1 * y1[o] : 0;
                n2[q] = o < n ? o2[q] + u.A2 * x2[o] + u.B2 * y2[o] : 0;
            }
#pragma unroll
            for (int q = 0; q < kBatch; ++q) {
                const int o = base + 32 * q;
                if (o >= n || o == u.R1 || o == u.R2) continue;
                g1[o] = (int16_t)n1[q];
                G[(size_t)o * n + u.R1] = (int16_t)n1[q];
                g2[o] = (int16_t)n2[q];
                G[(size_t)o * n + u.R2] = (int16_t)n2[q];
                const int e1 = iabs(n1[q]) - iabs(o1[q]);
                res[o] += e1 + iabs(n2[q]) - iabs(o2[q]);
                s1 += e1;
            }
        }
    }
    const int S1 = __reduce_add_sync(FULL, s1);
    __syncwarp();
    if (lane == 0) {
        const int kind = (mv.x >> 1) & 3, r1 = (mv.x >> 3) & 1023, r2 = (mv.x >> 13) & 1023;
        const int c1 = mv.y & 1023, c2 = (mv.y >> 10) & 1023;
        const int nv1 = (int)((mv.y >> 20) & 3) - 1, nv2 = (int)((mv.y >> 22) & 3) - 1;
        const int p1 = mv.z & 1023, p2 = (mv.z >> 10) & 1023;
        const int o11 = (int)((mv.x >> 23) & 3) - 1, o22 = (int)((mv.x >> 25) & 3) - 1;
        if (u.pair) {
            const int op = G[(size_t)r1 * n + r2];
            const int np = l_pair_new(u, op, W, n);
            const int pd = iabs(np) - iabs(op);
            G[(size_t)r1 * n + r2] = (int16_t)np;
            G[(size_t)r2 * n + r1] = (int16_t)np;
            res[r1] += S1 + pd;
            res[r2] += ds - S1;
        } else if (u.R2 >= 0) {
            res[r1] += S1;
            res[r2] += ds - S1;
        } else {
            res[r1] += ds;
        }
        int8_t* w11 = W + (size_t)c1 * n + r1;
        int8_t* w22 = W + (size_t)c2 * n + r2;
        if (kind == 0) {
            *w11 = (int8_t)-o11;
        } else if (kind == 2) {
            *w11 = (int8_t)-o11;
            *w22 = (int8_t)-o22;
        } else if (kind == 1) {
            *w11 = 0;
            *w22 = 0;
            W[(size_t)c2 * n + r1] = (int8_t)nv1;
            W[(size_t)c1 * n + r2] = (int8_t)nv2;
            mino[(size_t)r1 * m + p1] = (uint16_t)(sparse ? c2 : c1);
            mino[(size_t)r2 * m + p2] = (uint16_t)(sparse ? c1 : c2);
            mask[(size_t)nw * r1 + (c1 >> 6)] &= ~(1ull << (c1 & 63));
            mask[(size_t)nw * r1 + (c2 >> 6)] |= 1ull << (c2 & 63);
            mask[(size_t)nw * r2 + (c2 >> 6)] &= ~(1ull << (c2 & 63));
            mask[(size_t)nw * r2 + (c1 >> 6)] |= 1ull << (c1 & 63);
        } else if (GEN) {
            *w11 = 0;
            W[(size_t)c2 * n + r1] = (int8_t)nv1;
            mino[(size_t)r1 * m + p1] = (uint16_t)(sparse ? c2 : c1);
            mask[(size_t)nw * r1 + (c1 >> 6)] &= ~(1ull << (c1 & 63));
            mask[(size_t)nw * r1 + (c2 >> 6)] |= 1ull << (c2 & 63);
        }
    }
    __syncwarp();
}

// tab[d-1] = ceil(exp(-d/T) * 2^32) (see build_thresholds, xw_anneal.cu)
__device__ __noinline__ void l_thresholds(uint64_t* tab, double T, int lane) {
    const double t = T > 1.0e-12 ? T : 1.0e-12;
    for (uint32_t d = lane + 1; d <= kThrTable; d += 32) {
        const double e = acceptance_exp(__ddiv_rn(-(double)d, t));
        tab[d - 1] = (uint64_t)ceil(__dmul_rn(e, 0x1p32));
    }
    __syncwarp();
}

__device__ __forceinline__ void l_copy16(void* dst, const void* src, uint32_t bytes, int lane) {
    const uint32_t chunks = xw_pad16(bytes) / 16u;
    uint4* d = reinterpret_cast<uint4*>(dst);
    const uint4* s = reinterpret_cast<const uint4*>(src);
    for (uint32_t i = lane; i < chunks; i += 32) d[i] = s[i];
}

__device__ __forceinline__ uint64_t l_globaltimer() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Support and sign masks of the lane's rows from W; G = W W^T from them:
// G[r][o] = |S_r & S_o| - 2 |S_r & S_o & (N_r ^ N_o)|.  Returns whether
// every row has weight w.
__device__ bool build_gram(const int8_t* W, int16_t* G, uint64_t* mask, uint64_t* sign, int n, int w, int nw,
                           int lane) {
    bool ok = true;
#pragma unroll 1
    for (int o = lane; o < n; o += 32) {
        int weight = 0;
#pragma unroll 1
        for (int q = 0; q < nw; ++q) {
            uint64_t nz = 0, ng = 0;
#pragma unroll 1
            for (int c = 64 * q; c < n && c < 64 * q + 64; ++c) {
                const int v = W[(size_t)c * n + o];
                if (v != 0) nz |= 1ull << (c & 63);
                if (v < 0) ng |= 1ull << (c & 63);
            }
            mask[(size_t)o * nw + q] = nz;
            sign[(size_t)o * nw + q] = ng;
            weight += __popcll(nz);
        }
        if (weight != w) ok = false;
    }
    __syncwarp();
#pragma unroll 1
    for (int o = lane; o < n; o += 32) {
        const uint64_t* so = mask + (size_t)o * nw;
        const uint64_t* no = sign + (size_t)o * nw;
#pragma unroll 1
        for (int r = 0; r < n; ++r) {
            const uint64_t* sr = mask + (size_t)r * nw;
            const uint64_t* nr = sign + (size_t)r * nw;
            int dot = 0;
#pragma unroll 1
            for (int q = 0; q < nw; ++q) {
                const uint64_t both = sr[q] & so[q];
                dot += __popcll(both) - 2 * __popcll(both & (nr[q] ^ no[q]));
            }
            G[(size_t)r * n + o] = (int16_t)dot;
        }
    }
    __syncwarp();
    return ok;
}

template <bool GEN>
__device__ void run_large(const AnnealArgs& a, uint32_t rid, uint8_t* slot, int lane, uint64_t chunk_iters) {
    uint8_t* rec = a.arena + a.rec_off[rid];
    RepHeader* H = reinterpret_cast<RepHeader*>(rec);
    const uint32_t jid = H->job;
    XwJob* J = a.jobs + jid;
    if (*(volatile int32_t*)&J->done) return;
    if (a.stop_on_solve == 1 && *(volatile int32_t*)&J->solved) return;

    const int n = J->n, w = J->w, m = J->m, sparse = J->sparse;
    const int nw = (n + 63) / 64;
    const LSlot L = large_slot(n);
    const LGram LG = large_gram(n);
    int8_t* W = reinterpret_cast<int8_t*>(rec + J->off_w);
    uint16_t* mino = reinterpret_cast<uint16_t*>(rec + J->off_mino);
    uint8_t* gbase = a.gram + a.gram_off[rid];
    int16_t* G = reinterpret_cast<int16_t*>(gbase);
    uint64_t* mask = reinterpret_cast<uint64_t*>(gbase + LG.off_mask);
    uint64_t* sign = reinterpret_cast<uint64_t*>(gbase + LG.off_sign);
    int32_t* sRes = reinterpret_cast<int32_t*>(slot);
    uint4* sDraw = reinterpret_cast<uint4*>(slot + L.off_draws);
    const uint32_t* sDw = reinterpret_cast<const uint32_t*>(sDraw);
    LView* sView = reinterpret_cast<LView*>(slot + L.off_view);
    uint64_t* sThr = reinterpret_cast<uint64_t*>(slot + L.off_thr);

    uint64_t it = H->it;
    uint64_t iters = chunk_iters;
    if (J->budget_iters) {
        if (it >= J->budget_iters) return;
        if (iters > J->budget_iters - it) iters = J->budget_iters - it;
    }

    // ---- Gram and masks (once per W the host wrote), minority lists ----
    const uint32_t status0 = H->status;
    if (!(status0 & XW_STATUS_GRAM)) {
        const bool ok = build_gram(W, G, mask, sign, n, w, nw, lane);
        if (__any_sync(FULL, !ok)) {
            if (lane == 0) H->err |= XW_ERR_MINORITY;
            return;
        }
    }
    if (m > 0 && !(status0 & XW_STATUS_INIT)) {
        int bad = 0;
#pragma unroll 1
        for (int o = lane; o < n; o += 32) {
            int pos = 0;
#pragma unroll 1
            for (int c = 0; c < n; ++c) {
                if ((W[(size_t)c * n + o] != 0) == (sparse != 0)) {
                    if (pos < m) mino[(size_t)o * m + pos] = (uint16_t)c;
                    ++pos;
                }
            }
            if (pos != m) bad = 1;
        }
        if (__any_sync(FULL, bad)) {
            if (lane == 0) H->err |= XW_ERR_MINORITY;
            return;
        }
        __syncwarp();
    }

    // ---- residuals and totals from G ----
    int p_score = 0, p_conf = 0, p_par = 0;
    long long p_sq = 0;
#pragma unroll 1
    for (int o = lane; o < n; o += 32) {
        int r_sum = 0;
#pragma unroll 4
        for (int r = 0; r < n; ++r) {
            const int g = G[(size_t)r * n + o];
            if (r != o) {
                const int ag = iabs(g);
                r_sum += ag;
                p_conf += g != 0;
                p_sq += (long long)(g * g);
                p_par += ag & 1;
            }
        }
        sRes[o] = r_sum;
        p_score += r_sum;
    }
    const int score0 = __reduce_add_sync(FULL, p_score) / 2;
    const int conf0 = __reduce_add_sync(FULL, p_conf) / 2;
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) p_sq += __shfl_xor_sync(FULL, p_sq, off);
    const long long sq0 = p_sq / 2;
    const int par0 = __reduce_add_sync(FULL, p_par) / 2;
    __syncwarp();

    const int obj_kind = GEN ? H->obj_kind : 0;
    if (!GEN && (H->obj_kind != 0 || J->move_set != 0)) {
        if (lane == 0) H->err |= XW_ERR_KERNEL;
        return;
    }
    const int64_t obj0 = obj_kind == 1 ? sq0 : obj_kind == 2 ? par0 : score0;
    int score, conflicts, best_s, best_c, msi, cool;
    int64_t obj_total;
    uint64_t moves, cand_evals;
    uint32_t accepted = H->accepted, accepted_rows = H->accepted_rows, two_row_evals = H->two_row_evals;
    double T = H->temperature;
    const double reheat_T = H->reheat_temperature;
    bool at_best;  // W equals the best state and the best copy is pending
    if (status0 & XW_STATUS_INIT) {
        if (H->score != score0 || H->conflicts != conf0 || H->obj_total != obj0) {
            if (lane == 0) H->err |= XW_ERR_SCORE;
            return;
        }
        best_s = H->best_score;
        best_c = H->best_conflicts;
        msi = H->msi;
        cool = H->cool_ctr;
        moves = H->moves;
        cand_evals = H->cand_evals;
        at_best = false;
    } else {
        best_s = score0;
        best_c = conf0;
        msi = 0;
        cool = 0;
        moves = 0;
        cand_evals = 0;
        accepted = accepted_rows = two_row_evals = 0;
        at_best = true;
    }
    score = score0;
    conflicts = conf0;
    obj_total = obj0;

    const int tempering = J->tempering;
    const int cs = J->candidate_samples, ts = J->target_samples;
    const int mpc = J->moves_per_cool, stuck = J->stuck_threshold;
    const uint32_t k0 = J->key0, k1 = J->key1, stream = H->stream;
    const uint64_t thr_greedy = J->thr_greedy;
    const double t_min = J->t_min, cooling = J->cooling, reheat = J->reheat;
    const int bpc = 4 + (ts <= 4 ? 1 : 2);
    const bool coop = ts <= 8;
    if (lane == 0) {
        LView v;
        v.W = W; v.mino = mino; v.res = sRes; v.mask = mask; v.dw = sDw;
        v.thr_target = J->thr_target; v.thr_dbl = J->thr_double; v.thr_sign = J->thr_sign;
        v.thr_swsign = J->thr_swsign;
        v.n = n; v.w = w; v.m = m; v.sparse = sparse; v.ts = ts; v.bpc = bpc; v.cc = 31 / bpc;
        v.move_set = J->move_set; v.nw = nw;
        v.stream = stream; v.k0 = k0; v.k1 = k1; v.pad = 0;
        *sView = v;
    }
    __syncwarp();
    l_thresholds(sThr, T, lane);

    uint32_t my_slot = 0;
    if (lane > 0) {
        const int q = lane - 1, c = q / bpc, b = q - c * bpc;
        my_slot = cand_slot(c, b);
    }
    uint8_t* best_dst = rec + J->off_best;
    const uint32_t nn = (uint32_t)(n * n);

    uint64_t done = 0;
#pragma unroll 1
    for (; done < iters; ++done) {
        if (a.stop_on_solve) {
            if (best_s == 0) break;
            if (a.stop_on_solve == 1 && (done & 63) == 63 && *(volatile int32_t*)&J->solved) break;
        }
        sDraw[lane] = draw_block(my_slot, it, stream, k0, k1);
        __syncwarp();
        const uint4 mblk = sDraw[0];
        const int count = (uint64_t)mblk.x < thr_greedy ? cs : 1;

        // cooperative hot-row tournaments for candidates 0..3: the largest
        // residual, the first sample among equals
        unsigned long long hot_key = 0;
        if (coop) {
            const int c = lane >> 3, s = lane & 7;
            if (c < count && s < ts) {
                const uint32_t wd = sDw[(1 + c * bpc + 4 + (s >> 2)) * 4 + (s & 3)];
                const uint32_t row = draw_index(wd, (uint32_t)n, cand_slot(c, 4 + (s >> 2)), it, stream, k0, k1, s & 3);
                hot_key = ((unsigned long long)(uint32_t)sRes[row] << 15) | ((unsigned long long)(31 - s) << 10) |
                          (unsigned long long)row;
            }
#pragma unroll
            for (int off = 1; off < 8; off <<= 1) {
                const unsigned long long o = __shfl_xor_sync(FULL, hot_key, off);
                hot_key = o > hot_key ? o : hot_key;
            }
        }
        const int coop_row = (int)(__shfl_sync(FULL, hot_key, (lane & 3) << 3) & 1023ull);

        LMove desc = none();
        if (lane < count) desc = l_propose<GEN>(sView, it, lane, coop && lane < 4, coop_row);
        __syncwarp();

        bool have = false;
        LMove best_mv = none();
        int bds = 0, bdc = 0, bprim = 0;
#pragma unroll 1
        for (int c = 0; c < count; ++c) {
            LMove e;
            e.x = __shfl_sync(FULL, desc.x, c);
            if (!(e.x & 1u)) continue;
            e.y = __shfl_sync(FULL, desc.y, c);
            e.z = __shfl_sync(FULL, desc.z, c);
            const LUpdate u = l_decode(e);
            const LDeltas d = l_eval<GEN>(u, W, G, n, lane);
            const int ds = __reduce_add_sync(FULL, d.ds);
            const int dc = __reduce_add_sync(FULL, d.dc);
            int prim = ds;
            if (GEN) {
                if (obj_kind == 1) prim = __reduce_add_sync(FULL, d.dsq);
                else if (obj_kind == 2) prim = __reduce_add_sync(FULL, d.dpar);
            }
            ++cand_evals;
            two_row_evals += u.R2 >= 0;
            bool better = !have;
            if (!better) {
                if (prim != bprim) better = prim < bprim;
                else if (ds != bds) better = ds < bds;
                else better = dc < bdc;
            }
            if (better) {
                have = true; best_mv = e; bds = ds; bdc = dc; bprim = prim;
            }
        }
        if (!have) {
            ++it;
            continue;
        }
        ++moves;

        bool accept = bprim <= 0;
        if (!accept)
            accept = bprim <= (int64_t)kThrTable ? (uint64_t)mblk.y < sThr[bprim - 1]
                                                 : metropolis_accept(bprim, T, mblk.y);

        if (accept) {
            // leaving a best state without improving on it: its copy is due
            if (at_best && !(bds < 0 || (bds == 0 && bdc < 0))) {
                l_copy16(best_dst, W, nn, lane);
                __syncwarp();
                at_best = false;
            }
            const LUpdate u = l_decode(best_mv);
            l_commit<GEN>(best_mv, u, bds, W, G, sRes, mino, mask, n, m, nw, sparse, lane);
            score += bds;
            conflicts += bdc;
            obj_total += bprim;
            ++accepted;
            accepted_rows += u.R2 >= 0 ? 2u : 1u;
        }

        if (score < best_s || (score == best_s && conflicts < best_c)) {
            best_s = score;
            best_c = conflicts;
            msi = 0;
            at_best = true;
            if (best_s == 0 && lane == 0) {
                H->solve_it = it;
                H->solve_ns = l_globaltimer();
                if (atomicCAS(&J->solved, 0, 1) == 0) {
                    J->solved_replica = (int32_t)H->stream;
                    J->solved_it = it;
                    J->solve_ns = H->solve_ns;
                }
            }
        } else {
            ++msi;
        }
        if (!tempering) {
            const double T0 = T;
            if (++cool >= mpc) {
                cool = 0;
                T = __dmul_rn(T, cooling);
                if (T < t_min) T = t_min;
            }
            if (msi >= stuck) {
                msi = 0;
                T = __dmul_rn(reheat_T, reheat);
                if (T < t_min) T = t_min;
            }
            if (T != T0) l_thresholds(sThr, T, lane);
        }
        ++it;
    }

    __syncwarp();
    if (at_best) l_copy16(best_dst, W, nn, lane);
    if (lane == 0) {
        H->it = it;
        H->moves = moves;
        H->cand_evals = cand_evals;
        H->accepted = accepted;
        H->accepted_rows = accepted_rows;
        H->two_row_evals = two_row_evals;
        H->score = score;
        H->conflicts = conflicts;
        H->best_score = best_s;
        H->best_conflicts = best_c;
        H->obj_total = obj_total;
        H->temperature = T;
        H->msi = msi;
        H->cool_ctr = cool;
        H->status = status0 | XW_STATUS_INIT | XW_STATUS_GRAM | (best_s == 0 ? XW_STATUS_SOLVED : 0u);
    }
    __syncwarp();
}

// CTAs of four warps per SM the register budget is sized for
#ifndef XW_LARGE_MIN_BLOCKS
#define XW_LARGE_MIN_BLOCKS 4
#endif
template <bool GEN>
__global__ void __launch_bounds__(128, XW_LARGE_MIN_BLOCKS) anneal_large_kernel(AnnealArgs a) {
    extern __shared__ __align__(16) uint8_t smem[];
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    uint8_t* slot = smem + (size_t)warp * a.slot_bytes;
    // work items as in anneal_kernel (xw_anneal.cu): whole replicas, or
    // chunks of their iterations in chunk-major order
    const uint64_t total = (uint64_t)a.n_items * a.chunks;
    for (;;) {
        uint32_t item = 0;
        if (lane == 0) item = atomicAdd(a.counter, 1u);
        item = __shfl_sync(FULL, item, 0);
        if (item >= total) break;
        if (a.chunks == 1) {
            run_large<GEN>(a, a.items[item], slot, lane, a.iters);
            continue;
        }
        const uint32_t c = item / a.n_items;
        const uint32_t rid = a.items[item - c * a.n_items];
        const uint64_t lo = a.iters * c / a.chunks, hi = a.iters * (c + 1) / a.chunks;
        RepHeader* H = reinterpret_cast<RepHeader*>(a.arena + a.rec_off[rid]);
        const bool ok = chunk_begin(a.chunk_done + rid, c, a.chunk_wait_ns, &H->err, lane, FULL);
        if (ok) run_large<GEN>(a, rid, slot, lane, hi - lo);
        chunk_end(a.chunk_done + rid, c, ok, lane, FULL);
    }
}

}  // namespace

uint32_t anneal_large_slot_bytes(int n) { return large_slot(n).bytes; }

uint64_t anneal_large_gram_bytes(int n) { return (large_gram(n).bytes + 255u) & ~uint64_t(255); }

const void* anneal_large_kernel_fn(bool general) {
    return general ? reinterpret_cast<const void*>(&anneal_large_kernel<true>)
                   : reinterpret_cast<const void*>(&anneal_large_kernel<false>);
}

cudaError_t launch_anneal_large(const AnnealArgs& args, bool general, int warps_per_block, int blocks,
                                cudaStream_t stream) {
    const size_t smem = (size_t)warps_per_block * args.slot_bytes;
    const dim3 grid(blocks), block(32 * warps_per_block);
    void* kargs[] = {const_cast<AnnealArgs*>(&args)};
    return cudaLaunchKernel(anneal_large_kernel_fn(general), grid, block, kargs, smem, stream);
}

}  // namespace xw
