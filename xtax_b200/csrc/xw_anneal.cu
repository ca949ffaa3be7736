// xw_anneal.cu -- the population annealing kernel for weighing matrices.
//
// One warp owns one replica at a time.  The replica's int8 W (column-major),
// int32 Gram, row residuals, minority lists and row support masks live in the
// warp's shared-memory slot; lane o owns "other" rows o, o+32, ... of every
// O(n) delta, so a candidate's exact change to W W^T and to the score is one
// pass over shared memory plus one redux.sync.  The whole iteration is
// warp-synchronous: no __syncthreads, no block-wide reductions.
//
// Per iteration (the semantics of the reference kernel anneal_kernel,
// src/xweigh_cuda.cu:988-1130, with cuRAND replaced by counter-based Philox):
//   A  every lane computes one Philox block of this iteration's draws
//      (move-level block + the common blocks of the first candidates) into
//      shared memory;
//   C  8 lanes per candidate run the hot-row tournament (xweigh_cuda.cu:291-300)
//      and a segmented max picks the first best sample;
//   D  lane c proposes candidate c (propose_move, xweigh_cuda.cu:423-447);
//   E  the warp evaluates the candidates in order and keeps the first best
//      (device_better_evaluation, xweigh_cuda.cu:227-244);
//   F  Metropolis on the replica's objective with the integer draw and the
//      deterministic acceptance exponential;
//   G  the warp commits the move (commit_*, xweigh_cuda.cu:607-877);
//   H  best tracking, cooling and reheat (xweigh_cuda.cu:1087-1129).
//
// Every move kind changes at most two rows of W, and each changed Gram row
// is old + a*W[:,x] + b*W[:,y] for two columns x, y; evaluation and commit
// run that one form (plus the row1-row2 pair term of a double flip over two
// rows), so the hot loop has one code path instead of one per move kind.
// Instruction-cache misses, not arithmetic, bound this kernel when the
// per-kind paths are specialised and inlined; the proposal helpers are kept
// out of line for the same reason.
//
// Work distribution is persistent: each warp takes replica ids from a
// global counter until the launch's item list is exhausted, so replicas of
// different orders and weights share one launch.
#include <cuda_runtime.h>

#include <type_traits>

#include <cooperative_groups.h>

#include "xw_device.cuh"
#include "xw_kernels.h"

namespace xw {

namespace {

constexpr unsigned FULL = 0xffffffffu;

// Lane groups.  A replica is owned by a group of GW lanes: the whole warp
// (GW = 32), or one half of it (GW = 16, orders up to 16: two replicas per
// warp, each half with its own shared-memory slot and its own work items).
// Warp collectives name only the group's lanes; the two halves' replicas
// are independent and the hardware runs them side by side wherever their
// control flow agrees.
template <int GW>
__device__ __forceinline__ unsigned group_mask() {
    if constexpr (GW == 32) return FULL;
    else return 0xffffu << (threadIdx.x & 16);
}

// Move statistics in the replica header (accepted moves, the rows they
// changed, two-row candidate evaluations); a build with XW_MOVE_STATS=0
// leaves them at zero and drops their counting from the hot loop.
#ifndef XW_MOVE_STATS
#define XW_MOVE_STATS 1
#endif
constexpr bool kMoveStats = XW_MOVE_STATS != 0;

// Metropolis thresholds kept per replica for objective increases 1..kThrTable.
constexpr uint32_t kThrTable = 64;

// Replica-constant fields the proposal code reads, kept in the warp's slot.
struct View {
    const int8_t* W;
    const uint8_t* mino;
    const int32_t* res;
    const uint64_t* mask;      // MW words per row: nonzero support
    const uint32_t* dw;        // cached draw words of this iteration
    uint64_t valid[4];         // columns < n
    uint64_t thr_target, thr_dbl, thr_sign, thr_swsign;
    int n, w, m, sparse, ts, bpc, cc, move_set;
    uint32_t stream, k0, k1, pad;
};

struct SlotLayout {
    uint32_t off_g, off_res, off_mino, off_mask, off_draws, off_view, off_thr, bytes;
    int ld;
};

// The eight-rows-per-lane kernel (orders above 128) keeps G as int16
// (|G_ij| <= w <= 256, as the reference does) and 256-bit row masks, so that
// W(256,255) still fits one CTA's shared memory; `wide` selects that layout
// for every replica of such a launch, whatever its own order.
__host__ __device__ inline SlotLayout slot_layout(int n, int m, bool wide) {
    SlotLayout L;
    L.ld = n | 1;
    const uint32_t nn = (uint32_t)(n * n);
    const uint32_t gsz = wide ? 2u : 4u, mw = wide ? 4u : 2u;
    L.off_g = xw_pad16(nn);
    L.off_res = L.off_g + xw_pad16((uint32_t)(n * L.ld) * gsz);
    L.off_mino = L.off_res + xw_pad16((uint32_t)n * 4u);
    L.off_mask = L.off_mino + xw_pad16((uint32_t)(n * m));
    L.off_draws = L.off_mask + xw_pad16((uint32_t)n * 8u * mw);
    L.off_view = L.off_draws + 32u * 16u;
    L.off_thr = L.off_view + xw_pad16((uint32_t)sizeof(View));
    L.bytes = L.off_thr + kThrTable * 8u;
    return L;
}

__device__ __forceinline__ int iabs(int v) { return v < 0 ? -v : v; }

// First set bit at or after `start`, cyclically, of a 128-bit row mask.
__device__ __forceinline__ int cyclic_first(uint64_t lo, uint64_t hi, int start) {
    const uint64_t a_lo = start < 64 ? (lo & (~0ull << start)) : 0ull;
    const uint64_t a_hi = start < 64 ? hi : (hi & (~0ull << (start - 64)));
    if (a_lo) return __ffsll((long long)a_lo) - 1;
    if (a_hi) return 64 + __ffsll((long long)a_hi) - 1;
    if (lo) return __ffsll((long long)lo) - 1;
    if (hi) return 64 + __ffsll((long long)hi) - 1;
    return -1;
}

__device__ __forceinline__ int cyclic_first(const uint64_t (&m)[2], int start) {
    return cyclic_first(m[0], m[1], start);
}

// the same over a 256-bit row mask
__device__ __forceinline__ int cyclic_first(const uint64_t (&m)[4], int start) {
    const int ws = start >> 6;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        if (k < ws) continue;
        const uint64_t x = k == ws ? (m[k] & (~0ull << (start & 63))) : m[k];
        if (x) return 64 * k + __ffsll((long long)x) - 1;
    }
#pragma unroll
    for (int k = 0; k < 4; ++k)
        if (m[k]) return 64 * k + __ffsll((long long)m[k]) - 1;
    return -1;
}

template <int MW>
__device__ __forceinline__ void row_mask(const uint64_t* mask, int row, uint64_t (&m)[MW]) {
#pragma unroll
    for (int k = 0; k < MW; ++k) m[k] = mask[MW * row + k];
}

// Draw words outside the cached blocks (rare: attempts past the first,
// tournaments past 8 samples, candidates past the cached ones).
__device__ __noinline__ uint32_t slow_word(uint32_t slot, uint64_t it, uint32_t stream, uint32_t k0, uint32_t k1,
                                           int j) {
    return pick(draw_block(slot, it, stream, k0, k1), j);
}

__device__ __forceinline__ uint32_t word(const View* v, uint64_t it, int c, int b, int j) {
    if (c < v->cc && b < v->bpc) return v->dw[(1 + c * v->bpc + b) * 4 + j];
    return slow_word(cand_slot(c, b), it, v->stream, v->k0, v->k1, j);
}

__device__ __forceinline__ uint32_t index(const View* v, uint64_t it, int c, int b, int j, uint32_t count) {
    return draw_index(word(v, it, c, b, j), count, cand_slot(c, b), it, v->stream, v->k0, v->k1, j);
}

__device__ __forceinline__ int at(const View* v, int r, int c) { return v->W[c * v->n + r]; }

// The same replica context in registers, for the inlined common path of a
// proposal: reading it from shared memory would put two dependent loads in
// front of every draw.
struct Reg {
    const int8_t* W;
    const uint8_t* mino;
    const uint64_t* mask;
    const uint32_t* cw;        // this candidate's cached draw words
    uint64_t it;
    uint64_t thr_target, thr_dbl, thr_sign, thr_swsign;
    int n, w, m, sparse, move_set;
    bool cached;               // candidate's blocks 0..bpc-1 are in cw
    uint32_t stream, k0, k1;

    __device__ __forceinline__ uint32_t word(int c, int b, int j) const {
        if (cached) return cw[b * 4 + j];
        return slow_word(cand_slot(c, b), it, stream, k0, k1, j);
    }
    __device__ __forceinline__ uint32_t index(int c, int b, int j, uint32_t count) const {
        return draw_index(word(c, b, j), count, cand_slot(c, b), it, stream, k0, k1, j);
    }
    __device__ __forceinline__ int at(int r, int c) const { return W[c * n + r]; }
};

// Move descriptor, two words (8-bit rows, columns and minority positions):
//   d0 = valid | kind<<1 | r1<<3 | r2<<11 | c1<<19
//   d1 = c2 | (v1+1)<<8 | (v2+1)<<10 | p1<<12 | p2<<20
// kinds: 0 sign flip (r1,c1); 1 support switch with new values v1 at
// (r1,c2) and v2 at (r2,c1); 2 double flip (r1,c1),(r2,c2); 3 within-row
// swap: the nonzero at (r1,c1) moves to (r1,c2) with value v1.
__device__ __forceinline__ uint2 pack(int kind, int r1, int r2, int c1, int c2, int v1, int v2, int p1, int p2) {
    return make_uint2(1u | ((uint32_t)kind << 1) | ((uint32_t)r1 << 3) | ((uint32_t)r2 << 11) | ((uint32_t)c1 << 19),
                      (uint32_t)c2 | ((uint32_t)(v1 + 1) << 8) | ((uint32_t)(v2 + 1) << 10) | ((uint32_t)p1 << 12) |
                          ((uint32_t)p2 << 20));
}

// propose_sign_flip (xweigh_cuda.cu:302-325): a nonzero column of `row`,
// from the minority list when the row is sparse, else the first nonzero at
// or after a random column; -1 when the row has none.
template <int MW>
__device__ __noinline__ int d_flip_col(const View* v, uint64_t it, int c, int b, int j, int row) {
    if (v->sparse && v->m > 0) return v->mino[row * v->m + (int)index(v, it, c, b, j, (uint32_t)v->m)];
    const int start = (int)index(v, it, c, b, j, (uint32_t)v->n);
    uint64_t mk[MW];
    row_mask<MW>(v->mask, row, mk);
    return cyclic_first(mk, start);
}

// hot_row (xweigh_cuda.cu:291-300), serial form
__device__ __noinline__ int d_hot_row(const View* v, uint64_t it, int c) {
    int best = (int)index(v, it, c, 4, 0, (uint32_t)v->n);
#pragma unroll 1
    for (int k = 1; k < v->ts; ++k) {
        const int cand = (int)index(v, it, c, 4 + k / 4, k % 4, (uint32_t)v->n);
        if (v->res[cand] > v->res[best]) best = cand;
    }
    return best;
}

// propose_double_sign_flip (xweigh_cuda.cu:389-421), second-flip attempts
// 1..15 (attempt 0 is evaluated inline by d_propose)
template <int MW>
__device__ __noinline__ uint2 d_double_rest(const View* v, uint64_t it, int c, int row1, int col1) {
#pragma unroll 1
    for (int a = 1; a < 16; ++a) {
        const int b = 20 + (a - 1);
        const int row2 = word(v, it, c, b, 0) < 0x80000000u ? row1 : (int)index(v, it, c, b, 1, (uint32_t)v->n);
        const int col2 = d_flip_col<MW>(v, it, c, b, 2, row2);
        if (col2 < 0 || (row2 == row1 && col2 == col1)) continue;
        return pack(2, row1, row2, col1, col2, 0, 0, 0, 0);
    }
    return make_uint2(0u, 0u);
}

// propose_support_switch (xweigh_cuda.cu:327-387), new signs per
// switch_sign_fraction (xweigh_cuda.cu:378-383); attempts a0..23
__device__ __noinline__ uint2 d_switch(const View* v, uint64_t it, int c, int row1, int a0) {
    if (v->m == 0 || v->n < 2) return make_uint2(0u, 0u);
#pragma unroll 1
    for (int a = a0; a < 24; ++a) {
        // attempt 0 in cached blocks 1-2, attempt a>0 in blocks 36+2(a-1), +1
        const int B = a == 0 ? 1 : 36 + 2 * (a - 1);
        const int o = a == 0 ? 1 : 0;
        int row2 = (int)index(v, it, c, B, o, (uint32_t)(v->n - 1));
        if (row2 >= row1) ++row2;
        const int p1 = (int)index(v, it, c, B, o + 1, (uint32_t)v->m);
        const int p2 = (int)index(v, it, c, B, o + 2, (uint32_t)v->m);
        const int q1 = v->mino[row1 * v->m + p1], q2 = v->mino[row2 * v->m + p2];
        const int c1 = v->sparse ? q1 : q2, c2 = v->sparse ? q2 : q1;
        if (c1 == c2 || at(v, row1, c2) != 0 || at(v, row2, c1) != 0) continue;
        const int v1 = at(v, row1, c1), v2 = at(v, row2, c2);
        if (v1 == 0 || v2 == 0) continue;
        const uint32_t s1 = a == 0 ? word(v, it, c, 2, 0) : word(v, it, c, B, 3);
        const uint32_t s2 = a == 0 ? word(v, it, c, 2, 1) : word(v, it, c, B + 1, 0);
        return pack(1, row1, row2, c1, c2, (uint64_t)s1 < v->thr_swsign ? -v1 : v1,
                    (uint64_t)s2 < v->thr_swsign ? -v2 : v2, p1, p2);
    }
    return make_uint2(0u, 0u);
}

// within-row swap: a nonzero of the row moves to one of its zeros
template <int MW>
__device__ __noinline__ uint2 d_row_swap(const View* v, uint64_t it, int c, int row) {
    if (v->m == 0) return make_uint2(0u, 0u);
    uint64_t nz[MW];
    row_mask<MW>(v->mask, row, nz);
    int c1, c2, pos;
    if (v->sparse) {
        pos = (int)index(v, it, c, 1, 1, (uint32_t)v->m);
        c1 = v->mino[row * v->m + pos];
        uint64_t zero[MW];
#pragma unroll
        for (int k = 0; k < MW; ++k) zero[k] = ~nz[k] & v->valid[k];
        c2 = cyclic_first(zero, (int)index(v, it, c, 1, 2, (uint32_t)v->n));
    } else {
        pos = (int)index(v, it, c, 1, 2, (uint32_t)v->m);
        c2 = v->mino[row * v->m + pos];
        c1 = cyclic_first(nz, (int)index(v, it, c, 1, 1, (uint32_t)v->n));
    }
    if (c1 < 0 || c2 < 0) return make_uint2(0u, 0u);
    return pack(3, row, 0, c1, c2, word(v, it, c, 1, 3) < 0x80000000u ? 1 : -1, 0, pos, 0);
}

template <int MW>
__device__ __forceinline__ uint2 flip_move(const View* v, uint64_t it, int c, int b, int j, int row) {
    const int col = d_flip_col<MW>(v, it, c, b, j, row);
    return col < 0 ? make_uint2(0u, 0u) : pack(0, row, 0, col, 0, 0, 0, 0, 0);
}

// flip column from a draw word without the out-of-line call: minority pick
// for a sparse row, else the cyclic first nonzero from a random column
template <int MW>
__device__ __forceinline__ int flip_col_w(const Reg& r, int c, int b, int j, int row) {
    if (r.sparse && r.m > 0) return r.mino[row * r.m + (int)r.index(c, b, j, (uint32_t)r.m)];
    const int start = (int)r.index(c, b, j, (uint32_t)r.n);
    uint64_t mk[MW];
    row_mask<MW>(r.mask, row, mk);
    return cyclic_first(mk, start);
}

// propose_move (xweigh_cuda.cu:423-447).  The first attempt of every move
// kind is computed unconditionally from the cached draw words and the
// choice is made afterwards, so the candidate lanes of a warp run one
// instruction stream whatever kinds they pick; only the rare further
// attempts (a second flip that repeats the first, a switch whose 2x2 is not
// legal) branch into out-of-line code.  Move set 1 replaces the switch by
// the within-row swap and has no double flips.  The result equals the
// sequential reference order of draws and tests.
template <int MW, bool GEN>
__device__ __forceinline__ uint2 d_propose(const Reg& r, const View* v, int c, bool coop_ok, int coop_row) {
    const int n = r.n, m = r.m;
    const uint64_t it = r.it;
    const bool targeted = (uint64_t)r.word(c, 0, 0) < r.thr_target;
    const int row = targeted ? (coop_ok ? coop_row : d_hot_row(v, it, c)) : (int)r.index(c, 0, 1, (uint32_t)n);
    const bool want_dbl = (!GEN || r.move_set == 0) && (uint64_t)r.word(c, 0, 2) < r.thr_dbl;
    const bool want_flip = r.w == n || (uint64_t)r.word(c, 0, 3) < r.thr_sign;

    // double flip, attempt 0: first flip (2,3), second row/flip from block 3
    const int dcol1 = flip_col_w<MW>(r, c, 2, 3, row);
    const int drow2 = r.word(c, 3, 0) < 0x80000000u ? row : (int)r.index(c, 3, 1, (uint32_t)n);
    const int dcol2 = flip_col_w<MW>(r, c, 3, 2, drow2);
    const bool dbl_ok = dcol1 >= 0 && dcol2 >= 0 && !(drow2 == row && dcol2 == dcol1);
    // plain flip
    const int fcol = flip_col_w<MW>(r, c, 1, 0, row);

    uint2 mv = make_uint2(0u, 0u);
    if (want_dbl && dcol1 >= 0) {
        if (dbl_ok) return pack(2, row, drow2, dcol1, dcol2, 0, 0, 0, 0);
        mv = d_double_rest<MW>(v, it, c, row, dcol1);
        if (mv.x) return mv;
    }
    if (want_flip) return fcol < 0 ? make_uint2(0u, 0u) : pack(0, row, 0, fcol, 0, 0, 0, 0, 0);
    if (GEN && r.move_set == 1) {
        mv = d_row_swap<MW>(v, it, c, row);
    } else {
        // support switch, attempt 0 (blocks 1 and 2)
        const int mm = m > 0 ? m : 1;
        int row2 = (int)r.index(c, 1, 1, (uint32_t)(n > 1 ? n - 1 : 1));
        if (row2 >= row) ++row2;
        if (row2 >= n) row2 = 0;
        const int p1 = (int)r.index(c, 1, 2, (uint32_t)mm);
        const int p2 = (int)r.index(c, 1, 3, (uint32_t)mm);
        const int q1 = m > 0 ? r.mino[row * m + p1] : 0, q2 = m > 0 ? r.mino[row2 * m + p2] : 0;
        const int c1 = r.sparse ? q1 : q2, c2 = r.sparse ? q2 : q1;
        const int v1 = r.at(row, c1), v2 = r.at(row2, c2);
        const bool ok = m > 0 && n > 1 && c1 != c2 && r.at(row, c2) == 0 && r.at(row2, c1) == 0 && v1 != 0 &&
                        v2 != 0;
        if (ok) {
            const int nv1 = (uint64_t)r.word(c, 2, 0) < r.thr_swsign ? -v1 : v1;
            const int nv2 = (uint64_t)r.word(c, 2, 1) < r.thr_swsign ? -v2 : v2;
            return pack(1, row, row2, c1, c2, nv1, nv2, p1, p2);
        }
        mv = d_switch(v, it, c, row, 1);
    }
    if (mv.x) return mv;
    return flip_move<MW>(v, it, c, 2, 2, row);
}

// A decoded move as at most two row updates: row R1 gets
// A1*W[:,X1] + B1*W[:,Y1], row R2 (when >= 0) gets A2*W[:,X2] + B2*W[:,Y2];
// `pair` marks the double flip over two rows whose G[r1][r2] also changes.
struct Update {
    int R1, X1, Y1, A1, B1;
    int R2, X2, Y2, A2, B2;
    int pair;
};

__device__ __forceinline__ Update decode(uint32_t d0, uint32_t d1, const int8_t* W, int n) {
    const int kind = (d0 >> 1) & 3, r1 = (d0 >> 3) & 255, r2 = (d0 >> 11) & 255;
    const int c1 = (d0 >> 19) & 255, c2 = d1 & 255;
    const int nv1 = (int)((d1 >> 8) & 3) - 1, nv2 = (int)((d1 >> 10) & 3) - 1;
    const int w11 = W[c1 * n + r1], w22 = W[c2 * n + r2];
    Update u;
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

struct Deltas {
    int ds, dc, dsq, dpar;
};

// GEN: the general kernel, whose replicas may use the squared or parity
// objective; the lean one tracks the L1 score and conflicts only
template <bool GEN>
__device__ __forceinline__ void acc(Deltas& d, int old, int nw) {
    const int ao = iabs(old), an = iabs(nw);
    d.ds += an - ao;
    d.dc += (nw != 0) - (old != 0);
    if (GEN) {
        d.dsq += nw * nw - old * old;
        d.dpar += (an & 1) - (ao & 1);
    }
}

// the pair entry G[r1][r2] after a double flip over rows r1 != r2
// (xweigh_cuda.cu:564-583)
__device__ __forceinline__ int pair_new(const Update& u, int op, const int8_t* W, int n, int c1, int c2) {
    return op + u.A1 * W[c1 * n + u.R2] + u.A2 * W[c2 * n + u.R1] + (c1 == c2 ? u.A1 * u.A2 : 0);
}

// evaluate_move_warp (xweigh_cuda.cu:449-599): lane-partial deltas over the
// lane's own rows; the caller reduces them across the warp.
template <int OPL, typename GT, bool GEN, int GW = 32>
__device__ __forceinline__ Deltas eval_lane(const Update& u, const int8_t* W, const GT* G, int n, int ld,
                                            int lane) {
    Deltas d = {0, 0, 0, 0};
#pragma unroll
    for (int k = 0; k < OPL; ++k) {
        const int o = lane + GW * k;
        if (o < n && o != u.R1 && o != u.R2) {
            const int o1 = G[u.R1 * ld + o];
            acc<GEN>(d, o1, o1 + u.A1 * W[u.X1 * n + o] + u.B1 * W[u.Y1 * n + o]);
            if (u.R2 >= 0) {
                const int o2 = G[u.R2 * ld + o];
                acc<GEN>(d, o2, o2 + u.A2 * W[u.X2 * n + o] + u.B2 * W[u.Y2 * n + o]);
            }
        }
    }
    if (u.pair && lane == 0) {
        const int op = G[u.R1 * ld + u.R2];
        acc<GEN>(d, op, pair_new(u, op, W, n, u.X1, u.X2));
    }
    return d;
}

// commit_sign_flip / commit_support_switch / commit_double_sign_flip
// (xweigh_cuda.cu:607-877) and the within-row swap, in the two-row form.
template <int OPL, int MW, typename GT, bool GEN, int GW = 32>
__device__ void commit(uint32_t d0, uint32_t d1, const Update& u, int ds, int8_t* W, GT* G, int32_t* res,
                       uint8_t* mino, uint64_t* mask, int n, int ld, int m, int sparse, int lane) {
    const unsigned gm = group_mask<GW>();
    int s1 = 0;
#pragma unroll
    for (int k = 0; k < OPL; ++k) {
        const int o = lane + GW * k;
        if (o < n && o != u.R1 && o != u.R2) {
            const int o1 = G[u.R1 * ld + o];
            const int n1 = o1 + u.A1 * W[u.X1 * n + o] + u.B1 * W[u.Y1 * n + o];
            const int e1 = iabs(n1) - iabs(o1);
            G[u.R1 * ld + o] = (GT)n1;
            G[o * ld + u.R1] = (GT)n1;
            int e = e1;
            if (u.R2 >= 0) {
                const int o2 = G[u.R2 * ld + o];
                const int n2 = o2 + u.A2 * W[u.X2 * n + o] + u.B2 * W[u.Y2 * n + o];
                G[u.R2 * ld + o] = (GT)n2;
                G[o * ld + u.R2] = (GT)n2;
                e += iabs(n2) - iabs(o2);
            }
            res[o] += e;
            s1 += e1;
        }
    }
    const int S1 = __reduce_add_sync(gm, s1);
    __syncwarp(gm);
    if (lane == 0) {
        const int kind = (d0 >> 1) & 3, r1 = (d0 >> 3) & 255, r2 = (d0 >> 11) & 255;
        const int c1 = (d0 >> 19) & 255, c2 = d1 & 255;
        const int nv1 = (int)((d1 >> 8) & 3) - 1, nv2 = (int)((d1 >> 10) & 3) - 1;
        const int p1 = (d1 >> 12) & 255, p2 = (d1 >> 20) & 255;
        if (u.pair) {
            const int op = G[r1 * ld + r2];
            const int np = pair_new(u, op, W, n, c1, c2);
            const int pd = iabs(np) - iabs(op);
            G[r1 * ld + r2] = (GT)np;
            G[r2 * ld + r1] = (GT)np;
            res[r1] += S1 + pd;
            res[r2] += ds - S1;
        } else if (u.R2 >= 0) {
            res[r1] += S1;
            res[r2] += ds - S1;
        } else {
            res[r1] += ds;
        }
        if (kind == 0) {
            W[c1 * n + r1] = (int8_t)-W[c1 * n + r1];
        } else if (kind == 2) {
            W[c1 * n + r1] = (int8_t)-W[c1 * n + r1];
            W[c2 * n + r2] = (int8_t)-W[c2 * n + r2];
        } else if (kind == 1) {
            W[c1 * n + r1] = 0;
            W[c2 * n + r2] = 0;
            W[c2 * n + r1] = (int8_t)nv1;
            W[c1 * n + r2] = (int8_t)nv2;
            mino[r1 * m + p1] = (uint8_t)(sparse ? c2 : c1);
            mino[r2 * m + p2] = (uint8_t)(sparse ? c1 : c2);
            mask[MW * r1 + (c1 >> 6)] &= ~(1ull << (c1 & 63));
            mask[MW * r1 + (c2 >> 6)] |= 1ull << (c2 & 63);
            mask[MW * r2 + (c2 >> 6)] &= ~(1ull << (c2 & 63));
            mask[MW * r2 + (c1 >> 6)] |= 1ull << (c1 & 63);
        } else if (GEN) {
            W[c1 * n + r1] = 0;
            W[c2 * n + r1] = (int8_t)nv1;
            mino[r1 * m + p1] = (uint8_t)(sparse ? c2 : c1);
            mask[MW * r1 + (c1 >> 6)] &= ~(1ull << (c1 & 63));
            mask[MW * r1 + (c2 >> 6)] |= 1ull << (c2 & 63);
        }
    }
    __syncwarp(gm);
}

// tab[d-1] = ceil(exp(-d/T) * 2^32), computed with the same division and
// exponential as metropolis_accept, so that for a 32-bit draw u
//   u * 2^-32 < exp(-d/T)  <=>  u < tab[d-1]
// exactly (both sides scaled by 2^32 without rounding; u is an integer).
// Rebuilt whenever the replica's temperature changes.
template <int GW = 32>
__device__ __noinline__ void build_thresholds(uint64_t* tab, double T, int lane) {
    const double t = T > 1.0e-12 ? T : 1.0e-12;
    for (uint32_t d = lane + 1; d <= kThrTable; d += GW) {
        const double e = acceptance_exp(__ddiv_rn(-(double)d, t));
        tab[d - 1] = (uint64_t)ceil(__dmul_rn(e, 0x1p32));
    }
    __syncwarp(group_mask<GW>());
}

template <int GW = 32>
__device__ __forceinline__ void copy16(void* dst, const void* src, uint32_t bytes, int lane) {
    const uint32_t chunks = xw_pad16(bytes) / 16u;
    uint4* d = reinterpret_cast<uint4*>(dst);
    const uint4* s = reinterpret_cast<const uint4*>(src);
    for (uint32_t i = lane; i < chunks; i += GW) d[i] = s[i];
}

__device__ __forceinline__ uint64_t globaltimer() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Phase C: the hot-row tournaments of candidates 0..3 (hot_row,
// xweigh_cuda.cu:291-300), 8 lanes (samples) per candidate with a segmented
// maximum: one pass of a warp, two of a half-warp.  Returns the row of the
// lane's candidate for lanes 0..3.
template <int GW>
__device__ __forceinline__ int coop_hot_row(const uint32_t* sDw, const int32_t* sRes, int bpc, int count, int ts,
                                            bool coop, int n, uint64_t it, uint32_t stream, uint32_t k0,
                                            uint32_t k1, int lane) {
    const unsigned gm = group_mask<GW>();
    if constexpr (GW == 32) {
        int hot_key = 0;
        if (coop) {
            const int c = lane >> 3, s = lane & 7;
            if (c < count && s < ts) {
                const uint32_t wd = sDw[(1 + c * bpc + 4 + (s >> 2)) * 4 + (s & 3)];
                const uint32_t row =
                    draw_index(wd, (uint32_t)n, cand_slot(c, 4 + (s >> 2)), it, stream, k0, k1, s & 3);
                hot_key = (sRes[row] << 13) | ((31 - s) << 8) | (int)row;
            }
            hot_key = max(hot_key, __shfl_xor_sync(FULL, hot_key, 1));
            hot_key = max(hot_key, __shfl_xor_sync(FULL, hot_key, 2));
            hot_key = max(hot_key, __shfl_xor_sync(FULL, hot_key, 4));
        }
        return __shfl_sync(FULL, hot_key, (lane & 3) << 3) & 0xff;
    } else {
        int keys[2] = {0, 0};
        if (coop) {
#pragma unroll
            for (int pass = 0; pass < 2; ++pass) {
                const int c = 2 * pass + (lane >> 3), s = lane & 7;
                int hot_key = 0;
                if (c < count && s < ts) {
                    const uint32_t wd = sDw[(1 + c * bpc + 4 + (s >> 2)) * 4 + (s & 3)];
                    const uint32_t row =
                        draw_index(wd, (uint32_t)n, cand_slot(c, 4 + (s >> 2)), it, stream, k0, k1, s & 3);
                    hot_key = (sRes[row] << 13) | ((31 - s) << 8) | (int)row;
                }
                hot_key = max(hot_key, __shfl_xor_sync(gm, hot_key, 1, 16));
                hot_key = max(hot_key, __shfl_xor_sync(gm, hot_key, 2, 16));
                hot_key = max(hot_key, __shfl_xor_sync(gm, hot_key, 4, 16));
                keys[pass] = hot_key;
            }
        }
        // candidate c's winner sits in pass c/2 at lane (c%2)*8
        const int k0v = __shfl_sync(gm, keys[0], (lane & 1) << 3, 16);
        const int k1v = __shfl_sync(gm, keys[1], (lane & 1) << 3, 16);
        return ((lane >> 1) & 1 ? k1v : k0v) & 0xff;
    }
}

// A loaded replica: its shared-memory structures, the job's constants the
// iteration reads, and the scalar state the loop carries.
template <int OPL, int GW>
struct Replica {
    static constexpr int MW = OPL > 4 ? 4 : 2;
    using GT = typename std::conditional<(OPL > 4), int16_t, int32_t>::type;
    uint8_t* rec;
    RepHeader* H;
    XwJob* J;
    int8_t* sW;
    GT* sG;
    int32_t* sRes;
    uint8_t* sMino;
    uint64_t* sMask;
    uint64_t* sThr;
    int n, w, m, sparse, ld, obj_kind;
    uint32_t nn, status0;
    // scalar state
    uint64_t it, iters, moves, cand_evals;
    uint32_t accepted, accepted_rows, two_row_evals;
    int score, conflicts, best_s, best_c, msi, cool;
    int64_t obj_total;
    double T, reheat_T;
    // the copy that writes the record (a cluster's other CTAs keep an
    // identical copy in their own shared memory and write nothing)
    bool owner;
};

// Loads replica `rid` into the slot: W and the minority lists, the masks,
// Gram and residuals rebuilt from W and checked against the header.  False
// when the replica does not run (job done or solved, budget spent, or a
// failed self-check, which flags the header).  The group's lanes call it.
// `owner` false: a copy that writes nothing to the record; it also skips
// the exits on the job's done and solved flags, which other kernels may set
// while it loads (its owner decides whether the replica runs).
template <int OPL, bool GEN, int GW>
__device__ __forceinline__ bool load_replica(const AnnealArgs& a, uint32_t rid, uint8_t* slot, int lane,
                                             uint64_t chunk_iters, Replica<OPL, GW>& R, bool owner = true) {
    constexpr int MW = Replica<OPL, GW>::MW;
    using GT = typename Replica<OPL, GW>::GT;
    const unsigned gm = group_mask<GW>();
    uint8_t* rec = a.arena + a.rec_off[rid];
    RepHeader* H = reinterpret_cast<RepHeader*>(rec);
    const uint32_t jid = H->job;
    XwJob* J = a.jobs + jid;
    R.owner = owner;
    if (owner && *(volatile int32_t*)&J->done) return false;
    if (owner && a.stop_on_solve == 1 && *(volatile int32_t*)&J->solved) return false;

    // eight rows per lane: int16 Gram and 256-bit row masks (slot_layout)
    const int n = J->n, w = J->w, m = J->m, sparse = J->sparse;
    const SlotLayout L = slot_layout(n, m, OPL > 4);
    const int ld = L.ld;
    int8_t* sW = reinterpret_cast<int8_t*>(slot);
    GT* sG = reinterpret_cast<GT*>(slot + L.off_g);
    int32_t* sRes = reinterpret_cast<int32_t*>(slot + L.off_res);
    uint8_t* sMino = slot + L.off_mino;
    uint64_t* sMask = reinterpret_cast<uint64_t*>(slot + L.off_mask);

    uint64_t it = H->it;
    uint64_t iters = chunk_iters;
    if (J->budget_iters) {
        if (it >= J->budget_iters) return false;
        if (iters > J->budget_iters - it) iters = J->budget_iters - it;
    }

    // ---- load W and the minority lists; rebuild masks, Gram, residuals ----
    const uint32_t nn = (uint32_t)(n * n);
    copy16<GW>(sW, rec + J->off_w, nn, lane);
    const uint32_t status0 = H->status;
    if (m > 0 && (status0 & XW_STATUS_INIT)) copy16<GW>(sMino, rec + J->off_mino, (uint32_t)(n * m), lane);
    __syncwarp(gm);
    int bad_rows = 0;
#pragma unroll
    for (int k = 0; k < OPL; ++k) {
        const int o = lane + GW * k;
        if (o < n) {
            int pos = 0, weight = 0;
#pragma unroll
            for (int q = 0; q < MW; ++q) {
                uint64_t word = 0;
#pragma unroll 1
                for (int c = 64 * q; c < n && c < 64 * q + 64; ++c) {
                    const bool nz = sW[c * n + o] != 0;
                    if (nz) word |= 1ull << (c & 63);
                    if (m > 0 && !(status0 & XW_STATUS_INIT) && nz == (sparse != 0)) {
                        if (pos < m) sMino[o * m + pos] = (uint8_t)c;
                        ++pos;
                    }
                }
                sMask[MW * o + q] = word;
                weight += __popcll(word);
            }
            if (weight != w) bad_rows = 1;
            if (m > 0 && !(status0 & XW_STATUS_INIT) && pos != m) bad_rows = 1;
        }
    }
    if (__any_sync(gm, bad_rows)) {
        if (lane == 0) H->err |= XW_ERR_MINORITY;
        return false;
    }
    __syncwarp(gm);
    int p_score = 0, p_conf = 0, p_par = 0;
    long long p_sq = 0;
#pragma unroll
    for (int k = 0; k < OPL; ++k) {
        const int o = lane + GW * k;
        if (o < n) {
            int r_sum = 0;
#pragma unroll 1
            for (int r = 0; r < n; ++r) {
                int dot = 0;
#pragma unroll 1
                for (int c = 0; c < n; ++c) dot += sW[c * n + r] * sW[c * n + o];
                sG[r * ld + o] = (GT)dot;
                if (r != o) {
                    const int ad = iabs(dot);
                    r_sum += ad;
                    p_conf += dot != 0;
                    p_sq += (long long)(dot * dot);
                    p_par += ad & 1;
                }
            }
            sRes[o] = r_sum;
            p_score += r_sum;
        }
    }
    const int score0 = __reduce_add_sync(gm, p_score) / 2;
    const int conf0 = __reduce_add_sync(gm, p_conf) / 2;
#pragma unroll
    for (int off = GW / 2; off > 0; off >>= 1) p_sq += __shfl_xor_sync(gm, p_sq, off, GW);
    const long long sq0 = p_sq / 2;
    const int par0 = __reduce_add_sync(gm, p_par) / 2;
    __syncwarp(gm);

    const int obj_kind = GEN ? H->obj_kind : 0;
    if (!GEN && (H->obj_kind != 0 || J->move_set != 0)) {
        // the lean kernel was launched for a replica that needs the general one
        if (lane == 0) H->err |= XW_ERR_KERNEL;
        return false;
    }
    const int64_t obj0 = obj_kind == 1 ? sq0 : obj_kind == 2 ? par0 : score0;
    R.T = H->temperature;
    R.reheat_T = H->reheat_temperature;
    if (status0 & XW_STATUS_INIT) {
        if (H->score != score0 || H->conflicts != conf0 || H->obj_total != obj0) {
            if (lane == 0) H->err |= XW_ERR_SCORE;
            return false;
        }
        R.best_s = H->best_score;
        R.best_c = H->best_conflicts;
        R.msi = H->msi;
        R.cool = H->cool_ctr;
        R.moves = H->moves;
        R.cand_evals = H->cand_evals;
        R.accepted = H->accepted;
        R.accepted_rows = H->accepted_rows;
        R.two_row_evals = H->two_row_evals;
    } else {
        R.best_s = score0;
        R.best_c = conf0;
        R.msi = 0;
        R.cool = 0;
        R.moves = 0;
        R.cand_evals = 0;
        R.accepted = 0;
        R.accepted_rows = 0;
        R.two_row_evals = 0;
        if (owner) copy16<GW>(rec + J->off_best, sW, nn, lane);
    }
    R.score = score0;
    R.conflicts = conf0;
    R.obj_total = obj0;
    R.rec = rec;
    R.H = H;
    R.J = J;
    R.sW = sW;
    R.sG = sG;
    R.sRes = sRes;
    R.sMino = sMino;
    R.sMask = sMask;
    R.sThr = reinterpret_cast<uint64_t*>(slot + L.off_thr);
    R.n = n;
    R.w = w;
    R.m = m;
    R.sparse = sparse;
    R.ld = ld;
    R.obj_kind = obj_kind;
    R.nn = nn;
    R.status0 = status0;
    R.it = it;
    R.iters = iters;
    return true;
}

// Writes the replica's W, minority lists and scalar state back to its record.
template <int OPL, int GW>
__device__ __forceinline__ void store_replica(const Replica<OPL, GW>& R, int lane) {
    const unsigned gm = group_mask<GW>();
    __syncwarp(gm);
    copy16<GW>(R.rec + R.J->off_w, R.sW, R.nn, lane);
    if (R.m > 0) copy16<GW>(R.rec + R.J->off_mino, R.sMino, (uint32_t)(R.n * R.m), lane);
    if (lane == 0) {
        RepHeader* H = R.H;
        H->it = R.it;
        H->moves = R.moves;
        H->cand_evals = R.cand_evals;
        H->accepted = R.accepted;
        H->accepted_rows = R.accepted_rows;
        H->two_row_evals = R.two_row_evals;
        H->score = R.score;
        H->conflicts = R.conflicts;
        H->best_score = R.best_s;
        H->best_conflicts = R.best_c;
        H->obj_total = R.obj_total;
        H->temperature = R.T;
        H->msi = R.msi;
        H->cool_ctr = R.cool;
        H->status = R.status0 | XW_STATUS_INIT | (R.best_s == 0 ? XW_STATUS_SOLVED : 0u);
    }
    __syncwarp(gm);
}

// The proposing side of an iteration: the job constants the draws and
// proposals read, this group's draw buffer and View, and the lane's
// cached-block slots and register context.
template <int GW>
struct Proposer {
    uint4* sDraw;
    const uint32_t* sDw;
    View* sView;
    Reg rg;
    uint32_t my_slot, my_slot2;
    uint32_t k0, k1, stream;
    uint64_t thr_greedy;
    int cs, ts, bpc;
    bool coop;
};

// Sets up the proposer of a loaded replica with the draw buffer and View at
// `draws` and `view` (the group's own).  The group's lanes call it.
template <int OPL, int GW>
__device__ __forceinline__ void setup_proposer(const Replica<OPL, GW>& R, uint4* draws, View* view, int lane,
                                               Proposer<GW>& P) {
    const XwJob* J = R.J;
    const int n = R.n;
    P.sDraw = draws;
    P.sDw = reinterpret_cast<const uint32_t*>(draws);
    P.sView = view;
    P.cs = J->candidate_samples;
    P.ts = J->target_samples;
    P.k0 = J->key0;
    P.k1 = J->key1;
    P.stream = R.H->stream;
    P.thr_greedy = J->thr_greedy;
    P.bpc = 4 + (P.ts <= 4 ? 1 : 2);          // cached blocks per candidate
    P.coop = P.ts <= 8;                       // cooperative hot-row tournament
    if (lane == 0) {
        View v;
        v.W = R.sW; v.mino = R.sMino; v.res = R.sRes; v.mask = R.sMask; v.dw = P.sDw;
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const int lo = 64 * q;
            v.valid[q] = n >= lo + 64 ? ~0ull : n <= lo ? 0ull : ((1ull << (n - lo)) - 1ull);
        }
        v.thr_target = J->thr_target; v.thr_dbl = J->thr_double; v.thr_sign = J->thr_sign;
        v.thr_swsign = J->thr_swsign;
        v.n = n; v.w = R.w; v.m = R.m; v.sparse = R.sparse; v.ts = P.ts; v.bpc = P.bpc; v.cc = 31 / P.bpc;
        v.move_set = J->move_set;
        v.stream = P.stream; v.k0 = P.k0; v.k1 = P.k1; v.pad = 0;
        *view = v;
    }
    __syncwarp(group_mask<GW>());

    // lane -> cached Philox blocks of an iteration (block 0 is the
    // move-level block, 1 + c*bpc + b block b of candidate c); a half-warp
    // group computes two blocks per lane
    const int bpc = P.bpc;
    P.my_slot = 0;
    P.my_slot2 = 0;
    if (lane > 0) {
        const int q = lane - 1, c = q / bpc, b = q - c * bpc;
        P.my_slot = cand_slot(c, b);
    }
    if constexpr (GW == 16) {
        const int q = lane + 15, c = q / bpc, b = q - c * bpc;
        P.my_slot2 = cand_slot(c, b);
    }
    // register context of candidate `lane` for the inlined proposal path
    Reg& rg = P.rg;
    rg.W = R.sW; rg.mino = R.sMino; rg.mask = R.sMask;
    rg.cw = P.sDw + (1 + lane * bpc) * 4;
    rg.cached = lane < 31 / bpc;
    rg.thr_target = J->thr_target; rg.thr_dbl = J->thr_double; rg.thr_sign = J->thr_sign;
    rg.thr_swsign = J->thr_swsign;
    rg.n = n; rg.w = R.w; rg.m = R.m; rg.sparse = R.sparse; rg.move_set = J->move_set;
    rg.stream = P.stream; rg.k0 = P.k0; rg.k1 = P.k1;
}

// The move an iteration puts to the Metropolis test: the first best of its
// candidates (b0 = 0: none was valid), its deltas, the iteration's
// acceptance draw and the number of candidates evaluated.
struct Choice {
    uint32_t b0, b1;
    int bds, bdc, bprim;
    uint32_t u;
    uint32_t evals, evals2;   // candidates evaluated; those changing two rows
};

// Phases A-E of iteration `it` against the replica's current state: draws,
// hot-row tournaments, proposals, and the evaluation of the candidates in
// order.  Reads the state and writes only the group's draw buffer.
template <int OPL, bool GEN, int GW>
__device__ __forceinline__ Choice choose_move(const Replica<OPL, GW>& R, Proposer<GW>& P, uint64_t it, int lane) {
    constexpr int MW = Replica<OPL, GW>::MW;
    using GT = typename Replica<OPL, GW>::GT;
    const unsigned gm = group_mask<GW>();
    const int n = R.n, ts = P.ts, bpc = P.bpc;
    const uint32_t k0 = P.k0, k1 = P.k1, stream = P.stream;
    const uint32_t* sDw = P.sDw;
    const int32_t* sRes = R.sRes;
    // A: draws
    P.sDraw[lane] = draw_block(P.my_slot, it, stream, k0, k1);
    if constexpr (GW == 16) P.sDraw[lane + 16] = draw_block(P.my_slot2, it, stream, k0, k1);
    __syncwarp(gm);
    const uint4 mblk = P.sDraw[0];
    const int count = (uint64_t)mblk.x < P.thr_greedy ? P.cs : 1;

    // C: cooperative hot-row tournaments
    const int coop_row = coop_hot_row<GW>(sDw, sRes, bpc, count, ts, P.coop, n, it, stream, k0, k1, lane);

    // D: proposals, lane c proposes candidate c
    uint2 desc = make_uint2(0u, 0u);
    P.rg.it = it;
    if (lane < count) desc = d_propose<MW, GEN>(P.rg, P.sView, lane, P.coop && lane < 4, coop_row);
    __syncwarp(gm);

    // E: evaluate in candidate order, keep the first best
    Choice ch;
    ch.b0 = 0; ch.b1 = 0; ch.bds = 0; ch.bdc = 0; ch.bprim = 0;
    ch.u = mblk.y;
    ch.evals = 0;
    ch.evals2 = 0;
#pragma unroll 1
    for (int c = 0; c < count; ++c) {
        const uint32_t e0 = __shfl_sync(gm, desc.x, c, GW);
        const uint32_t e1 = __shfl_sync(gm, desc.y, c, GW);
        if (!(e0 & 1u)) continue;
        const Update u = decode(e0, e1, R.sW, n);
        const Deltas d = eval_lane<OPL, GT, GEN, GW>(u, R.sW, R.sG, n, R.ld, lane);
        const int packed = __reduce_add_sync(gm, d.ds * 4096 + d.dc);
        const int dc = ((packed + 2048) & 4095) - 2048;
        const int ds = (packed - dc) >> 12;
        int prim = ds;
        if (GEN) {
            if (R.obj_kind == 1) prim = __reduce_add_sync(gm, d.dsq);
            else if (R.obj_kind == 2) prim = __reduce_add_sync(gm, d.dpar);
        }
        ++ch.evals;
        if constexpr (kMoveStats) ch.evals2 += u.R2 >= 0;
        bool better = ch.b0 == 0;
        if (!better) {
            if (prim != ch.bprim) better = prim < ch.bprim;
            else if (ds != ch.bds) better = ds < ch.bds;
            else better = dc < ch.bdc;
        }
        if (better) {
            ch.b0 = e0; ch.b1 = e1; ch.bds = ds; ch.bdc = dc; ch.bprim = prim;
        }
    }
    return ch;
}

// Phases F-H of an iteration whose choice is valid: Metropolis on the
// replica's objective, the commit of an accepted move, best tracking
// (the best W copied to the record on improvement, the job's solve flag),
// cooling and reheat.  Returns whether the move was accepted.  The group's
// lanes call it.
template <int OPL, bool GEN, int GW>
__device__ __forceinline__ bool apply_move(Replica<OPL, GW>& R, const Choice& ch, int tempering, int mpc, int stuck,
                                           double t_min, double cooling, double reheat, int lane) {
    constexpr int MW = Replica<OPL, GW>::MW;
    using GT = typename Replica<OPL, GW>::GT;
    ++R.moves;
    // F: Metropolis
    bool accept = ch.bprim <= 0;
    if (!accept)
        accept = ch.bprim <= (int64_t)kThrTable ? (uint64_t)ch.u < R.sThr[ch.bprim - 1]
                                                : metropolis_accept(ch.bprim, R.T, ch.u);

    // G: commit
    if (accept) {
        const Update u = decode(ch.b0, ch.b1, R.sW, R.n);
        commit<OPL, MW, GT, GEN, GW>(ch.b0, ch.b1, u, ch.bds, R.sW, R.sG, R.sRes, R.sMino, R.sMask, R.n, R.ld,
                                     R.m, R.sparse, lane);
        R.score += ch.bds;
        R.conflicts += ch.bdc;
        R.obj_total += ch.bprim;
        if constexpr (kMoveStats) {
            ++R.accepted;
            R.accepted_rows += u.R2 >= 0 ? 2u : 1u;
        }
    }

    // H: best tracking, cooling, reheat
    if (R.score < R.best_s || (R.score == R.best_s && R.conflicts < R.best_c)) {
        R.best_s = R.score;
        R.best_c = R.conflicts;
        R.msi = 0;
        if (R.owner) copy16<GW>(R.rec + R.J->off_best, R.sW, R.nn, lane);
        if (R.best_s == 0 && lane == 0 && R.owner) {
            RepHeader* H = R.H;
            XwJob* J = R.J;
            H->solve_it = R.it;
            H->solve_ns = globaltimer();
            if (atomicCAS(&J->solved, 0, 1) == 0) {
                J->solved_replica = (int32_t)H->stream;
                J->solved_it = R.it;
                J->solve_ns = H->solve_ns;
            }
        }
    } else {
        ++R.msi;
    }
    if (!tempering) {
        const double T0 = R.T;
        if (++R.cool >= mpc) {
            R.cool = 0;
            R.T = __dmul_rn(R.T, cooling);
            if (R.T < t_min) R.T = t_min;
        }
        if (R.msi >= stuck) {
            R.msi = 0;
            R.T = __dmul_rn(R.reheat_T, reheat);
            if (R.T < t_min) R.T = t_min;
        }
        if (R.T != T0) build_thresholds<GW>(R.sThr, R.T, lane);
    }
    return accept;
}

// The one-warp (or half-warp) replica loop.  Its phases A-H are those of
// choose_move and apply_move above, written out in one body: as separate
// functions, even inlined, they hold more values live across the loop and
// spill more under the lean kernel's 96-register budget (measured 6%
// slower on W(26,25) populations).
// ONEZ: every row has one zero (w = n - 1: minority lists of one entry,
// the dense side), so the minority size and side are constants; NFIX > 0:
// the order is NFIX as well.  A replica of another shape is flagged
// (XW_ERR_KERNEL) and not annealed.
template <int OPL, bool GEN, int GW = 32, bool ONEZ = false, int NFIX = 0>
__device__ void run_replica(const AnnealArgs& a, uint32_t rid, uint8_t* slot, int lane, uint64_t chunk_iters) {
    const unsigned gm = group_mask<GW>();
    uint8_t* rec = a.arena + a.rec_off[rid];
    RepHeader* H = reinterpret_cast<RepHeader*>(rec);
    const uint32_t jid = H->job;
    XwJob* J = a.jobs + jid;
    if (*(volatile int32_t*)&J->done) return;
    if (a.stop_on_solve == 1 && *(volatile int32_t*)&J->solved) return;
    if ((ONEZ && (J->m != 1 || J->sparse != 0)) || (NFIX && J->n != NFIX)) {
        if (lane == 0) H->err |= XW_ERR_KERNEL;
        return;
    }

    // eight rows per lane: int16 Gram and 256-bit row masks (slot_layout)
    constexpr int MW = OPL > 4 ? 4 : 2;
    using GT = typename std::conditional<(OPL > 4), int16_t, int32_t>::type;
    // one zero per row: m = n - w = 1, so w = n - 1
    const int n = NFIX ? NFIX : J->n, w = ONEZ ? n - 1 : J->w, m = ONEZ ? 1 : J->m, sparse = ONEZ ? 0 : J->sparse;
    const SlotLayout L = slot_layout(n, m, OPL > 4);
    const int ld = L.ld;
    int8_t* sW = reinterpret_cast<int8_t*>(slot);
    GT* sG = reinterpret_cast<GT*>(slot + L.off_g);
    int32_t* sRes = reinterpret_cast<int32_t*>(slot + L.off_res);
    uint8_t* sMino = slot + L.off_mino;
    uint64_t* sMask = reinterpret_cast<uint64_t*>(slot + L.off_mask);
    uint4* sDraw = reinterpret_cast<uint4*>(slot + L.off_draws);
    const uint32_t* sDw = reinterpret_cast<const uint32_t*>(sDraw);
    View* sView = reinterpret_cast<View*>(slot + L.off_view);
    uint64_t* sThr = reinterpret_cast<uint64_t*>(slot + L.off_thr);

    uint64_t it = H->it;
    uint64_t iters = chunk_iters;
    if (J->budget_iters) {
        if (it >= J->budget_iters) return;
        if (iters > J->budget_iters - it) iters = J->budget_iters - it;
    }

    // ---- load W and the minority lists; rebuild masks, Gram, residuals ----
    const uint32_t nn = (uint32_t)(n * n);
    copy16<GW>(sW, rec + J->off_w, nn, lane);
    const uint32_t status0 = H->status;
    if (m > 0 && (status0 & XW_STATUS_INIT)) copy16<GW>(sMino, rec + J->off_mino, (uint32_t)(n * m), lane);
    __syncwarp(gm);
    int bad_rows = 0;
#pragma unroll
    for (int k = 0; k < OPL; ++k) {
        const int o = lane + GW * k;
        if (o < n) {
            int pos = 0, weight = 0;
#pragma unroll
            for (int q = 0; q < MW; ++q) {
                uint64_t word = 0;
#pragma unroll 1
                for (int c = 64 * q; c < n && c < 64 * q + 64; ++c) {
                    const bool nz = sW[c * n + o] != 0;
                    if (nz) word |= 1ull << (c & 63);
                    if (m > 0 && !(status0 & XW_STATUS_INIT) && nz == (sparse != 0)) {
                        if (pos < m) sMino[o * m + pos] = (uint8_t)c;
                        ++pos;
                    }
                }
                sMask[MW * o + q] = word;
                weight += __popcll(word);
            }
            if (weight != w) bad_rows = 1;
            if (m > 0 && !(status0 & XW_STATUS_INIT) && pos != m) bad_rows = 1;
        }
    }
    if (__any_sync(gm, bad_rows)) {
        if (lane == 0) H->err |= XW_ERR_MINORITY;
        return;
    }
    __syncwarp(gm);
    int p_score = 0, p_conf = 0, p_par = 0;
    long long p_sq = 0;
#pragma unroll
    for (int k = 0; k < OPL; ++k) {
        const int o = lane + GW * k;
        if (o < n) {
            int r_sum = 0;
#pragma unroll 1
            for (int r = 0; r < n; ++r) {
                int dot = 0;
#pragma unroll 1
                for (int c = 0; c < n; ++c) dot += sW[c * n + r] * sW[c * n + o];
                sG[r * ld + o] = (GT)dot;
                if (r != o) {
                    const int ad = iabs(dot);
                    r_sum += ad;
                    p_conf += dot != 0;
                    p_sq += (long long)(dot * dot);
                    p_par += ad & 1;
                }
            }
            sRes[o] = r_sum;
            p_score += r_sum;
        }
    }
    const int score0 = __reduce_add_sync(gm, p_score) / 2;
    const int conf0 = __reduce_add_sync(gm, p_conf) / 2;
#pragma unroll
    for (int off = GW / 2; off > 0; off >>= 1) p_sq += __shfl_xor_sync(gm, p_sq, off, GW);
    const long long sq0 = p_sq / 2;
    const int par0 = __reduce_add_sync(gm, p_par) / 2;
    __syncwarp(gm);

    const int obj_kind = GEN ? H->obj_kind : 0;
    if (!GEN && (H->obj_kind != 0 || J->move_set != 0)) {
        // the lean kernel was launched for a replica that needs the general one
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
    } else {
        best_s = score0;
        best_c = conf0;
        msi = 0;
        cool = 0;
        moves = 0;
        cand_evals = 0;
        accepted = accepted_rows = two_row_evals = 0;
        copy16<GW>(rec + J->off_best, sW, nn, lane);
    }
    score = score0;
    conflicts = conf0;
    obj_total = obj0;

    // ---- job constants ----
    const int tempering = J->tempering;
    const int cs = J->candidate_samples, ts = J->target_samples;
    const int mpc = J->moves_per_cool, stuck = J->stuck_threshold;
    const uint32_t k0 = J->key0, k1 = J->key1, stream = H->stream;
    const uint64_t thr_greedy = J->thr_greedy;
    const double t_min = J->t_min, cooling = J->cooling, reheat = J->reheat;
    const int bpc = 4 + (ts <= 4 ? 1 : 2);          // cached blocks per candidate
    const bool coop = ts <= 8;                      // cooperative hot-row tournament
    if (lane == 0) {
        View v;
        v.W = sW; v.mino = sMino; v.res = sRes; v.mask = sMask; v.dw = sDw;
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const int lo = 64 * q;
            v.valid[q] = n >= lo + 64 ? ~0ull : n <= lo ? 0ull : ((1ull << (n - lo)) - 1ull);
        }
        v.thr_target = J->thr_target; v.thr_dbl = J->thr_double; v.thr_sign = J->thr_sign;
        v.thr_swsign = J->thr_swsign;
        v.n = n; v.w = w; v.m = m; v.sparse = sparse; v.ts = ts; v.bpc = bpc; v.cc = 31 / bpc;
        v.move_set = J->move_set;
        v.stream = stream; v.k0 = k0; v.k1 = k1; v.pad = 0;
        *sView = v;
    }
    __syncwarp(gm);

    build_thresholds<GW>(sThr, T, lane);

    // lane -> cached Philox blocks of this iteration (block 0 is the
    // move-level block, 1 + c*bpc + b block b of candidate c); a half-warp
    // group computes two blocks per lane
    uint32_t my_slot = 0, my_slot2 = 0;
    if (lane > 0) {
        const int q = lane - 1, c = q / bpc, b = q - c * bpc;
        my_slot = cand_slot(c, b);
    }
    if constexpr (GW == 16) {
        const int q = lane + 15, c = q / bpc, b = q - c * bpc;
        my_slot2 = cand_slot(c, b);
    }
    // register context of candidate `lane` for the inlined proposal path
    Reg rg;
    rg.W = sW; rg.mino = sMino; rg.mask = sMask;
    rg.cw = sDw + (1 + lane * bpc) * 4;
    rg.cached = lane < 31 / bpc;
    rg.thr_target = J->thr_target; rg.thr_dbl = J->thr_double; rg.thr_sign = J->thr_sign;
    rg.thr_swsign = J->thr_swsign;
    rg.n = n; rg.w = w; rg.m = m; rg.sparse = sparse; rg.move_set = J->move_set;
    rg.stream = stream; rg.k0 = k0; rg.k1 = k1;

    uint64_t done = 0;
#pragma unroll 1
    for (; done < iters; ++done) {
        // 1: every replica of the job stops soon after any solve;
        // 2: a replica stops at its own solve only, so that each replica's
        //    trajectory is independent of how the launches are scheduled
        if (a.stop_on_solve) {
            if (best_s == 0) break;
            if (a.stop_on_solve == 1 && (done & 63) == 63 && *(volatile int32_t*)&J->solved) break;
        }
        // A: draws
        sDraw[lane] = draw_block(my_slot, it, stream, k0, k1);
        if constexpr (GW == 16) sDraw[lane + 16] = draw_block(my_slot2, it, stream, k0, k1);
        __syncwarp(gm);
        const uint4 mblk = sDraw[0];
        const int count = (uint64_t)mblk.x < thr_greedy ? cs : 1;

        // C: cooperative hot-row tournaments for candidates 0..3, 8 lanes
        // (samples) per candidate: one pass of the warp, two of a half-warp
        const int coop_row = coop_hot_row<GW>(sDw, sRes, bpc, count, ts, coop, n, it, stream, k0, k1, lane);

        // D: proposals, lane c proposes candidate c
        uint2 desc = make_uint2(0u, 0u);
        rg.it = it;
        if (lane < count) desc = d_propose<MW, GEN>(rg, sView, lane, coop && lane < 4, coop_row);
        __syncwarp(gm);

        // E: evaluate in candidate order, keep the first best
        bool have = false;
        uint32_t b0 = 0, b1 = 0;
        int bds = 0, bdc = 0, bprim = 0;
#pragma unroll 1
        for (int c = 0; c < count; ++c) {
            const uint32_t e0 = __shfl_sync(gm, desc.x, c, GW);
            const uint32_t e1 = __shfl_sync(gm, desc.y, c, GW);
            if (!(e0 & 1u)) continue;
            const Update u = decode(e0, e1, sW, n);
            const Deltas d = eval_lane<OPL, GT, GEN, GW>(u, sW, sG, n, ld, lane);
            const int packed = __reduce_add_sync(gm, d.ds * 4096 + d.dc);
            const int dc = ((packed + 2048) & 4095) - 2048;
            const int ds = (packed - dc) >> 12;
            int prim = ds;
            if (GEN) {
                if (obj_kind == 1) prim = __reduce_add_sync(gm, d.dsq);
                else if (obj_kind == 2) prim = __reduce_add_sync(gm, d.dpar);
            }
            ++cand_evals;
            if constexpr (kMoveStats) two_row_evals += u.R2 >= 0;
            bool better = !have;
            if (!better) {
                if (prim != bprim) better = prim < bprim;
                else if (ds != bds) better = ds < bds;
                else better = dc < bdc;
            }
            if (better) {
                have = true; b0 = e0; b1 = e1; bds = ds; bdc = dc; bprim = prim;
            }
        }
        if (!have) {
            ++it;
            continue;
        }
        ++moves;

        // F: Metropolis
        bool accept = bprim <= 0;
        if (!accept)
            accept = bprim <= (int64_t)kThrTable ? (uint64_t)mblk.y < sThr[bprim - 1]
                                                 : metropolis_accept(bprim, T, mblk.y);

        // G: commit
        if (accept) {
            const Update u = decode(b0, b1, sW, n);
            commit<OPL, MW, GT, GEN, GW>(b0, b1, u, bds, sW, sG, sRes, sMino, sMask, n, ld, m, sparse, lane);
            score += bds;
            conflicts += bdc;
            obj_total += bprim;
            if constexpr (kMoveStats) {
                ++accepted;
                accepted_rows += u.R2 >= 0 ? 2u : 1u;
            }
        }

        // H: best tracking, cooling, reheat
        if (score < best_s || (score == best_s && conflicts < best_c)) {
            best_s = score;
            best_c = conflicts;
            msi = 0;
            copy16<GW>(rec + J->off_best, sW, nn, lane);
            if (best_s == 0 && lane == 0) {
                H->solve_it = it;
                H->solve_ns = globaltimer();
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
            if (T != T0) build_thresholds<GW>(sThr, T, lane);
        }
        ++it;
    }

    // ---- write back ----
    __syncwarp(gm);
    copy16<GW>(rec + J->off_w, sW, nn, lane);
    if (m > 0) copy16<GW>(rec + J->off_mino, sMino, (uint32_t)(n * m), lane);
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
        H->status = status0 | XW_STATUS_INIT | (best_s == 0 ? XW_STATUS_SOLVED : 0u);
    }
    __syncwarp(gm);
}

// ---------------------------------------------------------------------------
// Latency mode: one replica per CTA of K warps, speculating K iterations at
// a time.  Warp k computes iteration it + k (phases A-E) against the
// replica's current state, each with its own draw buffer: the draws of an
// iteration depend only on its number, and its proposals and deltas only on
// the state, which no iteration changes before one is accepted.  Warp 0
// then takes the iterations in order through phases F-H until the first
// accepted one, commits it, and discards the iterations after it, whose
// proposals read the state it changed; the next round starts after the
// accepted iteration.  The trajectory is the one-warp kernel's, move for
// move; a round advances by the run of rejections up to the next accept
// (about 2-4 iterations at the acceptance rates of cooling runs) in about
// the time of one iteration, so a lone search runs that much faster.

// Per-warp results and the round's control word, after the slot's own
// (warp 0's) structures and the other warps' draw buffers and Views.
struct SpecOut {
    Choice ch;
    int32_t acc;        // the Metropolis outcome at the round's starting temperature
    int32_t pad;
};
struct SpecCtl {
    uint64_t it;        // first iteration of the round
    int32_t count;      // iterations of the round (0: the replica stops)
    int32_t pad;
    double T;           // the temperature at the round's start
};

// Per round buffer (two, used in turn): the outcomes of all the round's
// warps (K per CTA, CL CTAs), and the job's solved flag as the cluster's
// owner read it.
struct SpecLayout {
    SlotLayout L;
    uint32_t off_extra, per_warp, off_out, out_stride, off_flag, off_ctl, bytes;
};

// the latency-mode regions after a slot of `slot_bytes` (the one-warp
// layout of the replica, or the largest of a launch's replicas), for K
// warps per CTA and CL CTAs per replica
__host__ __device__ inline void spec_regions(uint32_t slot_bytes, int K, int CL, SpecLayout& S) {
    S.per_warp = 32u * 16u + xw_pad16((uint32_t)sizeof(View));
    S.off_extra = xw_pad16(slot_bytes);
    S.off_out = S.off_extra + (uint32_t)(K - 1) * S.per_warp;
    S.out_stride = xw_pad16((uint32_t)(K * CL) * (uint32_t)sizeof(SpecOut));
    S.off_flag = S.off_out + 2u * S.out_stride;
    S.off_ctl = xw_pad16(S.off_flag + 2u * 4u);
    S.bytes = S.off_ctl + (uint32_t)sizeof(SpecCtl);
}

__host__ __device__ inline SpecLayout spec_layout(int n, int m, int K, int CL) {
    SpecLayout S;
    S.L = slot_layout(n, m, false);
    spec_regions(S.L.bytes, K, CL, S);
    return S;
}

// The replica loop of a CTA of the latency mode.  With CL > 1 the replica
// runs on a cluster of CL CTAs (on CL SMs): every CTA loads its own copy,
// the cluster's warps speculate CL * K iterations, every warp writes its
// outcome into every CTA's round buffer (distributed shared memory), and
// after a cluster barrier each CTA's warp 0 makes the same walk and the
// same commit on its own copy, so the copies stay identical; only rank 0
// writes the record.  Everything that steers the walk is either the
// CTAs' identical state or read by rank 0 alone and exchanged (whether
// the replica runs at all, and the job's solved flag each round), so the
// CTAs take the same branches and meet at every barrier.
template <bool GEN, int CL>
__device__ void run_replica_spec(const AnnealArgs& a, uint32_t rid, uint8_t* slot, int warp, int K, int lane) {
    namespace cg = cooperative_groups;
    const int rank = CL > 1 ? (int)cg::this_cluster().block_rank() : 0;
    const bool owner = rank == 0;
    SpecCtl* ctl = nullptr;
    Replica<1, 32> R;
    bool ok = false;
    // warp 0 loads the replica; the round size goes to the others through
    // shared memory
    if (warp == 0) ok = load_replica<1, GEN, 32>(a, rid, slot, lane, a.iters, R, owner);
    // every warp reads the order to find the layout
    const XwJob* J = a.jobs + reinterpret_cast<const RepHeader*>(a.arena + a.rec_off[rid])->job;
    const SpecLayout S = spec_layout(J->n, J->m, K, CL);
    ctl = reinterpret_cast<SpecCtl*>(slot + S.off_ctl);
    const int tempering = J->tempering;
    const int mpc = J->moves_per_cool, stuck = J->stuck_threshold;
    const double t_min = J->t_min, cooling = J->cooling, reheat = J->reheat;
    const int KT = K * CL;
    uint64_t done = 0;
    if (warp == 0) {
        if (ok) build_thresholds<32>(R.sThr, R.T, lane);
        if (lane == 0 && owner) {
            SpecCtl c;
            c.it = ok ? R.it : 0;
            c.T = ok ? R.T : 0.0;
            c.pad = 0;
            const bool stop = !ok || R.iters == 0 || (a.stop_on_solve && R.best_s == 0);
            c.count = stop ? 0 : (int32_t)(R.iters < (uint64_t)KT ? R.iters : (uint64_t)KT);
            *ctl = c;
            if constexpr (CL > 1) {
                for (int q = 1; q < CL; ++q) *cg::this_cluster().map_shared_rank(ctl, q) = c;
            }
        }
    }
    if constexpr (CL > 1) cg::this_cluster().sync();
    else __syncthreads();
    if (ctl->count == 0) {
        // nothing to run: the loaded replica's record still gets its
        // rebuilt state, as the one-warp kernel writes it
        if (warp == 0 && ok && owner) store_replica<1, 32>(R, lane);
        return;
    }
    // every warp: the replica's structures (read-only until warp 0 commits)
    // and its own proposer
    if (warp != 0) {
        const SlotLayout& L = S.L;
        R.J = const_cast<XwJob*>(J);
        R.rec = a.arena + a.rec_off[rid];
        R.H = reinterpret_cast<RepHeader*>(R.rec);
        R.n = J->n; R.w = J->w; R.m = J->m; R.sparse = J->sparse; R.ld = L.ld;
        R.obj_kind = GEN ? R.H->obj_kind : 0;
        R.owner = owner;
        R.sW = reinterpret_cast<int8_t*>(slot);
        R.sG = reinterpret_cast<int32_t*>(slot + L.off_g);
        R.sRes = reinterpret_cast<int32_t*>(slot + L.off_res);
        R.sMino = slot + L.off_mino;
        R.sMask = reinterpret_cast<uint64_t*>(slot + L.off_mask);
        R.sThr = reinterpret_cast<uint64_t*>(slot + L.off_thr);
    }
    uint8_t* mine = warp == 0 ? slot + S.L.off_draws : slot + S.off_extra + (uint32_t)(warp - 1) * S.per_warp;
    View* view = warp == 0 ? reinterpret_cast<View*>(slot + S.L.off_view)
                           : reinterpret_cast<View*>(mine + 32u * 16u);
    Proposer<32> P;
    setup_proposer<1, 32>(R, reinterpret_cast<uint4*>(mine), view, lane, P);

    const int g = rank * K + warp;   // this warp's iteration within the round
#pragma unroll 1
    for (int round = 0;; ++round) {
        const int buf = round & 1;
        SpecOut* outs = reinterpret_cast<SpecOut*>(slot + S.off_out + (uint32_t)buf * S.out_stride);
        int32_t* flag = reinterpret_cast<int32_t*>(slot + S.off_flag) + buf;
        const uint64_t it0 = ctl->it;
        const int cnt = ctl->count;
        if (g < cnt) {
            const Choice ch = choose_move<1, GEN, 32>(R, P, it0 + (uint64_t)g, lane);
            // the Metropolis test at the round's starting temperature: the
            // one warp 0 would make if no cooling or reheat step falls
            // between the round's start and this iteration
            bool acc = false;
            if (ch.b0) {
                acc = ch.bprim <= 0;
                if (!acc)
                    acc = ch.bprim <= (int64_t)kThrTable ? (uint64_t)ch.u < R.sThr[ch.bprim - 1]
                                                         : metropolis_accept(ch.bprim, ctl->T, ch.u);
            }
            if (lane == 0) {
                SpecOut o;
                o.ch = ch;
                o.acc = acc ? 1 : 0;
                o.pad = 0;
                outs[g] = o;
                if constexpr (CL > 1) {
                    for (int q = 0; q < CL; ++q)
                        if (q != rank) cg::this_cluster().map_shared_rank(outs, q)[g] = o;
                }
            }
        }
        if constexpr (CL > 1) {
            if (owner && warp == 0 && lane == 0) {
                const int32_t sv = a.stop_on_solve == 1 ? *(volatile int32_t*)&R.J->solved : 0;
                for (int q = 0; q < CL; ++q) *cg::this_cluster().map_shared_rank(flag, q) = sv;
            }
            cg::this_cluster().sync();
        } else {
            __syncthreads();
        }
        if (warp == 0) {
            // Iterations in order until the first accepted move.  Fast path:
            // the rejected calls before it change only counters (moves, msi,
            // cool) unless one of them reaches a cooling or reheat step, so
            // when none can, they are counted in bulk and only the accepted
            // move goes through apply_move.  Otherwise the ordered walk.
            // The job's solved flag: read here on one CTA, as the owner read
            // it this round on a cluster.
            auto solved = [&]() -> bool {
                if constexpr (CL > 1) return *flag != 0;
                else return *(volatile int32_t*)&R.J->solved != 0;
            };
            // lane l holds the outcomes of iterations l and 32 + l (up to 64
            // iterations a round, on a cluster of four)
            Choice cl0 = {}, cl1 = {};
            int al0 = 0, al1 = 0;
            if (lane < cnt) {
                cl0 = outs[lane].ch;
                al0 = outs[lane].acc;
            }
            if (32 + lane < cnt) {
                cl1 = outs[32 + lane].ch;
                al1 = outs[32 + lane].acc;
            }
            const uint64_t have_m = (uint64_t)__ballot_sync(FULL, cl0.b0 != 0) |
                                    ((uint64_t)__ballot_sync(FULL, cl1.b0 != 0) << 32);
            const uint64_t acc_m = (uint64_t)__ballot_sync(FULL, cl0.b0 != 0 && al0 != 0) |
                                   ((uint64_t)__ballot_sync(FULL, cl1.b0 != 0 && al1 != 0) << 32);
            // calls (iterations with a candidate) that leave the temperature
            // unchanged: fewer than `room`
            const int room = tempering ? 0x7fffffff : min(mpc - R.cool, stuck - R.msi);
            const int ja = acc_m ? __ffsll((long long)acc_m) - 1 : -1;
            const int jend = ja >= 0 ? ja + 1 : cnt;
            const uint64_t span = jend >= 64 ? ~0ull : ((1ull << jend) - 1ull);
            const int calls = __popcll(have_m & span);
            const int rejects = ja >= 0 ? calls - 1 : calls;
            bool fast = rejects < room;
            // a check of the job's solved flag (every 64th iteration) that
            // falls in the span and finds it set: take the span in order
            if (fast && a.stop_on_solve == 1 && (done | 63) < done + (uint64_t)jend && solved()) fast = false;
            int j = 0;
            bool stop = false;
            if (fast) {
                const bool in0 = (span >> lane) & 1ull, in1 = (span >> (32 + lane)) & 1ull;
                R.cand_evals += __reduce_add_sync(FULL, (in0 ? cl0.evals : 0u) + (in1 ? cl1.evals : 0u));
                R.two_row_evals += __reduce_add_sync(FULL, (in0 ? cl0.evals2 : 0u) + (in1 ? cl1.evals2 : 0u));
                R.moves += (uint64_t)rejects;
                R.msi += rejects;
                if (!tempering) R.cool += rejects;
                if (ja >= 0) {
                    R.it += (uint64_t)ja;
                    const Choice ch = outs[ja].ch;
                    apply_move<1, GEN, 32>(R, ch, tempering, mpc, stuck, t_min, cooling, reheat, lane);
                    ++R.it;
                } else {
                    R.it += (uint64_t)cnt;
                }
                j = jend;
            } else {
#pragma unroll 1
                for (; j < cnt; ++j) {
                    if (a.stop_on_solve == 1 && ((done + (uint64_t)j) & 63) == 63 && solved()) {
                        stop = true;
                        break;
                    }
                    const Choice ch = outs[j].ch;
                    R.cand_evals += ch.evals;
                    R.two_row_evals += ch.evals2;
                    if (!ch.b0) {
                        ++R.it;
                        continue;
                    }
                    const bool accept =
                        apply_move<1, GEN, 32>(R, ch, tempering, mpc, stuck, t_min, cooling, reheat, lane);
                    ++R.it;
                    if (accept) {
                        ++j;
                        break;
                    }
                }
            }
            done += (uint64_t)j;
            if (a.stop_on_solve && R.best_s == 0) stop = true;
            if (lane == 0) {
                ctl->it = R.it;
                ctl->T = R.T;
                const uint64_t left = R.iters - done;
                ctl->count = stop || left == 0 ? 0 : (int32_t)(left < (uint64_t)KT ? left : (uint64_t)KT);
            }
        }
        __syncthreads();
        if (ctl->count == 0) break;
    }
    if (warp == 0 && owner) store_replica<1, 32>(R, lane);
    // the other CTAs' copies stay in their shared memory until every CTA
    // of the cluster has made its last remote write into this one
    if constexpr (CL > 1) cg::this_cluster().sync();
}

// Register budget per thread; it sets how many replica warps an SM holds.
// An SM's registers are split between its four schedulers (16384 each), so
// 128 registers per thread give 4 warps per scheduler and 96 give 5.  The
// lean one-row-per-lane kernel gains from the fifth warp (W(26,25) with
// 4096 replicas: 0.82 -> 0.87 G moves/s); the general and the wider kernels
// lose more to the spills of a 96-register budget than they gain (measured
// 6-18% slower), and keep 128.
#ifndef XW_ANNEAL_MAXNREG
#define XW_ANNEAL_MAXNREG 128
#endif
#ifndef XW_ANNEAL_MAXNREG_LEAN1
#define XW_ANNEAL_MAXNREG_LEAN1 96
#endif
#ifndef XW_ANNEAL_MAXNREG_PAIR
#define XW_ANNEAL_MAXNREG_PAIR 96
#endif
constexpr int anneal_maxnreg(int opl, bool general, int gw) {
    return gw == 16 ? XW_ANNEAL_MAXNREG_PAIR
                    : opl == 1 && !general ? XW_ANNEAL_MAXNREG_LEAN1 : XW_ANNEAL_MAXNREG;
}
// Each lane group (the warp, or each half of it) takes work items from the
// launch's counter on its own: a replica (all of its launch iterations) or
// one chunk of them.
template <int OPL, bool GEN, int GW, bool ONEZ = false, int NFIX = 0>
__global__ void __maxnreg__(anneal_maxnreg(OPL, GEN, GW)) anneal_kernel(AnnealArgs a) {
    extern __shared__ __align__(16) uint8_t smem[];
    const int lane = threadIdx.x & (GW - 1);
    const int group = threadIdx.x / GW;
    const unsigned gm = group_mask<GW>();
    uint8_t* slot = smem + (size_t)group * a.slot_bytes;
    const uint64_t total = (uint64_t)a.n_items * a.chunks;
    for (;;) {
        uint32_t item = 0;
        if (lane == 0) item = atomicAdd(a.counter, 1u);
        item = __shfl_sync(gm, item, 0, GW);
        if (item >= total) break;
        if (a.chunks == 1) {
            run_replica<OPL, GEN, GW, ONEZ, NFIX>(a, a.items[item], slot, lane, a.iters);
            continue;
        }
        const uint32_t c = item / a.n_items;
        const uint32_t rid = a.items[item - c * a.n_items];
        const uint64_t lo = a.iters * c / a.chunks, hi = a.iters * (c + 1) / a.chunks;
        RepHeader* H = reinterpret_cast<RepHeader*>(a.arena + a.rec_off[rid]);
        const bool ok = chunk_begin(a.chunk_done + rid, c, a.chunk_wait_ns, &H->err, lane, gm);
        if (ok) run_replica<OPL, GEN, GW, ONEZ, NFIX>(a, rid, slot, lane, hi - lo);
        chunk_end(a.chunk_done + rid, c, ok, lane, gm);
    }
}

// Latency mode: each CTA of K warps owns one replica at a time (orders up
// to 32), taken from the launch's counter.
// The latency mode: one CTA (CL = 1, a persistent loop over the launch's
// replicas) or one cluster of CL CTAs (one replica per cluster) per replica.
template <bool GEN, int CL>
__global__ void __launch_bounds__(512, 1) anneal_spec_kernel(AnnealArgs a, int K) {
    extern __shared__ __align__(16) uint8_t smem[];
    __shared__ uint32_t s_item;
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    if constexpr (CL > 1) {
        const uint32_t item = blockIdx.x / CL;
        if (item < a.n_items) run_replica_spec<GEN, CL>(a, a.items[item], smem, warp, K, lane);
    } else {
        for (;;) {
            if (threadIdx.x == 0) s_item = atomicAdd(a.counter, 1u);
            __syncthreads();
            const uint32_t item = s_item;
            if (item >= a.n_items) break;
            run_replica_spec<GEN, 1>(a, a.items[item], smem, warp, K, lane);
            __syncthreads();
        }
    }
}

// One thread per tempering job: adjacent-rung sweep of
// xweigh_anneal.hpp:1187-1221 on the device draw stream.
__global__ void exchange_kernel(XwJob* jobs, int njobs, uint8_t* arena, const uint64_t* rec_off,
                                const double* ladder, int stop_on_solve) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= njobs) return;
    XwJob& J = jobs[j];
    if (!J.tempering || J.done || (stop_on_solve && J.solved) || J.replicas < 2 || J.replicas > XW_MAX_RUNGS) return;
    const int R = J.replicas;
    if (J.exchange_iters) {
        // served jobs run launches shorter than the exchange interval: swap
        // only at the interval's boundaries of the job's own iteration count
        const uint64_t it0 = reinterpret_cast<const RepHeader*>(arena + rec_off[J.rep_begin])->it;
        if (it0 == 0 || it0 % J.exchange_iters) return;
    }
    int owner[XW_MAX_RUNGS];
    int64_t E[XW_MAX_RUNGS];
    for (int k = 0; k < R; ++k) {
        const RepHeader* H = reinterpret_cast<const RepHeader*>(arena + rec_off[J.rep_begin + k]);
        if (H->rung < 0 || H->rung >= R) return;
        owner[H->rung] = k;
        E[k] = H->obj_total;
    }
    const double* lad = ladder + J.ladder_off;
    const uint64_t round = J.exch_round;
    for (int rung = 0; rung + 1 < R; ++rung) {
        const int ra = owner[rung], rb = owner[rung + 1];
        const double x = __dmul_rn(__dsub_rn(__ddiv_rn(1.0, lad[rung]), __ddiv_rn(1.0, lad[rung + 1])),
                                   (double)(E[ra] - E[rb]));
        bool accept = x >= 0.0;
        if (!accept) {
            const uint4 blk = philox4x32_10(
                make_uint4((uint32_t)rung / 4u, (uint32_t)round, (uint32_t)(round >> 32), 0x80000000u),
                J.key0, J.key1);
            accept = __dmul_rn((double)pick(blk, rung % 4), 0x1p-32) < acceptance_exp(x);
        }
        if (accept) {
            owner[rung] = rb;
            owner[rung + 1] = ra;
        }
    }
    for (int rung = 0; rung < R; ++rung) {
        RepHeader* H = reinterpret_cast<RepHeader*>(arena + rec_off[J.rep_begin + owner[rung]]);
        H->rung = rung;
        H->temperature = lad[rung];
    }
    J.exch_round = round + 1;
}

// One warp per job: best replica by (best score, best conflicts, replica
// index) -- select_best_replica, xweigh_cuda.cu:1342-1354 -- summed
// counters, and a copy of the best replica's best W into a compact buffer.
// The first solver -- least (solve iteration, replica index) among replicas
// whose best score is 0 -- does not depend on how long the job ran after
// it; with first_solver_state its best W is the one copied out.
__global__ void collect_kernel(const XwJob* jobs, int njobs, const uint8_t* arena, const uint64_t* rec_off,
                               const uint64_t* best_out_off, JobOut* out, int8_t* best_out,
                               int first_solver_state) {
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (warp >= njobs) return;
    const XwJob& J = jobs[warp];
    int64_t bs = INT64_MAX, bc = INT64_MAX;
    int br = 0x7fffffff;
    uint64_t moves = 0, evals = 0, iters = 0, acc = 0, acc_rows = 0, evals2 = 0;
    uint64_t fs_it = UINT64_MAX, fs_ns = 0;
    int fs = 0x7fffffff;
    uint32_t err = 0;
    for (int r = lane; r < J.replicas; r += 32) {
        const RepHeader* H = reinterpret_cast<const RepHeader*>(arena + rec_off[J.rep_begin + r]);
        const int64_t s = H->best_score, c = H->best_conflicts;
        if (s < bs || (s == bs && (c < bc || (c == bc && r < br)))) { bs = s; bc = c; br = r; }
        if (s == 0 && (H->solve_it < fs_it || (H->solve_it == fs_it && r < fs))) {
            fs_it = H->solve_it; fs_ns = H->solve_ns; fs = r;
        }
        moves += H->moves;
        evals += H->cand_evals;
        acc += H->accepted;
        acc_rows += H->accepted_rows;
        evals2 += H->two_row_evals;
        iters = iters > H->it ? iters : H->it;
        err |= H->err;
    }
    for (int off = 16; off > 0; off >>= 1) {
        const int64_t s2 = __shfl_xor_sync(FULL, bs, off), c2 = __shfl_xor_sync(FULL, bc, off);
        const int r2 = __shfl_xor_sync(FULL, br, off);
        if (s2 < bs || (s2 == bs && (c2 < bc || (c2 == bc && r2 < br)))) { bs = s2; bc = c2; br = r2; }
        moves += __shfl_xor_sync(FULL, moves, off);
        evals += __shfl_xor_sync(FULL, evals, off);
        acc += __shfl_xor_sync(FULL, acc, off);
        acc_rows += __shfl_xor_sync(FULL, acc_rows, off);
        evals2 += __shfl_xor_sync(FULL, evals2, off);
        const uint64_t i2 = __shfl_xor_sync(FULL, iters, off);
        iters = iters > i2 ? iters : i2;
        err |= __shfl_xor_sync(FULL, err, off);
        const uint64_t fi2 = __shfl_xor_sync(FULL, fs_it, off), fn2 = __shfl_xor_sync(FULL, fs_ns, off);
        const int f2 = __shfl_xor_sync(FULL, fs, off);
        if (fi2 < fs_it || (fi2 == fs_it && f2 < fs)) { fs_it = fi2; fs_ns = fn2; fs = f2; }
    }
    if (first_solver_state && fs < J.replicas) br = fs;
    if (lane == 0) {
        JobOut o;
        o.score = bs; o.conflicts = bc; o.best_replica = br;
        o.solved = J.solved; o.err = (int32_t)err;
        o.first_solver = fs < J.replicas ? fs : -1;
        o.moves = moves; o.cand_evals = evals; o.iters = iters;
        o.accepted = acc; o.accepted_rows = acc_rows; o.two_row_evals = evals2;
        o.solved_it = fs < J.replicas ? fs_it : 0;
        o.solve_ns = fs < J.replicas ? fs_ns : 0;
        out[warp] = o;
    }
    if (best_out && br >= 0 && br < J.replicas) {
        const uint8_t* src = arena + rec_off[J.rep_begin + br] + J.off_best;
        int8_t* dst = best_out + best_out_off[warp];
        const int nn = J.n * J.n;
        for (int i = lane; i < nn; i += 32) dst[i] = (int8_t)src[i];
    }
}

__global__ void mark_t0_kernel(uint64_t* t0) {
    if (*t0 == 0) *t0 = globaltimer();
}

__global__ void stamp_kernel(uint64_t* t) { *t = globaltimer(); }

}  // namespace

uint32_t anneal_slot_bytes(int n, int m, int opl) { return slot_layout(n, m, opl > 4).bytes; }

int anneal_opl(int n) { return n <= 32 ? 1 : n <= 64 ? 2 : n <= 128 ? 4 : 8; }

template <int N>
const void* one_zero_order_fn() {
    return reinterpret_cast<const void*>(&anneal_kernel<1, false, 32, true, N>);
}

// the one-zero kernel compiled for one order: the even orders 6..26 (W(n, n-1)
// does not exist for odd n), nullptr for the others.  28, 30 and 32 compile
// with 380 bytes of spills a thread (40 for the kernel of any order) and are
// left to that kernel.
const void* one_zero_fixed_fn(int n) {
    switch (n) {
    case 6: return one_zero_order_fn<6>();
    case 8: return one_zero_order_fn<8>();
    case 10: return one_zero_order_fn<10>();
    case 12: return one_zero_order_fn<12>();
    case 14: return one_zero_order_fn<14>();
    case 16: return one_zero_order_fn<16>();
    case 18: return one_zero_order_fn<18>();
    case 20: return one_zero_order_fn<20>();
    case 22: return one_zero_order_fn<22>();
    case 24: return one_zero_order_fn<24>();
    case 26: return one_zero_order_fn<26>();
    default: return nullptr;
    }
}

const void* anneal_kernel_fn(int opl, bool general, int rpw, bool one_zero, int fixed_order) {
    if (one_zero && opl == 1 && !general && rpw == 1) {
        if (const void* f = fixed_order > 0 ? one_zero_fixed_fn(fixed_order) : nullptr) return f;
        return reinterpret_cast<const void*>(&anneal_kernel<1, false, 32, true>);
    }
    if (rpw == 2) {
        return general ? reinterpret_cast<const void*>(&anneal_kernel<1, true, 16>)
                       : reinterpret_cast<const void*>(&anneal_kernel<1, false, 16>);
    }
    if (general) {
        if (opl == 1) return reinterpret_cast<const void*>(&anneal_kernel<1, true, 32>);
        if (opl == 2) return reinterpret_cast<const void*>(&anneal_kernel<2, true, 32>);
        if (opl == 4) return reinterpret_cast<const void*>(&anneal_kernel<4, true, 32>);
        return reinterpret_cast<const void*>(&anneal_kernel<8, true, 32>);
    }
    if (opl == 1) return reinterpret_cast<const void*>(&anneal_kernel<1, false, 32>);
    if (opl == 2) return reinterpret_cast<const void*>(&anneal_kernel<2, false, 32>);
    if (opl == 4) return reinterpret_cast<const void*>(&anneal_kernel<4, false, 32>);
    return reinterpret_cast<const void*>(&anneal_kernel<8, false, 32>);
}

cudaError_t launch_anneal(const AnnealArgs& args, int opl, bool general, int warps_per_block, int blocks,
                          cudaStream_t stream, int rpw) {
    if (rpw != 1 && (rpw != 2 || opl != 1)) return cudaErrorInvalidValue;
    const size_t smem = (size_t)warps_per_block * rpw * args.slot_bytes;
    const dim3 grid(blocks), block(32 * warps_per_block);
    void* kargs[] = {const_cast<AnnealArgs*>(&args)};
    return cudaLaunchKernel(anneal_kernel_fn(opl, general, rpw, args.one_zero != 0, args.fixed_order), grid, block,
                            kargs, smem, stream);
}

// wpr warps per replica on `ctas` CTAs (1, 2 or 4; a cluster above 1) of
// wpr / ctas warps each
uint32_t anneal_spec_cta_bytes(uint32_t slot_bytes, int wpr, int ctas) {
    SpecLayout S;
    spec_regions(slot_bytes, wpr / ctas, ctas, S);
    return S.bytes;
}

const void* anneal_spec_kernel_fn(bool general, int ctas) {
    if (ctas == 4)
        return general ? reinterpret_cast<const void*>(&anneal_spec_kernel<true, 4>)
                       : reinterpret_cast<const void*>(&anneal_spec_kernel<false, 4>);
    if (ctas == 2)
        return general ? reinterpret_cast<const void*>(&anneal_spec_kernel<true, 2>)
                       : reinterpret_cast<const void*>(&anneal_spec_kernel<false, 2>);
    return general ? reinterpret_cast<const void*>(&anneal_spec_kernel<true, 1>)
                   : reinterpret_cast<const void*>(&anneal_spec_kernel<false, 1>);
}

cudaError_t launch_anneal_spec(const AnnealArgs& args, bool general, int wpr, int ctas, int blocks,
                               cudaStream_t stream) {
    const int CL = ctas;
    if ((CL != 1 && CL != 2 && CL != 4) || wpr % CL != 0 || wpr / CL < 2 || wpr / CL > 16 || args.chunks != 1)
        return cudaErrorInvalidValue;
    int k = wpr / CL;
    void* kargs[] = {const_cast<AnnealArgs*>(&args), &k};
    if (CL == 1)
        return cudaLaunchKernel(anneal_spec_kernel_fn(general, 1), dim3(blocks), dim3(32 * k), kargs,
                                args.slot_bytes, stream);
    // one cluster of CL CTAs per replica
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(CL * args.n_items);
    cfg.blockDim = dim3(32 * k);
    cfg.dynamicSmemBytes = args.slot_bytes;
    cfg.stream = stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = CL;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelExC(&cfg, anneal_spec_kernel_fn(general, CL), kargs);
}

cudaError_t launch_exchange(XwJob* jobs, int njobs, uint8_t* arena, const uint64_t* rec_off, const double* ladder,
                            int stop_on_solve, cudaStream_t stream) {
    if (njobs <= 0) return cudaSuccess;
    exchange_kernel<<<(njobs + 127) / 128, 128, 0, stream>>>(jobs, njobs, arena, rec_off, ladder, stop_on_solve);
    return cudaGetLastError();
}

cudaError_t launch_collect(const XwJob* jobs, int njobs, const uint8_t* arena, const uint64_t* rec_off,
                           const uint64_t* best_out_off, JobOut* out, int8_t* best_out, cudaStream_t stream,
                           int first_solver_state) {
    if (njobs <= 0) return cudaSuccess;
    collect_kernel<<<(njobs + 3) / 4, 128, 0, stream>>>(jobs, njobs, arena, rec_off, best_out_off, out, best_out,
                                                        first_solver_state);
    return cudaGetLastError();
}

cudaError_t launch_stamp(uint64_t* t, cudaStream_t stream) {
    stamp_kernel<<<1, 1, 0, stream>>>(t);
    return cudaGetLastError();
}

cudaError_t launch_mark_t0(uint64_t* t0, cudaStream_t stream) {
    mark_t0_kernel<<<1, 1, 0, stream>>>(t0);
    return cudaGetLastError();
}

}  // namespace xw
