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
// For orders up to 448 W can instead sit in the warp's slot as support and
// sign bit planes, which the proposals read without touching global
// memory.  Two forms do that: the hybrid (the default there) keeps G in
// HBM and stages each candidate's Gram rows in shared memory with all their
// loads in flight at once; the bit-plane form stores no G and recomputes
// each Gram entry it needs by popcounts, so a move makes no HBM traffic.
// Their arena keeps residuals, planes and the best state's planes between
// launches.
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
// Support mask word k of row r is mask[r * mrs + k * mks] (in u64 words):
// the Gram arena's row-major masks (mrs = nw, mks = 1), or the bit planes
// in shared memory (mrs = 2, mks = 2n; the sign word follows each support
// word), from which `planes` replicas also read W's entries.
struct LView {
    const int8_t* W;
    const uint16_t* mino;
    const int32_t* res;
    const uint64_t* mask;
    const uint32_t* dw;
    uint64_t thr_target, thr_dbl, thr_sign, thr_swsign;
    int n, w, m, sparse, ts, bpc, cc, move_set, nw;
    int mrs, mks, planes;
    uint32_t stream, k0, k1;
};

// The large-order kernel's forms: the Gram matrix and masks in HBM; bit
// planes in shared memory with every Gram entry recomputed; and the hybrid
// of the two, bit planes in shared memory (proposals and W's entries) with
// the Gram matrix in HBM (evaluation and commit), each candidate's Gram
// rows staged in shared memory with all their loads in flight at once.
enum LargeForm : int { kFormGram = 0, kFormPlanes = 1, kFormHybrid = 2 };

// Row stride of the hybrid form's Gram matrix: rows start on 16 bytes.
__host__ __device__ inline int gram_ld(int n) { return (n + 7) & ~7; }

// Shared memory per warp.  Every replica: residuals (int32 x n), the
// iteration's draw blocks, the view, the Metropolis thresholds.  A replica
// in bit-plane mode adds W as support and sign planes, planes[q * n + o] =
// {support word q of row o, sign word q of row o} (16 bytes; consecutive
// rows consecutive, so a warp reading word q of its 32 rows reads 512
// contiguous bytes), and its minority lists when they take at most
// kMinoSmemBytes (off_mino 0: they stay in the record); the hybrid form
// adds two staging buffers of two Gram rows each.
struct LSlot {
    uint32_t off_draws, off_view, off_thr, off_planes, off_mino, off_stage, bytes;
};

constexpr uint32_t kMinoSmemBytes = 8192;

__host__ __device__ inline LSlot large_slot(int n, int m, int form) {
    LSlot L;
    L.off_draws = xw_pad16((uint32_t)n * 4u);
    L.off_view = L.off_draws + 32u * 16u;
    L.off_thr = L.off_view + xw_pad16((uint32_t)sizeof(LView));
    L.bytes = L.off_thr + kThrTable * 8u;
    L.off_planes = L.off_mino = L.off_stage = 0;
    if (form != kFormGram) {
        const uint32_t nw = (uint32_t)(n + 63) / 64u;
        L.off_planes = xw_pad16(L.bytes);
        L.bytes = L.off_planes + nw * (uint32_t)n * 16u;
        const uint32_t mb = (uint32_t)n * (uint32_t)m * 2u;
        if (mb <= kMinoSmemBytes) {
            L.off_mino = L.bytes;
            L.bytes += xw_pad16(mb);
        }
    }
    if (form == kFormHybrid) {
        L.off_stage = L.bytes;
        L.bytes += 4u * (uint32_t)gram_ld(n) * 2u;
    }
    return L;
}

// Bit-plane mode: orders whose warp slot fits kPlanesSlotMax (four warps
// per CTA within the 227 KiB a CTA may hold), which bounds the plane words
// per row by kPlanesNw (n <= 448).
constexpr uint32_t kPlanesSlotMax = 227u * 1024u / 4u;
constexpr int kPlanesNw = 7;

__host__ __device__ inline bool large_planes_fit(int n, int m) {
    return n <= 64 * kPlanesNw && large_slot(n, m, kFormHybrid).bytes <= kPlanesSlotMax;
}

// Arena per replica.  Stored-Gram form: G (int16, row-major), support and
// sign masks.  Bit-plane form: the residuals, the planes and the best
// state's planes, so that a launch resumes without rebuilding them and a
// best state is saved with 16-byte copies (expanded to the record's int8
// layout once, at the end of the launch).  XW_STATUS_GRAM: the arena holds
// the record's W in that form.
struct LGram {
    uint64_t off_mask, off_sign, bytes;
};

struct LPArena {
    uint64_t off_planes, off_best, off_g, bytes;
};

// residuals, planes and the best state's planes (and, in the hybrid form,
// G: int16 row-major, rows gram_ld(n) entries apart)
__host__ __device__ inline LPArena planes_arena(int n, bool stored_gram) {
    const uint64_t nw = (uint64_t)(n + 63) / 64;
    LPArena A;
    A.off_planes = ((uint64_t)n * 4u + 15u) & ~uint64_t(15);
    A.off_best = A.off_planes + nw * (uint64_t)n * 16u;
    A.off_g = A.off_best + nw * (uint64_t)n * 16u;
    A.bytes = A.off_g + (stored_gram ? (uint64_t)n * gram_ld(n) * 2u : 0u);
    return A;
}

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

// entry (r, c) of a bit-plane pair: 0, +1 or -1
__device__ __forceinline__ int plane_entry(const uint64_t* e, int c) {
    const int s = (int)((e[0] >> (c & 63)) & 1ull), g = (int)((e[1] >> (c & 63)) & 1ull);
    return s - 2 * (s & g);
}

__device__ __forceinline__ int l_at(const LView* v, int r, int c) {
    if (v->planes) return plane_entry(v->mask + (size_t)r * v->mrs + (size_t)(c >> 6) * v->mks, c);
    return v->W[(size_t)c * v->n + r];
}

// word k of a row's support mask, or of its zero set (columns < n)
__device__ __forceinline__ uint64_t mask_word(const LView* v, int row, int k, bool zeros) {
    const int nw = v->nw, n = v->n;
    uint64_t x = v->mask[(size_t)row * v->mrs + (size_t)k * v->mks];
    if (zeros) {
        x = ~x;
        if (k == nw - 1 && (n & 63)) x &= (1ull << (n & 63)) - 1ull;
    }
    return x;
}

// first set bit at or after `start`, cyclically
__device__ __noinline__ int l_cyclic_first(const LView* v, int row, int start, bool zeros) {
    const int nw = v->nw;
    const int ws = start >> 6;
#pragma unroll 1
    for (int k = ws; k < nw; ++k) {
        uint64_t x = mask_word(v, row, k, zeros);
        if (k == ws) x &= ~0ull << (start & 63);
        if (x) return 64 * k + __ffsll((long long)x) - 1;
    }
#pragma unroll 1
    for (int k = 0; k <= ws && k < nw; ++k) {
        const uint64_t x = mask_word(v, row, k, zeros);
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
    return l_cyclic_first(v, row, start, false);
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
    int c1, c2, pos;
    if (v->sparse) {
        pos = (int)l_index(v, it, c, 1, 1, (uint32_t)v->m);
        c1 = v->mino[(size_t)row * v->m + pos];
        c2 = l_cyclic_first(v, row, (int)l_index(v, it, c, 1, 2, (uint32_t)v->n), true);
    } else {
        pos = (int)l_index(v, it, c, 1, 2, (uint32_t)v->m);
        c2 = v->mino[(size_t)row * v->m + pos];
        c1 = l_cyclic_first(v, row, (int)l_index(v, it, c, 1, 1, (uint32_t)v->n), false);
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

// ---------------------------------------------------------------------------
// Bit-plane mode.  No Gram matrix is stored: the entries an evaluation or a
// commit needs are recomputed from the planes in shared memory,
// G[r][o] = |S_r & S_o| - 2 |S_r & S_o & (N_r ^ N_o)| (S: support, N: sign
// bits), and a commit changes only the planes, the residuals and the
// minority lists.  A move costs no HBM traffic and no scattered stores; the
// price is the popcount arithmetic, about 12 instructions per 64 columns of
// each Gram entry read.  The deltas, ties and trajectory are those of the
// stored-Gram form.

__device__ __forceinline__ int p_at(const ulonglong2* P, int n, int r, int c) {
    return plane_entry(reinterpret_cast<const uint64_t*>(&P[(size_t)(c >> 6) * n + r]), c);
}

__device__ __forceinline__ void p_set(ulonglong2* P, int n, int r, int c, int v) {
    ulonglong2& e = P[(size_t)(c >> 6) * n + r];
    const uint64_t bit = 1ull << (c & 63);
    e.x = v != 0 ? (e.x | bit) : (e.x & ~bit);
    e.y = v < 0 ? (e.y | bit) : (e.y & ~bit);
}

__device__ __forceinline__ int p_dot(const ulonglong2* P, int n, int nw, int r, int o) {
    int d = 0;
#pragma unroll 1
    for (int q = 0; q < nw; ++q) {
        const ulonglong2 a = P[(size_t)q * n + r], b = P[(size_t)q * n + o];
        const uint64_t both = a.x & b.x;
        d += __popcll(both) - 2 * __popcll(both & (a.y ^ b.y));
    }
    return d;
}

__device__ __forceinline__ int p_pair_new(const LUpdate& u, int op, const ulonglong2* P, int n) {
    return op + u.A1 * p_at(P, n, u.R2, u.X1) + u.A2 * p_at(P, n, u.R1, u.X2) + (u.X1 == u.X2 ? u.A1 * u.A2 : 0);
}

// One pass over the lane's rows o = lane, lane + 32, ... for a move's
// updated rows R1 (and R2 when two): G[R1][o] (and G[R2][o]) by popcounts
// over the plane words (row o's words read once for both rows; the updated
// rows' words are broadcast reads), the new entries G + A W[o][X] + B W[o][Y],
// and then either the objective deltas (evaluation) or the residual
// updates (commit: res[o] changes, and the returned S1 sums R1's changes).
// One small loop serves both, so that it stays in the instruction cache
// and in registers.
struct PRows {
    LDeltas d;   // evaluation: the lane's objective deltas
    int s1;      // commit: the lane's sum of R1's residual changes
};

// Hybrid form: copy the stored Gram rows r1 (and r2) into the warp's
// staging buffer S (rows gram_ld(n) entries apart, 16-byte chunks, at most
// two per lane and row), every load issued before the first store, so that
// staging costs one round trip to L2/HBM
__device__ __forceinline__ void p_stage(const int16_t* G, int n, int r1, int r2, bool two, int16_t* S, int lane) {
    const int ldg = gram_ld(n), chunks = ldg / 8;
    const uint4* a = reinterpret_cast<const uint4*>(G + (size_t)r1 * ldg);
    const uint4* b = reinterpret_cast<const uint4*>(G + (size_t)r2 * ldg);
    const int k0 = lane, k1 = lane + 32;
    uint4 x0 = make_uint4(0, 0, 0, 0), x1 = x0, y0 = x0, y1 = x0;
    if (k0 < chunks) x0 = a[k0];
    if (k1 < chunks) x1 = a[k1];
    if (two) {
        if (k0 < chunks) y0 = b[k0];
        if (k1 < chunks) y1 = b[k1];
    }
    uint4* sa = reinterpret_cast<uint4*>(S);
    uint4* sb = reinterpret_cast<uint4*>(S + ldg);
    if (k0 < chunks) sa[k0] = x0;
    if (k1 < chunks) sa[k1] = x1;
    if (two) {
        if (k0 < chunks) sb[k0] = y0;
        if (k1 < chunks) sb[k1] = y1;
    }
    __syncwarp();
}

// The same copy issued as cp.async (global -> shared, bypassing L1, no
// registers held) and committed as one group: the caller overlaps it with
// the evaluation of the previous candidate and waits with cp.async.wait_group.
__device__ __forceinline__ void p_stage_async(const int16_t* G, int n, int r1, int r2, bool two, int16_t* S,
                                              int lane) {
    const int ldg = gram_ld(n), chunks = ldg / 8;
#pragma unroll
    for (int h = 0; h < 2; ++h) {
        const int k = lane + 32 * h;
        if (k < chunks) {
            asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(
                             (uint32_t)__cvta_generic_to_shared(S + 8 * k)),
                         "l"(G + (size_t)r1 * ldg + 8 * k)
                         : "memory");
            if (two)
                asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(
                                 (uint32_t)__cvta_generic_to_shared(S + ldg + 8 * k)),
                             "l"(G + (size_t)r2 * ldg + 8 * k)
                             : "memory");
        }
    }
    asm volatile("cp.async.commit_group;" ::: "memory");
}

// the updated rows of candidate c's move (from its descriptor word x)
__device__ __forceinline__ void move_rows(uint32_t x, int& r1, int& r2, bool& two) {
    const int kind = (x >> 1) & 3;
    r1 = (x >> 3) & 1023;
    r2 = (x >> 13) & 1023;
    two = kind == 1 || (kind == 2 && r1 != r2);
}

template <bool GEN, bool TWO, bool SG>
__device__ __forceinline__ PRows p_rows(const LUpdate& u, const ulonglong2* P, int16_t* G, const int16_t* S,
                                        int32_t* res, int n, int nw, int lane, bool commit) {
    PRows out = {{0, 0, 0, 0}, 0};
    const int ldg = gram_ld(n);
    const ulonglong2* pa = P + u.R1;
    const ulonglong2* pb = P + (TWO ? u.R2 : u.R1);
#pragma unroll 1
    for (int o = lane; o < n; o += 32) {
        int g1 = 0, g2 = 0;
        if constexpr (SG) {
            g1 = S[o];
            if constexpr (TWO) g2 = S[ldg + o];
        } else {
#pragma unroll 1
        for (int q = 0; q < nw; ++q) {
            const size_t off = (size_t)q * n;
            const ulonglong2 e = P[off + o], a = pa[off];
            const uint64_t b1 = a.x & e.x;
            g1 += __popcll(b1) - 2 * __popcll(b1 & (a.y ^ e.y));
            if constexpr (TWO) {
                const ulonglong2 b = pb[off];
                const uint64_t b2 = b.x & e.x;
                g2 += __popcll(b2) - 2 * __popcll(b2 & (b.y ^ e.y));
            }
        }
        }
        if (o == u.R1 || (TWO && o == u.R2)) continue;
        int n1 = g1 + u.A1 * p_at(P, n, o, u.X1);
        if (u.B1) n1 += u.B1 * p_at(P, n, o, u.Y1);
        int n2 = g2;
        if constexpr (TWO) {
            n2 += u.A2 * p_at(P, n, o, u.X2);
            if (u.B2) n2 += u.B2 * p_at(P, n, o, u.Y2);
        }
        if (commit) {
            const int e1 = iabs(n1) - iabs(g1);
            res[o] += TWO ? e1 + iabs(n2) - iabs(g2) : e1;
            out.s1 += e1;
            if constexpr (SG) {
                G[(size_t)u.R1 * ldg + o] = (int16_t)n1;
                G[(size_t)o * ldg + u.R1] = (int16_t)n1;
                if constexpr (TWO) {
                    G[(size_t)u.R2 * ldg + o] = (int16_t)n2;
                    G[(size_t)o * ldg + u.R2] = (int16_t)n2;
                }
            }
        } else {
            lacc<GEN>(out.d, g1, n1);
            if constexpr (TWO) lacc<GEN>(out.d, g2, n2);
        }
    }
    return out;
}

template <bool GEN, bool SG>
__device__ __forceinline__ PRows p_rows_any(const LUpdate& u, const ulonglong2* P, int16_t* G, const int16_t* S,
                                            int32_t* res, int n, int nw, int lane, bool commit) {
    return u.R2 >= 0 ? p_rows<GEN, true, SG>(u, P, G, S, res, n, nw, lane, commit)
                     : p_rows<GEN, false, SG>(u, P, G, S, res, n, nw, lane, commit);
}

// l_eval on the planes (and, SG, the move's stored Gram rows staged in S)
template <bool GEN, bool SG>
__device__ __forceinline__ LDeltas p_eval(const LUpdate& u, const ulonglong2* P, int16_t* G, const int16_t* S, int n,
                                          int nw, int lane) {
    LDeltas d = p_rows_any<GEN, SG>(u, P, G, S, nullptr, n, nw, lane, false).d;
    if (u.pair && lane == 0) {
        const int op = SG ? (int)S[u.R2] : p_dot(P, n, nw, u.R1, u.R2);
        lacc<GEN>(d, op, p_pair_new(u, op, P, n));
    }
    return d;
}

// l_commit on the planes: residuals from the recomputed rows, then the
// changed entries (lane 0, after every lane has read the old planes)
template <bool GEN, bool SG>
__device__ void p_commit(const LMove& mv, const LUpdate& u, int ds, ulonglong2* P, int16_t* G, const int16_t* S,
                         int32_t* res, uint16_t* mino, int n, int m, int nw, int sparse, int lane) {
    const int s1 = p_rows_any<GEN, SG>(u, P, G, S, res, n, nw, lane, true).s1;
    const int S1 = __reduce_add_sync(FULL, s1);
    __syncwarp();
    if (lane == 0) {
        const int kind = (mv.x >> 1) & 3, r1 = (mv.x >> 3) & 1023, r2 = (mv.x >> 13) & 1023;
        const int c1 = mv.y & 1023, c2 = (mv.y >> 10) & 1023;
        const int nv1 = (int)((mv.y >> 20) & 3) - 1, nv2 = (int)((mv.y >> 22) & 3) - 1;
        const int p1 = mv.z & 1023, p2 = (mv.z >> 10) & 1023;
        const int o11 = (int)((mv.x >> 23) & 3) - 1, o22 = (int)((mv.x >> 25) & 3) - 1;
        if (u.pair) {
            const int op = SG ? (int)S[r2] : p_dot(P, n, nw, r1, r2);
            const int np = p_pair_new(u, op, P, n);
            const int pd = iabs(np) - iabs(op);
            if constexpr (SG) {
                const int ldg = gram_ld(n);
                G[(size_t)r1 * ldg + r2] = (int16_t)np;
                G[(size_t)r2 * ldg + r1] = (int16_t)np;
            }
            res[r1] += S1 + pd;
            res[r2] += ds - S1;
        } else if (u.R2 >= 0) {
            res[r1] += S1;
            res[r2] += ds - S1;
        } else {
            res[r1] += ds;
        }
        if (kind == 0) {
            p_set(P, n, r1, c1, -o11);
        } else if (kind == 2) {
            p_set(P, n, r1, c1, -o11);
            p_set(P, n, r2, c2, -o22);
        } else if (kind == 1) {
            p_set(P, n, r1, c1, 0);
            p_set(P, n, r2, c2, 0);
            p_set(P, n, r1, c2, nv1);
            p_set(P, n, r2, c1, nv2);
            mino[(size_t)r1 * m + p1] = (uint16_t)(sparse ? c2 : c1);
            mino[(size_t)r2 * m + p2] = (uint16_t)(sparse ? c1 : c2);
        } else if (GEN) {
            p_set(P, n, r1, c1, 0);
            p_set(P, n, r1, c2, nv1);
            mino[(size_t)r1 * m + p1] = (uint16_t)(sparse ? c2 : c1);
        }
    }
    __syncwarp();
}

// Residuals and the totals of the lane's rows from the planes (a replica
// whose planes were just built): every G[r][o], r != o; G, when given,
// receives the Gram matrix
__device__ __noinline__ void p_totals(const ulonglong2* P, int16_t* G, int32_t* res, int n, int nw, int lane,
                                      int& score, int& conf, long long& sq, int& par) {
#pragma unroll 1
    for (int o = lane; o < n; o += 32) {
        int r_sum = 0;
#pragma unroll 1
        for (int r = 0; r < n; ++r) {
            int g = 0;
#pragma unroll 1
            for (int q = 0; q < nw; ++q) {
                const ulonglong2 x = P[(size_t)q * n + r], e = P[(size_t)q * n + o];
                const uint64_t both = x.x & e.x;
                g += __popcll(both) - 2 * __popcll(both & (x.y ^ e.y));
            }
            if (G) G[(size_t)r * gram_ld(n) + o] = (int16_t)g;
            if (r != o) {
                const int ag = iabs(g);
                r_sum += ag;
                conf += g != 0;
                sq += (long long)(g * g);
                par += ag & 1;
            }
        }
        res[o] = r_sum;
        score += r_sum;
    }
}

// W (column-major int8, as in the record) from the planes (in shared
// memory or in the arena): each lane expands its rows' words, the warp's
// stores for one column are 32 consecutive bytes
__device__ void p_store_w(int8_t* dst, const ulonglong2* P, int n, int lane) {
    const int nw = (n + 63) / 64;
#pragma unroll 1
    for (int q = 0; q < nw; ++q) {
        const int c1 = min(n, 64 * q + 64);
#pragma unroll 1
        for (int o = lane; o < n; o += 32) {
            const ulonglong2 e = P[(size_t)q * n + o];
#pragma unroll 4
            for (int c = 64 * q; c < c1; ++c) {
                const int s = (int)((e.x >> (c & 63)) & 1ull), g = (int)((e.y >> (c & 63)) & 1ull);
                dst[(size_t)c * n + o] = (int8_t)(s - 2 * (s & g));
            }
        }
    }
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

template <bool GEN, int FORM>
__device__ void run_large(const AnnealArgs& a, uint32_t rid, uint8_t* slot, int lane, uint64_t chunk_iters) {
    constexpr bool PM = FORM != kFormGram;     // W as bit planes in the slot
    constexpr bool SG = FORM != kFormPlanes;   // the Gram matrix stored in HBM
    uint8_t* rec = a.arena + a.rec_off[rid];
    RepHeader* H = reinterpret_cast<RepHeader*>(rec);
    const uint32_t jid = H->job;
    XwJob* J = a.jobs + jid;
    if (*(volatile int32_t*)&J->done) return;
    if (a.stop_on_solve == 1 && *(volatile int32_t*)&J->solved) return;

    const int n = J->n, w = J->w, m = J->m, sparse = J->sparse;
    const int nw = (n + 63) / 64;
    const LSlot L = large_slot(n, m, FORM);
    int8_t* W = reinterpret_cast<int8_t*>(rec + J->off_w);
    uint16_t* const mino_rec = reinterpret_cast<uint16_t*>(rec + J->off_mino);
    // bit-plane mode: W as planes in the slot; the arena keeps residuals,
    // planes and the best state's planes between launches
    ulonglong2* const P = PM ? reinterpret_cast<ulonglong2*>(slot + L.off_planes) : nullptr;
    uint16_t* const mino = PM && L.off_mino ? reinterpret_cast<uint16_t*>(slot + L.off_mino) : mino_rec;
    uint8_t* const parena = PM ? a.gram + a.gram_off[rid] : nullptr;
    const LPArena PA = planes_arena(n, SG);
    const uint32_t plane_bytes = (uint32_t)nw * (uint32_t)n * 16u;
    int16_t* G = PM && SG ? reinterpret_cast<int16_t*>(parena + PA.off_g) : nullptr;
    int16_t* const S = PM && SG ? reinterpret_cast<int16_t*>(slot + L.off_stage) : nullptr;
    uint64_t *mask = nullptr, *sign = nullptr;
    if constexpr (!PM) {
        const LGram LG = large_gram(n);
        uint8_t* gbase = a.gram + a.gram_off[rid];
        G = reinterpret_cast<int16_t*>(gbase);
        mask = reinterpret_cast<uint64_t*>(gbase + LG.off_mask);
        sign = reinterpret_cast<uint64_t*>(gbase + LG.off_sign);
    }
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

    // ---- Gram and masks (once per W the host wrote), or the planes (every
    // load); minority lists ----
    const uint32_t status0 = H->status;
    const bool cached = PM && (status0 & XW_STATUS_GRAM);
    if constexpr (PM) {
        if (!large_planes_fit(n, m)) {
            if (lane == 0) H->err |= XW_ERR_KERNEL;
            return;
        }
    }
    if (cached) {
        l_copy16(P, parena + PA.off_planes, plane_bytes, lane);
        l_copy16(sRes, parena, (uint32_t)n * 4u, lane);
        if (m > 0 && mino != mino_rec) l_copy16(mino, mino_rec, (uint32_t)(n * m) * 2u, lane);
        __syncwarp();
    } else if constexpr (PM) {
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
                P[(size_t)q * n + o] = make_ulonglong2(nz, ng);
                weight += __popcll(nz);
            }
            if (weight != w) ok = false;
        }
        if (__any_sync(FULL, !ok)) {
            if (lane == 0) H->err |= XW_ERR_MINORITY;
            return;
        }
        if (m > 0 && (status0 & XW_STATUS_INIT) && mino != mino_rec)
            l_copy16(mino, mino_rec, (uint32_t)(n * m) * 2u, lane);
        __syncwarp();
    } else if (!(status0 & XW_STATUS_GRAM)) {
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

    // ---- residuals and totals from G (a cached bit-plane replica: the
    // score from its saved residuals, the other totals from its header) ----
    int p_score = 0, p_conf = 0, p_par = 0;
    long long p_sq = 0;
    if (cached) {
#pragma unroll 1
        for (int o = lane; o < n; o += 32) p_score += sRes[o];
    } else if constexpr (PM) {
        p_totals(P, G, sRes, n, nw, lane, p_score, p_conf, p_sq, p_par);
    } else {
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
    }
    const int score0 = __reduce_add_sync(FULL, p_score) / 2;
    const int conf0 = cached ? H->conflicts : __reduce_add_sync(FULL, p_conf) / 2;
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
    const int64_t obj0 = cached && obj_kind != 0 ? H->obj_total
                         : obj_kind == 1         ? sq0
                         : obj_kind == 2         ? par0
                                                 : score0;
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
        v.W = W; v.mino = mino; v.res = sRes; v.dw = sDw;
        if constexpr (PM) {
            v.mask = reinterpret_cast<const uint64_t*>(P);
            v.mrs = 2;
            v.mks = 2 * n;
            v.planes = 1;
        } else {
            v.mask = mask;
            v.mrs = nw;
            v.mks = 1;
            v.planes = 0;
        }
        v.thr_target = J->thr_target; v.thr_dbl = J->thr_double; v.thr_sign = J->thr_sign;
        v.thr_swsign = J->thr_swsign;
        v.n = n; v.w = w; v.m = m; v.sparse = sparse; v.ts = ts; v.bpc = bpc; v.cc = 31 / bpc;
        v.move_set = J->move_set; v.nw = nw;
        v.stream = stream; v.k0 = k0; v.k1 = k1;
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
    bool best_saved = false;   // bit-plane form: a best state saved in the arena this run

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
        // hybrid form: candidate c's Gram rows are staged into one of two
        // buffers while the candidate before it is evaluated; held[b] is
        // the candidate whose rows buffer b holds
        int best_cand = -1, held0 = -1, held1 = -1, cur = 0;
        uint32_t vmask = 0;
        const int ldg = gram_ld(n);
        if constexpr (PM && SG) {
            vmask = __ballot_sync(FULL, lane < count && (desc.x & 1u));
            if (vmask) {
                const int c0 = __ffs(vmask) - 1;
                int r1, r2;
                bool two;
                move_rows(__shfl_sync(FULL, desc.x, c0), r1, r2, two);
                p_stage_async(G, n, r1, r2, two, S, lane);
                held0 = c0;
            }
        }
#pragma unroll 1
        for (int c = 0; c < count; ++c) {
            LMove e;
            e.x = __shfl_sync(FULL, desc.x, c);
            if (!(e.x & 1u)) continue;
            e.y = __shfl_sync(FULL, desc.y, c);
            e.z = __shfl_sync(FULL, desc.z, c);
            const LUpdate u = l_decode(e);
            LDeltas d;
            int16_t* Sc = S;
            if constexpr (PM && SG) {
                // c is in buffer cur; the next valid candidate goes to the other
                const uint32_t rest = vmask & ~((2u << c) - 1u);
                if (rest) {
                    const int cn = __ffs(rest) - 1;
                    int r1, r2;
                    bool two;
                    move_rows(__shfl_sync(FULL, desc.x, cn), r1, r2, two);
                    p_stage_async(G, n, r1, r2, two, S + (cur ^ 1) * 2 * ldg, lane);
                    if (cur) held0 = cn;
                    else held1 = cn;
                    asm volatile("cp.async.wait_group 1;" ::: "memory");
                } else {
                    asm volatile("cp.async.wait_group 0;" ::: "memory");
                }
                __syncwarp();
                Sc = S + cur * 2 * ldg;
                cur ^= 1;
            }
            if constexpr (PM) d = p_eval<GEN, SG>(u, P, G, Sc, n, nw, lane);
            else d = l_eval<GEN>(u, W, G, n, lane);
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
                have = true; best_mv = e; bds = ds; bdc = dc; bprim = prim; best_cand = c;
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
                if constexpr (PM) {
                    l_copy16(parena + PA.off_best, P, plane_bytes, lane);
                    best_saved = true;
                } else {
                    l_copy16(best_dst, W, nn, lane);
                }
                __syncwarp();
                at_best = false;
            }
            const LUpdate u = l_decode(best_mv);
            int16_t* Sb = S;
            if constexpr (PM && SG) {
                // the buffers hold the last two evaluated candidates' rows
                if (held0 == best_cand) {
                    Sb = S;
                } else if (held1 == best_cand) {
                    Sb = S + 2 * ldg;
                } else {
                    p_stage(G, n, u.R1, u.R2, u.R2 >= 0, S, lane);
                    Sb = S;
                }
            }
            if constexpr (PM) p_commit<GEN, SG>(best_mv, u, bds, P, G, Sb, sRes, mino, n, m, nw, sparse, lane);
            else l_commit<GEN>(best_mv, u, bds, W, G, sRes, mino, mask, n, m, nw, sparse, lane);
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
    if constexpr (PM) {
        // the arena's planes and residuals, the record's W, best W and
        // minority lists from the slot
        l_copy16(parena + PA.off_planes, P, plane_bytes, lane);
        l_copy16(parena, sRes, (uint32_t)n * 4u, lane);
        if (at_best) {
            p_store_w(reinterpret_cast<int8_t*>(best_dst), P, n, lane);
        } else if (best_saved) {
            __syncwarp();
            p_store_w(reinterpret_cast<int8_t*>(best_dst),
                      reinterpret_cast<const ulonglong2*>(parena + PA.off_best), n, lane);
        }
        p_store_w(W, P, n, lane);
        if (m > 0 && mino != mino_rec) l_copy16(mino_rec, mino, (uint32_t)(n * m) * 2u, lane);
        __syncwarp();
    } else {
        if (at_best) l_copy16(best_dst, W, nn, lane);
    }
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

// CTAs of four warps per SM the register budget is sized for: the
// stored-Gram form hides HBM latency with warps; the bit-plane form holds
// two CTAs (its slots fill shared memory) and spends the registers on its
// per-lane Gram rows
#ifndef XW_LARGE_MIN_BLOCKS
#define XW_LARGE_MIN_BLOCKS 4
#endif
template <bool GEN, int FORM>
__global__ void __launch_bounds__(128, FORM != kFormGram ? 2 : XW_LARGE_MIN_BLOCKS) anneal_large_kernel(AnnealArgs a) {
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
            run_large<GEN, FORM>(a, a.items[item], slot, lane, a.iters);
            continue;
        }
        const uint32_t c = item / a.n_items;
        const uint32_t rid = a.items[item - c * a.n_items];
        const uint64_t lo = a.iters * c / a.chunks, hi = a.iters * (c + 1) / a.chunks;
        RepHeader* H = reinterpret_cast<RepHeader*>(a.arena + a.rec_off[rid]);
        const bool ok = chunk_begin(a.chunk_done + rid, c, a.chunk_wait_ns, &H->err, lane, FULL);
        if (ok) run_large<GEN, FORM>(a, rid, slot, lane, hi - lo);
        chunk_end(a.chunk_done + rid, c, ok, lane, FULL);
    }
}

}  // namespace

bool anneal_large_planes_fit(int n, int m) { return large_planes_fit(n, m); }

uint32_t anneal_large_slot_bytes(int n, int m, int form) { return large_slot(n, m, form).bytes; }

uint64_t anneal_large_arena_bytes(int n, int form) {
    const uint64_t b = form == kFormGram ? large_gram(n).bytes : planes_arena(n, form == kFormHybrid).bytes;
    return (b + 255u) & ~uint64_t(255);
}

const void* anneal_large_kernel_fn(bool general, int form) {
    if (form == kFormPlanes)
        return general ? reinterpret_cast<const void*>(&anneal_large_kernel<true, kFormPlanes>)
                       : reinterpret_cast<const void*>(&anneal_large_kernel<false, kFormPlanes>);
    if (form == kFormHybrid)
        return general ? reinterpret_cast<const void*>(&anneal_large_kernel<true, kFormHybrid>)
                       : reinterpret_cast<const void*>(&anneal_large_kernel<false, kFormHybrid>);
    return general ? reinterpret_cast<const void*>(&anneal_large_kernel<true, kFormGram>)
                   : reinterpret_cast<const void*>(&anneal_large_kernel<false, kFormGram>);
}

cudaError_t launch_anneal_large(const AnnealArgs& args, bool general, int form, int warps_per_block, int blocks,
                                cudaStream_t stream) {
    const size_t smem = (size_t)warps_per_block * args.slot_bytes;
    const dim3 grid(blocks), block(32 * warps_per_block);
    void* kargs[] = {const_cast<AnnealArgs*>(&args)};
    return cudaLaunchKernel(anneal_large_kernel_fn(general, form), grid, block, kargs, smem, stream);
}

}  // namespace xw
