// xw_anneal.cu -- the population annealing kernel for weighing matrices.
//
// One warp owns one replica at a time.  The replica's int8 W (column-major),
// int32 Gram, row residuals, minority lists and row support masks live in the
// warp's shared-memory slot; lane o owns "other" rows o, o+32, ... of every
// O(n) delta, so a candidate's exact change to W W^T and to the score is one
// pass over registers and shared memory plus one redux.sync.  The whole
// iteration is warp-synchronous: no __syncthreads, no block-wide reductions.
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
// Work distribution is persistent: each warp takes replica ids from a
// global counter until the launch's item list is exhausted, so replicas of
// different orders and weights share one launch.
#include <cuda_runtime.h>

#include "xw_device.cuh"
#include "xw_kernels.h"

namespace xw {

namespace {

constexpr unsigned FULL = 0xffffffffu;

struct SlotLayout {
    uint32_t off_g, off_res, off_mino, off_mask, off_draws, bytes;
    int ld;
};

__host__ __device__ inline SlotLayout slot_layout(int n, int m) {
    SlotLayout L;
    L.ld = n | 1;
    const uint32_t nn = (uint32_t)(n * n);
    L.off_g = xw_pad16(nn);
    L.off_res = L.off_g + xw_pad16((uint32_t)(n * L.ld) * 4u);
    L.off_mino = L.off_res + xw_pad16((uint32_t)n * 4u);
    L.off_mask = L.off_mino + xw_pad16((uint32_t)(n * m));
    L.off_draws = L.off_mask + xw_pad16((uint32_t)n * 16u);
    L.bytes = L.off_draws + 32u * 16u;
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

// Per-lane view of a replica for the scalar proposal code.
struct View {
    const int8_t* W;
    const uint8_t* mino;
    const int32_t* res;
    const uint64_t* mask;      // 2 words per row: nonzero support
    const uint32_t* dw;        // cached draw words
    int n, w, m, sparse, ts, bpc, cc;
    uint64_t it;
    uint32_t stream, k0, k1;
    uint64_t valid_lo, valid_hi;

    __device__ __forceinline__ int at(int r, int c) const { return W[c * n + r]; }

    __device__ __forceinline__ uint32_t word(int c, int b, int j) const {
        if (c < cc && b < bpc) return dw[(1 + c * bpc + b) * 4 + j];
        return pick(draw_block(cand_slot(c, b), it, stream, k0, k1), j);
    }

    __device__ __forceinline__ uint32_t index(int c, int b, int j, uint32_t count) const {
        uint32_t out;
        if (lemire_ok(word(c, b, j), count, out)) return out;
        return lemire_retry(cand_slot(c, b), it, stream, k0, k1, j, count);
    }
};

struct Move {
    int kind, r1, r2, c1, c2, p1, p2, v1, v2;
};

__device__ __forceinline__ uint32_t pack0(const Move& mv) {
    return 1u | ((uint32_t)mv.kind << 1) | ((uint32_t)mv.r1 << 3) | ((uint32_t)mv.r2 << 10) |
           ((uint32_t)mv.c1 << 17) | ((uint32_t)mv.c2 << 24);
}
__device__ __forceinline__ uint32_t pack1(const Move& mv) {
    return (uint32_t)(mv.v1 + 1) | ((uint32_t)(mv.v2 + 1) << 2) | ((uint32_t)mv.p1 << 4) |
           ((uint32_t)mv.p2 << 11);
}

// propose_sign_flip (xweigh_cuda.cu:302-325): a nonzero of `row`, from the
// minority list when the row is sparse, else the first nonzero at or after
// a random column.
__device__ bool d_flip(const View& v, int c, int b, int j, int row, Move& mv) {
    int col;
    if (v.sparse && v.m > 0) {
        col = v.mino[row * v.m + (int)v.index(c, b, j, (uint32_t)v.m)];
    } else {
        const int start = (int)v.index(c, b, j, (uint32_t)v.n);
        col = cyclic_first(v.mask[2 * row], v.mask[2 * row + 1], start);
        if (col < 0) return false;
    }
    mv.kind = 0; mv.r1 = row; mv.c1 = col; mv.r2 = 0; mv.c2 = 0;
    mv.p1 = 0; mv.p2 = 0; mv.v1 = 0; mv.v2 = 0;
    return true;
}

// hot_row (xweigh_cuda.cu:291-300), serial form
__device__ int d_hot_row(const View& v, int c) {
    int best = (int)v.index(c, 4, 0, (uint32_t)v.n);
    for (int k = 1; k < v.ts; ++k) {
        const int cand = (int)v.index(c, 4 + k / 4, k % 4, (uint32_t)v.n);
        if (v.res[cand] > v.res[best]) best = cand;
    }
    return best;
}

// propose_double_sign_flip (xweigh_cuda.cu:389-421)
__device__ bool d_double(const View& v, int c, int row1, Move& mv) {
    Move first;
    if (!d_flip(v, c, 2, 3, row1, first)) return false;
    for (int a = 0; a < 16; ++a) {
        const int b = a == 0 ? 3 : 20 + (a - 1);
        const int row2 = v.word(c, b, 0) < 0x80000000u ? row1 : (int)v.index(c, b, 1, (uint32_t)v.n);
        Move second;
        if (!d_flip(v, c, b, 2, row2, second)) continue;
        if (first.r1 == second.r1 && first.c1 == second.c1) continue;
        mv.kind = 2; mv.r1 = first.r1; mv.c1 = first.c1; mv.r2 = second.r1; mv.c2 = second.c1;
        mv.p1 = 0; mv.p2 = 0; mv.v1 = 0; mv.v2 = 0;
        return true;
    }
    return false;
}

// propose_support_switch (xweigh_cuda.cu:327-387)
__device__ bool d_switch(const View& v, int c, int row1, uint64_t thr_swsign, Move& mv) {
    if (v.m == 0 || v.n < 2) return false;
    for (int a = 0; a < 24; ++a) {
        int br, jr, bp1, jp1, bp2, jp2, bs1, js1, bs2, js2;
        if (a == 0) {
            br = 1; jr = 1; bp1 = 1; jp1 = 2; bp2 = 1; jp2 = 3; bs1 = 2; js1 = 0; bs2 = 2; js2 = 1;
        } else {
            const int B = 36 + 2 * (a - 1);
            br = B; jr = 0; bp1 = B; jp1 = 1; bp2 = B; jp2 = 2; bs1 = B; js1 = 3; bs2 = B + 1; js2 = 0;
        }
        int row2 = (int)v.index(c, br, jr, (uint32_t)(v.n - 1));
        if (row2 >= row1) ++row2;
        const int p1 = (int)v.index(c, bp1, jp1, (uint32_t)v.m);
        const int p2 = (int)v.index(c, bp2, jp2, (uint32_t)v.m);
        int c1, c2;
        if (v.sparse) { c1 = v.mino[row1 * v.m + p1]; c2 = v.mino[row2 * v.m + p2]; }
        else { c2 = v.mino[row1 * v.m + p1]; c1 = v.mino[row2 * v.m + p2]; }
        if (c1 == c2 || v.at(row1, c2) != 0 || v.at(row2, c1) != 0) continue;
        const int v1 = v.at(row1, c1), v2 = v.at(row2, c2);
        if (v1 == 0 || v2 == 0) continue;
        mv.kind = 1; mv.r1 = row1; mv.r2 = row2; mv.c1 = c1; mv.c2 = c2; mv.p1 = p1; mv.p2 = p2;
        mv.v1 = (uint64_t)v.word(c, bs1, js1) < thr_swsign ? -v1 : v1;
        mv.v2 = (uint64_t)v.word(c, bs2, js2) < thr_swsign ? -v2 : v2;
        return true;
    }
    return false;
}

// within-row swap: a nonzero of the row moves to one of its zeros
__device__ bool d_row_swap(const View& v, int c, int row, Move& mv) {
    if (v.m == 0) return false;
    const uint64_t nz_lo = v.mask[2 * row], nz_hi = v.mask[2 * row + 1];
    int c1, c2, pos;
    if (v.sparse) {
        pos = (int)v.index(c, 1, 1, (uint32_t)v.m);
        c1 = v.mino[row * v.m + pos];
        c2 = cyclic_first(~nz_lo & v.valid_lo, ~nz_hi & v.valid_hi, (int)v.index(c, 1, 2, (uint32_t)v.n));
        if (c2 < 0) return false;
    } else {
        pos = (int)v.index(c, 1, 2, (uint32_t)v.m);
        c2 = v.mino[row * v.m + pos];
        c1 = cyclic_first(nz_lo, nz_hi, (int)v.index(c, 1, 1, (uint32_t)v.n));
        if (c1 < 0) return false;
    }
    mv.kind = 3; mv.r1 = row; mv.r2 = 0; mv.c1 = c1; mv.c2 = c2; mv.p1 = pos; mv.p2 = 0;
    mv.v1 = v.word(c, 1, 3) < 0x80000000u ? 1 : -1;
    mv.v2 = 0;
    return true;
}

struct Thresholds {
    uint64_t target, dbl, sign, swsign;
};

__device__ bool d_propose(const View& v, int c, int move_set, const Thresholds& th,
                          bool coop_ok, int coop_row, Move& mv) {
    const bool targeted = (uint64_t)v.word(c, 0, 0) < th.target;
    const int row = targeted ? (coop_ok ? coop_row : d_hot_row(v, c))
                             : (int)v.index(c, 0, 1, (uint32_t)v.n);
    if (move_set == 1) {
        if (v.w == v.n || (uint64_t)v.word(c, 0, 3) < th.sign) return d_flip(v, c, 1, 0, row, mv);
        if (d_row_swap(v, c, row, mv)) return true;
        return d_flip(v, c, 2, 2, row, mv);
    }
    if ((uint64_t)v.word(c, 0, 2) < th.dbl && d_double(v, c, row, mv)) return true;
    if (v.w == v.n || (uint64_t)v.word(c, 0, 3) < th.sign) return d_flip(v, c, 1, 0, row, mv);
    if (d_switch(v, c, row, th.swsign, mv)) return true;
    return d_flip(v, c, 2, 2, row, mv);
}

struct Deltas {
    int ds, dc, dsq, dpar;
};

__device__ __forceinline__ void acc(Deltas& d, int old, int nw) {
    const int ao = iabs(old), an = iabs(nw);
    d.ds += an - ao;
    d.dc += (nw != 0) - (old != 0);
    d.dsq += nw * nw - old * old;
    d.dpar += (an & 1) - (ao & 1);
}

// evaluate_move_warp (xweigh_cuda.cu:449-599): lane-partial deltas over the
// lane's own rows; the caller reduces them across the warp.
template <int OPL>
__device__ __forceinline__ Deltas eval_lane(int kind, int r1, int r2, int c1, int c2, int nv1, int nv2,
                                            const int8_t* W, const int32_t* G, int n, int ld, int lane) {
    Deltas d = {0, 0, 0, 0};
    if (kind == 0) {
        const int ch = -2 * W[c1 * n + r1];
#pragma unroll
        for (int k = 0; k < OPL; ++k) {
            const int o = lane + 32 * k;
            if (o < n && o != r1) {
                const int old = G[r1 * ld + o];
                acc(d, old, old + ch * W[c1 * n + o]);
            }
        }
    } else if (kind == 1) {
        const int v1 = W[c1 * n + r1], v2 = W[c2 * n + r2];
#pragma unroll
        for (int k = 0; k < OPL; ++k) {
            const int o = lane + 32 * k;
            if (o < n && o != r1 && o != r2) {
                const int o1 = G[r1 * ld + o], o2 = G[r2 * ld + o];
                const int w1 = W[c1 * n + o], w2 = W[c2 * n + o];
                acc(d, o1, o1 + nv1 * w2 - v1 * w1);
                acc(d, o2, o2 + nv2 * w1 - v2 * w2);
            }
        }
    } else if (kind == 2) {
        const int ch1 = -2 * W[c1 * n + r1], ch2 = -2 * W[c2 * n + r2];
        if (r1 == r2) {
#pragma unroll
            for (int k = 0; k < OPL; ++k) {
                const int o = lane + 32 * k;
                if (o < n && o != r1) {
                    const int old = G[r1 * ld + o];
                    acc(d, old, old + ch1 * W[c1 * n + o] + ch2 * W[c2 * n + o]);
                }
            }
        } else {
#pragma unroll
            for (int k = 0; k < OPL; ++k) {
                const int o = lane + 32 * k;
                if (o < n && o != r1 && o != r2) {
                    const int o1 = G[r1 * ld + o], o2 = G[r2 * ld + o];
                    acc(d, o1, o1 + ch1 * W[c1 * n + o]);
                    acc(d, o2, o2 + ch2 * W[c2 * n + o]);
                }
            }
            if (lane == 0) {
                const int op = G[r1 * ld + r2];
                acc(d, op, op + ch1 * W[c1 * n + r2] + ch2 * W[c2 * n + r1] + (c1 == c2 ? ch1 * ch2 : 0));
            }
        }
    } else {
        const int v = W[c1 * n + r1];
#pragma unroll
        for (int k = 0; k < OPL; ++k) {
            const int o = lane + 32 * k;
            if (o < n && o != r1) {
                const int old = G[r1 * ld + o];
                acc(d, old, old + nv1 * W[c2 * n + o] - v * W[c1 * n + o]);
            }
        }
    }
    return d;
}

__device__ __forceinline__ void set_pair(int32_t* G, int32_t* res, int ld, int a, int o, int old, int nw, int& d) {
    d = iabs(nw) - iabs(old);
    G[a * ld + o] = nw;
    G[o * ld + a] = nw;
    res[o] += d;
}

__device__ __forceinline__ void mask_move(uint64_t* mask, int row, int from, int to) {
    mask[2 * row + (from >> 6)] &= ~(1ull << (from & 63));
    mask[2 * row + (to >> 6)] |= 1ull << (to & 63);
}

// commit_sign_flip / commit_support_switch / commit_double_sign_flip
// (xweigh_cuda.cu:607-877) and the within-row swap.
template <int OPL>
__device__ void commit(int kind, int r1, int r2, int c1, int c2, int nv1, int nv2, int p1, int p2,
                       int ds, int8_t* W, int32_t* G, int32_t* res, uint8_t* mino, uint64_t* mask,
                       int n, int ld, int m, int sparse, int lane) {
    if (kind == 0) {
        const int ch = -2 * W[c1 * n + r1];
#pragma unroll
        for (int k = 0; k < OPL; ++k) {
            const int o = lane + 32 * k;
            if (o < n && o != r1) {
                const int old = G[r1 * ld + o];
                int d;
                set_pair(G, res, ld, r1, o, old, old + ch * W[c1 * n + o], d);
            }
        }
        __syncwarp();
        if (lane == 0) {
            res[r1] += ds;
            W[c1 * n + r1] = (int8_t)-W[c1 * n + r1];
        }
    } else if (kind == 1) {
        const int v1 = W[c1 * n + r1], v2 = W[c2 * n + r2];
        int s1 = 0;
#pragma unroll
        for (int k = 0; k < OPL; ++k) {
            const int o = lane + 32 * k;
            if (o < n && o != r1 && o != r2) {
                const int o1 = G[r1 * ld + o], o2 = G[r2 * ld + o];
                const int w1 = W[c1 * n + o], w2 = W[c2 * n + o];
                int d1, d2;
                set_pair(G, res, ld, r1, o, o1, o1 + nv1 * w2 - v1 * w1, d1);
                set_pair(G, res, ld, r2, o, o2, o2 + nv2 * w1 - v2 * w2, d2);
                s1 += d1;
            }
        }
        const int S1 = __reduce_add_sync(FULL, s1);
        __syncwarp();
        if (lane == 0) {
            res[r1] += S1;
            res[r2] += ds - S1;
            W[c1 * n + r1] = 0;
            W[c2 * n + r2] = 0;
            W[c2 * n + r1] = (int8_t)nv1;
            W[c1 * n + r2] = (int8_t)nv2;
            if (sparse) { mino[r1 * m + p1] = (uint8_t)c2; mino[r2 * m + p2] = (uint8_t)c1; }
            else { mino[r1 * m + p1] = (uint8_t)c1; mino[r2 * m + p2] = (uint8_t)c2; }
            mask_move(mask, r1, c1, c2);
            mask_move(mask, r2, c2, c1);
        }
    } else if (kind == 2) {
        const int ch1 = -2 * W[c1 * n + r1], ch2 = -2 * W[c2 * n + r2];
        if (r1 == r2) {
#pragma unroll
            for (int k = 0; k < OPL; ++k) {
                const int o = lane + 32 * k;
                if (o < n && o != r1) {
                    const int old = G[r1 * ld + o];
                    int d;
                    set_pair(G, res, ld, r1, o, old, old + ch1 * W[c1 * n + o] + ch2 * W[c2 * n + o], d);
                }
            }
            __syncwarp();
            if (lane == 0) res[r1] += ds;
        } else {
            int s1 = 0;
#pragma unroll
            for (int k = 0; k < OPL; ++k) {
                const int o = lane + 32 * k;
                if (o < n && o != r1 && o != r2) {
                    const int o1 = G[r1 * ld + o], o2 = G[r2 * ld + o];
                    int d1, d2;
                    set_pair(G, res, ld, r1, o, o1, o1 + ch1 * W[c1 * n + o], d1);
                    set_pair(G, res, ld, r2, o, o2, o2 + ch2 * W[c2 * n + o], d2);
                    s1 += d1;
                }
            }
            const int S1 = __reduce_add_sync(FULL, s1);
            __syncwarp();
            if (lane == 0) {
                const int op = G[r1 * ld + r2];
                const int np = op + ch1 * W[c1 * n + r2] + ch2 * W[c2 * n + r1] + (c1 == c2 ? ch1 * ch2 : 0);
                const int pd = iabs(np) - iabs(op);
                G[r1 * ld + r2] = np;
                G[r2 * ld + r1] = np;
                res[r1] += S1 + pd;
                res[r2] += ds - S1;
            }
        }
        if (lane == 0) {
            W[c1 * n + r1] = (int8_t)-W[c1 * n + r1];
            W[c2 * n + r2] = (int8_t)-W[c2 * n + r2];
        }
    } else {
        const int v = W[c1 * n + r1];
#pragma unroll
        for (int k = 0; k < OPL; ++k) {
            const int o = lane + 32 * k;
            if (o < n && o != r1) {
                const int old = G[r1 * ld + o];
                int d;
                set_pair(G, res, ld, r1, o, old, old + nv1 * W[c2 * n + o] - v * W[c1 * n + o], d);
            }
        }
        __syncwarp();
        if (lane == 0) {
            res[r1] += ds;
            W[c1 * n + r1] = 0;
            W[c2 * n + r1] = (int8_t)nv1;
            mino[r1 * m + p1] = (uint8_t)(sparse ? c2 : c1);
            mask_move(mask, r1, c1, c2);
        }
    }
    __syncwarp();
}

__device__ __forceinline__ void copy16(void* dst, const void* src, uint32_t bytes, int lane) {
    const uint32_t chunks = xw_pad16(bytes) / 16u;
    uint4* d = reinterpret_cast<uint4*>(dst);
    const uint4* s = reinterpret_cast<const uint4*>(src);
    for (uint32_t i = lane; i < chunks; i += 32) d[i] = s[i];
}

__device__ __forceinline__ uint64_t globaltimer() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

template <int OPL>
__device__ void run_replica(const AnnealArgs& a, uint32_t rid, uint8_t* slot, int lane) {
    uint8_t* rec = a.arena + a.rec_off[rid];
    RepHeader* H = reinterpret_cast<RepHeader*>(rec);
    const uint32_t jid = H->job;
    XwJob* J = a.jobs + jid;
    if (*(volatile int32_t*)&J->done) return;
    if (a.stop_on_solve && *(volatile int32_t*)&J->solved) return;

    const int n = J->n, w = J->w, m = J->m, sparse = J->sparse;
    const SlotLayout L = slot_layout(n, m);
    const int ld = L.ld;
    int8_t* sW = reinterpret_cast<int8_t*>(slot);
    int32_t* sG = reinterpret_cast<int32_t*>(slot + L.off_g);
    int32_t* sRes = reinterpret_cast<int32_t*>(slot + L.off_res);
    uint8_t* sMino = slot + L.off_mino;
    uint64_t* sMask = reinterpret_cast<uint64_t*>(slot + L.off_mask);
    uint4* sDraw = reinterpret_cast<uint4*>(slot + L.off_draws);
    const uint32_t* sDw = reinterpret_cast<const uint32_t*>(sDraw);

    uint64_t it = H->it;
    uint64_t iters = a.iters;
    if (J->budget_iters) {
        if (it >= J->budget_iters) return;
        if (iters > J->budget_iters - it) iters = J->budget_iters - it;
    }

    // ---- load W and the minority lists; rebuild masks, Gram, residuals ----
    const uint32_t nn = (uint32_t)(n * n);
    copy16(sW, rec + J->off_w, nn, lane);
    const uint32_t status0 = H->status;
    if (m > 0 && (status0 & XW_STATUS_INIT)) copy16(sMino, rec + J->off_mino, (uint32_t)(n * m), lane);
    __syncwarp();
    int bad_rows = 0;
#pragma unroll
    for (int k = 0; k < OPL; ++k) {
        const int o = lane + 32 * k;
        if (o < n) {
            uint64_t lo = 0, hi = 0;
            int pos = 0;
            for (int c = 0; c < n; ++c) {
                const bool nz = sW[c * n + o] != 0;
                if (nz) { if (c < 64) lo |= 1ull << c; else hi |= 1ull << (c - 64); }
                if (m > 0 && !(status0 & XW_STATUS_INIT) && nz == (sparse != 0)) {
                    if (pos < m) sMino[o * m + pos] = (uint8_t)c;
                    ++pos;
                }
            }
            sMask[2 * o] = lo;
            sMask[2 * o + 1] = hi;
            if (__popcll(lo) + __popcll(hi) != w) bad_rows = 1;
            if (m > 0 && !(status0 & XW_STATUS_INIT) && pos != m) bad_rows = 1;
        }
    }
    if (__any_sync(FULL, bad_rows)) {
        if (lane == 0) H->err |= XW_ERR_MINORITY;
        return;
    }
    __syncwarp();
    int p_score = 0, p_conf = 0, p_sq = 0, p_par = 0;
#pragma unroll
    for (int k = 0; k < OPL; ++k) {
        const int o = lane + 32 * k;
        if (o < n) {
            int r_sum = 0;
            for (int r = 0; r < n; ++r) {
                int dot = 0;
                for (int c = 0; c < n; ++c) dot += sW[c * n + r] * sW[c * n + o];
                sG[r * ld + o] = dot;
                if (r != o) {
                    const int ad = iabs(dot);
                    r_sum += ad;
                    p_conf += dot != 0;
                    p_sq += dot * dot;
                    p_par += ad & 1;
                }
            }
            sRes[o] = r_sum;
            p_score += r_sum;
        }
    }
    const int score0 = __reduce_add_sync(FULL, p_score) / 2;
    const int conf0 = __reduce_add_sync(FULL, p_conf) / 2;
    const int sq0 = __reduce_add_sync(FULL, p_sq) / 2;
    const int par0 = __reduce_add_sync(FULL, p_par) / 2;
    __syncwarp();

    const int obj_kind = H->obj_kind;
    const int64_t obj0 = obj_kind == 1 ? sq0 : obj_kind == 2 ? par0 : score0;
    int score, conflicts, best_s, best_c, msi, cool;
    int64_t obj_total;
    uint64_t moves, cand_evals;
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
        copy16(rec + J->off_best, sW, nn, lane);
    }
    score = score0;
    conflicts = conf0;
    obj_total = obj0;

    // ---- job constants ----
    const int tempering = J->tempering, move_set = J->move_set;
    const int cs = J->candidate_samples, ts = J->target_samples;
    const int mpc = J->moves_per_cool, stuck = J->stuck_threshold;
    const uint32_t k0 = J->key0, k1 = J->key1, stream = H->stream;
    const uint64_t thr_greedy = J->thr_greedy;
    Thresholds th;
    th.target = J->thr_target; th.dbl = J->thr_double; th.sign = J->thr_sign; th.swsign = J->thr_swsign;
    const double t_min = J->t_min, cooling = J->cooling, reheat = J->reheat;
    const int bpc = 4 + (ts <= 4 ? 1 : 2);          // cached blocks per candidate
    const int cc = 31 / bpc;                        // cached candidates
    const bool coop = ts <= 8;                      // cooperative hot-row tournament

    View v;
    v.W = sW; v.mino = sMino; v.res = sRes; v.mask = sMask; v.dw = sDw;
    v.n = n; v.w = w; v.m = m; v.sparse = sparse; v.ts = ts; v.bpc = bpc; v.cc = cc;
    v.stream = stream; v.k0 = k0; v.k1 = k1;
    v.valid_lo = n >= 64 ? ~0ull : ((1ull << n) - 1ull);
    v.valid_hi = n <= 64 ? 0ull : (n == 128 ? ~0ull : ((1ull << (n - 64)) - 1ull));

    // lane -> cached Philox block of this iteration
    uint32_t my_slot = 0;
    if (lane > 0) {
        const int q = lane - 1, c = q / bpc, b = q - c * bpc;
        my_slot = cand_slot(c, b);
    }

    uint64_t done = 0;
    for (; done < iters; ++done) {
        if (a.stop_on_solve) {
            if (best_s == 0) break;
            if ((done & 63) == 63 && *(volatile int32_t*)&J->solved) break;
        }
        v.it = it;
        // A: draws
        sDraw[lane] = draw_block(my_slot, it, stream, k0, k1);
        __syncwarp();
        const uint4 mblk = sDraw[0];
        const int count = (uint64_t)mblk.x < thr_greedy ? cs : 1;

        // C: cooperative hot-row tournaments for candidates 0..3
        int hot_key = 0;
        if (coop) {
            const int c = lane >> 3, s = lane & 7;
            if (c < count && s < ts) {
                const uint32_t word = sDw[(1 + c * bpc + 4 + (s >> 2)) * 4 + (s & 3)];
                uint32_t row;
                if (!lemire_ok(word, (uint32_t)n, row))
                    row = lemire_retry(cand_slot(c, 4 + (s >> 2)), it, stream, k0, k1, s & 3, (uint32_t)n);
                hot_key = (sRes[row] << 13) | ((31 - s) << 8) | (int)row;
            }
            hot_key = max(hot_key, __shfl_xor_sync(FULL, hot_key, 1));
            hot_key = max(hot_key, __shfl_xor_sync(FULL, hot_key, 2));
            hot_key = max(hot_key, __shfl_xor_sync(FULL, hot_key, 4));
        }
        const int coop_row = __shfl_sync(FULL, hot_key, (lane & 3) << 3) & 0xff;

        // D: proposals, lane c proposes candidate c
        uint32_t d0 = 0, d1 = 0;
        if (lane < count) {
            Move mv;
            if (d_propose(v, lane, move_set, th, coop && lane < 4, coop_row, mv)) {
                d0 = pack0(mv);
                d1 = pack1(mv);
            }
        }
        __syncwarp();

        // E: evaluate in candidate order, keep the first best
        bool have = false;
        uint32_t b0 = 0, b1 = 0;
        int bds = 0, bdc = 0, bprim = 0;
        for (int c = 0; c < count; ++c) {
            const uint32_t e0 = __shfl_sync(FULL, d0, c);
            const uint32_t e1 = __shfl_sync(FULL, d1, c);
            if (!(e0 & 1u)) continue;
            const int kind = (e0 >> 1) & 3, r1 = (e0 >> 3) & 127, r2 = (e0 >> 10) & 127;
            const int c1 = (e0 >> 17) & 127, c2 = (e0 >> 24) & 127;
            const int nv1 = (int)(e1 & 3) - 1, nv2 = (int)((e1 >> 2) & 3) - 1;
            const Deltas d = eval_lane<OPL>(kind, r1, r2, c1, c2, nv1, nv2, sW, sG, n, ld, lane);
            const int packed = __reduce_add_sync(FULL, d.ds * 4096 + d.dc);
            const int dc = ((packed + 2048) & 4095) - 2048;
            const int ds = (packed - dc) >> 12;
            int prim = ds;
            if (obj_kind == 1) prim = __reduce_add_sync(FULL, d.dsq);
            else if (obj_kind == 2) prim = __reduce_add_sync(FULL, d.dpar);
            ++cand_evals;
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
        const bool accept = bprim <= 0 || metropolis_accept(bprim, T, mblk.y);

        // G: commit
        if (accept) {
            const int kind = (b0 >> 1) & 3, r1 = (b0 >> 3) & 127, r2 = (b0 >> 10) & 127;
            const int c1 = (b0 >> 17) & 127, c2 = (b0 >> 24) & 127;
            const int nv1 = (int)(b1 & 3) - 1, nv2 = (int)((b1 >> 2) & 3) - 1;
            const int p1 = (b1 >> 4) & 127, p2 = (b1 >> 11) & 127;
            commit<OPL>(kind, r1, r2, c1, c2, nv1, nv2, p1, p2, bds, sW, sG, sRes, sMino, sMask,
                        n, ld, m, sparse, lane);
            score += bds;
            conflicts += bdc;
            obj_total += bprim;
        }

        // H: best tracking, cooling, reheat
        if (score < best_s || (score == best_s && conflicts < best_c)) {
            best_s = score;
            best_c = conflicts;
            msi = 0;
            copy16(rec + J->off_best, sW, nn, lane);
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
        }
        ++it;
    }

    // ---- write back ----
    __syncwarp();
    copy16(rec + J->off_w, sW, nn, lane);
    if (m > 0) copy16(rec + J->off_mino, sMino, (uint32_t)(n * m), lane);
    if (lane == 0) {
        H->it = it;
        H->moves = moves;
        H->cand_evals = cand_evals;
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
    __syncwarp();
}

template <int OPL>
__global__ void __launch_bounds__(128, 6) anneal_kernel(AnnealArgs a) {
    extern __shared__ __align__(16) uint8_t smem[];
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    uint8_t* slot = smem + (size_t)warp * a.slot_bytes;
    for (;;) {
        uint32_t item = 0;
        if (lane == 0) item = atomicAdd(a.counter, 1u);
        item = __shfl_sync(FULL, item, 0);
        if (item >= a.n_items) break;
        run_replica<OPL>(a, a.items[item], slot, lane);
    }
}

// One thread per tempering job: adjacent-rung sweep of
// xweigh_anneal.hpp:1187-1221 on the device draw stream.
__global__ void exchange_kernel(XwJob* jobs, int njobs, uint8_t* arena, const uint64_t* rec_off,
                                const double* ladder) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= njobs) return;
    XwJob& J = jobs[j];
    if (!J.tempering || J.done || J.solved || J.replicas < 2 || J.replicas > XW_MAX_RUNGS) return;
    const int R = J.replicas;
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

}  // namespace

uint32_t anneal_slot_bytes(int n, int m) { return slot_layout(n, m).bytes; }

int anneal_opl(int n) { return n <= 32 ? 1 : n <= 64 ? 2 : 4; }

const void* anneal_kernel_fn(int opl) {
    if (opl == 1) return reinterpret_cast<const void*>(&anneal_kernel<1>);
    if (opl == 2) return reinterpret_cast<const void*>(&anneal_kernel<2>);
    return reinterpret_cast<const void*>(&anneal_kernel<4>);
}

cudaError_t launch_anneal(const AnnealArgs& args, int opl, int warps_per_block, int blocks,
                          cudaStream_t stream) {
    const size_t smem = (size_t)warps_per_block * args.slot_bytes;
    const dim3 grid(blocks), block(32 * warps_per_block);
    if (opl == 1) anneal_kernel<1><<<grid, block, smem, stream>>>(args);
    else if (opl == 2) anneal_kernel<2><<<grid, block, smem, stream>>>(args);
    else anneal_kernel<4><<<grid, block, smem, stream>>>(args);
    return cudaGetLastError();
}

cudaError_t launch_exchange(XwJob* jobs, int njobs, uint8_t* arena, const uint64_t* rec_off,
                            const double* ladder, cudaStream_t stream) {
    if (njobs <= 0) return cudaSuccess;
    exchange_kernel<<<(njobs + 127) / 128, 128, 0, stream>>>(jobs, njobs, arena, rec_off, ladder);
    return cudaGetLastError();
}

}  // namespace xw

// ---- result collection --------------------------------------------------
namespace xw {

namespace {

// One warp per job: best replica by (best score, best conflicts, replica
// index) -- select_best_replica, xweigh_cuda.cu:1342-1354 -- summed
// counters, and a copy of the best replica's best W into a compact buffer.
__global__ void collect_kernel(const XwJob* jobs, int njobs, const uint8_t* arena,
                               const uint64_t* rec_off, const uint64_t* best_out_off,
                               JobOut* out, int8_t* best_out) {
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (warp >= njobs) return;
    const XwJob& J = jobs[warp];
    int64_t bs = INT64_MAX, bc = INT64_MAX;
    int br = 0x7fffffff;
    uint64_t moves = 0, evals = 0, iters = 0;
    uint32_t err = 0;
    for (int r = lane; r < J.replicas; r += 32) {
        const RepHeader* H = reinterpret_cast<const RepHeader*>(arena + rec_off[J.rep_begin + r]);
        const int64_t s = H->best_score, c = H->best_conflicts;
        if (s < bs || (s == bs && (c < bc || (c == bc && r < br)))) { bs = s; bc = c; br = r; }
        moves += H->moves;
        evals += H->cand_evals;
        iters = iters > H->it ? iters : H->it;
        err |= H->err;
    }
    for (int off = 16; off > 0; off >>= 1) {
        const int64_t s2 = __shfl_xor_sync(FULL, bs, off), c2 = __shfl_xor_sync(FULL, bc, off);
        const int r2 = __shfl_xor_sync(FULL, br, off);
        if (s2 < bs || (s2 == bs && (c2 < bc || (c2 == bc && r2 < br)))) { bs = s2; bc = c2; br = r2; }
        moves += __shfl_xor_sync(FULL, moves, off);
        evals += __shfl_xor_sync(FULL, evals, off);
        const uint64_t i2 = __shfl_xor_sync(FULL, iters, off);
        iters = iters > i2 ? iters : i2;
        err |= __shfl_xor_sync(FULL, err, off);
    }
    if (lane == 0) {
        JobOut o;
        o.score = bs; o.conflicts = bc; o.best_replica = br;
        o.solved = J.solved; o.err = (int32_t)err; o.pad = 0;
        o.moves = moves; o.cand_evals = evals; o.iters = iters;
        o.solved_it = J.solved_it; o.solve_ns = J.solve_ns;
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

}  // namespace

cudaError_t launch_collect(const XwJob* jobs, int njobs, const uint8_t* arena, const uint64_t* rec_off,
                           const uint64_t* best_out_off, JobOut* out, int8_t* best_out,
                           cudaStream_t stream) {
    if (njobs <= 0) return cudaSuccess;
    collect_kernel<<<(njobs + 3) / 4, 128, 0, stream>>>(jobs, njobs, arena, rec_off, best_out_off, out,
                                                         best_out);
    return cudaGetLastError();
}

cudaError_t launch_mark_t0(uint64_t* t0, cudaStream_t stream) {
    mark_t0_kernel<<<1, 1, 0, stream>>>(t0);
    return cudaGetLastError();
}

}  // namespace xw
