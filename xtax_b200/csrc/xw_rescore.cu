// xw_rescore.cu -- exact batched W W^T on the 5th-generation tensor cores.
//
// Full rescoring and verification of a batch of ternary matrices (the
// reference does this on the CPU, one matrix at a time: rebuild_gram_bits /
// verify_weighing, xweigh_anneal.hpp:239-264 and 429-453).  Per matrix it
// returns the L1 score sum_{i<j}|G_ij|, the conflicts #{i<j: G_ij != 0},
// the squared score sum_{i<j} G_ij^2 and the exact flag (G = wI), and
// optionally G itself, with G = W W^T computed in int32 by
// tcgen05.mma.kind::i8 -- exact, since |G_ij| <= n.
//
// Input: `count` row-major n x n int8 matrices, contiguous.  A tile is 128
// rows of that array (4 matrices of n=32, 2 of n=64, 1 of n=96 or 128),
// loaded by TMA with 128-byte swizzle into shared memory, the K (column)
// extent zero-filled to 128.  One MMA chain computes D = A A^T (M = 128,
// N = rows of the tile, K in ceil(n/32) steps of 32: the zero-filled
// columns past n are not multiplied) into a TMEM
// accumulator; the diagonal n x n blocks of D are the tile's Gram matrices.
// The epilogue warps read their TMEM lane quarter (one row per thread) and
// reduce the row statistics per matrix.  The kernel is persistent (two
// CTAs per SM) and warp-specialised: per CTA a producer warp keeps a 6-tile
// TMA ring full, an MMA warp fills two TMEM accumulators in turn, and two
// groups of four epilogue warps drain them, each step waiting only on the
// mbarrier of its stage or accumulator, so that loads, MMAs and epilogues of
// successive tiles overlap.  The bound is HBM: n^2 bytes read per matrix against 2n^3
// MACs.
//
// Every wait on an mbarrier has an iteration limit; on expiry the kernel
// records an error code, waits (bounded) for its own loads still in flight,
// releases its TMEM and returns.
#include <cuda.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/xw.h"
#include "xw_host_internal.h"

namespace xw {

namespace {

// Pipeline shape: CTAs per SM, TMA ring depth (tiles), TMEM accumulators
// (128 columns each) and epilogue groups (four warps each) per CTA.  The
// shared-memory ring must admit no more CTAs per SM than the TMEM columns
// do (kCtasPerSm x kAccs x 128 <= 512).  Measured on B200, 65536 matrices,
// ms at n = 32 / 64 / 96 / 128 (CTAs x stages x accumulators x groups):
//   2 x 6 x 2 x 2   0.047 / 0.121 / 0.234 / 0.278   (the default; 0.045 / 0.110 /
//                   0.224 / 0.276 with the diagonal entry taken by a select
//                   tree and the extra block alternating at n = 64)
//   4 x 3 x 1 x 1   0.049 / 0.133 / 0.256 / 0.307
//   1 x 8 x 4 x 4   0.070 / 0.141 / 0.311 / 0.346
//   1 x 8 x 4 x 2   0.070 / 0.168 / 0.305 / 0.412
//   2 x 6 x 2 x 1   0.057 / 0.165 / 0.320 / 0.381
// against 0.053 / 0.125 / 0.238 / 0.317 for one CTA-wide barrier per tile
// step (4 CTAs per SM, 3 stages).
#ifndef XW_RESCORE_CTAS
#define XW_RESCORE_CTAS 2
#endif
#ifndef XW_RESCORE_STAGES
#define XW_RESCORE_STAGES 6
#endif
#ifndef XW_RESCORE_ACCS
#define XW_RESCORE_ACCS 2
#endif
#ifndef XW_RESCORE_GROUPS
#define XW_RESCORE_GROUPS 2
#endif
constexpr int kCtasPerSm = XW_RESCORE_CTAS;
constexpr int kStages = XW_RESCORE_STAGES;
constexpr int kTileRows = 128;
constexpr int kTileBytes = kTileRows * 128;   // 128 rows x 128 bytes (K padded to 128)
constexpr int kAccs = XW_RESCORE_ACCS;
constexpr int kAccCols = 128;                 // columns of one accumulator (N <= 128)
constexpr uint32_t kTmemCols = kAccs * kAccCols;
constexpr int kGroups = XW_RESCORE_GROUPS;
constexpr int kThreads = 64 + 128 * kGroups;
constexpr int kCombineSlots = 8;
static_assert(kAccs % kGroups == 0, "an accumulator belongs to one epilogue group");
static_assert(kCombineSlots >= kAccs / kGroups + 1, "a combine slot outlives its tile");
static_assert(kCtasPerSm * kAccs * kAccCols <= 512, "TMEM columns of the resident CTAs");
static_assert(kTmemCols == 128 || kTmemCols == 256 || kTmemCols == 512, "TMEM allocation size");
constexpr long long kSpinLimit = 1ll << 22;

struct RescoreParams {
    int count;          // matrices
    int n, w;
    int rows_per_tile;  // matrices per tile * n
    int mpt;            // matrices per tile
    int ntiles;
    int4* stats;        // per matrix {score, conflicts, squared, exact}
    int32_t* gram;      // nullable: per matrix n*n row-major
    int* error;         // nonzero after a timed-out wait
    const int2* dims;   // nullable: per matrix {order, weight} of a matrix zero-padded to n
};

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count));
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
                 : "memory");
}

// bounded wait for the phase with parity `parity` to complete
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity) {
    const uint32_t addr = smem_addr(bar);
    for (long long i = 0; i < kSpinLimit; ++i) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(done)
            : "r"(addr), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}

__device__ __forceinline__ void tma_load_2d(void* dst, const CUtensorMap* map, int x, int y, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cta.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4}], [%2];"
        ::"r"(smem_addr(dst)), "l"(map), "r"(smem_addr(bar)), "r"(x), "r"(y)
        : "memory");
}

// K-major operand with 128-byte swizzle: 8-row groups 1024 bytes apart.
// (The 32- and 64-byte swizzles with boxes of n bytes per row, tried for
// n = 32 and 64, were slower: 0.055 against 0.047 ms at n = 32.)
__device__ __forceinline__ uint64_t smem_desc(const void* tile) {
    const uint64_t addr = smem_addr(tile);
    uint64_t d = 0;
    d |= (addr >> 4) & 0x3fffull;           // start address
    d |= (uint64_t)1 << 16;                  // leading byte offset (unused for this layout)
    d |= (uint64_t)(1024 >> 4) << 32;        // stride byte offset
    d |= (uint64_t)1 << 46;                  // descriptor version for sm_100
    d |= (uint64_t)2 << 61;                  // SWIZZLE_128B
    return d;
}

// kind::i8, signed A and B, int32 D, both K-major, M = 128, N = n_cols
__device__ __forceinline__ uint32_t instr_desc(int n_cols) {
    return (2u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n_cols >> 3) << 17) | ((uint32_t)(128 >> 4) << 24);
}

__device__ __forceinline__ void mma_i8(uint32_t tmem_d, uint64_t a, uint64_t b, uint32_t idesc, uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n\t}"
        ::"r"(tmem_d), "l"(a), "l"(b), "r"(idesc), "r"(accumulate));
}

__device__ __forceinline__ void mma_commit(uint64_t* bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_addr(bar))
                 : "memory");
}

// 32 consecutive int32 columns of this warp's TMEM lane quarter, one row per thread
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, int (&v)[32]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
        "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
        "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
        : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
          "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15]),
          "=r"(v[16]), "=r"(v[17]), "=r"(v[18]), "=r"(v[19]), "=r"(v[20]), "=r"(v[21]), "=r"(v[22]), "=r"(v[23]),
          "=r"(v[24]), "=r"(v[25]), "=r"(v[26]), "=r"(v[27]), "=r"(v[28]), "=r"(v[29]), "=r"(v[30]), "=r"(v[31])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

// Warp roles.  Warp 0 (one thread): TMA producer over a kStages ring of
// tiles.  Warp 1: allocates TMEM; one thread issues each tile's MMA chain
// into the next of kAccs accumulators (128 columns each) and commits it to
// the tile's stage (free again) and to the accumulator (ready).  Warps
// 2..2+4*kGroups-1: epilogue groups of four warps, one per TMEM lane
// quarter (warp w reads lanes 32*(w%4)..); group g takes the tiles
// it = g, g + kGroups, ... of this CTA and frees the accumulator as soon as
// its rows are read.  No CTA-wide barrier inside the tile loop: a tile's
// load, MMA and epilogue each wait only on the mbarrier of the stage or
// accumulator they use, so loads run kStages tiles ahead and the MMA of the
// next tiles overlaps the epilogue of this one.
__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_addr(bar)) : "memory");
}

__device__ __forceinline__ void rescore_fail(const RescoreParams& p, volatile int* abort_flag, int code) {
    atomicExch(p.error, code);
    *abort_flag = 1;
}

// Per-row statistics of one tile's accumulator rows 32q..32q+31 (this
// warp's lane quarter); see the epilogue comment below.  rot is the
// group's count of tiles before this one.  Returns the warp's sums and
// whether every row's diagonal entry is right.
__device__ __forceinline__ void tile_rows(const RescoreParams& p, uint32_t tacc, int t, int rot, int q, int lane,
                                          int4& part, int& diag_ok, int& mat) {
    const int row0 = 32 * q;
    const int b = row0 / p.n;       // matrix of this warp within the tile
    const int i0 = row0 - b * p.n;  // first row of the warp within the matrix
    const int i = i0 + lane;
    mat = t * p.mpt + b;
    const int col0 = b * p.n;
    const int nb = p.n / 32, rb = i0 / 32;
    int s_abs = 0, s_nz = 0, s_sq = 0, dg = 0;
    int o_abs = 0, o_nz = 0, o_sq = 0;
    auto block = [&](int c, int& a_abs, int& a_nz, int& a_sq) {
        int v[32];
        tmem_ld32(tacc + ((uint32_t)row0 << 16) + (uint32_t)(col0 + c), v);
#pragma unroll
        for (int j = 0; j < 32; j += 2) {
            const int a0 = abs(v[j]), a1 = abs(v[j + 1]);
            a_abs += a0 + a1;
            a_nz += min(a0, 1) + min(a1, 1);
            a_sq += v[j] * v[j] + v[j + 1] * v[j + 1];
        }
        if (c == i0) {
            // v[lane] by a five-level select tree on the lane's bits (a
            // chain of 31 selects measured 4-9% slower per launch)
            int u[16];
#pragma unroll
            for (int j = 0; j < 16; ++j) u[j] = (lane & 16) ? v[j + 16] : v[j];
#pragma unroll
            for (int j = 0; j < 8; ++j) u[j] = (lane & 8) ? u[j + 8] : u[j];
#pragma unroll
            for (int j = 0; j < 4; ++j) u[j] = (lane & 4) ? u[j + 4] : u[j];
#pragma unroll
            for (int j = 0; j < 2; ++j) u[j] = (lane & 2) ? u[j + 2] : u[j];
            dg = (lane & 1) ? u[1] : u[0];
        }
        if (p.gram && mat < p.count) {
            int32_t* dst = p.gram + (size_t)mat * p.n * p.n + (size_t)i * p.n + c;
            if (((uintptr_t)p.gram & 15u) == 0) {   // 16-byte stores need a 16-byte aligned base
                int4* d4 = reinterpret_cast<int4*>(dst);
#pragma unroll
                for (int j = 0; j < 32; j += 4) d4[j / 4] = make_int4(v[j], v[j + 1], v[j + 2], v[j + 3]);
            } else {
#pragma unroll
                for (int j = 0; j < 32; ++j) dst[j] = v[j];
            }
        }
    };
    // G is symmetric: without a Gram output each unordered pair of
    // off-diagonal 32x32 blocks is read once, by the warp of one of its two
    // row blocks (offsets d = 1..nb/2 cyclically), and counted twice; the
    // diagonal entry (lane j of the warp's diagonal block) is taken out after.
    // At d = nb/2 the two row blocks rb and rb + d name the same pair: one
    // of them reads it, the one with rb / d even.  For n = 64 (nb = 2, two
    // warps per matrix, warp q issuing on scheduler q) the choice
    // alternates from tile to tile, (rb + rot) / d even, so that schedulers
    // 0 and 2 do not take the extra block on every tile (measured 5% at
    // n = 64; at n = 128 alternating measured 4% slower)
    if (p.gram) {
        for (int c = 0; c < p.n; c += 32) block(c, s_abs, s_nz, s_sq);
    } else {
        block(i0, s_abs, s_nz, s_sq);
        for (int d = 1; 2 * d <= nb; ++d) {
            if (2 * d == nb && ((nb == 2 ? rb + rot : rb) / d & 1)) continue;
            block(((rb + d) % nb) * 32, o_abs, o_nz, o_sq);
        }
    }
    s_abs += 2 * o_abs - abs(dg);
    s_nz += 2 * o_nz - min(abs(dg), 1);
    s_sq += 2 * o_sq - dg * dg;
    // a zero-padded matrix: its own rows carry w on the diagonal, the
    // padding rows 0 (their off-diagonal entries are 0 anyway)
    int nv = p.n, wv = p.w;
    if (p.dims && mat < p.count) {
        const int2 d = p.dims[mat];
        nv = d.x;
        wv = d.y;
    }
    diag_ok = i < nv ? dg == wv : dg == 0;
    part.x = __reduce_add_sync(0xffffffffu, s_abs);
    part.y = __reduce_add_sync(0xffffffffu, s_nz);
    part.z = __reduce_add_sync(0xffffffffu, s_sq);
    diag_ok = (int)__reduce_and_sync(0xffffffffu, (unsigned)diag_ok);
}

// symmetric G: the off-diagonal sums count each pair twice
__device__ __forceinline__ int4 matrix_stats(int abs_sum, int nz_sum, int sq_sum, int diag_ok) {
    return make_int4(abs_sum / 2, nz_sum / 2, sq_sum / 2, (nz_sum == 0 && diag_ok) ? 1 : 0);
}

__global__ void __launch_bounds__(kThreads, kCtasPerSm) rescore_tc_kernel(const __grid_constant__ CUtensorMap tmap,
                                                                 RescoreParams p) {
    extern __shared__ uint8_t smem_raw[];
    // tiles on a 1024-byte boundary (the 128-byte swizzle pattern repeats every 1024 bytes)
    uint8_t* tiles = reinterpret_cast<uint8_t*>(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
    __shared__ __align__(8) uint64_t full_bar[kStages];
    __shared__ __align__(8) uint64_t empty_bar[kStages];
    __shared__ __align__(8) uint64_t accf_bar[kAccs];
    __shared__ __align__(8) uint64_t acce_bar[kAccs];
    __shared__ uint32_t tmem_base_sh;
    __shared__ volatile int abort_sh;
    // cross-warp sums of matrices that span several lane quarters (n >= 64):
    // per group, kCombineSlots tiles in flight, two matrices per tile at
    // most; fields abs, nonzero, squared, diagonal-ok, arrivals
    __shared__ int comb_sh[kGroups][kCombineSlots][2][5];

    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    if (warp == 1) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(&tmem_base_sh)),
                     "r"(kTmemCols));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    if (tid == 0) {
        for (int s = 0; s < kStages; ++s) {
            mbar_init(&full_bar[s], 1);
            mbar_init(&empty_bar[s], 1);
        }
        for (int a = 0; a < kAccs; ++a) {
            mbar_init(&accf_bar[a], 1);
            mbar_init(&acce_bar[a], 4);   // the four warps of the group that owns the accumulator
        }
        abort_sh = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    for (int k = tid; k < kGroups * kCombineSlots * 2; k += blockDim.x) {
        int* f = &comb_sh[0][0][0][0] + 5 * k;
        f[0] = f[1] = f[2] = f[4] = 0;
        f[3] = 1;
    }
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;");
    const uint32_t tmem = tmem_base_sh;

    const int grid = gridDim.x;
    // this CTA's tiles: blockIdx.x, blockIdx.x + grid, ...
    const int ntl = (int)blockIdx.x < p.ntiles ? (p.ntiles - 1 - (int)blockIdx.x) / grid + 1 : 0;
    // a TMA box delivers rows_per_tile rows of 128 bytes (zero fill included)
    const uint32_t box_bytes = 128u * (uint32_t)p.rows_per_tile;
    constexpr int S = kStages;

    if (warp == 0) {
        if (lane == 0) {
            int it = 0;
            for (; it < ntl && !abort_sh; ++it) {
                const int s = it % S;
                if (it >= S && !mbar_wait(&empty_bar[s], (uint32_t)(it / S - 1) & 1u)) {
                    rescore_fail(p, &abort_sh, 3);
                    break;
                }
                mbar_expect_tx(&full_bar[s], box_bytes);
                tma_load_2d(tiles + s * kTileBytes, &tmap, 0, ((int)blockIdx.x + it * grid) * p.rows_per_tile,
                            &full_bar[s]);
            }
            // drain: the loads still in flight are among the last S
            // issued (earlier ones were consumed before their stage came back)
            for (int k = it > S ? it - S : 0; k < it; ++k)
                mbar_wait(&full_bar[k % S], (uint32_t)(k / S) & 1u);
        }
    } else if (warp == 1) {
        if (lane == 0) {
            const uint32_t idesc = instr_desc(p.rows_per_tile);
            // K steps of 32 columns that hold matrix entries; the box's
            // columns past n are zero-filled by the TMA load and add nothing
            const int ksteps = (p.n + 31) / 32;
            int it = 0;
            for (; it < ntl && !abort_sh; ++it) {
                const int s = it % S, a = it % kAccs;
                if (!mbar_wait(&full_bar[s], (uint32_t)(it / S) & 1u)) {
                    rescore_fail(p, &abort_sh, 1);
                    break;
                }
                if (it >= kAccs && !mbar_wait(&acce_bar[a], (uint32_t)(it / kAccs - 1) & 1u)) {
                    rescore_fail(p, &abort_sh, 4);
                    break;
                }
                asm volatile("tcgen05.fence::after_thread_sync;");
                const uint64_t d = smem_desc(tiles + s * kTileBytes);
                const uint32_t tacc = tmem + (uint32_t)(a * kAccCols);
#pragma unroll 1
                for (int k = 0; k < ksteps; ++k)
                    mma_i8(tacc, d + (uint64_t)(2 * k), d + (uint64_t)(2 * k), idesc, k > 0);
                mma_commit(&empty_bar[s]);
                mma_commit(&accf_bar[a]);
            }
            // every MMA issued has completed once the last commit arrived
            if (it > 0) mbar_wait(&accf_bar[(it - 1) % kAccs], (uint32_t)((it - 1) / kAccs) & 1u);
        }
    } else {
        const int e = warp - 2, g = e >> 2, q = warp & 3;
        const bool active = 32 * q < p.rows_per_tile;
        const int wpm = (p.n + 31) / 32;   // warps (lane quarters) per matrix
        for (int it = g; it < ntl; it += kGroups) {
            if (abort_sh) break;
            const int a = it % kAccs;
            if (!mbar_wait(&accf_bar[a], (uint32_t)(it / kAccs) & 1u)) {
                rescore_fail(p, &abort_sh, 2);
                break;
            }
            asm volatile("tcgen05.fence::after_thread_sync;");
            const int t = (int)blockIdx.x + it * grid;
            int4 part = make_int4(0, 0, 0, 0);
            int diag_ok = 1, mat = 0;
            if (active) tile_rows(p, tmem + (uint32_t)(a * kAccCols), t, it / kGroups, q, lane, part, diag_ok, mat);
            // the accumulator is free for the MMA of a later tile
            asm volatile("tcgen05.fence::before_thread_sync;");
            __syncwarp();
            if (lane == 0) mbar_arrive(&acce_bar[a]);
            if (!active || lane != 0 || mat >= p.count) continue;
            if (wpm == 1) {
                p.stats[mat] = matrix_stats(part.x, part.y, part.z, diag_ok);
                continue;
            }
            // the last of the matrix's warps to arrive writes its stats and
            // resets the slot; a slot is reused kCombineSlots tiles later,
            // when every warp of the group has long finished this tile
            int* f = comb_sh[g][(it / kGroups) % kCombineSlots][(32 * q) / p.n];
            atomicAdd(&f[0], part.x);
            atomicAdd(&f[1], part.y);
            atomicAdd(&f[2], part.z);
            atomicAnd(&f[3], diag_ok);
            __threadfence_block();
            if (atomicAdd(&f[4], 1) == wpm - 1) {
                __threadfence_block();
                const int sa = atomicExch(&f[0], 0), sn = atomicExch(&f[1], 0), sq = atomicExch(&f[2], 0),
                          ok = atomicExch(&f[3], 1);
                atomicExch(&f[4], 0);
                p.stats[mat] = matrix_stats(sa, sn, sq, ok);
            }
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;");
    if (warp == 1)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTmemCols));
}

// SIMT path for orders that do not fill 32-row tensor-core blocks: one warp
// per matrix, lane o accumulates column o of G.
__global__ void rescore_simt_kernel(const int8_t* W, int count, int n, int w, int4* stats, int32_t* gram,
                                    const int2* dims) {
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (warp >= count) return;
    const int nv = dims ? dims[warp].x : n;
    if (dims) w = dims[warp].y;
    const int8_t* M = W + (size_t)warp * n * n;
    int s_abs = 0, s_nz = 0, s_sq = 0, diag_ok = 1;
    for (int o = lane; o < n; o += 32) {
        for (int r = 0; r < n; ++r) {
            int dot = 0;
            for (int c = 0; c < n; ++c) dot += M[r * n + c] * M[o * n + c];
            if (gram) gram[(size_t)warp * n * n + (size_t)r * n + o] = dot;
            if (r == o) {
                diag_ok &= dot == (o < nv ? w : 0);
            } else {
                const int a = dot < 0 ? -dot : dot;
                s_abs += a;
                s_nz += a != 0;
                s_sq += dot * dot;
            }
        }
    }
    s_abs = __reduce_add_sync(0xffffffffu, s_abs);
    s_nz = __reduce_add_sync(0xffffffffu, s_nz);
    s_sq = __reduce_add_sync(0xffffffffu, s_sq);
    diag_ok = (int)__reduce_and_sync(0xffffffffu, (unsigned)diag_ok);
    if (lane == 0) stats[warp] = make_int4(s_abs / 2, s_nz / 2, s_sq / 2, (s_nz == 0 && diag_ok) ? 1 : 0);
}

typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                  const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiledFn encode_tiled() {
    static std::once_flag once;
    static EncodeTiledFn fn = nullptr;
    std::call_once(once, []() {
        void* ptr = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &ptr, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<EncodeTiledFn>(ptr);
    });
    return fn;
}

int32_t rfail(int32_t code, const std::string& msg) {
    set_last_error(msg);
    return code;
}

// timed-out-wait flag of the rescoring kernel (one int per device)
static __device__ int g_rescore_error;

int* error_flag_ptr() {
    static std::mutex mu;
    static int* ptr[64] = {};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return nullptr;
    std::lock_guard<std::mutex> lock(mu);
    if (!ptr[dev]) {
        void* p = nullptr;
        if (cudaGetSymbolAddress(&p, g_rescore_error) != cudaSuccess) return nullptr;
        ptr[dev] = static_cast<int*>(p);
    }
    return ptr[dev];
}

}  // namespace

// Enqueue the rescoring of `count` row-major n x n matrices at W (device).
int32_t rescore_device(const int8_t* W, int64_t count, int n, int w, int32_t* stats, int32_t* gram,
                       cudaStream_t stream, int* err_flag, bool force_simt, const int2* dims) {
    if (count < 0 || count > INT32_MAX / 4) return rfail(XW_ERR_INVALID, "rescore: count out of range");
    if (n < 1 || n > XW_MAX_ORDER_SHARED) return rfail(XW_ERR_INVALID, "rescore: order must be in [1, 256]");
    if (count == 0) return XW_OK;
    cudaError_t e;
    // tensor cores for n in {32, 64, 96, 128}: a tile row is one 128-byte TMA row
    const bool tc = !force_simt && n % 32 == 0 && n <= 128 && ((uintptr_t)W % 16) == 0;
    if (!tc) {
        const int blocks = (int)((count * 32 + 255) / 256);
        rescore_simt_kernel<<<blocks, 256, 0, stream>>>(W, (int)count, n, w, reinterpret_cast<int4*>(stats), gram,
                                                        dims);
        e = cudaGetLastError();
        return e == cudaSuccess ? XW_OK : rfail(XW_ERR_CUDA, std::string("rescore launch: ") + cudaGetErrorString(e));
    }
    EncodeTiledFn enc = encode_tiled();
    if (!enc) return rfail(XW_ERR_CUDA, "rescore: cuTensorMapEncodeTiled is unavailable");
    RescoreParams p;
    p.count = (int)count;
    p.n = n;
    p.w = w;
    p.mpt = n <= 64 ? 128 / n : 1;
    p.rows_per_tile = p.mpt * n;
    p.ntiles = (int)((count + p.mpt - 1) / p.mpt);
    p.stats = reinterpret_cast<int4*>(stats);
    p.gram = gram;
    p.error = err_flag;
    p.dims = dims;
    CUtensorMap map;
    const cuuint64_t extent[2] = {(cuuint64_t)n, (cuuint64_t)count * n};
    const cuuint64_t strides[1] = {(cuuint64_t)n};
    const cuuint32_t box[2] = {128u, (cuuint32_t)p.rows_per_tile};
    const cuuint32_t estr[2] = {1u, 1u};
    const CUresult r = enc(&map, CU_TENSOR_MAP_DATA_TYPE_UINT8, 2, const_cast<int8_t*>(W), extent, strides, box, estr,
                           CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                           CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return rfail(XW_ERR_CUDA, "rescore: cuTensorMapEncodeTiled failed");
    int dev = 0, sms = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const size_t smem = (size_t)kStages * kTileBytes + 1024;
    e = cudaFuncSetAttribute(rescore_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return rfail(XW_ERR_CUDA, std::string("rescore attribute: ") + cudaGetErrorString(e));
    // kCtasPerSm persistent CTAs per SM; the tile loop is grid-strided, so
    // fewer resident CTAs only serialise, never skip, tiles
    const int blocks = (int)std::min<int64_t>(p.ntiles, (int64_t)kCtasPerSm * sms);
    rescore_tc_kernel<<<blocks, kThreads, smem, stream>>>(map, p);
    e = cudaGetLastError();
    return e == cudaSuccess ? XW_OK : rfail(XW_ERR_CUDA, std::string("rescore launch: ") + cudaGetErrorString(e));
}

// Copies each matrix of a verification batch into its zero-padded
// row-major slot (block b: matrix b of the group; the source is the
// column-major W of the search) and writes its {order, weight}.
__global__ void verify_gather_kernel(const VerifyItem* items, const int32_t* index, int N, int8_t* dst, int2* dims) {
    const VerifyItem it = items[index[blockIdx.x]];
    int8_t* out = dst + (size_t)blockIdx.x * N * N;
    for (int e = threadIdx.x; e < N * N; e += blockDim.x) {
        const int r = e / N, c = e - r * N;
        out[e] = r < it.n && c < it.n ? it.W[(size_t)c * it.n + r] : (int8_t)0;
    }
    if (threadIdx.x == 0) dims[blockIdx.x] = make_int2(it.n, it.w);
}

DeviceVerifier& shared_verifier(int device, std::mutex*& mu) {
    static std::mutex table_mu;
    static std::mutex use_mu[64];
    static DeviceVerifier* table[64] = {};   // kept until exit
    if (device < 0 || device >= 64) throw std::invalid_argument("device ordinal out of range");
    std::lock_guard<std::mutex> lock(table_mu);
    if (!table[device]) table[device] = new DeviceVerifier();
    mu = &use_mu[device];
    return *table[device];
}

DeviceVerifier::~DeviceVerifier() {
    for (void* ptr : {(void*)d_items, (void*)d_index, (void*)d_stage, (void*)d_dims, (void*)d_stats})
        if (ptr) cudaFree(ptr);
    if (h_stats) cudaFreeHost(h_stats);
    if (h_table) cudaFreeHost(h_table);
}

void DeviceVerifier::reserve(size_t items, size_t stage_bytes) {
    if (items > cap_items) {
        for (void* ptr : {(void*)d_items, (void*)d_index, (void*)d_dims, (void*)d_stats})
            if (ptr) check_cuda(cudaFree(ptr), "cudaFree");
        if (h_stats) check_cuda(cudaFreeHost(h_stats), "cudaFreeHost");
        if (h_table) check_cuda(cudaFreeHost(h_table), "cudaFreeHost");
        const size_t cap = std::max<size_t>(items, 64);
        check_cuda(cudaMalloc(&d_items, sizeof(VerifyItem) * cap), "cudaMalloc verification items");
        check_cuda(cudaMalloc(&d_index, sizeof(int32_t) * cap), "cudaMalloc verification index");
        check_cuda(cudaMalloc(&d_dims, sizeof(int2) * cap), "cudaMalloc verification dims");
        check_cuda(cudaMalloc(&d_stats, sizeof(int4) * cap), "cudaMalloc verification stats");
        check_cuda(cudaMallocHost(&h_stats, sizeof(int4) * cap), "cudaMallocHost verification stats");
        check_cuda(cudaMallocHost(&h_table, (sizeof(VerifyItem) + sizeof(int32_t)) * cap),
                   "cudaMallocHost verification table");
        cap_items = cap;
    }
    if (stage_bytes > cap_stage) {
        if (d_stage) check_cuda(cudaFree(d_stage), "cudaFree");
        check_cuda(cudaMalloc(&d_stage, stage_bytes), "cudaMalloc verification staging");
        cap_stage = stage_bytes;
    }
}

void DeviceVerifier::run(const std::vector<VerifyItem>& items, cudaStream_t stream, std::vector<VerifyStats>& out) {
    out.assign(items.size(), VerifyStats{});
    if (items.empty()) return;
    // groups of one padded order: a multiple of 32 up to 128 (tensor cores),
    // the order itself above (SIMT)
    auto padded = [](int n) { return n <= 128 ? 32 * ((n + 31) / 32) : n; };
    std::vector<int32_t> index(items.size());
    for (size_t k = 0; k < items.size(); ++k) {
        if (items[k].n < 1 || items[k].n > XW_MAX_ORDER_SHARED)
            throw std::invalid_argument("device verification covers orders 1..256");
        index[k] = (int32_t)k;
    }
    std::stable_sort(index.begin(), index.end(),
                     [&](int32_t a, int32_t b) { return padded(items[a].n) < padded(items[b].n); });
    size_t stage = 0;
    for (size_t k = 0; k < items.size(); ++k) {
        const size_t N = (size_t)padded(items[index[k]].n);
        stage = (stage + N * N + 127) & ~size_t(127);
    }
    reserve(items.size(), stage);
    VerifyItem* hi = reinterpret_cast<VerifyItem*>(h_table);
    int32_t* hx = reinterpret_cast<int32_t*>(hi + items.size());
    std::memcpy(hi, items.data(), sizeof(VerifyItem) * items.size());
    std::memcpy(hx, index.data(), sizeof(int32_t) * items.size());
    check_cuda(cudaMemcpyAsync(d_items, hi, sizeof(VerifyItem) * items.size(), cudaMemcpyHostToDevice, stream),
               "upload verification items");
    check_cuda(cudaMemcpyAsync(d_index, hx, sizeof(int32_t) * items.size(), cudaMemcpyHostToDevice, stream),
               "upload verification index");
    int* flag = error_flag_ptr();
    if (!flag) throw std::runtime_error("rescore: cannot resolve the error flag");
    size_t off = 0;
    for (size_t g0 = 0; g0 < index.size();) {
        const int N = padded(items[index[g0]].n);
        size_t g1 = g0;
        while (g1 < index.size() && padded(items[index[g1]].n) == N) ++g1;
        const int cnt = (int)(g1 - g0);
        int8_t* dst = d_stage + off;
        verify_gather_kernel<<<cnt, 256, 0, stream>>>(d_items, d_index + g0, N, dst, d_dims + g0);
        check_cuda(cudaGetLastError(), "launch verify_gather_kernel");
        const int32_t rc = rescore_device(dst, cnt, N, 0, reinterpret_cast<int32_t*>(d_stats + g0), nullptr, stream,
                                          flag, false, d_dims + g0);
        if (rc != XW_OK) throw std::runtime_error("device verification launch failed");
        off = (off + (size_t)cnt * N * N + 127) & ~size_t(127);
        g0 = g1;
    }
    check_cuda(cudaMemcpyAsync(h_stats, d_stats, sizeof(int4) * items.size(), cudaMemcpyDeviceToHost, stream),
               "read verification stats");
    check_cuda(cudaStreamSynchronize(stream), "cudaStreamSynchronize verification");
    if (xw_rescore_status() != XW_OK) throw std::runtime_error("device verification: a rescoring wait expired");
    for (size_t k = 0; k < items.size(); ++k) {
        const int4 v = reinterpret_cast<const int4*>(h_stats)[k];
        out[index[k]] = VerifyStats{v.x, v.y, v.z, v.w};
    }
}

}  // namespace xw

using namespace xw;

extern "C" int32_t xw_rescore_device(const int8_t* W, int64_t count, int32_t n, int32_t w, int32_t* stats,
                                     int32_t* gram, int32_t simt, void* stream) {
    if (!W || !stats) return rfail(XW_ERR_INVALID, "rescore: null argument");
    int* flag = error_flag_ptr();
    if (!flag) return rfail(XW_ERR_CUDA, "rescore: cannot resolve the error flag");
    return rescore_device(W, count, n, w, stats, gram, static_cast<cudaStream_t>(stream), flag, simt != 0, nullptr);
}

extern "C" int32_t xw_rescore_status(void) {
    int* flag = error_flag_ptr();
    if (!flag) return rfail(XW_ERR_CUDA, "rescore: cannot resolve the error flag");
    int v = 0;
    if (cudaMemcpy(&v, flag, sizeof v, cudaMemcpyDeviceToHost) != cudaSuccess)
        return rfail(XW_ERR_CUDA, "rescore: cannot read the error flag");
    if (v == 0) return XW_OK;
    const int zero = 0;
    cudaMemcpy(flag, &zero, sizeof zero, cudaMemcpyHostToDevice);
    return rfail(XW_ERR_TIMEOUT, "rescore: a pipeline wait expired (code " + std::to_string(v) + ")");
}

extern "C" int32_t xw_rescore(const int8_t* W, int64_t count, int32_t n, int32_t w, int32_t* stats, int32_t* gram) {
    if (!W || !stats || count < 0 || n < 1 || n > XW_MAX_ORDER_SHARED) return rfail(XW_ERR_INVALID, "rescore: bad arguments");
    if (count == 0) return XW_OK;
    const size_t in_bytes = (size_t)count * n * n, st_bytes = (size_t)count * 16,
                 g_bytes = gram ? (size_t)count * n * n * 4 : 0;
    int8_t* dW = nullptr;
    int32_t *dS = nullptr, *dG = nullptr;
    auto cleanup = [&]() {
        if (dW) cudaFree(dW);
        if (dS) cudaFree(dS);
        if (dG) cudaFree(dG);
    };
    if (cudaMalloc(&dW, in_bytes) != cudaSuccess || cudaMalloc(&dS, st_bytes) != cudaSuccess ||
        (gram && cudaMalloc(&dG, g_bytes) != cudaSuccess)) {
        cleanup();
        return rfail(XW_ERR_CAPACITY, "rescore: device allocation failed");
    }
    int32_t rc = XW_OK;
    if (cudaMemcpy(dW, W, in_bytes, cudaMemcpyHostToDevice) != cudaSuccess)
        rc = rfail(XW_ERR_CUDA, "rescore: copy to device failed");
    if (rc == XW_OK) rc = xw_rescore_device(dW, count, n, w, dS, dG, 0, nullptr);
    if (rc == XW_OK && cudaDeviceSynchronize() != cudaSuccess) rc = rfail(XW_ERR_CUDA, "rescore: kernel failed");
    if (rc == XW_OK) rc = xw_rescore_status();
    if (rc == XW_OK && cudaMemcpy(stats, dS, st_bytes, cudaMemcpyDeviceToHost) != cudaSuccess)
        rc = rfail(XW_ERR_CUDA, "rescore: copy to host failed");
    if (rc == XW_OK && gram && cudaMemcpy(gram, dG, g_bytes, cudaMemcpyDeviceToHost) != cudaSuccess)
        rc = rfail(XW_ERR_CUDA, "rescore: copy to host failed");
    cleanup();
    return rc;
}
