// xw_kernels.h -- host-side declarations of the annealing kernels.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "xw_layout.h"

#define XW_MAX_RUNGS 256

namespace xw {

struct AnnealArgs {
    XwJob* jobs;
    uint8_t* arena;            // replica records
    const uint64_t* rec_off;   // byte offset of each replica record
    const uint32_t* items;     // replica ids this launch runs
    uint32_t n_items;
    uint32_t slot_bytes;       // shared memory per warp
    uint32_t* counter;         // persistent work counter, zeroed per launch
    uint64_t iters;            // iterations per replica this launch
    int32_t stop_on_solve;
    // 1: every replica of the launch has one zero per row (w = n - 1); the
    // lean one-row, one-replica-per-warp kernel then runs its instantiation
    // with the minority size and side as constants (other kernels ignore it)
    int32_t one_zero;
    uint8_t* gram = nullptr;            // large-order kernel: Gram and mask arena
    const uint64_t* gram_off = nullptr; // byte offset of each replica's Gram there
    // The shared-memory kernel can split each replica's `iters` into `chunks`
    // consecutive work items, scheduled chunk-major, so that a launch with
    // more replicas than resident warps does not end in a part-filled wave.
    // chunk_done[rid] (zeroed per launch) counts a replica's finished chunks.
    uint32_t chunks = 1;
    uint32_t* chunk_done = nullptr;
    // device-time limit of a chunk's wait for its predecessor, 0 = 30 s
    uint64_t chunk_wait_ns = 0;
    // with one_zero: the launch's single order, whose instantiation (the even
    // orders 6..26) then runs with the order as a constant; 0 = any order
    int32_t fixed_order = 0;
    int32_t fixed_pad = 0;
};

// shared-memory bytes one warp needs for a replica of order n, minority m,
// in a launch of the `opl` rows-per-lane kernel
uint32_t anneal_slot_bytes(int n, int m, int opl);
// lanes' rows per lane: 1 for n <= 32, 2 for n <= 64, 4 for n <= 128, 8 for n <= 256
int anneal_opl(int n);
// `general`: some replica of the launch uses the squared or parity objective
// or the within-row swap move set; otherwise the lean kernel (L1 score,
// the reference's moves) runs, which drops that work from the hot loop.
// `rpw`: replicas per warp, 1, or 2 for orders up to 16 (opl 1; each half
// of a warp owns a replica and a shared-memory slot of args.slot_bytes, so
// a CTA holds warps_per_block * rpw slots).
// `one_zero`: the instantiation for launches whose replicas all have one zero
// per row (AnnealArgs::one_zero); it applies to opl 1, lean, rpw 1 only;
// `fixed_order` > 0: all of them have that order (AnnealArgs::fixed_order).
const void* anneal_kernel_fn(int opl, bool general, int rpw = 1, bool one_zero = false, int fixed_order = 0);
cudaError_t launch_anneal(const AnnealArgs& args, int opl, bool general, int warps_per_block, int blocks,
                          cudaStream_t stream, int rpw = 1);
// Latency mode (orders up to 32): one replica per CTA of K warps (2..16),
// which speculate K iterations at a time and keep the first accepted one;
// the trajectory is the one-warp kernel's.  Shared memory per CTA for
// replicas whose one-warp slot (anneal_slot_bytes at one row per lane) is
// at most slot_bytes; the kernel and its launch (a.slot_bytes: the CTA's
// dynamic shared memory; a.chunks must be 1).
// wpr warps per replica on `ctas` CTAs of wpr / ctas warps (2..16) each:
// one CTA, or a cluster of two or four (one replica per cluster, `blocks`
// unused)
uint32_t anneal_spec_cta_bytes(uint32_t slot_bytes, int wpr, int ctas);
const void* anneal_spec_kernel_fn(bool general, int ctas);
cudaError_t launch_anneal_spec(const AnnealArgs& args, bool general, int wpr, int ctas, int blocks,
                               cudaStream_t stream);
// Orders above XW_MAX_N (xw_anneal_large.cu), in one of three forms:
// 0 the Gram matrix and masks in an HBM arena; 1 bit planes in shared
// memory, no Gram matrix stored (its entries recomputed by popcounts);
// 2 bit planes in shared memory and the Gram matrix in HBM.  Forms 1 and 2
// take orders whose W fits a warp's slot as bit planes.  Whether (n, m)
// fits them, shared memory per warp, arena bytes per replica (a multiple of
// 256), the kernel, and its launch.
bool anneal_large_planes_fit(int n, int m);
uint32_t anneal_large_slot_bytes(int n, int m, int form);
uint64_t anneal_large_arena_bytes(int n, int form);
const void* anneal_large_kernel_fn(bool general, int form);
cudaError_t launch_anneal_large(const AnnealArgs& args, bool general, int form, int warps_per_block, int blocks,
                                cudaStream_t stream);
cudaError_t launch_exchange(XwJob* jobs, int njobs, uint8_t* arena, const uint64_t* rec_off,
                            const double* ladder, int stop_on_solve, cudaStream_t stream);

}  // namespace xw

namespace xw {

struct JobOut {
    int64_t score, conflicts;
    int32_t best_replica, solved, err;
    int32_t first_solver;           // least (solve iteration, index) with score 0, or -1
    uint64_t moves, cand_evals, iters;
    uint64_t solved_it, solve_ns;   // the first solver's solve iteration and %globaltimer
    uint64_t accepted, accepted_rows, two_row_evals;   // sums of the replicas' statistics
};

// One warp per job: results and (best_out nonnull) the chosen replica's best
// W at best_out + best_out_off[job].  first_solver_state chooses the first
// solver when there is one, else the least (score, conflicts, index).
cudaError_t launch_collect(const XwJob* jobs, int njobs, const uint8_t* arena, const uint64_t* rec_off,
                           const uint64_t* best_out_off, JobOut* out, int8_t* best_out,
                           cudaStream_t stream, int first_solver_state = 0);
cudaError_t launch_mark_t0(uint64_t* t0, cudaStream_t stream);
// *t = %globaltimer when the stream reaches it
cudaError_t launch_stamp(uint64_t* t, cudaStream_t stream);

}  // namespace xw
