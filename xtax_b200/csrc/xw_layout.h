// xw_layout.h -- HBM layout of annealing jobs and replica records, shared by
// the host orchestrator and the kernels.
//
// A job is one independent search W(n,w) with its own Philox key: one
// xweigh_cuda run, one tempering instance, or one served request.  Its
// replicas are records in one byte arena:
//
//   [RepHeader 128 B][W: n*n int8, column-major][best W: n*n int8][minority: n*m u8]
//
// each section padded to 16 bytes.  The Gram matrix, the row residuals and
// the row support masks are not stored: the kernel rebuilds them in shared
// memory from W when it loads a replica (O(n^3/32) per lane, negligible next
// to the thousands of moves per launch) and checks the rebuilt score against
// the tracked one.
//
// Orders above XW_MAX_N keep 16-bit minority lists (n*m u16) and a Gram
// arena beside the records (int16 G, support and sign masks per replica)
// that persists between launches; see xw_anneal_large.cu.
#pragma once

#include <stdint.h>

#define XW_MAX_N 256           // largest order of the shared-memory kernel
#define XW_MAX_ORDER_LARGE 1024 // largest order of the HBM-resident kernel
#define XW_MAX_CANDIDATES 32
#define XW_MAX_TARGET_SAMPLES 64
#define XW_NOALLOC_SCRATCH_BYTES (4 * 1024 * 1024)

#define XW_STATUS_INIT 1u      // record holds incremental state (score etc.)
#define XW_STATUS_SOLVED 2u    // best score reached 0
#define XW_STATUS_GRAM 4u      // large orders: the arena holds this W's Gram and masks (or, in
                               // bit-plane mode, its planes and residuals)
#define XW_ERR_SCORE 1u        // rebuilt score differs from the tracked one
#define XW_ERR_MINORITY 2u     // W row weights disagree with the minority lists
#define XW_ERR_KERNEL 4u       // a lean launch met a replica that needs the general kernel
#define XW_ERR_CHUNK 8u        // a chunk's wait for its replica's previous chunk timed out
// (the same values as XW_DEVERR_* of include/xw.h)

struct XwJob {
    int32_t n, w, m, sparse;        // m = min(w, n-w); sparse = (w <= n-w)
    int32_t tempering;              // 0 cooling/reheat, 1 fixed rung temperatures
    int32_t move_set;               // 0 flip/switch/double, 1 flip/within-row swap
    int32_t candidate_samples, target_samples;
    int32_t moves_per_cool, stuck_threshold;
    int32_t objective;              // -1 hash rule, else forced objective
    int32_t replicas;               // R
    uint32_t key0, key1;            // Philox key
    uint32_t rep_begin;             // first replica id of the job
    uint32_t record_bytes;
    uint32_t off_w, off_best, off_mino;
    int32_t general;                // needs the general kernel (objectives, move set 1)
    uint64_t thr_greedy, thr_target, thr_double, thr_sign, thr_swsign;
    double t_min, cooling, reheat;
    uint64_t budget_iters;          // per-replica iteration cap, 0 = none
    uint64_t exch_round;            // tempering exchange rounds done
    uint64_t ladder_off;            // index of the first rung temperature
    int32_t solved;                 // set on device when a replica solves
    int32_t solved_replica;
    uint64_t solved_it;
    uint64_t solve_ns;              // %globaltimer at the solve
    int32_t done;                   // host: job retired, skip its replicas
    int32_t large;                  // runs on the HBM-resident kernel (u16 minority lists)
    uint64_t exchange_iters;        // tempering: exchange only when the job's
                                    // iteration count is a multiple of this
                                    // (0 = after every anneal launch)
};

struct RepHeader {
    uint64_t it;                    // iterations run (the Philox counter)
    uint64_t moves;                 // iterations with a valid candidate
    uint64_t cand_evals;
    int32_t score, conflicts;       // L1 score and conflicts of W
    int32_t best_score, best_conflicts;
    int64_t obj_total;              // total of the replica's own objective
    double temperature, reheat_temperature;
    int32_t msi, cool_ctr, rung, obj_kind;
    uint32_t job, stream;           // job id; replica index within the job
    uint32_t status, err;
    uint64_t solve_it;
    uint64_t solve_ns;
    // move statistics (32-bit, wrapping): accepted moves, rows those moves
    // changed (1 or 2 each), and candidates evaluated that change two rows
    uint32_t accepted, accepted_rows, two_row_evals;
    uint32_t pad;
};

#ifdef __cplusplus
static_assert(sizeof(RepHeader) == 128, "replica header is 128 bytes");
#endif

#ifdef __CUDACC__
#define XW_HD __host__ __device__
#else
#define XW_HD
#endif

static inline XW_HD uint32_t xw_pad16(uint32_t v) { return (v + 15u) & ~15u; }
