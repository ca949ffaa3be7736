/* xw.h -- C ABI of the B200-native weighing-matrix population annealer.
 *
 * Drop-in boundary for the xweigh_cuda path of flinty-mathematics/xtax.
 * Every entry point names the reference interface it replaces
 * (src/xweigh_cuda.hpp, src/xweigh_cuda.cu, src/xweigh_anneal.hpp,
 * src/xweigh_cuda_main.cpp).  Plain C types only; no exceptions cross the
 * ABI.  Each call returns an xw status code; on failure xw_last_error()
 * gives the message (thread-local), worded like the reference's exception
 * text where one exists.
 *
 * Matrices are n*n int8 arrays in the reference's column-major order:
 * entry (row r, column c) at [c*n + r] (xweigh_anneal.hpp:290-296), except
 * the batched rescoring input, which is row-major (see xw_rescore).
 */
#ifndef XW_H
#define XW_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* status codes */
#define XW_OK 0
#define XW_ERR_INVALID 1   /* an argument or parameter is out of range */
#define XW_ERR_CUDA 2      /* a CUDA runtime call failed */
#define XW_ERR_CAPACITY 3  /* shared memory, device memory or a size limit */
#define XW_ERR_INTERNAL 4  /* an invariant failed (score mismatch, ...) */
#define XW_ERR_NOT_FOUND 5 /* unknown request id */
#define XW_ERR_TIMEOUT 6   /* a wait ended before the request finished */
#define XW_ERR_IO 7        /* file read or write failed */

/* Device error bits of a replica (xw_replica_state.error, OR-ed over a
 * job's replicas in xw_job_result.error). */
#define XW_DEVERR_SCORE 1u     /* the Gram rebuilt from W disagrees with the tracked score */
#define XW_DEVERR_MINORITY 2u  /* a row's weight is not w, or disagrees with its minority list */
#define XW_DEVERR_KERNEL 4u    /* a lean launch met a replica that needs the general kernel */
#define XW_DEVERR_CHUNK 8u     /* a chunk's wait for the replica's previous chunk ran out;
                                  the replica's later chunks of that launch did not run */

#define XW_MAX_ORDER_CUDA 1024      /* largest n the device path anneals */
#define XW_MAX_ORDER_SHARED 256     /* largest n whose replica state sits in shared memory; larger
                                       orders keep it in HBM (no counterpart in the reference,
                                       whose kernel stops where shared memory ends, about n = 276).
                                       Also the limit of the server, the rescoring kernel and
                                       xw_anneal_noalloc. */
#define XW_MAX_CANDIDATE_SAMPLES 32 /* xweigh_cuda.hpp:11 */
#define XW_MAX_TARGET_SAMPLES 64    /* xweigh_cuda.hpp:12 */

/* Mirrors xweigh_cuda::Params (xweigh_cuda.hpp:14-44) field for field, in
 * the same order, followed by the extensions of this implementation. */
typedef struct xw_params {
    int32_t device;
    int32_t replicas;             /* 0 = occupancy-based */
    int32_t moves_per_launch;     /* iterations per replica between host checks */
    uint64_t seed;                /* 0 = random_device */
    double max_seconds;
    double save_interval;
    double sign_fraction;
    double double_sign_fraction;
    double switch_sign_fraction;
    double squared_objective_fraction;
    double parity_objective_fraction;
    double greedy_fraction;
    int32_t candidate_samples;
    double target_fraction;
    int32_t target_samples;
    double t_init;
    double t_min;
    double cooling;
    int32_t moves_per_cool;
    int32_t stuck_threshold;
    double reheat;
    double restart_interval;      /* seconds without improvement before an elite restart (0 = off) */
    double restart_fraction;
    int32_t restart_kick_min;
    int32_t restart_kick_max;
    /* ---- extensions ---- */
    uint64_t max_moves;           /* total move budget over all replicas, 0 = none */
    int32_t tempering;            /* 1: replicas form a parallel-tempering ladder t_min..t_init */
    int32_t exchange_interval;    /* iterations between exchanges when tempering */
    int32_t objective;            /* -1 reference per-replica mix, 0 L1, 1 squared, 2 parity */
    int32_t move_set;             /* 0 flip/switch/double flip, 1 flip/within-row swap */
    int32_t start_kind;           /* 0 regular random start, 1 row-only random start */
    int32_t stop_on_solve;        /* 1: stop every replica once one solves; 2: a replica stops at
                                     its own solve and the others finish the launch, so that
                                     results do not depend on launch timing */
    int32_t warps_per_block;      /* 0 = autotuned */
    int32_t replicas_per_warp;    /* 0 = autotuned; 2: orders up to 16 run two replicas per warp,
                                     one per half-warp (needs candidate_samples <= 16) */
    int32_t warps_per_replica;    /* orders up to 32: 0 = autotuned (the latency mode when a
                                     launch class has at most one replica per SM), 1 = one warp
                                     per replica, 2..16 = that many warps per replica, which
                                     speculate as many iterations at once and keep the first
                                     accepted one (same trajectory, lower latency per move),
                                     18..32 (even) = a cluster of two CTAs on two SMs per
                                     replica, half the warps on each, 36..64 (multiples of 4)
                                     = a cluster of four */
    int32_t restart_kicks;        /* elite restarts: 0 = kicks on the host with the reference's
                                     mt19937 streams (xweigh_cuda.cu:2089-2193), after reading
                                     the job's records back; 1 = kicks on the device with a
                                     Philox stream per (job, restart round, replica), records
                                     rewritten in place (no record crosses to the host) */
} xw_params;

/* xweigh_cuda::DeviceInfo (xweigh_cuda.hpp:46-54) */
typedef struct xw_device_info {
    char name[256];
    int32_t ordinal;
    int32_t compute_major;
    int32_t compute_minor;
    int32_t multiprocessors;
    uint64_t global_memory;
    uint64_t max_shared_memory_per_block;
} xw_device_info;

/* xweigh_cuda::RunResult (xweigh_cuda.hpp:56-65) plus the best state's
 * scores, solve time and exact verification */
typedef struct xw_result {
    int64_t score;
    int64_t conflicts;
    int32_t replicas;
    int32_t solved;               /* best score is 0 */
    int32_t verified;             /* W W^T = wI checked exactly in int64 */
    int32_t best_replica;
    uint64_t moves;
    uint64_t candidate_evaluations;
    uint64_t restarted_replicas;
    uint64_t iterations;          /* per-replica iterations of the longest replica */
    double initialization_seconds;
    double search_seconds;
    double time_to_solution_seconds; /* -1 when unsolved */
    xw_device_info device;
} xw_result;

typedef void (*xw_log_fn)(const char* line, void* user);
typedef void (*xw_checkpoint_fn)(const int8_t* best_colmajor, int32_t n, void* user);

/* Reference defaults (xweigh_cuda.hpp:14-44) and extension defaults. */
void xw_params_default(xw_params* p);

/* Thread-local message of the last failed call on this thread. */
const char* xw_last_error(void);

/* validate_params (xweigh_cuda.cu:1160-1241): XW_OK or XW_ERR_INVALID with
 * the reference's message. */
int32_t xw_validate_params(int32_t n, int32_t w, const xw_params* p);

/* xweigh_cuda::query_device (xweigh_cuda.cu:1382-1417) */
int32_t xw_query_device(int32_t ordinal, xw_device_info* out);

/* xweigh_cuda::run_annealer (xweigh_cuda.cu:1419-2436).  start_colmajor
 * (nullable, n*n) starts every replica from one validated state, as
 * initial_state does.  best_colmajor (caller-owned, n*n) receives the best
 * state.  log receives the reference's progress lines; checkpoint receives
 * the best state at most every save_interval seconds.  Stops on
 * xw_request_stop(), max_seconds, max_moves or a solve. */
int32_t xw_run(int32_t n, int32_t w, const xw_params* p, const int8_t* start_colmajor,
               xw_log_fn log, xw_checkpoint_fn checkpoint, void* user,
               xw_result* out, int8_t* best_colmajor);

/* The stop flag (g_stop, stop_signal.hpp:44).  Async-signal-safe. */
void xw_request_stop(void);
void xw_clear_stop(void);

/* ---- host-side helpers of the drop-in ------------------------------- */
/* State::random_start (xweigh_anneal.hpp:117-131) */
int32_t xw_random_start(int32_t n, int32_t w, uint32_t seed, int8_t* out_colmajor);
/* row-only start: w nonzeros per row at uniform positions, uniform signs */
int32_t xw_row_start(int32_t n, int32_t w, uint64_t seed, uint32_t replica, int8_t* out_colmajor);
/* State::sylvester_blocks (xweigh_anneal.hpp:133-149) */
int32_t xw_sylvester(int32_t n, int32_t w, int8_t* out_colmajor);
/* full recompute: stats = {L1 score, conflicts, squared, parity} over i<j */
int32_t xw_score(int32_t n, int32_t w, const int8_t* W_colmajor, int64_t stats[4]);
/* verify_support / verify_weighing (xweigh_anneal.hpp:221-264):
 * bit0 support, bit1 W W^T = wI */
int32_t xw_verify(int32_t n, int32_t w, const int8_t* W_colmajor);
/* read_state_csv (xweigh_anneal.hpp:669-756) */
int32_t xw_read_csv(const char* path, int32_t n, int32_t w, int8_t* out_colmajor);
/* write_entries_csv (xweigh_anneal.hpp:758-797), atomic temp + rename */
int32_t xw_write_csv(const char* path, int32_t n, const int8_t* W_colmajor);
/* impossibility_reason (xweigh_cuda_main.cpp:32-52); "" when none */
const char* xw_impossibility_reason(int32_t n, int32_t w);
/* calibrate_temperature (xweigh_anneal.hpp:881-899) on State s with seed */
double xw_calibrate(int32_t n, int32_t w, const int8_t* W_colmajor, const xw_params* p, uint32_t seed);

/* ---- batched populations (many independent searches, one device) ---- */
/* One search W(n,w): `replicas` replicas with starts derived from `seed`
 * (regular start of replica r: State::random_start(n, w, seed + r*0x9e3779b9)). */
typedef struct xw_job_spec {
    int32_t n, w;
    uint64_t seed;
    int32_t replicas;
    int32_t reserved;
    uint64_t max_moves;           /* per-job total move budget, 0 = the params' */
} xw_job_spec;

typedef struct xw_job_result {
    int64_t score, conflicts;     /* best over the job's replicas */
    int32_t best_replica;
    int32_t solved;
    int32_t verified;
    int32_t error;                /* nonzero: a replica failed a device self-check */
    uint64_t moves;
    uint64_t candidate_evaluations;
    uint64_t iterations;          /* max over replicas */
    uint64_t solved_iteration;    /* iteration of the first solve */
    double time_to_solution_seconds; /* device clock, from the first launch */
    uint64_t accepted_moves;      /* Metropolis acceptances (sum of 32-bit per-replica counters) */
    uint64_t accepted_rows;       /* rows of W those accepted moves changed (1 or 2 each) */
    uint64_t two_row_evaluations; /* candidate evaluations of moves that change two rows */
} xw_job_result;

typedef struct xw_batch xw_batch;

/* Build the jobs' start states (or copy `starts`, sum of R*n*n bytes in job
 * order, nullable) and upload them.  Tempering jobs form one ladder each. */
int32_t xw_batch_create(const xw_job_spec* jobs, int32_t njobs, const xw_params* p,
                        const int8_t* starts, xw_batch** out);
/* Bind the batch's work to a CUDA stream (cudaStream_t; NULL = its own). */
int32_t xw_batch_set_stream(xw_batch* b, void* cuda_stream);
/* Restore the uploaded start states on the device (no host transfer). */
int32_t xw_batch_reset(xw_batch* b);
/* Enqueue `iters` iterations per replica: rounds of exchange_interval (or
 * moves_per_launch) iterations, each one persistent launch (plus an
 * exchange launch when tempering), as one captured CUDA graph.  Returns
 * without waiting. */
int32_t xw_batch_run(xw_batch* b, uint64_t iters);
/* Same work as xw_batch_run, as plain stream launches with a CUDA event
 * pair around every anneal launch (for per-launch timing). */
int32_t xw_batch_run_timed(xw_batch* b, uint64_t iters);
int32_t xw_batch_synchronize(xw_batch* b);
/* Device milliseconds of each anneal launch of the last xw_batch_run_timed,
 * or of the whole graph launch of the last xw_batch_run (count 1). */
int32_t xw_batch_launch_times(xw_batch* b, float* ms, int32_t cap, int32_t* count);
/* Results per job; best (nullable) receives each job's best W in job order. */
int32_t xw_batch_results(xw_batch* b, xw_job_result* results, int8_t* best);
/* Snapshot of one replica (the per-replica state of DeviceStorage,
 * xweigh_cuda.cu:197-215, plus this implementation's Philox position). */
typedef struct xw_replica_state {
    uint64_t iterations;          /* Philox iteration counter */
    uint64_t moves;
    uint64_t candidate_evaluations;
    int64_t score, conflicts;
    int64_t best_score, best_conflicts;
    int64_t objective_total;
    double temperature, reheat_temperature;
    int32_t moves_since_improvement, cooling_counter, rung, objective_kind;
    uint32_t status, error;
    uint32_t accepted_moves, accepted_rows, two_row_evaluations;   /* 32-bit, wrapping */
    uint32_t reserved;
} xw_replica_state;

/* Read replica `replica` of job `job`: state, current W, best W (n*n each,
 * nullable) and the minority lists (n*min(w,n-w) entries, nullable: one
 * byte each for n <= XW_MAX_ORDER_SHARED, a native-endian uint16 each above). */
int32_t xw_batch_read_replica(xw_batch* b, int32_t job, int32_t replica, xw_replica_state* st,
                              int8_t* W, int8_t* best_W, uint8_t* minority);

/* Exact population snapshot (checkpoint / resume): the job table and every
 * replica record as they are on the device, with the batch's parameters,
 * ladders and initial temperatures, written atomically (temporary file +
 * rename).  A batch loaded from it continues bit-exactly where the saved one
 * stood: running K iterations, saving, loading and running L more gives the
 * state of K + L iterations in one batch.  `over` (nullable) replaces the
 * run-time settings (device, moves_per_launch, stop_on_solve,
 * warps_per_block, max_seconds); the file is specific to this build's struct
 * layout and is rejected otherwise.  No counterpart in the reference, which
 * checkpoints only the best W as CSV (write_entries_csv). */
int32_t xw_batch_save(xw_batch* b, const char* path);
int32_t xw_batch_load(const char* path, const xw_params* over, xw_batch** out);

/* Bytes the batch moves between host and device: h2d at creation (replica
 * records, job table, offsets, ladder), d2h per xw_batch_results call. */
int32_t xw_batch_bytes(xw_batch* b, uint64_t* h2d, uint64_t* d2h);

/* One elite restart of job `job` now, as xw_run makes one after
 * restart_interval seconds without improvement (xweigh_cuda.cu:1817-2289):
 * the job's best replica is the elite; restart_fraction of the others,
 * from a cursor that persists between calls, get kicked copies of its best
 * W (on the host or the device per params.restart_kicks).  *restarted
 * receives how many.  Cooling jobs only (a tempering job restarts none). */
int32_t xw_batch_restart(xw_batch* b, int32_t job, int32_t* restarted);

/* Launch shape of the batch's class with the most replicas: warps per
 * block, blocks, shared bytes per replica slot. */
int32_t xw_batch_shape(xw_batch* b, int32_t* warps_per_block, int32_t* blocks, int32_t* slot_bytes);

/* One launch of a batch's round.  Replicas of one rows-per-lane class (or
 * of the orders up to 16, which may share a warp two by two) run in one
 * launch with one shape; the launches of a round run side by side.  No
 * counterpart in the reference, which launches one search at a time. */
typedef struct xw_launch_class {
    int32_t min_order, max_order;
    int32_t large;                 /* orders above 256: 1 Gram matrix in HBM; 2 W as bit planes in
                                      shared memory, Gram entries recomputed; 3 bit planes and the
                                      Gram matrix in HBM; 0 below */
    int32_t rows_per_lane;         /* 1, 2, 4 or 8 (shared-memory kernel) */
    int32_t replicas_per_warp;     /* 1, or 2 (half-warp replicas, orders up to 16) */
    int32_t warps_per_block;
    int32_t blocks;
    int32_t slot_bytes;            /* shared memory per replica */
    int32_t chunks;                /* work items per replica and launch */
    int32_t replicas;
    int32_t general;               /* the general kernel (squared/parity objectives, row swaps) */
    int32_t warps_per_replica;     /* 1, or 2..64 in the latency mode (one replica per CTA, or
                                      per cluster of two CTAs above 16, four above 32) */
} xw_launch_class;
/* Up to `cap` launch classes of the batch into out; *count receives how
 * many there are. */
int32_t xw_batch_classes(xw_batch* b, xw_launch_class* out, int32_t cap, int32_t* count);
void xw_batch_destroy(xw_batch* b);

/* Launch-shape autotuner (the tunable is warps per CTA; each replica is one
 * warp): builds the batch, times `iters` iterations per replica at 1, 2, 4,
 * 8 and 16 warps per CTA (those that fit shared memory), records the fastest
 * for the batch's rows-per-lane class and shared-memory slot size in the
 * tuning cache (XW_TUNE_CACHE, default ~/.cache/xw_tune.txt), which later
 * batches and servers with warps_per_block = 0 use.  best_ms (nullable)
 * receives the winner's device milliseconds. */
int32_t xw_autotune(const xw_job_spec* jobs, int32_t njobs, const xw_params* p, uint64_t iters,
                    int32_t* best_wpb, float* best_ms);

/* Whole batched search through host buffers: upload, run until every job
 * is solved or out of budget (or `iters` per replica when nonzero), read
 * back.  The end-to-end call of the served-batch benchmark. */
int32_t xw_batch_solve(const xw_job_spec* jobs, int32_t njobs, const xw_params* p,
                       const int8_t* starts, uint64_t iters,
                       xw_job_result* results, int8_t* best);

/* ---- batched exact rescoring and verification ------------------------- */
/* Full recompute of G = W W^T for `count` row-major n x n int8 matrices
 * (contiguous), the batched form of rebuild_gram_bits + verify_weighing
 * (xweigh_anneal.hpp:429-453, 239-264).  stats receives 4 int32 per matrix:
 * L1 score sum_{i<j}|G_ij|, conflicts #{i<j: G_ij != 0}, squared score
 * sum_{i<j} G_ij^2, and 1 when G = wI exactly (else 0).  gram (nullable)
 * receives each G as n*n row-major int32.  n a multiple of 32 runs on the
 * tensor cores (tcgen05 kind::i8, int32 accumulation, exact since
 * |G_ij| <= n); other n <= 128 on a SIMT kernel.  Host buffers. */
int32_t xw_rescore(const int8_t* W_rowmajor, int64_t count, int32_t n, int32_t w, int32_t* stats,
                   int32_t* gram);
/* Same on device buffers, enqueued on `stream` (cudaStream_t); simt != 0
 * forces the SIMT kernel.  Allocates nothing.  Check xw_rescore_status()
 * after the stream completes. */
int32_t xw_rescore_device(const int8_t* W_rowmajor, int64_t count, int32_t n, int32_t w, int32_t* stats,
                          int32_t* gram, int32_t simt, void* stream);
/* XW_OK, or XW_ERR_TIMEOUT when a rescoring pipeline wait expired since the
 * last call (the flag is cleared).  Synchronous. */
int32_t xw_rescore_status(void);

/* ---- elite restarts --------------------------------------------------- */
/* The escape-move scan of an elite restart (xweigh_cuda.cu:1870-2057), on
 * the device: every support switch out of W (rows r1 < r2, a column c1
 * nonzero in r1 and zero in r2, a column c2 nonzero in r2 and zero in r1,
 * new signs new1 at (r1,c2) and new2 at (r2,c1)) with its exact change of
 * the L1 score and of the conflicts; `out` receives the `limit` best by
 * (score delta, conflict delta), ties in scan order (r1, r2, c1, c2, new1,
 * new2), and *count how many (fewer when there are fewer switches).
 * xw_run's restarts use it.  W: n*n column-major, rows of weight w. */
typedef struct xw_escape_move {
    int32_t row1, row2, col1, col2, new1, new2;
    int64_t score_delta, conflict_delta;
} xw_escape_move;
int32_t xw_escape_scan(int32_t n, int32_t w, const int8_t* W_colmajor, int32_t limit, xw_escape_move* out,
                       int32_t* count);

/* ---- serving: continuous batching of search requests ------------------ */
/* The reference serves one search per process: xweigh_cuda_main.cpp:281-285
 * calls run_annealer (xweigh_cuda.cu:1419-2436), which allocates, anneals
 * and frees one population.  A server instead keeps one device's
 * population resident and admits requests while earlier ones run.  Each
 * request is one W(n,w) search (an xw_job_spec with its own parameters):
 * host worker threads build its start states and records; the engine
 * thread admits it when its replicas fit the resident cap and its records
 * fit the device arena (first come, first served), and every engine round
 * advances resident requests by `quantum_iters` iterations per replica:
 * all of them, or (the default) those with the least attained iterations,
 * so that requests that solve early are not queued behind long searches.
 * A request ends at the end of the round in which its first replica solved,
 * its move budget or time limit ran out, or it was cancelled.
 *
 * Replicas of a served request stop at their own solve (stop_on_solve 2)
 * and run rounds of a fixed length from the request's own start, so the
 * first solution, its iteration, the best W and the move counts of a
 * request are the same whether it ran alone or among other requests; only
 * times differ.  Thread safety: any thread may submit, poll, wait, cancel
 * and read stats concurrently. */
#define XW_REQ_QUEUED 0    /* accepted, not yet on the device */
#define XW_REQ_RUNNING 1   /* resident on the device */
#define XW_REQ_DONE 2      /* solved, out of budget or out of time */
#define XW_REQ_CANCELLED 3
#define XW_REQ_FAILED 4    /* see status and error */

typedef struct xw_server_config {
    int32_t device;
    int32_t quantum_iters;         /* iterations per replica per engine round (default 2000) */
    int32_t max_requests;          /* resident requests (job slots, default 1024) */
    int32_t max_resident_replicas; /* admission cap on resident replicas (0 = the replica id
                                      space) */
    int32_t max_replica_ids;       /* replica id space (default 262144) */
    int32_t warps_per_block;       /* 0 = tuned */
    int32_t prep_threads;          /* host threads building start states (0 = half the cores) */
    int32_t sylvester_shortcut;    /* 1: a power-of-two w dividing n is answered by Sylvester
                                      blocks without search (xweigh_cuda_main.cpp:270-277) */
    uint64_t arena_bytes;          /* device bytes for resident replica records (default 1 GiB) */
    int32_t schedule;              /* XW_SCHED_ALL: every resident request advances every round;
                                      XW_SCHED_LEAST_ATTAINED (default): each round advances the
                                      requests with the fewest iterations so far, oldest first,
                                      up to max_active_replicas */
    int32_t max_active_replicas;   /* replicas advanced per round under XW_SCHED_LEAST_ATTAINED
                                      (0 = eight waves of the device's resident warps) */
    int32_t replicas_per_warp;     /* orders up to 16: 1 or 2 replicas per warp, 0 = tuned */
    int32_t reserved[5];
} xw_server_config;

#define XW_SCHED_ALL 0
#define XW_SCHED_LEAST_ATTAINED 1

typedef struct xw_request {
    int32_t n, w;
    uint64_t seed;                 /* Philox key and start seeds, as xw_job_spec */
    int32_t replicas;
    int32_t reserved;
    uint64_t max_moves;            /* total move budget, 0 = params->max_moves (0 = none) */
    const xw_params* params;       /* nullable: xw_params_default; device, replicas,
                                      moves_per_launch and stop_on_solve are the server's;
                                      max_seconds limits the request's time on the device */
    const int8_t* starts;          /* nullable: replicas*n*n column-major start states */
} xw_request;

typedef struct xw_request_result {
    int32_t state;                 /* XW_REQ_* */
    int32_t status;                /* XW_OK, or the failure's code */
    int32_t n, w;
    int32_t replicas;
    int32_t solved;                /* a replica reached score 0 */
    int32_t verified;              /* the returned W satisfies W W^T = wI (int64 check) */
    int32_t sylvester;             /* answered without search */
    int32_t best_replica;          /* the first solver, else least (score, conflicts, index) */
    int32_t reserved;
    int64_t score, conflicts;      /* of the returned W */
    uint64_t moves;
    uint64_t candidate_evaluations;
    uint64_t iterations;           /* per replica, max over replicas */
    uint64_t solved_iteration;     /* the first solver's solve iteration */
    double submit_seconds;         /* server clock (seconds since creation) */
    double admit_seconds;          /* -1 until resident */
    double finish_seconds;         /* -1 until finished */
    double time_to_solution_seconds; /* submit -> first exact solution (device clock), -1 if none */
    double t_init;                 /* initial temperature used */
    char error[192];
} xw_request_result;

typedef struct xw_server_stats {
    uint64_t submitted, admitted, finished, solved, cancelled, failed, sylvester;
    uint64_t queued, running;      /* now */
    uint64_t resident_replicas;    /* now */
    uint64_t rounds;               /* engine rounds run */
    uint64_t moves;                /* moves of finished requests */
    double device_seconds;         /* device time of all rounds */
    double busy_seconds;           /* engine wall time with requests resident */
    uint64_t arena_bytes, arena_bytes_used;
    int32_t quantum_iters, max_resident_replicas;
    int32_t schedule, max_active_replicas;
} xw_server_stats;

typedef struct xw_server xw_server;

void xw_server_config_default(xw_server_config* c);
/* Allocates the device arena and tables and starts the engine and worker
 * threads. */
int32_t xw_server_create(const xw_server_config* c, xw_server** out);
/* Queue a request.  Fails at once (XW_ERR_INVALID with the reference's
 * validation or impossibility message, XW_ERR_CAPACITY when it can never
 * fit) instead of failing later. */
int32_t xw_submit(xw_server* s, const xw_request* r, uint64_t* id);
/* Current state of a request; best (nullable, n*n column-major) receives
 * the returned W once the request has finished. */
int32_t xw_poll(xw_server* s, uint64_t id, xw_request_result* res, int8_t* best_colmajor);
/* Wait until the request finishes or timeout_seconds pass (< 0: no limit);
 * XW_ERR_TIMEOUT when it is still unfinished. */
int32_t xw_wait(xw_server* s, uint64_t id, double timeout_seconds, xw_request_result* res,
                int8_t* best_colmajor);
/* Checkpoint of a request: the reference writes its best W to best_W.csv
 * every save_interval during a run (xweigh_cuda.cu:2350-2362).  For a
 * running request this waits (timeout_seconds < 0: no limit) until the end
 * of the next engine round that it is resident for and returns its progress
 * then (moves, iterations, the score and conflicts of its best W) with
 * best (nullable, n*n column-major) receiving that W: the first solver's,
 * else the least (score, conflicts, replica).  A finished request: as
 * xw_poll.  XW_ERR_TIMEOUT when no round ended in time (a queued request
 * waits for its admission). */
int32_t xw_checkpoint(xw_server* s, uint64_t id, double timeout_seconds, xw_request_result* res,
                      int8_t* best_colmajor);
/* Exact snapshot of a running request's population -- its job entry, every
 * replica record, its ladder and initial temperature -- as the next engine
 * round leaves them, written atomically to `path` in the format of
 * xw_batch_save (one job).  Resume it in a server with xw_submit_snapshot
 * or as a batch with xw_batch_load: the search continues move for move.
 * Fails with XW_ERR_INVALID for a finished request, XW_ERR_IO when the file
 * cannot be written, XW_ERR_TIMEOUT when no round ended in time (the
 * snapshot is then still written, its result dropped).  The engine thread
 * writes the file, which delays the next round by that long.  No
 * counterpart in the reference, which can only restart from a CSV. */
int32_t xw_request_save(xw_server* s, uint64_t id, const char* path, double timeout_seconds);
/* Queue a request that continues the population of a one-job snapshot
 * (xw_request_save, or xw_batch_save of a batch of one job of an order the
 * server takes).  Its parameters are the snapshot's; device, replicas and
 * stop rule are the server's, as for xw_submit. */
int32_t xw_submit_snapshot(xw_server* s, const char* path, uint64_t* id);
/* Cancel: a queued request ends at once, a resident one at the end of the
 * current round with its best W so far.  No effect on finished requests. */
int32_t xw_cancel(xw_server* s, uint64_t id);
/* Forget a finished request (its result and W). */
int32_t xw_release(xw_server* s, uint64_t id);
int32_t xw_server_get_stats(xw_server* s, xw_server_stats* out);
/* Stops the threads (unfinished requests end cancelled) and frees the
 * device memory. */
void xw_server_destroy(xw_server* s);

/* ---- the CPU annealer ------------------------------------------------- */
/* The reference's CPU tool xweigh (src/xweigh_main.cpp, engine
 * src/xweigh_anneal.hpp:909-1291): one worker thread per core, each
 * annealing its own state, a parallel-tempering ladder over the workers
 * when there are two or more, the monitor's exchanges and best-matrix
 * writes.  The fallback for hosts without a B200.  xw_cpu_params mirrors
 * xweigh::Params (xweigh_anneal.hpp:42-67) field for field, without the
 * Windows pinning switches. */
typedef struct xw_cpu_params {
    int32_t threads;              /* worker threads (default: hardware threads) */
    int32_t tempering;            /* 1: parallel tempering for two or more workers */
    uint64_t seed;                /* 0 = random_device */
    double max_seconds;
    double save_interval;
    double sign_fraction;
    double greedy_fraction;
    int32_t candidate_samples;
    double target_fraction;
    int32_t target_samples;
    int32_t exchange_interval;    /* moves per worker between exchanges */
    double t_init;                /* 0 = calibrate */
    double t_min;
    double cooling;
    int32_t moves_per_cool;
    int32_t stuck_threshold;
    double reheat;
    double reseed_factor;
} xw_cpu_params;

typedef struct xw_cpu_result {
    int64_t score, conflicts;     /* of the best W */
    int32_t solved, verified;
    uint64_t moves;
    double seconds;               /* search time */
    double t_init;                /* the (calibrated) initial temperature */
    int32_t threads;
    int32_t reserved;
} xw_cpu_result;

void xw_cpu_params_default(xw_cpu_params* p);
/* run_annealer (xweigh_anneal.hpp:1106-1291) from `start` (nullable:
 * State::random_start with the seed), with the reference's log lines through
 * `log`, best-matrix writes through `checkpoint` every save_interval, and
 * xw_request_stop as the stop flag.  best_out (nullable) receives the best
 * W, column-major. */
int32_t xw_cpu_run(int32_t n, int32_t w, const xw_cpu_params* p, const int8_t* start, xw_log_fn log,
                   xw_checkpoint_fn checkpoint, void* user, xw_cpu_result* out, int8_t* best_out);

/* ---- annealing without device allocation ------------------------------ */
/* No counterpart in the reference: an entry point for callers that cannot
 * call cudaMalloc -- hosts whose device memory belongs to their own pool
 * allocator or fixed budget, and loops that cannot take the device
 * synchronisation that cudaMalloc/cudaFree imply.  It anneals one W(n,w)
 * search of `replicas` replicas for `iters` iterations with the batch
 * engine's kernels (cooling, or a tempering ladder when p->tempering),
 * keeping all scratch state in a static device array of
 * XW_NOALLOC_SCRATCH_BYTES (4 MiB) that every GPU loading this library holds
 * until exit; a request that needs more is rejected with XW_ERR_CAPACITY.
 * Inputs and outputs are the caller's device buffers:
 *   starts  replicas*n*n int8, column-major start states
 *   best    replicas*n*n int8, each replica's best state
 *   stats   replicas*4 int64: best score, best conflicts, score, moves;
 *           a replica the kernel refused (a start row whose weight is not
 *           w, a failed device self-check) reports best score -1, best
 *           conflicts -(its XW_ERR_* device error bits) and score -1
 * p->t_init must be positive (no host calibration).  Work is enqueued on
 * `stream` (cudaStream_t, NULL = legacy default) and the call returns
 * without waiting.  The first call on a device looks up the array's device
 * address (cudaGetSymbolAddress) with that device current; make it before
 * any stream capture.  Calls share the array: calls that overlap on the GPU
 * race, so serialise them; each call rewrites the array from its inputs. */
#define XW_NOALLOC_SCRATCH_BYTES (4 * 1024 * 1024)
int32_t xw_anneal_noalloc(int32_t n, int32_t w, const xw_params* p, int32_t replicas, uint64_t iters,
                          const int8_t* starts, int8_t* best, int64_t* stats, void* stream);

#ifdef __cplusplus
}
#endif
#endif
