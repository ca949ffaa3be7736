/* xw_oracle.h -- CPU restatement of the weighing-matrix annealer.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker that the parity
 * tests, smoke() and the bench's cpu_baseline leg compare the CUDA path with.
 * The product never links, loads or calls it.
 *
 * Two families of functions:
 *  - reference mode: the CPU engine of flinty-mathematics/xtax
 *    (src/xweigh_anneal.hpp), restated in C with its mt19937 stream and the
 *    libstdc++ distributions it draws through.  Pinned against the reference
 *    itself (oracle/_ref/ref_harness, tests/golden/).
 *  - device mode: the population algorithm of the reference's xweigh_cuda
 *    kernel (src/xweigh_cuda.cu:291-1130) with the counter-based Philox draw
 *    layout the CUDA kernel uses, replayed one replica at a time.
 */
#ifndef XW_ORACLE_H
#define XW_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define XWO_MAX_N 1024

/* ---- random streams ---------------------------------------------------- */
void xwo_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]);
/* first `count` outputs of std::mt19937(seed) */
void xwo_mt_stream(uint32_t seed, int count, uint32_t* out);
/* std::uniform_int_distribution<int>(0, range-1) draws (libstdc++ >= 11) */
void xwo_mt_uniform_stream(uint32_t seed, uint32_t range, int count, uint32_t* out);
/* std::generate_canonical<double,53> draws */
void xwo_mt_canonical_stream(uint32_t seed, int count, double* out);
/* the acceptance exponential shared bit-for-bit with the device */
double xwo_exp(double x);

/* ---- states and scores -------------------------------------------------- */
void xwo_random_start(int n, int w, uint32_t seed, int8_t* W_colmajor);
void xwo_sylvester(int n, int w, int8_t* W_colmajor);
/* row-only start: w nonzeros per row at uniform positions, uniform signs,
 * drawn from the init stream of (key, stream) */
void xwo_row_start(int n, int w, uint32_t key0, uint32_t key1, uint32_t stream,
                   int8_t* W_colmajor);
/* full recompute in int64: stats = {L1 score, conflicts, squared, parity}
 * over pairs i<j; G (n*n row-major, nullable), row residuals (nullable) */
void xwo_rescore(int n, int w, const int8_t* W_colmajor, int64_t stats[4],
                 int64_t* G, int64_t* residual);
/* bit0: row and column weights are w and entries ternary; bit1: W W^T = wI */
int xwo_verify(int n, int w, const int8_t* W_colmajor);

/* ---- reference mode (xweigh CPU engine) --------------------------------- */
typedef struct {
    double sign_fraction, greedy_fraction, target_fraction;
    int32_t candidate_samples, target_samples;
    double t_init, t_min, cooling, reheat, reseed_factor;
    int32_t moves_per_cool, stuck_threshold;
} xwo_ref_params;

void xwo_ref_params_default(xwo_ref_params* p);
/* calibrate_temperature on random_start(n, w, seed) with that seed, as
 * run_annealer does (anneal.hpp:1110-1114) */
double xwo_calibrate(int n, int w, uint32_t seed, const xwo_ref_params* p);

typedef struct {
    int64_t moves, accepted, score, conflicts, best_score, best_conflicts;
    double initial_temperature, temperature;
    uint32_t worker_seed;
    uint64_t hash;
} xwo_walk_result;

/* run_annealer with one thread: random start from `seed`, calibration,
 * anneal_worker until solved or max_moves moves */
void xwo_ref_walk(int n, int w, uint32_t seed, int64_t max_moves,
                  const xwo_ref_params* p, xwo_walk_result* r,
                  int8_t* start_out, int8_t* final_out, int8_t* best_out);

/* ---- device mode -------------------------------------------------------- */
typedef struct {
    int32_t n, w;
    int32_t tempering;          /* 0: cooling/reheat per replica; 1: fixed rung temperatures */
    int32_t move_set;           /* 0: flip, switch (signed), double flip; 1: flip, within-row swap */
    int32_t candidate_samples, target_samples;
    int32_t moves_per_cool, stuck_threshold;
    uint32_t key0, key1;
    int32_t objective;          /* -1: per-replica hash rule; 0 L1, 1 squared, 2 parity */
    int32_t pad_;
    double greedy_fraction, target_fraction, double_sign_fraction,
           sign_fraction, switch_sign_fraction;
    double squared_objective_fraction, parity_objective_fraction;
    double t_min, cooling, reheat;
} xwo_job;

typedef struct {
    uint64_t it, moves, cand_evals;
    int64_t score, conflicts, obj_total, best_score, best_conflicts;
    double temperature, reheat_temperature;
    int32_t msi, cool_ctr, rung, obj_kind;
} xwo_replica_scalars;

typedef struct xwo_replica xwo_replica;

/* replica `index` of the job, starting from W0 at temperature t0 (rung for
 * tempering); all incremental structures are built by full recompute */
xwo_replica* xwo_rep_create(const xwo_job* job, uint32_t index, const int8_t* W0,
                            double t0, int32_t rung);
void xwo_rep_destroy(xwo_replica* r);
/* run `iters` device iterations; stop early when best score reaches 0 and
 * stop_on_solve; returns iterations run */
int64_t xwo_rep_run(xwo_replica* r, int64_t iters, int stop_on_solve);
void xwo_rep_get(const xwo_replica* r, xwo_replica_scalars* s, int8_t* W,
                 int8_t* best_W, uint16_t* minority, int32_t* G, int32_t* residual);
void xwo_rep_set_temperature(xwo_replica* r, double t, int32_t rung);
/* incremental state vs full recompute: 0 when consistent */
int xwo_rep_check(const xwo_replica* r);

/* one adjacent-rung exchange sweep over a job's R replicas (ladder[R]),
 * round number `round`; updates rungs and temperatures; returns swaps */
int xwo_exchange(const xwo_job* job, xwo_replica** reps, int R,
                 const double* ladder, uint64_t round);

/* one move of kind 0 flip, 1 switch (new values v1,v2), 2 double flip,
 * 3 within-row swap (new value v1) on W; deltas in out[4]; commits into W
 * when `commit`; returns the full-recompute consistency flags after commit */
int xwo_move_eval(int n, int w, int8_t* W, int kind, int r1, int r2, int c1, int c2,
                  int v1, int v2, int commit, int64_t out[4]);

/* The device kick of an elite restart (restart mode 1): replica `replica`,
 * the index-th restarted in restart round `round`, from the elite E
 * (column-major), with the escape move esc = {row1, row2, col1, col2,
 * new1, new2} (NULL: none), `kick` steps and the sign-flip threshold
 * thr_sign on a 32-bit draw.  Writes the kicked W to K. */
void xwo_kick(int n, int w, const int8_t* E, const int32_t* esc, uint32_t key0, uint32_t key1, uint64_t round,
              uint32_t replica, uint32_t index, int kick, uint64_t thr_sign, int8_t* K);

#ifdef __cplusplus
}
#endif
#endif
