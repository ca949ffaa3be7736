// xw_host_internal.h -- the batch engine shared by the C ABI entry points.
#pragma once

#include <cuda_runtime.h>

#include <string>
#include <vector>

#include "../../include/xw.h"
#include "xw_cpu.h"
#include "xw_kernels.h"

namespace xw {

std::string validate(int n, int w, const xw_params& p);
// the parameters need the general anneal kernel: the squared or parity
// objective on some replica, or the within-row swap move set
bool needs_general_kernel(const xw_params& p);
void set_last_error(const std::string& msg);
// The least order that runs on the HBM-resident kernel: XW_MAX_N + 1, or
// the value of XW_LARGE_MIN_ORDER in [1, XW_MAX_N + 1] (tests run small
// orders through that kernel to compare it with the shared-memory one).
int large_min_order();
std::string strfmt(const char* f, ...);
// throws std::runtime_error naming `what` when e is an error
void check_cuda(cudaError_t e, const char* what);

// One job's table entry (every field but rep_begin and ladder_off), its
// replicas' records (replicas * J.record_bytes bytes, headers naming job
// `job_index`), its rung temperatures and its initial temperature.  starts
// (nullable) holds replicas*n*n column-major start states; otherwise the
// starts follow params.start_kind.  parallel: build the starts on all host
// threads.
void prepare_job(const xw_job_spec& spec, const xw_params& params, const int8_t* starts, uint32_t job_index,
                 bool parallel, XwJob& J, std::vector<uint8_t>& records, std::vector<double>& temps,
                 double& t_init);

// Enqueues the batched rescoring kernel (xw_rescore.cu).
int32_t rescore_device(const int8_t* W, int64_t count, int n, int w, int32_t* stats, int32_t* gram,
                       cudaStream_t stream, int* err_flag, bool force_simt);

// Warps per block for the anneal kernel of a given lanes-per-row class and
// shared-memory slot, from the autotuner's cache (xw_tune.cpp).
int tuned_warps_per_block(int opl, uint32_t slot_bytes, int device);
// Chunks per replica and launch for `replicas` on `slots` resident warps
// (XW_CHUNKS overrides: tests compare chunked and whole-replica launches).
uint32_t choose_chunks(uint32_t replicas, uint32_t slots);
// Record the fastest warps per block for that class in the tuning cache.
void record_tuned(int opl, uint32_t slot_bytes, int wpb);

struct Batch {
    xw_params params{};
    cudaDeviceProp props{};
    cudaStream_t stream = nullptr;
    bool own_stream = false;

    std::vector<XwJob> jobs;
    std::vector<uint32_t> rep_seed;
    std::vector<uint64_t> rec_off;
    std::vector<uint32_t> items;
    std::vector<double> ladder;
    std::vector<size_t> best_offsets;
    std::vector<double> t_init_used;
    uint32_t total_replicas = 0;
    size_t arena_bytes = 0;
    size_t best_bytes = 0;
    bool tempering = false;

    int opl = 1;
    bool general = false;      // some job needs the general kernel
    uint32_t slot_bytes = 0;
    int warps_per_block = 4;
    int blocks_per_sm = 1;
    int blocks = 1;
    // shared-memory kernel: work items per replica and launch (see
    // AnnealArgs::chunks), chosen so that the resident warps' waves fill
    uint32_t chunks = 1;
    void* d_chunk_done = nullptr;

    // jobs with J.large run on the HBM-resident kernel: items[0, n_large)
    // are their replicas; the rest run on the shared-memory kernel
    uint32_t n_large = 0;
    bool general_large = false;
    uint32_t large_slot_bytes = 0;
    int large_wpb = 4;
    int large_blocks = 1;
    uint32_t large_chunks = 1;
    std::vector<uint64_t> gram_off;   // per replica, into d_gram
    size_t gram_bytes = 0;

    void* d_jobs = nullptr;
    void* d_jobs0 = nullptr;
    void* d_arena = nullptr;
    void* d_arena0 = nullptr;
    void* d_rec_off = nullptr;
    void* d_items = nullptr;
    void* d_counters = nullptr;
    int counters_cap = 0;
    void* d_ladder = nullptr;
    void* d_out = nullptr;
    void* d_best_off = nullptr;
    void* d_best = nullptr;
    void* d_t0 = nullptr;
    void* d_gram = nullptr;
    void* d_gram_off = nullptr;
    uint64_t t0_host = 0;

    std::vector<cudaEvent_t> events;
    int last_rounds = 0;
    cudaGraphExec_t graph_exec = nullptr;
    uint64_t graph_iters = 0;

    Batch() = default;
    Batch(const Batch&) = delete;
    Batch& operator=(const Batch&) = delete;
    ~Batch();

    // device memory from the engine's per-device pool, in the batch's stream
    void dalloc(void** ptr, size_t bytes, const char* what);
    void build(const xw_job_spec* specs, int njobs, const xw_params& p, const int8_t* starts);
    void derive_layout();
    void upload(const std::vector<uint8_t>& host);
    void save(const std::string& path);
    // rebuild from a snapshot; `over` (nullable) replaces the run-time
    // settings (device, launch length, stop mode, shape, time limit)
    void load(const std::string& path, const xw_params* over);
    void configure_shape(int warps_per_block);
    void reset();
    uint64_t round_iters() const;
    void reserve_rounds(int rounds);
    void enqueue_rounds(uint64_t iters, bool timed);
    void run(uint64_t iters, bool use_graph);
    void collect(std::vector<JobOut>& out, int8_t* best_host, bool want_best);
    void fill_results(const std::vector<JobOut>& out, const int8_t* best_host, xw_job_result* res) const;
};

// Population snapshot: the job table and every replica record, with the
// parameters, ladder and initial temperatures.  File layout (native byte
// order, this build's struct sizes):
//   "XWPOP001" | u32 sizeof(XwJob), sizeof(RepHeader), sizeof(xw_params), njobs
//   | u64 replicas, arena bytes, ladder entries | xw_params | XwJob[njobs]
//   | u64 record offsets[replicas] | f64 ladder[] | f64 t_init[njobs] | arena
// written to a temporary file and renamed into place.  Batches and served
// requests write and read the same format.
struct Snapshot {
    xw_params params{};
    std::vector<XwJob> jobs;
    std::vector<uint64_t> rec_off;
    std::vector<double> ladder;
    std::vector<double> t_init;
    std::vector<uint8_t> arena;
};
void write_snapshot(const std::string& path, const Snapshot& sn);
// checks that every record lies in the arena and names its job; clears the
// records' Gram-arena bits
Snapshot read_snapshot(const std::string& path);

// The escape-move scan of an elite restart on the device (xw_restart.cu): the
// `limit` best support switches out of the column-major W (G its Gram,
// row-major) by (score delta, conflict delta, scan order).
std::vector<ScanResult> escape_scan(int n, const int8_t* W, const int32_t* G, size_t limit);

// Elite-restart bookkeeping of one job (the reference's restart_cursor,
// restart_round and restarted_replicas, xweigh_cuda.cu:1812-1814).
struct RestartState {
    size_t cursor = 0;
    uint64_t round = 0;
    uint64_t restarted = 0;
    int elite = 0;
};

// Escape-scan cost (operations) for an elite W, and the most a restart
// spends on it: above, restarts kick without an escape move.
double escape_scan_work(int n, const std::vector<int8_t>& W);
constexpr double kEscapeScanBudget = 1.0e12;

// Elite restart of job j's replicas (xweigh_cuda.cu:1817-2289); returns how
// many replicas were restarted and the reference's log line.
int restart_population(Batch& b, int j, const std::vector<int8_t>& elite_best, int64_t gbest, int64_t gconf,
                       RestartState& rs, double elapsed, std::string& line);

}  // namespace xw
