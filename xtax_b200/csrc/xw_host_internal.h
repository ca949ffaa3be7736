// xw_host_internal.h -- the batch engine shared by the C ABI entry points.
#pragma once

#include <cuda_runtime.h>

#include <atomic>
#include <mutex>
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
// the flag xw_request_stop sets
const std::atomic<int>& stop_flag();
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

// Enqueues the batched rescoring kernel (xw_rescore.cu).  dims (nullable,
// device): per matrix {order, weight} of a matrix zero-padded to n x n.
int32_t rescore_device(const int8_t* W, int64_t count, int n, int w, int32_t* stats, int32_t* gram,
                       cudaStream_t stream, int* err_flag, bool force_simt, const int2* dims = nullptr);

// Exact verification of search results on the device: column-major W of
// order n <= 256 and weight w, in device memory, each gathered into a
// zero-padded row-major matrix and rescored in one batch per padded order
// (tensor cores up to 128).  Per item {L1 score, conflicts, squared score,
// exact (W W^T = wI)}, the reference's rebuild_gram_bits + verify_weighing
// (xweigh_anneal.hpp:239-264, 429-453).  Keeps its scratch between calls.
struct VerifyItem {
    const int8_t* W;
    int32_t n, w;
};
struct VerifyStats {
    int32_t score, conflicts, squared, exact;
};
struct DeviceVerifier {
    VerifyItem* d_items = nullptr;
    int32_t* d_index = nullptr;
    int8_t* d_stage = nullptr;
    int2* d_dims = nullptr;
    int4* d_stats = nullptr;
    void* h_stats = nullptr;
    void* h_table = nullptr;
    size_t cap_items = 0, cap_stage = 0;
    DeviceVerifier() = default;
    DeviceVerifier(const DeviceVerifier&) = delete;
    DeviceVerifier& operator=(const DeviceVerifier&) = delete;
    ~DeviceVerifier();
    void reserve(size_t items, size_t stage_bytes);
    // enqueues on `stream`, waits, and returns the stats in item order
    void run(const std::vector<VerifyItem>& items, cudaStream_t stream, std::vector<VerifyStats>& out);
};
// The verifier batches share on a device (its scratch is allocated once and
// kept: a batch's own would pay pinned-memory allocations and a cudaFree
// per batch), with the mutex that serialises its users.
DeviceVerifier& shared_verifier(int device, std::mutex*& mu);

// Launch-shape classes of the autotuner (xw_tune.cpp): the rows-per-lane
// class of the order (1, 2, 4, 8), or kTunePairKind for orders up to 16
// (with at most 16 candidates per move), which may run two replicas per warp.
constexpr int kTunePairKind = 16;
int tune_kind(int n, int candidate_samples);
struct TunedShape {
    int wpb;   // warps per CTA
    int rpw;   // replicas per warp
};
// The tuned shape of a class and shared-memory slot size, from the cache
// (XW_WARPS_PER_BLOCK and XW_REPLICAS_PER_WARP override it).
TunedShape tuned_shape(int kind, uint32_t slot_bytes, int device);
// Warps per replica of the latency mode for a class of at most one replica
// per SM (1: the one-warp kernel), from the cache under kTuneLatencyKind
// (XW_WARPS_PER_REPLICA overrides it); 8 without an entry.
constexpr int kTuneLatencyKind = 32;
int tuned_warps_per_replica(uint32_t slot_bytes, int device);
// Warps per block alone (the serving loop's classes of rows per lane).
int tuned_warps_per_block(int opl, uint32_t slot_bytes, int device);
// Chunks per replica and launch for `replicas` on `slots` resident warps
// (XW_CHUNKS overrides: tests compare chunked and whole-replica launches).
uint32_t choose_chunks(uint32_t replicas, uint32_t slots);
// Device-time limit of a chunk's wait for its replica's previous chunk
// (AnnealArgs::chunk_wait_ns): 0, the kernel's 30 s, unless XW_CHUNK_WAIT_NS
// sets another (tests make the wait run out with a short one).
uint64_t chunk_wait_limit_ns();
// Raises the kernel's dynamic shared-memory limit to the device's opt-in
// maximum.  Every caller sets the same value, so no caller ever lowers the
// limit another one relies on (the attribute is per kernel and process-wide).
void raise_smem_limit(const void* fn, int device);
// The device's properties, queried once per device and kept (the query
// took from 8 to over 100 ms per call on a loaded B200 host).
const cudaDeviceProp& device_properties(int device);
// Record the fastest shape for that class in the tuning cache.
void record_tuned(int kind, uint32_t slot_bytes, int wpb, int rpw);

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

    // The shared-memory kernel runs one launch per class and round: the
    // replicas of one tuning kind (rows-per-lane class, or the orders up to
    // 16) share a kernel instantiation, a slot size (the class's largest
    // order's) and a CTA shape; items[item_begin, item_begin + item_count)
    // are the class's replicas.  Classes' launches of a round run side by
    // side on their own streams.
    struct LaunchClass {
        int kind = 1, opl = 1, rpw = 1;
        // warps per replica: 1, or 2..64 for the latency mode (orders up to
        // 32), whose `ctas` CTAs (one, or a cluster of two or four) of
        // wpr / ctas warps each hold a copy of one replica (spec_bytes)
        int wpr = 1, ctas = 1;
        uint32_t spec_bytes = 0;
        bool general = false;
        // every job of the class has one zero per row (w = n - 1): the lean
        // one-row kernel runs its instantiation for that shape
        bool one_zero = true;
        int min_n = 0, max_n = 0;
        uint32_t slot_bytes = 0;
        uint32_t item_begin = 0, item_count = 0;
        int wpb = 4, blocks = 1, blocks_per_sm = 1;
        // work items per replica and launch (see AnnealArgs::chunks), chosen
        // so that the resident groups' waves fill
        uint32_t chunks = 1;
    };
    std::vector<LaunchClass> classes;
    // launches of a round in issue order: class index, or -1 for the
    // large-order kernel
    std::vector<int> launch_order;
    // keep the orders up to 16 in a class of their own even at one replica
    // per warp (the autotuner times them apart)
    bool split_pair_class = false;
    void* d_chunk_done = nullptr;
    std::vector<cudaStream_t> side_streams;
    std::vector<cudaEvent_t> side_events;    // fork, then one join per launch

    // jobs with J.large run on the HBM-resident kernel: items[0, n_large)
    // are their replicas; the rest run on the shared-memory kernel
    uint32_t n_large = 0;
    bool general_large = false;
    int large_form = 0;          // the large-order class's kernel form (anneal_large_kernel_fn)
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
    int counters_per_round = 0;
    void* d_ladder = nullptr;
    void* d_out = nullptr;
    void* d_best_off = nullptr;
    void* d_best = nullptr;
    void* d_t0 = nullptr;
    void* d_gram = nullptr;
    void* d_gram_off = nullptr;
    uint64_t t0_host = 0;

    // collect() with the best states checks every job's best W of order
    // <= 256 on the device (score, conflicts, exact flag per job)
    std::vector<VerifyStats> vstats;
    std::vector<char> vstats_valid;

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
    // every class's shape: params' warps per block and replicas per warp
    // where set, else the tuned ones
    void configure_shape();
    // class k's shape; false when it does not fit the device
    bool configure_class(size_t k, int wpb, int rpw);
    // class k in the latency mode with `wpr` warps per replica
    bool configure_latency(size_t k, int wpr);
    // launches per round (classes plus the large-order kernel)
    int launches_per_round() const { return (int)classes.size() + (n_large ? 1 : 0); }
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

// Device kicks of an elite restart (xw_restart.cu): one restarted replica
// (its record, its position among the restarted, its kick steps, and the
// escape move it starts with, -1 for none) ...
struct KickJob {
    uint32_t rid;
    uint32_t index;
    int32_t kick;
    int32_t esc;
};
// ... and a launch over `count` of them: the job, the arena, the elite's
// best W (device, column-major), the escape moves as {row1, row2, col1,
// col2, new1, new2}, the restart round, the elite's score and conflicts,
// the reheat, and scratch of count * 1024 u16 (the row kicks' shuffles).
struct KickArgs {
    const XwJob* job;
    uint8_t* arena;
    const uint64_t* rec_off;
    const int8_t* elite;
    const int32_t* escapes;
    const KickJob* kicks;
    uint16_t* scratch;
    uint64_t round;
    int32_t gbest, gconf;
    double t_min, reheat;
};
void launch_kicks(const KickArgs& a, int count, cudaStream_t stream);

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
