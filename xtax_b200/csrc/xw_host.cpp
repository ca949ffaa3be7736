// xw_host.cpp -- host orchestration and the C ABI (include/xw.h).
//
// Replaces the host half of src/xweigh_cuda.cu (validate_params :1160,
// query_device :1382, run_annealer :1419) with a batch engine: any number of
// independent searches ("jobs") share one device arena of replica records
// and one persistent anneal launch per round; rounds are captured into a
// CUDA graph; results come back through a device-side collection kernel so
// the host reads a few bytes per job instead of whole populations.
#include <cuda_runtime.h>

#include <algorithm>
#include <array>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <memory>
#include <mutex>
#include <random>
#include <stdexcept>
#include <string>
#include <thread>
#include <vector>

#include "../../include/xw.h"
#include "xw_cpu.h"
#include "xw_host_internal.h"
#include "xw_kernels.h"

namespace {

thread_local std::string g_last_error;
std::atomic<int> g_stop{0};

int32_t fail(int32_t code, const std::string& msg) {
    g_last_error = msg;
    return code;
}

std::string fmt(const char* f, ...) {
    char buf[1024];
    va_list ap;
    va_start(ap, f);
    vsnprintf(buf, sizeof buf, f, ap);
    va_end(ap);
    return buf;
}

struct CudaError : std::runtime_error {
    using std::runtime_error::runtime_error;
};

void check(cudaError_t e, const char* what) {
    if (e != cudaSuccess)
        throw CudaError(fmt("%s failed: %s (%s)", what, cudaGetErrorName(e), cudaGetErrorString(e)));
}

uint64_t coin_threshold(double p) {
    if (!(p > 0.0)) return 0;
    if (p >= 1.0) return 4294967296ull;
    return (uint64_t)std::ceil(p * 4294967296.0);
}

template <typename F>
void parallel_for(int count, F f, int grain = 16) {
    const int threads = std::max(1, std::min<int>((int)std::thread::hardware_concurrency(), count / grain + 1));
    if (threads <= 1) {
        for (int i = 0; i < count; ++i) f(i);
        return;
    }
    std::vector<std::thread> pool;
    std::atomic<int> next{0};
    std::exception_ptr err;
    std::atomic<bool> failed{false};
    for (int t = 0; t < threads; ++t)
        pool.emplace_back([&]() {
            for (;;) {
                const int i = next.fetch_add(1);
                if (i >= count || failed.load()) return;
                try {
                    f(i);
                } catch (...) {
                    if (!failed.exchange(true)) err = std::current_exception();
                }
            }
        });
    for (auto& th : pool) th.join();
    if (err) std::rethrow_exception(err);
}

}  // namespace

namespace xw {

void set_last_error(const std::string& msg) { g_last_error = msg; }

const std::atomic<int>& stop_flag() { return g_stop; }

bool needs_general_kernel(const xw_params& p) {
    if (p.move_set != 0) return true;
    if (p.objective == 1 || p.objective == 2) return true;
    return p.objective == -1 && (p.squared_objective_fraction > 0.0 || p.parity_objective_fraction > 0.0);
}

std::string strfmt(const char* f, ...) {
    char buf[1024];
    va_list ap;
    va_start(ap, f);
    vsnprintf(buf, sizeof buf, f, ap);
    va_end(ap);
    return buf;
}

void check_cuda(cudaError_t e, const char* what) { check(e, what); }

static_assert(XW_MAX_ORDER_CUDA == XW_MAX_ORDER_LARGE, "public and device order limits agree");
static_assert(XW_MAX_ORDER_SHARED == XW_MAX_N, "public and shared-memory order limits agree");

uint64_t chunk_wait_limit_ns() {
    const char* e = std::getenv("XW_CHUNK_WAIT_NS");
    if (!e || !*e) return 0;
    return std::strtoull(e, nullptr, 10);
}

void raise_smem_limit(const void* fn, int device) {
    int optin = 0;
    check(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, device),
          "cudaDeviceGetAttribute max opt-in shared memory");
    // the opt-in maximum covers static and dynamic shared memory together
    cudaFuncAttributes attr{};
    check(cudaFuncGetAttributes(&attr, fn), "cudaFuncGetAttributes");
    check(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, optin - (int)attr.sharedSizeBytes),
          "cudaFuncSetAttribute max dynamic shared memory");
}

const cudaDeviceProp& device_properties(int device) {
    static std::mutex mu;
    static cudaDeviceProp props[64];
    static bool have[64] = {};
    if (device < 0 || device >= 64) throw std::invalid_argument("device ordinal out of range");
    std::lock_guard<std::mutex> lock(mu);
    if (!have[device]) {
        check(cudaGetDeviceProperties(&props[device], device), "cudaGetDeviceProperties");
        have[device] = true;
    }
    return props[device];
}

int large_min_order() {
    const char* e = std::getenv("XW_LARGE_MIN_ORDER");
    if (!e || !*e) return XW_MAX_N + 1;
    return std::clamp(std::atoi(e), 1, XW_MAX_N + 1);
}

// The large-order kernel's form for orders whose bit planes fit a warp's
// slot (n <= 448): by default 2, bit planes in shared memory with the Gram
// matrix in HBM (W(276,275) on B200: 104 M moves/s against 69 M for form 0
// and 60 M for form 1); XW_LARGE_PLANES=0 the Gram matrix and masks in HBM
// (the form of larger orders), 1 bit planes with every Gram entry
// recomputed (no Gram matrix: a quarter of the device memory per replica
// at n = 276, and no HBM traffic per move).
static int large_form_wanted() {
    const char* e = std::getenv("XW_LARGE_PLANES");
    if (!e || !*e) return 2;
    const int v = std::atoi(e);
    return v == 1 || v == 2 ? v : 0;
}

std::string validate(int n, int w, const xw_params& p) {
    if (n < 1 || n > 32767) return "CUDA xweigh order is out of range";
    if (w < 1 || w > n) return "CUDA xweigh weight must be in [1, n]";
    if (p.replicas < 0) return "CUDA replica count must be nonnegative";
    if (p.moves_per_launch < 1) return "CUDA moves per launch must be positive";
    if (p.max_seconds < 0.0) return "CUDA max seconds must be nonnegative";
    if (p.save_interval < 0.0) return "CUDA save interval must be nonnegative";
    if (p.sign_fraction < 0.0 || p.sign_fraction > 1.0) return "CUDA sign fraction must be in [0, 1]";
    if (p.double_sign_fraction < 0.0 || p.double_sign_fraction > 1.0)
        return "CUDA double-sign fraction must be in [0, 1]";
    if (p.switch_sign_fraction < 0.0 || p.switch_sign_fraction > 1.0)
        return "CUDA switch-sign fraction must be in [0, 1]";
    if (p.squared_objective_fraction < 0.0 || p.squared_objective_fraction > 1.0)
        return "CUDA squared-objective fraction must be in [0, 1]";
    if (p.parity_objective_fraction < 0.0 || p.parity_objective_fraction > 1.0)
        return "CUDA parity-objective fraction must be in [0, 1]";
    if (p.squared_objective_fraction + p.parity_objective_fraction > 1.0)
        return "CUDA alternate objective fractions must sum to at most 1";
    if (p.greedy_fraction < 0.0 || p.greedy_fraction > 1.0) return "CUDA greedy fraction must be in [0, 1]";
    if (p.target_fraction < 0.0 || p.target_fraction > 1.0) return "CUDA target fraction must be in [0, 1]";
    if (p.candidate_samples < 1 || p.candidate_samples > XW_MAX_CANDIDATE_SAMPLES)
        return "CUDA candidate samples must be in [1, MAX_CANDIDATE_SAMPLES]";
    if (p.target_samples < 1 || p.target_samples > XW_MAX_TARGET_SAMPLES)
        return "CUDA target samples must be in [1, MAX_TARGET_SAMPLES]";
    if (p.t_init < 0.0) return "CUDA initial temperature must be nonnegative";
    if (p.t_min <= 0.0) return "CUDA minimum temperature must be positive";
    if (p.cooling <= 0.0 || p.cooling >= 1.0) return "CUDA cooling factor must be in (0, 1)";
    if (p.moves_per_cool < 1) return "CUDA moves per cool must be positive";
    if (p.stuck_threshold < 1) return "CUDA stuck threshold must be positive";
    if (p.reheat <= 0.0) return "CUDA reheat factor must be positive";
    if (p.restart_interval < 0.0) return "CUDA restart interval must be nonnegative";
    if (p.restart_fraction <= 0.0 || p.restart_fraction > 1.0) return "CUDA restart fraction must be in (0, 1]";
    if (p.restart_kick_min < 0) return "CUDA minimum restart kick must be nonnegative";
    if (p.restart_kick_max < p.restart_kick_min) return "CUDA maximum restart kick must be at least the minimum";
    if (p.exchange_interval < 1) return "CUDA exchange interval must be positive";
    if (p.objective < -1 || p.objective > 2) return "CUDA objective must be -1, 0, 1 or 2";
    if (p.move_set < 0 || p.move_set > 1) return "CUDA move set must be 0 or 1";
    if (p.start_kind < 0 || p.start_kind > 1) return "CUDA start kind must be 0 or 1";
    if (p.warps_per_block < 0 || p.warps_per_block > 16) return "CUDA warps per block must be in [0, 16]";
    if (p.replicas_per_warp < 0 || p.replicas_per_warp > 2) return "CUDA replicas per warp must be 0, 1 or 2";
    if (p.warps_per_replica < 0 || p.warps_per_replica > 64 ||
        (p.warps_per_replica > 16 && p.warps_per_replica % (p.warps_per_replica > 32 ? 4 : 2) != 0))
        return "CUDA warps per replica must be in [0, 16], even up to 32, or a multiple of 4 up to 64";
    if (p.restart_kicks < 0 || p.restart_kicks > 1) return "CUDA restart kicks must be 0 (host) or 1 (device)";
    if (p.stop_on_solve < 0 || p.stop_on_solve > 2) return "CUDA stop-on-solve mode must be 0, 1 or 2";
    return {};
}

// ------------------------------------------------------------------------
// Batch: device arena of replica records for a set of jobs.

// Device memory of batches comes from one pool per device, in stream order,
// and goes back to that pool when a batch is destroyed: handing it back to
// the driver (cudaFree) stalled the next call for up to 0.8 s on B200.  The
// pool keeps what it has been given (release threshold: never), so memory a
// batch frees is the next batch's without a driver call.
cudaMemPool_t batch_pool(int device) {
    static std::mutex mu;
    static cudaMemPool_t pools[64] = {};
    if (device < 0 || device >= 64) throw std::invalid_argument("device ordinal out of range");
    std::lock_guard<std::mutex> lock(mu);
    if (!pools[device]) {
        cudaMemPoolProps props;
        std::memset(&props, 0, sizeof props);
        props.allocType = cudaMemAllocationTypePinned;
        props.location.type = cudaMemLocationTypeDevice;
        props.location.id = device;
        check(cudaMemPoolCreate(&pools[device], &props), "cudaMemPoolCreate");
        uint64_t keep = UINT64_MAX;
        check(cudaMemPoolSetAttribute(pools[device], cudaMemPoolAttrReleaseThreshold, &keep),
              "cudaMemPoolSetAttribute");
    }
    return pools[device];
}

void Batch::dalloc(void** ptr, size_t bytes, const char* what) {
    check(cudaMallocFromPoolAsync(ptr, std::max<size_t>(bytes, 16), batch_pool(params.device), stream), what);
}

Batch::~Batch() {
    if (graph_exec) cudaGraphExecDestroy(graph_exec);
    for (auto e : events) cudaEventDestroy(e);
    for (auto e : side_events) cudaEventDestroy(e);
    if (stream) cudaStreamSynchronize(stream);
    for (void* ptr : {d_jobs, d_jobs0, d_arena, d_arena0, d_rec_off, d_items, d_counters, d_ladder,
                      d_out, d_best_off, d_best, d_t0, d_gram, d_gram_off, d_chunk_done})
        if (ptr) cudaFreeAsync(ptr, stream);
    if (stream) cudaStreamSynchronize(stream);
    for (auto st : side_streams) cudaStreamDestroy(st);
    if (own_stream && stream) cudaStreamDestroy(stream);
}

// header, W, best W, minority lists (u16 on the HBM-resident kernel)
static size_t record_bytes(int n, int m, bool large) {
    const uint32_t nn = xw_pad16((uint32_t)(n * n));
    const size_t b = 128 + 2 * (size_t)nn + xw_pad16((uint32_t)(n * m) * (large ? 2u : 1u));
    return (b + 127) & ~size_t(127);
}

void prepare_job(const xw_job_spec& s, const xw_params& p, const int8_t* starts, uint32_t job_index, bool parallel,
                 XwJob& J, std::vector<uint8_t>& records, std::vector<double>& temps, double& t_init) {
    if (s.n < 1 || s.n > XW_MAX_ORDER_CUDA)
        throw std::invalid_argument(fmt("job %u: order %d is outside [1, %d] of the device path", job_index, s.n,
                                        XW_MAX_ORDER_CUDA));
    if (s.w < 1 || s.w > s.n) throw std::invalid_argument(fmt("job %u: weight must be in [1, n]", job_index));
    if (s.replicas < 1) throw std::invalid_argument(fmt("job %u: replica count must be positive", job_index));
    const bool tempering = p.tempering != 0;
    if (tempering && s.replicas > XW_MAX_RUNGS)
        throw std::invalid_argument(fmt("job %u: a tempering ladder has at most %d rungs", job_index, XW_MAX_RUNGS));
    std::memset(&J, 0, sizeof J);
    J.n = s.n;
    J.w = s.w;
    J.m = std::min(s.w, s.n - s.w);
    J.sparse = s.w <= s.n - s.w;
    J.tempering = tempering;
    J.move_set = p.move_set;
    J.candidate_samples = p.candidate_samples;
    J.target_samples = p.target_samples;
    J.moves_per_cool = p.moves_per_cool;
    J.stuck_threshold = p.stuck_threshold;
    J.objective = p.objective;
    J.general = needs_general_kernel(p) ? 1 : 0;
    J.large = s.n >= large_min_order() ? 1 : 0;
    J.replicas = s.replicas;
    // the Philox key follows the reference's curand seed derivation
    // (xweigh_cuda.cu:1724-1727)
    const uint32_t base = (uint32_t)s.seed;
    const uint64_t key = ((uint64_t)base << 32) ^ s.seed ^ 0xd1b54a32d192ed03ull;
    J.key0 = (uint32_t)key;
    J.key1 = (uint32_t)(key >> 32);
    const uint32_t nn = xw_pad16((uint32_t)(s.n * s.n));
    J.off_w = 128;
    J.off_best = 128 + nn;
    J.off_mino = 128 + 2 * nn;
    J.record_bytes = (uint32_t)record_bytes(s.n, J.m, J.large != 0);
    J.thr_greedy = coin_threshold(p.greedy_fraction);
    J.thr_target = coin_threshold(p.target_fraction);
    J.thr_double = p.move_set == 0 ? coin_threshold(p.double_sign_fraction) : 0;
    J.thr_sign = coin_threshold(p.sign_fraction);
    J.thr_swsign = coin_threshold(p.switch_sign_fraction);
    J.t_min = p.t_min;
    J.cooling = p.cooling;
    J.reheat = p.reheat;
    const uint64_t budget = s.max_moves ? s.max_moves : p.max_moves;
    J.budget_iters = budget ? (budget + (uint64_t)s.replicas - 1) / (uint64_t)s.replicas : 0;

    const int R = J.replicas, n = J.n, w = J.w;
    std::vector<std::vector<int8_t>> W(R);
    auto start_of = [&](int r) -> std::vector<int8_t> {
        if (starts) return std::vector<int8_t>(starts + (size_t)r * n * n, starts + (size_t)(r + 1) * n * n);
        if (p.start_kind == 1) return row_start(n, w, J.key0, J.key1, (uint32_t)r);
        return CpuState::random_start(n, w, base + (uint32_t)r * 0x9e3779b9u).entries();
    };
    // start states and their scores (so that results read before the first
    // launch are meaningful; the kernel rebuilds and checks them)
    std::vector<std::array<int64_t, 4>> start_stats(R);
    auto make_start = [&](int r) {
        W[r] = start_of(r);
        if (W[r].size() != (size_t)n * n) throw std::invalid_argument("start state size mismatch");
        xw_score(n, w, W[r].data(), start_stats[r].data());
    };
    if (parallel) {
        parallel_for(R, make_start);
    } else {
        for (int r = 0; r < R; ++r) make_start(r);
    }
    // calibrate_temperature on replica 0 (xweigh_cuda.cu:1563-1567)
    t_init = p.t_init;
    if (t_init <= 0.0) {
        CpuParams cp;
        cp.sign_fraction = p.sign_fraction;
        cp.target_fraction = p.target_fraction;
        cp.target_samples = p.target_samples;
        // the reference calibrates on replica 0's State as random_start
        // left it (minority lists in switch order) or as read from CSV
        const CpuState s0 = (!starts && p.start_kind == 0) ? CpuState::random_start(n, w, base)
                                                           : CpuState::from_entries(n, w, W[0]);
        t_init = calibrate_temperature(s0, cp, base);
    }
    // geometric ladder from min(t_min, t_init) to t_init (xweigh_cuda.cu:1580-1594)
    const double bottom = std::min(p.t_min, t_init);
    const double ratio = R > 1 ? std::pow(t_init / std::max(bottom, 1.0e-12), 1.0 / (double)(R - 1)) : 1.0;
    temps.assign(R, 0.0);
    double t = bottom;
    for (int r = 0; r < R; ++r) {
        temps[r] = t;
        t *= ratio;
    }
    records.assign((size_t)R * J.record_bytes, 0);
    for (int r = 0; r < R; ++r) {
        uint8_t* rec = records.data() + (size_t)r * J.record_bytes;
        RepHeader* H = reinterpret_cast<RepHeader*>(rec);
        H->job = job_index;
        H->stream = (uint32_t)r;
        H->temperature = temps[r];
        H->reheat_temperature = temps[r];
        H->rung = r;
        H->score = H->best_score = (int32_t)start_stats[r][0];
        H->conflicts = H->best_conflicts = (int32_t)start_stats[r][1];
        if (p.objective >= 0) {
            H->obj_kind = p.objective;
        } else {
            const uint32_t h = (uint32_t)r * 0x9e3779b9u + 0x85ebca6bu;
            const double choice = (double)h * (1.0 / 4294967296.0);
            H->obj_kind = choice < p.squared_objective_fraction ? 1
                : choice < p.squared_objective_fraction + p.parity_objective_fraction ? 2 : 0;
        }
        std::memcpy(rec + J.off_w, W[r].data(), (size_t)n * n);
        std::memcpy(rec + J.off_best, W[r].data(), (size_t)n * n);
    }
}

void Batch::build(const xw_job_spec* specs, int njobs, const xw_params& p, const int8_t* starts) {
    params = p;
    check(cudaSetDevice(p.device), "cudaSetDevice");
    props = device_properties(p.device);
    if (njobs < 1) throw std::invalid_argument("batch needs at least one job");
    jobs.resize(njobs);
    rep_seed.resize(njobs);
    best_offsets.resize(njobs);
    t_init_used.assign(njobs, 0.0);
    tempering = p.tempering != 0;
    std::vector<uint8_t> host;
    ladder.clear();
    rec_off.clear();
    uint32_t rep = 0;
    // jobs are built in parallel across jobs when there are enough of them,
    // else each job builds its replicas' starts in parallel
    std::vector<size_t> start_at((size_t)njobs, 0);
    for (int j = 1; j < njobs; ++j)
        start_at[j] = start_at[j - 1] + (size_t)specs[j - 1].replicas * specs[j - 1].n * specs[j - 1].n;
    std::vector<std::vector<uint8_t>> records((size_t)njobs);
    std::vector<std::vector<double>> temps((size_t)njobs);
    const bool across = njobs >= (int)std::max(2u, std::thread::hardware_concurrency());
    auto build_job = [&](int j) {
        prepare_job(specs[j], p, starts ? starts + start_at[j] : nullptr, (uint32_t)j, !across, jobs[j], records[j],
                    temps[j], t_init_used[j]);
    };
    if (across) {
        parallel_for(njobs, build_job, 1);
    } else {
        for (int j = 0; j < njobs; ++j) build_job(j);
    }
    for (int j = 0; j < njobs; ++j) {
        const xw_job_spec& s = specs[j];
        XwJob& J = jobs[j];
        J.rep_begin = rep;
        J.ladder_off = ladder.size();
        if (tempering) ladder.insert(ladder.end(), temps[j].begin(), temps[j].end());
        rep_seed[j] = (uint32_t)s.seed;
        for (int r = 0; r < s.replicas; ++r) rec_off.push_back(host.size() + (size_t)r * J.record_bytes);
        host.insert(host.end(), records[j].begin(), records[j].end());
        rep += (uint32_t)s.replicas;
    }
    if (ladder.empty()) ladder.push_back(0.0);
    derive_layout();
    upload(host);
}

// Work list, result offsets, launch classes and shared-memory slots from
// the job table.
void Batch::derive_layout() {
    const int njobs = (int)jobs.size();
    total_replicas = 0;
    best_offsets.assign(njobs, 0);
    size_t best_off = 0;
    n_large = 0;
    general_large = false;
    large_slot_bytes = 0;
    // the large-order launch runs in bit-plane mode when every large job's
    // W fits a warp's shared memory as bit planes
    large_form = large_form_wanted();
    for (const XwJob& J : jobs)
        if (J.large && !anneal_large_planes_fit(J.n, J.m)) large_form = 0;
    for (int j = 0; j < njobs; ++j) {
        const XwJob& J = jobs[j];
        total_replicas += (uint32_t)J.replicas;
        best_offsets[j] = best_off;
        best_off += (size_t)J.n * J.n;
        if (J.large) {
            n_large += (uint32_t)J.replicas;
            general_large = general_large || J.general != 0;
            large_slot_bytes = std::max(large_slot_bytes, anneal_large_slot_bytes(J.n, J.m, large_form));
        }
    }
    best_bytes = best_off;
    // work items: the HBM-resident replicas, then the others; longest
    // replicas first within each (cost grows with n), so that each launch
    // class is one range of items
    items.resize(total_replicas);
    std::vector<int> job_of(total_replicas);
    for (int j = 0; j < njobs; ++j)
        for (int r = 0; r < jobs[j].replicas; ++r) job_of[jobs[j].rep_begin + r] = j;
    for (uint32_t i = 0; i < total_replicas; ++i) items[i] = i;
    std::stable_sort(items.begin(), items.end(), [&](uint32_t a, uint32_t b) {
        const XwJob &A = jobs[job_of[a]], &B = jobs[job_of[b]];
        if (A.large != B.large) return A.large > B.large;
        return A.n > B.n;
    });
    // launch classes over the shared-memory items.  The orders up to 16 get
    // a launch of their own (two replicas per warp) only when it pays: at
    // one replica per warp they run the one-row-per-lane kernel and join
    // that class's launch, and so they do when the batch holds other orders
    // of that class and too few of them to fill the device alone -- a small
    // second launch would run its replicas beside the first at low
    // occupancy instead of sharing its chunked work list.
    uint32_t pair_count = 0, one_row_count = 0;
    for (uint32_t i = n_large; i < total_replicas; ++i) {
        const XwJob& J = jobs[job_of[items[i]]];
        const int kind = tune_kind(J.n, J.candidate_samples);
        pair_count += kind == kTunePairKind;
        one_row_count += kind == 1;
    }
    const uint32_t fill = 2u * 20u * (uint32_t)std::max(1, props.multiProcessorCount);
    const bool merge_pairs = one_row_count > 0 && pair_count < fill;
    classes.clear();
    for (uint32_t i = n_large; i < total_replicas; ++i) {
        const XwJob& J = jobs[job_of[items[i]]];
        int kind = tune_kind(J.n, J.candidate_samples);
        if (kind == kTunePairKind && !split_pair_class) {
            int rpw = params.replicas_per_warp;
            if (rpw == 0) rpw = tuned_shape(kTunePairKind, anneal_slot_bytes(J.n, J.m, 1), params.device).rpw;
            if (rpw == 1 || (merge_pairs && params.replicas_per_warp != 2)) kind = anneal_opl(J.n);
        }
        if (classes.empty() || classes.back().kind != kind) {
            LaunchClass c;
            c.kind = kind;
            c.opl = anneal_opl(J.n);
            c.min_n = c.max_n = J.n;
            c.item_begin = i;
            classes.push_back(c);
        }
        LaunchClass& c = classes.back();
        c.item_count += 1;
        c.min_n = std::min(c.min_n, J.n);
        c.max_n = std::max(c.max_n, J.n);
        c.general = c.general || J.general != 0;
        c.one_zero = c.one_zero && J.m == 1 && !J.sparse;
        c.slot_bytes = std::max(c.slot_bytes, anneal_slot_bytes(J.n, J.m, c.opl));
    }
    // arena offsets of the large-order replicas (Gram matrices, or planes
    // and residuals in bit-plane mode)
    gram_off.assign(total_replicas, 0);
    gram_bytes = 0;
    for (uint32_t i = 0; i < total_replicas; ++i) {
        const XwJob& J = jobs[job_of[i]];
        if (!J.large) continue;
        gram_off[i] = gram_bytes;
        gram_bytes += anneal_large_arena_bytes(J.n, large_form);
    }
}

// Device buffers for the batch; the records in `host` become the state that
// reset() restores.
void Batch::upload(const std::vector<uint8_t>& host) {
    const int njobs = (int)jobs.size();
    const size_t arena = host.size();
    arena_bytes = arena;
    auto dmalloc = [&](void** ptr, size_t bytes, const char* what) { dalloc(ptr, bytes, what); };
    size_t free_b = 0, total_b = 0;
    check(cudaMemGetInfo(&free_b, &total_b), "cudaMemGetInfo");
    {
        // memory the batch pool holds but no batch uses is free to this batch
        uint64_t reserved = 0, used = 0;
        cudaMemPool_t pool = batch_pool(params.device);
        check(cudaMemPoolGetAttribute(pool, cudaMemPoolAttrReservedMemCurrent, &reserved), "cudaMemPoolGetAttribute");
        check(cudaMemPoolGetAttribute(pool, cudaMemPoolAttrUsedMemCurrent, &used), "cudaMemPoolGetAttribute");
        if (reserved > used) free_b += (size_t)(reserved - used);
    }
    const size_t need = 2 * arena + 2 * sizeof(XwJob) * njobs + 16 * total_replicas + best_bytes + gram_bytes;
    if (need > free_b)
        throw std::length_error(fmt("CUDA replica state requires %g MiB, but only %g MiB is free",
                                    need / 1048576.0, free_b / 1048576.0));
    if (!stream) {
        check(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking), "cudaStreamCreate");
        own_stream = true;
    }
    dmalloc(&d_jobs, sizeof(XwJob) * njobs, "cudaMalloc jobs");
    dmalloc(&d_jobs0, sizeof(XwJob) * njobs, "cudaMalloc jobs");
    dmalloc(&d_arena, arena, "cudaMalloc replica records");
    dmalloc(&d_arena0, arena, "cudaMalloc replica records");
    dmalloc(&d_rec_off, sizeof(uint64_t) * total_replicas, "cudaMalloc record offsets");
    dmalloc(&d_items, sizeof(uint32_t) * total_replicas, "cudaMalloc items");
    dmalloc(&d_ladder, sizeof(double) * ladder.size(), "cudaMalloc ladder");
    dmalloc(&d_out, sizeof(JobOut) * njobs, "cudaMalloc results");
    dmalloc(&d_best_off, sizeof(uint64_t) * njobs, "cudaMalloc result offsets");
    dmalloc(&d_best, best_bytes, "cudaMalloc best states");
    dmalloc(&d_t0, sizeof(uint64_t), "cudaMalloc clock");
    if (n_large) {
        dmalloc(&d_gram, gram_bytes, "cudaMalloc Gram arena");
        dmalloc(&d_gram_off, sizeof(uint64_t) * total_replicas, "cudaMalloc Gram offsets");
        check(cudaMemcpyAsync(d_gram_off, gram_off.data(), sizeof(uint64_t) * total_replicas, cudaMemcpyHostToDevice,
                              stream),
              "upload Gram offsets");
    }
    check(cudaMemcpyAsync(d_jobs0, jobs.data(), sizeof(XwJob) * njobs, cudaMemcpyHostToDevice, stream), "upload jobs");
    check(cudaMemcpyAsync(d_arena0, host.data(), arena, cudaMemcpyHostToDevice, stream), "upload records");
    check(cudaMemcpyAsync(d_rec_off, rec_off.data(), sizeof(uint64_t) * total_replicas, cudaMemcpyHostToDevice, stream),
          "upload offsets");
    check(cudaMemcpyAsync(d_items, items.data(), sizeof(uint32_t) * total_replicas, cudaMemcpyHostToDevice, stream),
          "upload items");
    check(cudaMemcpyAsync(d_ladder, ladder.data(), sizeof(double) * ladder.size(), cudaMemcpyHostToDevice, stream),
          "upload ladder");
    check(cudaMemcpyAsync(d_best_off, best_offsets.data(), sizeof(uint64_t) * njobs, cudaMemcpyHostToDevice, stream),
          "upload result offsets");
    reset();
    check(cudaStreamSynchronize(stream), "cudaStreamSynchronize upload");
    // streams and fork/join events for side-by-side launches of a round
    const int launches = launches_per_round();
    while ((int)side_streams.size() < launches - 1) {
        cudaStream_t st;
        check(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking), "cudaStreamCreate");
        side_streams.push_back(st);
    }
    while ((int)side_events.size() < (launches > 1 ? launches + 1 : 0)) {
        cudaEvent_t e;
        check(cudaEventCreateWithFlags(&e, cudaEventDisableTiming), "cudaEventCreate");
        side_events.push_back(e);
    }
    configure_shape();
}

// Population snapshots (the format is described with Snapshot): a batch
// saves its job table and records as they are on the device now.
static const char kSnapMagic[8] = {'X', 'W', 'P', 'O', 'P', '0', '0', '1'};

void write_snapshot(const std::string& path, const Snapshot& sn) {
    const std::string tmp = path + ".tmp";
    FILE* f = std::fopen(tmp.c_str(), "wb");
    if (!f) throw std::runtime_error("cannot write snapshot " + tmp);
    bool ok = true;
    auto put = [&](const void* p, size_t n) { ok = ok && std::fwrite(p, 1, n, f) == n; };
    const uint32_t sizes[4] = {(uint32_t)sizeof(XwJob), (uint32_t)sizeof(RepHeader), (uint32_t)sizeof(xw_params),
                               (uint32_t)sn.jobs.size()};
    const uint64_t counts[3] = {sn.rec_off.size(), sn.arena.size(), sn.ladder.size()};
    put(kSnapMagic, 8);
    put(sizes, sizeof sizes);
    put(counts, sizeof counts);
    put(&sn.params, sizeof sn.params);
    put(sn.jobs.data(), sizeof(XwJob) * sn.jobs.size());
    put(sn.rec_off.data(), sizeof(uint64_t) * sn.rec_off.size());
    put(sn.ladder.data(), sizeof(double) * sn.ladder.size());
    put(sn.t_init.data(), sizeof(double) * sn.t_init.size());
    put(sn.arena.data(), sn.arena.size());
    ok = (std::fclose(f) == 0) && ok;
    if (!ok || std::rename(tmp.c_str(), path.c_str()) != 0) {
        std::remove(tmp.c_str());
        throw std::runtime_error("cannot write snapshot " + path);
    }
}

Snapshot read_snapshot(const std::string& path) {
    FILE* f = std::fopen(path.c_str(), "rb");
    if (!f) throw std::invalid_argument("cannot open snapshot " + path);
    bool ok = true;
    auto get = [&](void* p, size_t n) { ok = ok && std::fread(p, 1, n, f) == n; };
    char magic[8];
    uint32_t sizes[4];
    uint64_t counts[3];
    get(magic, 8);
    get(sizes, sizeof sizes);
    get(counts, sizeof counts);
    if (!ok || std::memcmp(magic, kSnapMagic, 8) != 0 || sizes[0] != sizeof(XwJob) ||
        sizes[1] != sizeof(RepHeader) || sizes[2] != sizeof(xw_params) || sizes[3] == 0 ||
        counts[0] > (1ull << 32) || counts[2] > (1ull << 32)) {
        std::fclose(f);
        throw std::invalid_argument("not a population snapshot of this build: " + path);
    }
    Snapshot sn;
    get(&sn.params, sizeof sn.params);
    sn.jobs.resize(sizes[3]);
    get(sn.jobs.data(), sizeof(XwJob) * sn.jobs.size());
    sn.rec_off.resize(counts[0]);
    get(sn.rec_off.data(), sizeof(uint64_t) * sn.rec_off.size());
    sn.ladder.resize(counts[2]);
    get(sn.ladder.data(), sizeof(double) * sn.ladder.size());
    sn.t_init.resize(sn.jobs.size());
    get(sn.t_init.data(), sizeof(double) * sn.t_init.size());
    sn.arena.resize(counts[1]);
    get(sn.arena.data(), sn.arena.size());
    std::fclose(f);
    if (!ok) throw std::invalid_argument("truncated population snapshot: " + path);
    // the saved records must lie inside the arena and name their own job
    uint64_t total = 0;
    for (size_t j = 0; j < sn.jobs.size(); ++j) {
        const XwJob& J = sn.jobs[j];
        if (J.n < 1 || J.n > XW_MAX_ORDER_CUDA || J.replicas < 1 ||
            (uint64_t)J.rep_begin + J.replicas > counts[0])
            throw std::invalid_argument("corrupt population snapshot: " + path);
        for (int r = 0; r < J.replicas; ++r) {
            const uint64_t off = sn.rec_off[J.rep_begin + r];
            if (off + J.record_bytes > sn.arena.size() ||
                reinterpret_cast<const RepHeader*>(sn.arena.data() + off)->job != (uint32_t)j)
                throw std::invalid_argument("corrupt population snapshot: " + path);
        }
        total += (uint64_t)J.replicas;
    }
    if (total != counts[0]) throw std::invalid_argument("corrupt population snapshot: " + path);
    // a snapshot holds no Gram arena: the large-order kernel rebuilds it
    for (size_t j = 0; j < sn.jobs.size(); ++j)
        for (int r = 0; r < sn.jobs[j].replicas; ++r)
            reinterpret_cast<RepHeader*>(sn.arena.data() + sn.rec_off[sn.jobs[j].rep_begin + r])->status &=
                ~XW_STATUS_GRAM;
    return sn;
}

void Batch::save(const std::string& path) {
    Snapshot sn;
    sn.params = params;
    sn.jobs.resize(jobs.size());
    sn.arena.resize(arena_bytes);
    check(cudaMemcpyAsync(sn.jobs.data(), d_jobs, sizeof(XwJob) * sn.jobs.size(), cudaMemcpyDeviceToHost, stream),
          "read job table");
    check(cudaMemcpyAsync(sn.arena.data(), d_arena, arena_bytes, cudaMemcpyDeviceToHost, stream), "read records");
    check(cudaStreamSynchronize(stream), "cudaStreamSynchronize snapshot");
    sn.rec_off = rec_off;
    sn.ladder = ladder;
    sn.t_init = t_init_used;
    write_snapshot(path, sn);
}

void Batch::load(const std::string& path, const xw_params* over) {
    Snapshot sn = read_snapshot(path);
    params = sn.params;
    jobs = std::move(sn.jobs);
    rec_off = std::move(sn.rec_off);
    ladder = std::move(sn.ladder);
    t_init_used = std::move(sn.t_init);
    std::vector<uint8_t> host = std::move(sn.arena);
    if (over) {
        // run-time settings may change on resume; the search itself may not
        params.device = over->device;
        params.moves_per_launch = over->moves_per_launch;
        params.stop_on_solve = over->stop_on_solve;
        params.warps_per_block = over->warps_per_block;
        params.replicas_per_warp = over->replicas_per_warp;
        params.warps_per_replica = over->warps_per_replica;
        params.max_seconds = over->max_seconds;
    }
    tempering = params.tempering != 0;
    rep_seed.assign(jobs.size(), 0);
    check(cudaSetDevice(params.device), "cudaSetDevice");
    props = device_properties(params.device);
    derive_layout();
    upload(host);
}

uint32_t choose_chunks(uint32_t replicas, uint32_t slots) {
    if (const char* e = std::getenv("XW_CHUNKS"); e && *e) return (uint32_t)std::clamp(std::atoi(e), 1, 64);
    if (slots == 0 || replicas <= slots) return 1;
    uint32_t best = 1;
    double best_waves = 0.0;
    for (uint32_t k = 1; k <= 8; ++k) {
        const double waves = (double)((uint64_t)replicas * k / slots + ((uint64_t)replicas * k % slots != 0)) / k;
        if (k == 1 || waves < best_waves - 1e-9) {
            best = k;
            best_waves = waves;
        }
    }
    return best;
}

void Batch::configure_shape() {
    if (graph_exec) {
        cudaGraphExecDestroy(graph_exec);
        graph_exec = nullptr;
    }
    if (n_large) {
        // four warps per CTA, as many CTAs as the SMs hold
        const void* lfn = anneal_large_kernel_fn(general_large, large_form);
        const size_t lsmem = (size_t)large_wpb * large_slot_bytes;
        raise_smem_limit(lfn, params.device);
        int per_sm = 0;
        check(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, lfn, 32 * large_wpb, lsmem),
              "cudaOccupancyMaxActiveBlocksPerMultiprocessor");
        if (per_sm < 1) throw std::length_error("CUDA large-order anneal kernel has zero occupancy");
        const int want = (int)((n_large + large_wpb - 1) / large_wpb);
        large_blocks = std::max(1, std::min(want, per_sm * props.multiProcessorCount));
        large_chunks = choose_chunks(n_large, (uint32_t)(large_blocks * large_wpb));
    }
    int optin = 0;
    check(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, params.device),
          "cudaDeviceGetAttribute max opt-in shared memory");
    for (size_t k = 0; k < classes.size(); ++k) {
        const LaunchClass& c = classes[k];
        if (c.slot_bytes > (uint32_t)optin)
            throw std::length_error(fmt("CUDA replica requires %.2f KiB of shared memory, but device %d permits "
                                        "%.2f KiB per opt-in block",
                                        c.slot_bytes / 1024.0, params.device, optin / 1024.0));
        // the latency mode: orders up to 32, and (unless set) classes of at
        // most one replica per SM, where a replica's speed is its latency
        if (c.max_n <= 32) {
            int wpr = params.warps_per_replica;
            if (wpr == 0 && c.item_count <= (uint32_t)props.multiProcessorCount) {
                wpr = tuned_warps_per_replica(c.slot_bytes, params.device);
                // a cluster of two or four SMs per replica only while every
                // replica has its SMs
                if (wpr > 32 && 4 * c.item_count > (uint32_t)props.multiProcessorCount) wpr = 32;
                if (wpr > 16 && 2 * c.item_count > (uint32_t)props.multiProcessorCount) wpr = 16;
            }
            if (wpr > 1 && configure_latency(k, wpr)) continue;
        }
        TunedShape t = tuned_shape(c.kind, c.slot_bytes, params.device);
        if (params.warps_per_block > 0) t.wpb = params.warps_per_block;
        if (params.replicas_per_warp > 0) t.rpw = params.replicas_per_warp;
        if (c.kind != kTunePairKind) t.rpw = 1;
        // the widest shape that fits the opt-in shared memory
        t.wpb = std::max(1, std::min(t.wpb, std::min(16, (int)(optin / (c.slot_bytes * (uint32_t)t.rpw)))));
        if (!configure_class(k, t.wpb, t.rpw) && !configure_class(k, 1, 1))
            throw std::length_error("CUDA anneal kernel has zero occupancy on the selected device");
    }
    uint32_t most_chunks = n_large ? large_chunks : 1;
    for (const LaunchClass& c : classes) most_chunks = std::max(most_chunks, c.chunks);
    if (most_chunks > 1 && !d_chunk_done)
        dalloc(&d_chunk_done, sizeof(uint32_t) * std::max<uint32_t>(total_replicas, 1), "cudaMalloc chunk counters");
    // launches of a round go out smallest estimated work first (replicas x
    // order, the large-order kernel's iterations counted four times): each
    // is a persistent kernel sized for the whole device, so the one issued
    // last takes the SMs the others leave and absorbs their tails
    std::vector<std::pair<double, int>> work;
    if (n_large) {
        int nmax = 0;
        for (const XwJob& J : jobs)
            if (J.large) nmax = std::max(nmax, J.n);
        work.push_back({4.0 * n_large * nmax, -1});
    }
    for (size_t k = 0; k < classes.size(); ++k) work.push_back({(double)classes[k].item_count * classes[k].max_n, (int)k});
    std::stable_sort(work.begin(), work.end(), [](const auto& x, const auto& y) { return x.first < y.first; });
    launch_order.clear();
    for (const auto& wv : work) launch_order.push_back(wv.second);
}

bool Batch::configure_latency(size_t k, int wpr) {
    if (graph_exec) {
        cudaGraphExecDestroy(graph_exec);
        graph_exec = nullptr;
    }
    LaunchClass& c = classes.at(k);
    if (c.max_n > 32 || wpr < 2 || wpr > 64) return false;
    // the warps spread over as many CTAs (a cluster of up to four, one per
    // SM) as the class's replicas leave SMs for, at 8 to 16 warps per CTA
    // (C1, W(12,11) per search: 32 warps as four CTAs of 8 5.50 M moves/s,
    // as two of 16 5.14 M; 8 warps as four CTAs of 2 1.61 M, as one CTA
    // 1.81 M).  Failing that, the fewest CTAs of 2 to 16 warps that hold
    // them (their clusters then run in turns).
    int cl = 0;
    for (int q : {4, 2, 1}) {
        if (wpr % q != 0 || wpr / q > 16 || (q > 1 && wpr / q < 8)) continue;
        if (q > 1 && (uint32_t)q * c.item_count > (uint32_t)props.multiProcessorCount) continue;
        cl = q;
        break;
    }
    for (int q : {1, 2, 4}) {
        if (cl != 0) break;
        if (wpr % q == 0 && wpr / q >= 2 && wpr / q <= 16) cl = q;
    }
    if (cl == 0) return false;
    const void* fn = anneal_spec_kernel_fn(c.general, cl);
    raise_smem_limit(fn, params.device);
    const uint32_t bytes = anneal_spec_cta_bytes(c.slot_bytes, wpr, cl);
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, 32 * (wpr / cl), bytes) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    if (per_sm < 1) return false;
    c.wpr = wpr;
    c.ctas = cl;
    c.spec_bytes = bytes;
    c.rpw = 1;
    c.wpb = wpr / cl;
    c.blocks_per_sm = per_sm;
    c.blocks = cl > 1 ? cl * (int)c.item_count
                      : std::max(1, std::min((int)c.item_count, per_sm * props.multiProcessorCount));
    c.chunks = 1;
    return true;
}

bool Batch::configure_class(size_t k, int wpb, int rpw) {
    if (graph_exec) {
        cudaGraphExecDestroy(graph_exec);
        graph_exec = nullptr;
    }
    LaunchClass& c = classes.at(k);
    if (rpw == 2 && c.kind != kTunePairKind) return false;
    c.wpr = 1;
    c.ctas = 1;
    const void* fn = anneal_kernel_fn(c.opl, c.general, rpw, c.one_zero, c.min_n == c.max_n ? c.min_n : 0);
    raise_smem_limit(fn, params.device);
    const size_t smem = (size_t)wpb * rpw * c.slot_bytes;
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, 32 * wpb, smem) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    if (per_sm < 1) return false;
    c.wpb = wpb;
    c.rpw = rpw;
    c.blocks_per_sm = per_sm;
    const uint32_t groups = (uint32_t)(wpb * rpw);
    const int want = (int)((c.item_count + groups - 1) / groups);
    c.blocks = std::max(1, std::min(want, per_sm * props.multiProcessorCount));
    // More replicas than resident groups: a launch of whole replicas ends in
    // a part-filled wave (4096 replicas on 2368 warps run 2 waves for 1.73
    // waves of work).  Split each replica's iterations into k chunks, k in
    // [1, 8] with the fewest waves per unit of work, the least k on ties.
    c.chunks = choose_chunks(c.item_count, (uint32_t)c.blocks * groups);
    if (c.chunks > 1 && !d_chunk_done)
        dalloc(&d_chunk_done, sizeof(uint32_t) * std::max<uint32_t>(total_replicas, 1), "cudaMalloc chunk counters");
    return true;
}

void Batch::reset() {
    check(cudaMemcpyAsync(d_jobs, d_jobs0, sizeof(XwJob) * jobs.size(), cudaMemcpyDeviceToDevice, stream),
          "reset jobs");
    check(cudaMemcpyAsync(d_arena, d_arena0, arena_bytes, cudaMemcpyDeviceToDevice, stream), "reset records");
    check(cudaMemsetAsync(d_t0, 0, sizeof(uint64_t), stream), "reset clock");
}

uint64_t Batch::round_iters() const {
    return tempering ? (uint64_t)params.exchange_interval : (uint64_t)params.moves_per_launch;
}

// Events and work counters for `rounds` rounds; allocated outside any
// stream capture.
void Batch::reserve_rounds(int rounds) {
    while ((int)events.size() < 2 * rounds) {
        cudaEvent_t e;
        check(cudaEventCreate(&e), "cudaEventCreate");
        events.push_back(e);
    }
    if (counters_cap < rounds || counters_per_round != launches_per_round()) {
        if (d_counters) check(cudaFreeAsync(d_counters, stream), "cudaFreeAsync counters");
        d_counters = nullptr;
        // one counter per round for each launch of the round
        dalloc(&d_counters, sizeof(uint32_t) * (size_t)launches_per_round() * rounds, "cudaMalloc counters");
        check(cudaStreamSynchronize(stream), "cudaStreamSynchronize");
        counters_cap = rounds;
        counters_per_round = launches_per_round();
    }
}

void Batch::enqueue_rounds(uint64_t iters, bool timed) {
    const uint64_t per = round_iters();
    const int rounds = (int)((iters + per - 1) / per);
    const int launches = launches_per_round();
    if ((int)events.size() < 2 * rounds || counters_cap < rounds || counters_per_round != launches)
        throw std::logic_error("round resources not reserved");
    uint32_t most_chunks = n_large ? large_chunks : 1;
    for (const LaunchClass& c : classes) most_chunks = std::max(most_chunks, c.chunks);
    check(launch_mark_t0(static_cast<uint64_t*>(d_t0), stream), "launch mark_t0");
    check(cudaMemsetAsync(d_counters, 0, sizeof(uint32_t) * (size_t)launches * rounds, stream),
          "cudaMemsetAsync counters");
    uint64_t left = iters;
    for (int k = 0; k < rounds; ++k) {
        AnnealArgs a;
        a.jobs = static_cast<XwJob*>(d_jobs);
        a.arena = static_cast<uint8_t*>(d_arena);
        a.rec_off = static_cast<const uint64_t*>(d_rec_off);
        a.iters = std::min(left, per);
        a.stop_on_solve = params.stop_on_solve;
        a.one_zero = 0;
        a.chunk_wait_ns = chunk_wait_limit_ns();
        left -= a.iters;
        uint32_t* counters = static_cast<uint32_t*>(d_counters) + (size_t)launches * k;
        if (timed) check(cudaEventRecord(events[2 * k], stream), "cudaEventRecord");
        // one chunk-counter reset for all of the round's launches (their
        // replicas are disjoint), before they fork
        if (a.iters >= 2 && most_chunks > 1)
            check(cudaMemsetAsync(d_chunk_done, 0, sizeof(uint32_t) * total_replicas, stream),
                  "cudaMemsetAsync chunk counters");
        // launch l runs on the batch's stream when it is alone, else on side
        // stream l, forked from and joined back into the batch's stream
        if (launches > 1) check(cudaEventRecord(side_events[0], stream), "cudaEventRecord");
        int l = 0;
        auto on = [&](int idx) {
            if (launches == 1) return stream;
            cudaStream_t st = idx == 0 ? stream : side_streams[idx - 1];
            if (idx > 0) check(cudaStreamWaitEvent(st, side_events[0], 0), "cudaStreamWaitEvent");
            return st;
        };
        auto join = [&](int idx, cudaStream_t st) {
            if (launches == 1 || idx == 0) return;
            check(cudaEventRecord(side_events[idx], st), "cudaEventRecord");
        };
        for (const int which : launch_order) {
            if (which < 0) {
                AnnealArgs la = a;
                la.items = static_cast<const uint32_t*>(d_items);
                la.n_items = n_large;
                la.slot_bytes = large_slot_bytes;
                la.counter = counters + l;
                la.gram = static_cast<uint8_t*>(d_gram);
                la.gram_off = static_cast<const uint64_t*>(d_gram_off);
                la.chunks = la.iters >= large_chunks ? large_chunks : 1;
                if (la.chunks > 1) la.chunk_done = static_cast<uint32_t*>(d_chunk_done);
                cudaStream_t st = on(l);
                check(launch_anneal_large(la, general_large, large_form, large_wpb, large_blocks, st),
                      "launch anneal_large_kernel");
                join(l, st);
                ++l;
                continue;
            }
            const LaunchClass& c = classes[(size_t)which];
            AnnealArgs ca = a;
            ca.items = static_cast<const uint32_t*>(d_items) + c.item_begin;
            ca.n_items = c.item_count;
            ca.slot_bytes = c.slot_bytes;
            ca.counter = counters + l;
            ca.one_zero = c.one_zero ? 1 : 0;
            ca.fixed_order = c.one_zero && c.min_n == c.max_n ? c.min_n : 0;
            ca.chunks = ca.iters >= c.chunks ? c.chunks : 1;
            if (ca.chunks > 1) ca.chunk_done = static_cast<uint32_t*>(d_chunk_done);
            cudaStream_t st = on(l);
            if (c.wpr > 1) {
                ca.slot_bytes = c.spec_bytes;
                ca.chunks = 1;
                ca.chunk_done = nullptr;
                check(launch_anneal_spec(ca, c.general, c.wpr, c.ctas, c.blocks, st), "launch anneal_spec_kernel");
            } else {
                check(launch_anneal(ca, c.opl, c.general, c.wpb, c.blocks, st, c.rpw), "launch anneal_kernel");
            }
            join(l, st);
            ++l;
        }
        for (int idx = 1; idx < launches; ++idx)
            check(cudaStreamWaitEvent(stream, side_events[idx], 0), "cudaStreamWaitEvent");
        if (timed) check(cudaEventRecord(events[2 * k + 1], stream), "cudaEventRecord");
        if (tempering)
            check(launch_exchange(static_cast<XwJob*>(d_jobs), (int)jobs.size(), static_cast<uint8_t*>(d_arena),
                                  static_cast<const uint64_t*>(d_rec_off), static_cast<const double*>(d_ladder),
                                  params.stop_on_solve, stream),
                  "launch exchange_kernel");
    }
    last_rounds = timed ? rounds : 0;
}

void Batch::run(uint64_t iters, bool use_graph) {
    if (iters == 0) return;
    const uint64_t per = round_iters();
    reserve_rounds((int)((iters + per - 1) / per));
    if (!use_graph) {
        enqueue_rounds(iters, true);
        return;
    }
    if (!graph_exec || graph_iters != iters) {
        if (graph_exec) {
            cudaGraphExecDestroy(graph_exec);
            graph_exec = nullptr;
        }
        cudaGraph_t g;
        check(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal), "cudaStreamBeginCapture");
        try {
            enqueue_rounds(iters, false);
        } catch (...) {
            cudaStreamEndCapture(stream, &g);
            if (g) cudaGraphDestroy(g);
            throw;
        }
        check(cudaStreamEndCapture(stream, &g), "cudaStreamEndCapture");
        const cudaError_t e = cudaGraphInstantiate(&graph_exec, g, 0);
        cudaGraphDestroy(g);
        check(e, "cudaGraphInstantiate");
        graph_iters = iters;
    }
    // events outside the graph: the time of the whole graph launch
    check(cudaEventRecord(events[0], stream), "cudaEventRecord");
    check(cudaGraphLaunch(graph_exec, stream), "cudaGraphLaunch");
    check(cudaEventRecord(events[1], stream), "cudaEventRecord");
    last_rounds = 1;
}

void Batch::collect(std::vector<JobOut>& out, int8_t* best_host, bool want_best) {
    check(launch_collect(static_cast<const XwJob*>(d_jobs), (int)jobs.size(), static_cast<const uint8_t*>(d_arena),
                         static_cast<const uint64_t*>(d_rec_off), static_cast<const uint64_t*>(d_best_off),
                         static_cast<JobOut*>(d_out), want_best ? static_cast<int8_t*>(d_best) : nullptr, stream),
          "launch collect_kernel");
    out.resize(jobs.size());
    check(cudaMemcpyAsync(out.data(), d_out, sizeof(JobOut) * jobs.size(), cudaMemcpyDeviceToHost, stream),
          "cudaMemcpy results to host");
    if (want_best && best_host)
        check(cudaMemcpyAsync(best_host, d_best, best_bytes, cudaMemcpyDeviceToHost, stream),
              "cudaMemcpy best states to host");
    check(cudaMemcpyAsync(&t0_host, d_t0, sizeof(uint64_t), cudaMemcpyDeviceToHost, stream), "cudaMemcpy clock");
    check(cudaStreamSynchronize(stream), "cudaStreamSynchronize results");
    vstats.assign(jobs.size(), VerifyStats{});
    vstats_valid.assign(jobs.size(), 0);
    if (want_best) {
        // every job's best W (orders up to 256) rescored and checked exactly
        // on the device, in one batch
        std::vector<VerifyItem> items;
        std::vector<size_t> of;
        for (size_t j = 0; j < jobs.size(); ++j) {
            if (jobs[j].n > XW_MAX_ORDER_SHARED) continue;
            items.push_back({static_cast<const int8_t*>(d_best) + best_offsets[j], jobs[j].n, jobs[j].w});
            of.push_back(j);
        }
        std::vector<VerifyStats> vs;
        std::mutex* mu = nullptr;
        DeviceVerifier& verifier = shared_verifier(params.device, mu);
        {
            std::lock_guard<std::mutex> lock(*mu);
            verifier.run(items, stream, vs);
        }
        for (size_t k = 0; k < of.size(); ++k) {
            vstats[of[k]] = vs[k];
            vstats_valid[of[k]] = 1;
        }
    }
}

void Batch::fill_results(const std::vector<JobOut>& out, const int8_t* best_host, xw_job_result* res) const {
    for (size_t j = 0; j < jobs.size(); ++j) {
        const JobOut& o = out[j];
        xw_job_result& r = res[j];
        std::memset(&r, 0, sizeof r);
        r.score = o.score;
        r.conflicts = o.conflicts;
        r.best_replica = o.best_replica;
        r.solved = o.score == 0;
        r.error = o.err;
        r.moves = o.moves;
        r.candidate_evaluations = o.cand_evals;
        r.accepted_moves = o.accepted;
        r.accepted_rows = o.accepted_rows;
        r.two_row_evaluations = o.two_row_evals;
        r.iterations = o.iters;
        r.solved_iteration = o.solved_it;
        r.time_to_solution_seconds = (o.solved && o.solve_ns >= t0_host) ? (o.solve_ns - t0_host) * 1e-9 : -1.0;
        if (best_host && r.solved) {
            const int n = jobs[j].n;
            if (j < vstats_valid.size() && vstats_valid[j]) {
                // the device check of this best W (collect)
                r.verified = vstats[j].exact == 1 && vstats[j].score == 0 ? 1 : 0;
            } else {
                // orders above 256: the int64 check on the host
                std::vector<int8_t> e(best_host + best_offsets[j], best_host + best_offsets[j] + (size_t)n * n);
                try {
                    r.verified = CpuState::from_entries(n, jobs[j].w, e).verify_weighing() ? 1 : 0;
                } catch (const std::exception&) {
                    r.verified = 0;
                }
            }
        }
    }
}

// Elite restart of job j (xweigh_cuda.cu:1817-2289): restart_count replicas,
// taken from a rotating cursor and skipping the elite, are replaced by kicked
// copies of the elite's best state; each gets the kicked state's score, the
// better of it and the global best as its best, and the reheat temperature.
// The job's records make one round trip through host memory.  Returns the
// number of replicas restarted; `line` receives the reference's log line.
// Operations of the escape scan of W: about 4 n per candidate switch, and a
// row pair (r1, r2) has k1 * k2 of them, k1 (k2) the columns that are
// nonzero in r1 (r2) and zero in the other row.
double escape_scan_work(int n, const std::vector<int8_t>& W) {
    const int nw = (n + 63) / 64;
    std::vector<uint64_t> S((size_t)n * nw, 0);
    for (int c = 0; c < n; ++c)
        for (int r = 0; r < n; ++r)
            if (W[(size_t)c * n + r]) S[(size_t)r * nw + c / 64] |= 1ull << (c % 64);
    double pairs = 0.0;
    for (int a = 0; a < n; ++a)
        for (int b2 = a + 1; b2 < n; ++b2) {
            int k1 = 0, k2 = 0;
            for (int q = 0; q < nw; ++q) {
                const uint64_t x = S[(size_t)a * nw + q], y = S[(size_t)b2 * nw + q];
                k1 += __builtin_popcountll(x & ~y);
                k2 += __builtin_popcountll(y & ~x);
            }
            pairs += (double)k1 * k2;
        }
    return pairs * 4.0 * n;
}

int restart_population(Batch& b, int j, const std::vector<int8_t>& elite_best, int64_t gbest, int64_t gconf,
                       RestartState& rs, double elapsed, std::string& line) {
    const xw_params& p = b.params;
    XwJob& J = b.jobs[j];
    const int R = J.replicas, n = J.n, w = J.w;
    if (p.restart_interval <= 0.0 || R < 2 || J.tempering) return 0;
    const int available = R - 1;
    const int count = std::clamp((int)std::ceil(p.restart_fraction * available), 1, available);
    const CpuState elite = CpuState::from_entries(n, w, elite_best);
    const size_t limit = std::max<size_t>((size_t)count * 4, 1);
    std::vector<int32_t> eg((size_t)n * n);
    for (int a = 0; a < n; ++a)
        for (int c = 0; c < n; ++c) eg[(size_t)a * n + c] = elite.gram_at(a, c);
    // Within the reference's orders the scan is at most ~1.4e11 operations
    // (W(256,128), 0.3 s); above them, with weights near n/2, it grows as
    // n^5 (W(300,150) ~3e11, W(1024,512) ~5e14).  Past kEscapeScanBudget
    // the restart kicks without an escape move rather than stall the run.
    std::vector<ScanResult> scan;
    if (escape_scan_work(n, elite_best) <= kEscapeScanBudget) scan = escape_scan(n, elite_best.data(), eg.data(), limit);
    const std::vector<EscapeMove> escapes = escape_moves_from(elite, scan);
    std::vector<int> selected;
    size_t scanned = 0;
    while ((int)selected.size() < count && scanned < (size_t)R * 2) {
        const int r = (int)((rs.cursor + scanned) % (size_t)R);
        ++scanned;
        if (r == rs.elite) continue;
        selected.push_back(r);
    }
    rs.cursor = (rs.cursor + scanned) % (size_t)R;
    auto kick_of = [&](size_t idx) {
        return selected.size() > 1 ? p.restart_kick_min + (int)(idx * (size_t)(p.restart_kick_max - p.restart_kick_min) /
                                                                (selected.size() - 1))
                                   : p.restart_kick_min;
    };
    auto done_line = [&]() {
        ++rs.round;
        rs.restarted += selected.size();
        line = fmt("[restart] seconds=%g elite_score=%lld replicas=%zu kicks=%d..%d min_escape_delta=%lld", elapsed,
                   (long long)gbest, selected.size(), p.restart_kick_min, p.restart_kick_max,
                   (long long)(escapes.empty() ? 0 : escapes.front().score_delta));
        return (int)selected.size();
    };

    if (p.restart_kicks == 1) {
        // device kicks: the records are rewritten in place by one CTA per
        // restarted replica (xw_restart.cu); only the job's small tables
        // cross to the device, no record comes back
        const size_t pool = std::min(scan.size(), std::max<size_t>(selected.size() * 4, 1));
        std::vector<int32_t> esc;
        for (size_t k = 0; k < pool; ++k) {
            const ScanResult& x = scan[k];
            esc.insert(esc.end(), {x.row1, x.row2, x.col1, x.col2, x.new1, x.new2});
        }
        std::vector<KickJob> kicks(selected.size());
        for (size_t idx = 0; idx < selected.size(); ++idx) {
            kicks[idx].rid = J.rep_begin + (uint32_t)selected[idx];
            kicks[idx].index = (uint32_t)idx;
            kicks[idx].kick = kick_of(idx);
            kicks[idx].esc = pool ? (int32_t)((idx + (size_t)rs.round * selected.size()) % pool) : -1;
        }
        void *d_kicks = nullptr, *d_esc = nullptr, *d_scratch = nullptr;
        b.dalloc(&d_kicks, sizeof(KickJob) * kicks.size(), "cudaMalloc kicks");
        b.dalloc(&d_esc, sizeof(int32_t) * std::max<size_t>(esc.size(), 1), "cudaMalloc escape moves");
        b.dalloc(&d_scratch, sizeof(uint16_t) * XW_MAX_ORDER_LARGE * kicks.size(), "cudaMalloc kick scratch");
        check(cudaMemcpyAsync(d_kicks, kicks.data(), sizeof(KickJob) * kicks.size(), cudaMemcpyHostToDevice, b.stream),
              "upload kicks");
        if (!esc.empty())
            check(cudaMemcpyAsync(d_esc, esc.data(), sizeof(int32_t) * esc.size(), cudaMemcpyHostToDevice, b.stream),
                  "upload escape moves");
        KickArgs ka;
        ka.job = static_cast<const XwJob*>(b.d_jobs) + j;
        ka.arena = static_cast<uint8_t*>(b.d_arena);
        ka.rec_off = static_cast<const uint64_t*>(b.d_rec_off);
        ka.elite = static_cast<const int8_t*>(b.d_best) + b.best_offsets[j];
        ka.escapes = static_cast<const int32_t*>(d_esc);
        ka.kicks = static_cast<const KickJob*>(d_kicks);
        ka.scratch = static_cast<uint16_t*>(d_scratch);
        ka.round = rs.round;
        ka.gbest = (int32_t)gbest;
        ka.gconf = (int32_t)gconf;
        ka.t_min = p.t_min;
        ka.reheat = p.reheat;
        launch_kicks(ka, (int)kicks.size(), b.stream);
        for (void* ptr : {d_kicks, d_esc, d_scratch}) check(cudaFreeAsync(ptr, b.stream), "cudaFreeAsync");
        check(cudaStreamSynchronize(b.stream), "cudaStreamSynchronize kicks");
        return done_line();
    }

    const size_t rb = J.record_bytes, base = b.rec_off[J.rep_begin];
    std::vector<uint8_t> host((size_t)R * rb);
    uint8_t* dev = static_cast<uint8_t*>(b.d_arena) + base;
    check(cudaMemcpyAsync(host.data(), dev, host.size(), cudaMemcpyDeviceToHost, b.stream), "read restart records");
    check(cudaStreamSynchronize(b.stream), "cudaStreamSynchronize");
    CpuParams cp;
    cp.sign_fraction = p.sign_fraction;
    cp.target_fraction = p.target_fraction;
    cp.target_samples = p.target_samples;
    const int m = J.m;
    const uint32_t base_seed = (uint32_t)p.seed;
    parallel_for((int)selected.size(), [&](int idx) {
        const int r = selected[(size_t)idx];
        const int kick = kick_of((size_t)idx);
        const CpuState k = kick_elite(elite, escapes, (size_t)idx, selected.size(), rs.round, r, base_seed, kick, cp);
        uint8_t* rec = host.data() + (size_t)r * rb;
        RepHeader* H = reinterpret_cast<RepHeader*>(rec);
        std::memcpy(rec + J.off_w, k.entries().data(), (size_t)n * n);
        if (J.large) {
            std::memcpy(rec + J.off_mino, k.minority().data(), sizeof(uint16_t) * n * m);
            H->status &= ~XW_STATUS_GRAM;   // the kernel rebuilds G from the new W
        } else {
            for (int i = 0; i < n * m; ++i) rec[J.off_mino + i] = (uint8_t)k.minority()[(size_t)i];
        }
        const bool kick_better = k.score() < gbest || (k.score() == gbest && k.conflicts() < gconf);
        std::memcpy(rec + J.off_best, kick_better ? k.entries().data() : elite_best.data(), (size_t)n * n);
        H->score = (int32_t)k.score();
        H->conflicts = (int32_t)k.conflicts();
        H->best_score = (int32_t)(kick_better ? k.score() : gbest);
        H->best_conflicts = (int32_t)(kick_better ? k.conflicts() : gconf);
        int64_t st[4];
        xw_score(n, w, k.entries().data(), st);
        H->obj_total = H->obj_kind == 1 ? st[2] : H->obj_kind == 2 ? st[3] : st[0];
        H->temperature = std::max(p.t_min, H->reheat_temperature * p.reheat);
        H->msi = 0;
        H->cool_ctr = 0;
    });
    check(cudaMemcpyAsync(dev, host.data(), host.size(), cudaMemcpyHostToDevice, b.stream), "write restart records");
    check(cudaStreamSynchronize(b.stream), "cudaStreamSynchronize");
    return done_line();
}

}  // namespace xw

// ==========================================================================
// C ABI
using namespace xw;

extern "C" {

void xw_params_default(xw_params* p) {
    std::memset(p, 0, sizeof *p);
    p->device = 0;
    p->replicas = 0;
    p->moves_per_launch = 4096;
    p->seed = 0;
    p->max_seconds = 0.0;
    p->save_interval = 2.0;
    p->sign_fraction = 0.5;
    p->double_sign_fraction = 0.25;
    p->switch_sign_fraction = 0.5;
    p->squared_objective_fraction = 0.25;
    p->parity_objective_fraction = 0.25;
    p->greedy_fraction = 0.5;
    p->candidate_samples = 4;
    p->target_fraction = 0.7;
    p->target_samples = 8;
    p->t_init = 0.0;
    p->t_min = 0.25;
    p->cooling = 0.999;
    p->moves_per_cool = 500;
    p->stuck_threshold = 50000;
    p->reheat = 1.0;
    p->restart_interval = 5.0;
    p->restart_fraction = 0.25;
    p->restart_kick_min = 2;
    p->restart_kick_max = 64;
    p->max_moves = 0;
    p->tempering = 0;
    p->exchange_interval = 10000;
    p->objective = -1;
    p->move_set = 0;
    p->start_kind = 0;
    p->stop_on_solve = 1;
    p->warps_per_block = 0;
    p->replicas_per_warp = 0;
    p->warps_per_replica = 0;
    p->restart_kicks = 0;
}

const char* xw_last_error(void) { return g_last_error.c_str(); }

int32_t xw_validate_params(int32_t n, int32_t w, const xw_params* p) {
    if (!p) return fail(XW_ERR_INVALID, "null params");
    const std::string e = validate(n, w, *p);
    return e.empty() ? XW_OK : fail(XW_ERR_INVALID, e);
}

int32_t xw_query_device(int32_t ordinal, xw_device_info* out) {
    if (!out) return fail(XW_ERR_INVALID, "null output");
    int count = 0;
    cudaError_t e = cudaGetDeviceCount(&count);
    if (e != cudaSuccess)
        return fail(XW_ERR_CUDA, fmt("cudaGetDeviceCount failed: %s (%s)", cudaGetErrorName(e), cudaGetErrorString(e)));
    if (ordinal < 0 || ordinal >= count)
        return fail(XW_ERR_INVALID,
                    fmt("CUDA device ordinal %d is out of range; found %d device(s)", ordinal, count));
    cudaDeviceProp prop{};
    e = cudaGetDeviceProperties(&prop, ordinal);
    if (e != cudaSuccess) return fail(XW_ERR_CUDA, fmt("cudaGetDeviceProperties failed: %s", cudaGetErrorString(e)));
    int optin = 0;
    cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, ordinal);
    if (optin <= 0) optin = (int)prop.sharedMemPerBlock;
    std::memset(out, 0, sizeof *out);
    std::snprintf(out->name, sizeof out->name, "%s", prop.name);
    out->ordinal = ordinal;
    out->compute_major = prop.major;
    out->compute_minor = prop.minor;
    out->multiprocessors = prop.multiProcessorCount;
    out->global_memory = prop.totalGlobalMem;
    out->max_shared_memory_per_block = (uint64_t)optin;
    return XW_OK;
}

void xw_request_stop(void) { g_stop.store(1, std::memory_order_relaxed); }
void xw_clear_stop(void) { g_stop.store(0, std::memory_order_relaxed); }

int32_t xw_random_start(int32_t n, int32_t w, uint32_t seed, int8_t* out) {
    if (n < 1 || w < 1 || w > n || !out) return fail(XW_ERR_INVALID, "invalid W(n,w) or output");
    const CpuState s = CpuState::random_start(n, w, seed);
    std::memcpy(out, s.entries().data(), (size_t)n * n);
    return XW_OK;
}

int32_t xw_row_start(int32_t n, int32_t w, uint64_t seed, uint32_t replica, int8_t* out) {
    if (n < 1 || w < 1 || w > n || !out) return fail(XW_ERR_INVALID, "invalid W(n,w) or output");
    const uint32_t base = (uint32_t)seed;
    const uint64_t key = ((uint64_t)base << 32) ^ seed ^ 0xd1b54a32d192ed03ull;
    const std::vector<int8_t> e = row_start(n, w, (uint32_t)key, (uint32_t)(key >> 32), replica);
    std::memcpy(out, e.data(), e.size());
    return XW_OK;
}

int32_t xw_sylvester(int32_t n, int32_t w, int8_t* out) {
    if (n < 1 || w < 1 || w > n || !out || (w & (w - 1)) != 0 || n % w != 0)
        return fail(XW_ERR_INVALID, "Sylvester blocks need w a power of two dividing n");
    const CpuState s = CpuState::sylvester_blocks(n, w);
    std::memcpy(out, s.entries().data(), (size_t)n * n);
    return XW_OK;
}

int32_t xw_score(int32_t n, int32_t w, const int8_t* W, int64_t stats[4]) {
    if (n < 1 || !W || !stats) return fail(XW_ERR_INVALID, "invalid arguments");
    (void)w;
    int64_t s = 0, c = 0, q = 0, par = 0;
    const size_t nn = (size_t)n * n;
    bool ternary = true;
    for (size_t i = 0; i < nn && ternary; ++i) ternary = W[i] >= -1 && W[i] <= 1;
    if (ternary) {
        // W_a . W_b = |S_a & S_b| - 2 |S_a & S_b & (N_a ^ N_b)| over the
        // support (S) and negative-sign (N) bit rows: O(n^3 / 64)
        const int nw = (n + 63) / 64;
        std::vector<uint64_t> S((size_t)n * nw, 0), N((size_t)n * nw, 0);
        for (int k = 0; k < n; ++k)
            for (int a = 0; a < n; ++a) {
                const int8_t v = W[(size_t)k * n + a];
                if (v) S[(size_t)a * nw + k / 64] |= 1ull << (k % 64);
                if (v < 0) N[(size_t)a * nw + k / 64] |= 1ull << (k % 64);
            }
        for (int a = 0; a < n; ++a)
            for (int b = a + 1; b < n; ++b) {
                int64_t d = 0;
                for (int k = 0; k < nw; ++k) {
                    const uint64_t both = S[(size_t)a * nw + k] & S[(size_t)b * nw + k];
                    d += __builtin_popcountll(both) -
                         2 * __builtin_popcountll(both & (N[(size_t)a * nw + k] ^ N[(size_t)b * nw + k]));
                }
                const int64_t ad = d < 0 ? -d : d;
                s += ad;
                c += d != 0;
                q += d * d;
                par += ad & 1;
            }
        stats[0] = s; stats[1] = c; stats[2] = q; stats[3] = par;
        return XW_OK;
    }
    for (int a = 0; a < n; ++a)
        for (int b = a + 1; b < n; ++b) {
            int64_t d = 0;
            for (int k = 0; k < n; ++k) d += (int64_t)W[(size_t)k * n + a] * W[(size_t)k * n + b];
            const int64_t ad = d < 0 ? -d : d;
            s += ad;
            c += d != 0;
            q += d * d;
            par += ad & 1;
        }
    stats[0] = s; stats[1] = c; stats[2] = q; stats[3] = par;
    return XW_OK;
}

int32_t xw_verify(int32_t n, int32_t w, const int8_t* W) {
    if (n < 1 || w < 1 || !W) return 0;
    try {
        const CpuState s = CpuState::from_entries(n, w, std::vector<int8_t>(W, W + (size_t)n * n));
        if (!s.verify_support()) return 0;
        return s.verify_weighing() ? 3 : 1;
    } catch (const std::exception&) {
        return 0;
    }
}

int32_t xw_read_csv(const char* path, int32_t n, int32_t w, int8_t* out) {
    if (!path || !out) return fail(XW_ERR_INVALID, "null argument");
    try {
        const std::vector<int8_t> e = read_csv(path, n, w);
        std::memcpy(out, e.data(), e.size());
        return XW_OK;
    } catch (const std::exception& ex) {
        return fail(XW_ERR_IO, ex.what());
    }
}

int32_t xw_write_csv(const char* path, int32_t n, const int8_t* W) {
    if (!path || !W || n < 1) return fail(XW_ERR_INVALID, "null argument");
    try {
        write_csv(std::vector<int8_t>(W, W + (size_t)n * n), n, path);
        return XW_OK;
    } catch (const std::exception& ex) {
        return fail(XW_ERR_IO, ex.what());
    }
}

const char* xw_impossibility_reason(int32_t n, int32_t w) {
    static thread_local std::string reason;
    reason = impossibility_reason(n, w);
    return reason.c_str();
}

double xw_calibrate(int32_t n, int32_t w, const int8_t* W, const xw_params* p, uint32_t seed) {
    try {
        CpuParams cp;
        cp.sign_fraction = p->sign_fraction;
        cp.target_fraction = p->target_fraction;
        cp.target_samples = p->target_samples;
        cp.t_init = p->t_init;
        const CpuState s = CpuState::from_entries(n, w, std::vector<int8_t>(W, W + (size_t)n * n));
        return calibrate_temperature(s, cp, seed);
    } catch (const std::exception& ex) {
        g_last_error = ex.what();
        return -1.0;
    }
}

// ---- batches ---------------------------------------------------------------

struct xw_batch {
    std::unique_ptr<Batch> b;
    std::vector<RestartState> restarts;   // per job, for xw_batch_restart
};

#define XW_GUARD(...)                                                         \
    try {                                                                     \
        __VA_ARGS__                                                           \
    } catch (const CudaError& ex) {                                           \
        return fail(XW_ERR_CUDA, ex.what());                                  \
    } catch (const std::length_error& ex) {                                   \
        return fail(XW_ERR_CAPACITY, ex.what());                              \
    } catch (const std::invalid_argument& ex) {                               \
        return fail(XW_ERR_INVALID, ex.what());                               \
    } catch (const std::bad_alloc&) {                                         \
        return fail(XW_ERR_CAPACITY, "insufficient host memory");             \
    } catch (const std::exception& ex) {                                      \
        return fail(XW_ERR_INTERNAL, ex.what());                              \
    }

int32_t xw_batch_create(const xw_job_spec* jobs, int32_t njobs, const xw_params* p, const int8_t* starts,
                        xw_batch** out) {
    if (!jobs || !p || !out || njobs < 1) return fail(XW_ERR_INVALID, "invalid batch arguments");
    for (int j = 0; j < njobs; ++j) {
        const std::string e = validate(jobs[j].n, jobs[j].w, *p);
        if (!e.empty()) return fail(XW_ERR_INVALID, e);
    }
    XW_GUARD({
        auto h = std::make_unique<xw_batch>();
        h->b = std::make_unique<Batch>();
        h->b->build(jobs, njobs, *p, starts);
        *out = h.release();
        return XW_OK;
    })
}

int32_t xw_batch_save(xw_batch* h, const char* path) {
    if (!h || !path) return fail(XW_ERR_INVALID, "null argument");
    XW_GUARD({
        h->b->save(path);
        return XW_OK;
    })
}

int32_t xw_batch_load(const char* path, const xw_params* over, xw_batch** out) {
    if (!path || !out) return fail(XW_ERR_INVALID, "null argument");
    if (over) {
        const std::string e = validate(1, 1, *over);
        if (!e.empty()) return fail(XW_ERR_INVALID, e);
    }
    XW_GUARD({
        auto h = std::make_unique<xw_batch>();
        h->b = std::make_unique<Batch>();
        h->b->load(path, over);
        *out = h.release();
        return XW_OK;
    })
}

int32_t xw_batch_set_stream(xw_batch* h, void* s) {
    if (!h) return fail(XW_ERR_INVALID, "null batch");
    XW_GUARD({
        Batch& b = *h->b;
        check(cudaStreamSynchronize(b.stream), "cudaStreamSynchronize");
        if (b.own_stream) cudaStreamDestroy(b.stream);
        b.own_stream = s == nullptr;
        if (s) b.stream = static_cast<cudaStream_t>(s);
        else check(cudaStreamCreateWithFlags(&b.stream, cudaStreamNonBlocking), "cudaStreamCreate");
        if (b.graph_exec) {
            cudaGraphExecDestroy(b.graph_exec);
            b.graph_exec = nullptr;
        }
        return XW_OK;
    })
}

int32_t xw_batch_reset(xw_batch* h) {
    if (!h) return fail(XW_ERR_INVALID, "null batch");
    XW_GUARD({
        h->b->reset();
        return XW_OK;
    })
}

int32_t xw_batch_run(xw_batch* h, uint64_t iters) {
    if (!h) return fail(XW_ERR_INVALID, "null batch");
    XW_GUARD({
        h->b->run(iters, true);
        return XW_OK;
    })
}

int32_t xw_batch_run_timed(xw_batch* h, uint64_t iters) {
    if (!h) return fail(XW_ERR_INVALID, "null batch");
    XW_GUARD({
        h->b->run(iters, false);
        return XW_OK;
    })
}

int32_t xw_batch_synchronize(xw_batch* h) {
    if (!h) return fail(XW_ERR_INVALID, "null batch");
    XW_GUARD({
        check(cudaStreamSynchronize(h->b->stream), "cudaStreamSynchronize");
        return XW_OK;
    })
}

int32_t xw_batch_launch_times(xw_batch* h, float* ms, int32_t cap, int32_t* count) {
    if (!h || !count) return fail(XW_ERR_INVALID, "null argument");
    XW_GUARD({
        Batch& b = *h->b;
        check(cudaStreamSynchronize(b.stream), "cudaStreamSynchronize");
        *count = b.last_rounds;
        for (int k = 0; k < b.last_rounds && k < cap; ++k)
            check(cudaEventElapsedTime(&ms[k], b.events[2 * k], b.events[2 * k + 1]), "cudaEventElapsedTime");
        return XW_OK;
    })
}

int32_t xw_autotune(const xw_job_spec* jobs, int32_t njobs, const xw_params* pin, uint64_t iters,
                    int32_t* best_wpb, float* best_ms) {
    if (!jobs || njobs < 1 || !pin || !best_wpb || iters == 0) return fail(XW_ERR_INVALID, "bad autotune arguments");
    XW_GUARD({
        for (int j = 0; j < njobs; ++j) {
            const std::string err = validate(jobs[j].n, jobs[j].w, *pin);
            if (!err.empty()) return fail(XW_ERR_INVALID, err);
        }
        Batch b;
        b.split_pair_class = true;   // the orders up to 16 are tuned apart
        b.build(jobs, njobs, *pin, nullptr);
        if (b.classes.empty())
            return fail(XW_ERR_INVALID, "autotune covers the shared-memory kernel; every job here is of larger order");
        int optin = 0;
        check(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, pin->device),
              "cudaDeviceGetAttribute max opt-in shared memory");
        // each class alone: the batch's other classes are left out of the
        // trial launches by timing only this class's items
        const std::vector<Batch::LaunchClass> all = b.classes;
        const uint32_t n_large = b.n_large;
        b.n_large = 0;   // the trials launch no large-order replicas
        float total_best = 0.0f;
        int first_wpb = 0;
        for (size_t k = 0; k < all.size(); ++k) {
            b.classes.assign(1, all[k]);
            int best = 0, best_rpw = 1;
            float best_t = 0.0f;
            auto time_trial = [&]() {
                b.reserve_rounds((int)((iters + b.round_iters() - 1) / b.round_iters()));
                float total = 0.0f;
                for (int rep = 0; rep < 2; ++rep) {   // the first pass warms up, the second is timed
                    b.reset();
                    b.run(iters, false);
                    check(cudaStreamSynchronize(b.stream), "cudaStreamSynchronize");
                    total = 0.0f;
                    for (int r = 0; r < b.last_rounds; ++r) {
                        float ms = 0.0f;
                        check(cudaEventElapsedTime(&ms, b.events[2 * r], b.events[2 * r + 1]), "cudaEventElapsedTime");
                        total += ms;
                    }
                }
                return total;
            };
            // the latency mode, for classes of at most one replica per SM
            int best_wpr = 1;
            float best_lat = 0.0f;
            if (all[k].max_n <= 32 && all[k].item_count <= (uint32_t)b.props.multiProcessorCount) {
                for (int wpr : {2, 4, 8, 16, 32, 64}) {
                    if (wpr > 16 && (uint32_t)(wpr / 16) * all[k].item_count > (uint32_t)b.props.multiProcessorCount)
                        continue;
                    if (!b.configure_latency(0, wpr)) continue;
                    const float t = time_trial();
                    if (best_wpr == 1 || t < best_lat) {
                        best_wpr = wpr;
                        best_lat = t;
                    }
                }
            }
            float default_t = 0.0f;   // four warps per CTA, one replica per warp
            for (int rpw : {1, 2}) {
                if (rpw == 2 && all[k].kind != kTunePairKind) continue;
                for (int wpb : {1, 2, 4, 8, 16}) {
                    if ((size_t)wpb * rpw * all[k].slot_bytes > (size_t)optin) break;
                    if (!b.configure_class(0, wpb, rpw)) continue;
                    const float total = time_trial();
                    if (wpb == 4 && rpw == 1) default_t = total;
                    if (best == 0 || total < best_t) {
                        best = wpb;
                        best_rpw = rpw;
                        best_t = total;
                    }
                }
            }
            if (best == 0) return fail(XW_ERR_CAPACITY, "no launch shape fits the device's shared memory");
            // a short trial's tail and chunking favour shapes that hold fewer
            // warps (W(18..30,n-1) x 4096: 16 warps per CTA won a 2000-
            // iteration trial and lost 10% over 20000 iterations), so the
            // default shape stays unless a trial beats it by more than 3%
            if (default_t > 0.0f && best_t > 0.97f * default_t) {
                best = 4;
                best_rpw = 1;
                best_t = default_t;
            }
            record_tuned(all[k].kind, all[k].slot_bytes, best, best_rpw);
            if (best_wpr > 1) {
                // the latency mode against the best one-warp shape
                const bool lat = best_lat < best_t;
                record_tuned(kTuneLatencyKind, all[k].slot_bytes, lat ? best_wpr : 1, 1);
                if (lat) best_t = best_lat;
            }
            if (k == 0) first_wpb = best;
            total_best += best_t;
        }
        b.classes = all;
        b.n_large = n_large;
        *best_wpb = first_wpb;
        if (best_ms) *best_ms = total_best;
        return XW_OK;
    })
}

int32_t xw_batch_restart(xw_batch* h, int32_t job, int32_t* restarted) {
    if (!h || !restarted) return fail(XW_ERR_INVALID, "null argument");
    XW_GUARD({
        Batch& b = *h->b;
        if (job < 0 || job >= (int)b.jobs.size()) return fail(XW_ERR_INVALID, "job index out of range");
        if (h->restarts.size() != b.jobs.size()) h->restarts.assign(b.jobs.size(), RestartState{});
        std::vector<JobOut> out;
        std::vector<int8_t> best(b.best_bytes);
        b.collect(out, best.data(), true);
        const XwJob& J = b.jobs[job];
        const std::vector<int8_t> elite(best.begin() + b.best_offsets[job],
                                        best.begin() + b.best_offsets[job] + (size_t)J.n * J.n);
        RestartState& rs = h->restarts[job];
        rs.elite = out[job].best_replica;
        std::string line;
        *restarted = restart_population(b, job, elite, out[job].score, out[job].conflicts, rs, 0.0, line);
        return XW_OK;
    })
}

int32_t xw_batch_results(xw_batch* h, xw_job_result* results, int8_t* best) {
    if (!h || !results) return fail(XW_ERR_INVALID, "null argument");
    XW_GUARD({
        Batch& b = *h->b;
        std::vector<JobOut> out;
        std::vector<int8_t> tmp;
        int8_t* dst = best;
        if (!dst) {
            tmp.resize(b.best_bytes);
            dst = tmp.data();
        }
        b.collect(out, dst, true);
        b.fill_results(out, dst, results);
        return XW_OK;
    })
}

int32_t xw_batch_read_replica(xw_batch* h, int32_t job, int32_t replica, xw_replica_state* st, int8_t* W,
                              int8_t* best_W, uint8_t* minority) {
    if (!h) return fail(XW_ERR_INVALID, "null batch");
    Batch& b = *h->b;
    if (job < 0 || job >= (int)b.jobs.size()) return fail(XW_ERR_INVALID, "job index out of range");
    const XwJob& J = b.jobs[job];
    if (replica < 0 || replica >= J.replicas) return fail(XW_ERR_INVALID, "replica index out of range");
    XW_GUARD({
        std::vector<uint8_t> rec(J.record_bytes);
        check(cudaStreamSynchronize(b.stream), "cudaStreamSynchronize");
        check(cudaMemcpy(rec.data(), static_cast<uint8_t*>(b.d_arena) + b.rec_off[J.rep_begin + replica],
                         J.record_bytes, cudaMemcpyDeviceToHost),
              "cudaMemcpy replica to host");
        const RepHeader* H = reinterpret_cast<const RepHeader*>(rec.data());
        if (st) {
            st->iterations = H->it;
            st->moves = H->moves;
            st->candidate_evaluations = H->cand_evals;
            st->score = H->score;
            st->conflicts = H->conflicts;
            st->best_score = H->best_score;
            st->best_conflicts = H->best_conflicts;
            st->objective_total = H->obj_total;
            st->temperature = H->temperature;
            st->reheat_temperature = H->reheat_temperature;
            st->moves_since_improvement = H->msi;
            st->cooling_counter = H->cool_ctr;
            st->rung = H->rung;
            st->objective_kind = H->obj_kind;
            st->status = H->status;
            st->error = H->err;
            st->accepted_moves = H->accepted;
            st->accepted_rows = H->accepted_rows;
            st->two_row_evaluations = H->two_row_evals;
            st->reserved = 0;
        }
        const size_t nn = (size_t)J.n * J.n;
        if (W) std::memcpy(W, rec.data() + J.off_w, nn);
        if (best_W) std::memcpy(best_W, rec.data() + J.off_best, nn);
        // one byte per entry up to XW_MAX_ORDER_SHARED, two above, whichever
        // kernel holds the replica
        const size_t nm = (size_t)J.n * J.m;
        if (minority && !J.large) {
            std::memcpy(minority, rec.data() + J.off_mino, nm);
        } else if (minority && J.n > XW_MAX_ORDER_SHARED) {
            std::memcpy(minority, rec.data() + J.off_mino, 2 * nm);
        } else if (minority) {
            const uint16_t* src = reinterpret_cast<const uint16_t*>(rec.data() + J.off_mino);
            for (size_t i = 0; i < nm; ++i) minority[i] = (uint8_t)src[i];
        }
        return XW_OK;
    })
}

int32_t xw_batch_bytes(xw_batch* h, uint64_t* h2d, uint64_t* d2h) {
    if (!h) return fail(XW_ERR_INVALID, "null batch");
    const Batch& b = *h->b;
    if (h2d)
        *h2d = b.arena_bytes + sizeof(XwJob) * b.jobs.size() + sizeof(uint64_t) * b.total_replicas +
               sizeof(uint32_t) * b.total_replicas + sizeof(double) * b.ladder.size() +
               sizeof(uint64_t) * b.jobs.size();
    if (d2h) *d2h = sizeof(JobOut) * b.jobs.size() + b.best_bytes + sizeof(uint64_t);
    return XW_OK;
}

int32_t xw_batch_shape(xw_batch* h, int32_t* wpb, int32_t* blocks, int32_t* slot) {
    if (!h) return fail(XW_ERR_INVALID, "null batch");
    // the class with the most replicas
    const Batch& b = *h->b;
    const Batch::LaunchClass* c = nullptr;
    for (const auto& k : b.classes)
        if (!c || k.item_count > c->item_count) c = &k;
    if (wpb) *wpb = c ? c->wpb : b.large_wpb;
    if (blocks) *blocks = c ? c->blocks : b.large_blocks;
    if (slot) *slot = (int32_t)(c ? c->slot_bytes : b.large_slot_bytes);
    return XW_OK;
}

int32_t xw_batch_classes(xw_batch* h, xw_launch_class* out, int32_t cap, int32_t* count) {
    if (!h || !count || (cap > 0 && !out)) return fail(XW_ERR_INVALID, "null argument");
    const Batch& b = *h->b;
    std::vector<xw_launch_class> all;
    if (b.n_large) {
        xw_launch_class c{};
        c.large = 1 + b.large_form;
        c.min_order = 0x7fffffff;
        for (const XwJob& J : b.jobs)
            if (J.large) {
                c.min_order = std::min(c.min_order, J.n);
                c.max_order = std::max(c.max_order, J.n);
                c.general = c.general || J.general;
            }
        c.rows_per_lane = 0;
        c.replicas_per_warp = 1;
        c.warps_per_block = b.large_wpb;
        c.blocks = b.large_blocks;
        c.slot_bytes = (int32_t)b.large_slot_bytes;
        c.chunks = (int32_t)b.large_chunks;
        c.replicas = (int32_t)b.n_large;
        c.warps_per_replica = 1;
        all.push_back(c);
    }
    for (const auto& k : b.classes) {
        xw_launch_class c{};
        c.min_order = k.min_n;
        c.max_order = k.max_n;
        c.rows_per_lane = k.opl;
        c.replicas_per_warp = k.rpw;
        c.warps_per_block = k.wpb;
        c.blocks = k.blocks;
        c.slot_bytes = (int32_t)k.slot_bytes;
        c.chunks = (int32_t)k.chunks;
        c.replicas = (int32_t)k.item_count;
        c.general = k.general ? 1 : 0;
        c.warps_per_replica = k.wpr;
        if (k.wpr > 1) c.slot_bytes = (int32_t)k.spec_bytes;
        all.push_back(c);
    }
    *count = (int32_t)all.size();
    for (int32_t i = 0; i < cap && i < (int32_t)all.size(); ++i) out[i] = all[i];
    return XW_OK;
}

void xw_batch_destroy(xw_batch* h) { delete h; }

int32_t xw_batch_solve(const xw_job_spec* jobs, int32_t njobs, const xw_params* p, const int8_t* starts,
                       uint64_t iters, xw_job_result* results, int8_t* best) {
    xw_batch* h = nullptr;
    int32_t rc = xw_batch_create(jobs, njobs, p, starts, &h);
    if (rc != XW_OK) return rc;
    std::unique_ptr<xw_batch> guard(h);
    XW_GUARD({
        Batch& b = *h->b;
        uint64_t target = iters;
        if (target == 0) {
            for (const XwJob& J : b.jobs) target = std::max<uint64_t>(target, J.budget_iters);
            if (target == 0) return fail(XW_ERR_INVALID, "xw_batch_solve needs iters or a move budget");
        }
        b.run(target, false);
        std::vector<JobOut> out;
        std::vector<int8_t> tmp;
        int8_t* dst = best;
        if (!dst) {
            tmp.resize(b.best_bytes);
            dst = tmp.data();
        }
        b.collect(out, dst, true);
        b.fill_results(out, dst, results);
        return XW_OK;
    })
}

// ---- xw_run: the xweigh_cuda run_annealer drop-in -------------------------

int32_t xw_run(int32_t n, int32_t w, const xw_params* pin, const int8_t* start, xw_log_fn log,
               xw_checkpoint_fn checkpoint, void* user, xw_result* out, int8_t* best_out) {
    if (!pin || !out) return fail(XW_ERR_INVALID, "null argument");
    xw_params p = *pin;
    {
        const std::string e = validate(n, w, p);
        if (!e.empty()) return fail(XW_ERR_INVALID, e);
    }
    auto say = [&](const std::string& line) {
        if (log) log(line.c_str(), user);
    };
    std::memset(out, 0, sizeof *out);
    if (start) {
        try {
            const CpuState s = CpuState::from_entries(n, w, std::vector<int8_t>(start, start + (size_t)n * n));
            if (!s.verify_support()) return fail(XW_ERR_INVALID, "CUDA initial state is not fixed-weight");
        } catch (const std::exception&) {
            return fail(XW_ERR_INVALID, "CUDA initial state is not fixed-weight");
        }
    }
    int32_t rc = xw_query_device(p.device, &out->device);
    if (rc != XW_OK) return rc;
    if (n > XW_MAX_ORDER_CUDA)
        return fail(XW_ERR_CAPACITY, fmt("CUDA replica of order %d is above the device path's maximum order %d", n,
                                         XW_MAX_ORDER_CUDA));
    XW_GUARD({
        check(cudaSetDevice(p.device), "cudaSetDevice");
        const auto t_init0 = std::chrono::steady_clock::now();
        if (p.seed == 0) p.seed = (uint64_t)std::random_device{}();
        Batch b;
        xw_job_spec spec{};
        spec.n = n;
        spec.w = w;
        spec.seed = p.seed;
        int replicas = p.replicas;
        const int m = std::min(w, n - w);
        const bool large = n >= large_min_order();
        const int form = large && anneal_large_planes_fit(n, m) ? large_form_wanted() : 0;
        const uint32_t slot = large ? anneal_large_slot_bytes(n, m, form) : anneal_slot_bytes(n, m, anneal_opl(n));
        if (replicas == 0) {
            // one resident wave: warp slots per SM times SMs
            const int wpb = large ? 4 : p.warps_per_block > 0 ? p.warps_per_block : 4;
            int per_sm = 0;
            const void* fn = large ? anneal_large_kernel_fn(needs_general_kernel(p), form)
                                   : anneal_kernel_fn(anneal_opl(n), needs_general_kernel(p));
            raise_smem_limit(fn, p.device);
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, 32 * wpb, (size_t)wpb * slot);
            replicas = std::max(1, per_sm * wpb * out->device.multiprocessors);
        }
        if (p.tempering && replicas > XW_MAX_RUNGS) replicas = XW_MAX_RUNGS;
        spec.replicas = replicas;
        spec.max_moves = p.max_moves;
        say(fmt("[cuda] device=%s compute=%d.%d multiprocessors=%d replicas=%d shared_kib=%g", out->device.name,
                out->device.compute_major, out->device.compute_minor, out->device.multiprocessors, replicas,
                slot / 1024.0));
        std::vector<int8_t> starts;
        if (start) {
            starts.resize((size_t)replicas * n * n);
            for (int r = 0; r < replicas; ++r) std::memcpy(starts.data() + (size_t)r * n * n, start, (size_t)n * n);
        }
        b.build(&spec, 1, p, start ? starts.data() : nullptr);
        const double init_s = std::chrono::duration<double>(std::chrono::steady_clock::now() - t_init0).count();
        const double rec_mib = b.jobs[0].record_bytes / 1048576.0;
        say(fmt("[init] seconds=%g replica_mib=%g total_replica_mib=%g", init_s, rec_mib, rec_mib * replicas));
        std::vector<JobOut> res;
        std::vector<int8_t> best((size_t)n * n);
        b.collect(res, best.data(), true);
        say(fmt("[t=0s] start score=%lld conflicts=%lld n=%d w=%d replicas=%d t_init=%g", (long long)res[0].score,
                (long long)res[0].conflicts, n, w, replicas, b.t_init_used[0]));
        int64_t gbest = res[0].score, gconf = res[0].conflicts;
        int best_rep = res[0].best_replica;
        const auto t0 = std::chrono::steady_clock::now();
        double last_save = -1e300, last_progress = 0.0, last_improvement = 0.0, last_restart = 0.0;
        RestartState rs;
        bool pending = true;
        double solve_s = -1.0;
        const uint64_t budget = b.jobs[0].budget_iters;
        uint64_t done_iters = 0;
        while (gbest != 0) {
            const double el = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
            if (g_stop.load(std::memory_order_relaxed) || (p.max_seconds > 0.0 && el >= p.max_seconds)) break;
            if (budget && done_iters >= budget) break;
            uint64_t it = b.round_iters();
            if (budget) it = std::min<uint64_t>(it, budget - done_iters);
            b.run(it, false);
            done_iters += it;
            b.collect(res, best.data(), true);
            const double now = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
            if (res[0].err) throw std::runtime_error("CUDA replica failed its device self-check");
            if (res[0].score < gbest || (res[0].score == gbest && res[0].conflicts < gconf)) {
                gbest = res[0].score;
                gconf = res[0].conflicts;
                best_rep = res[0].best_replica;
                pending = true;
                say(fmt("[t=%gs] new best score=%lld conflicts=%lld (replica %d)", now, (long long)gbest,
                        (long long)gconf, best_rep));
                if (gbest == 0) solve_s = now;
                last_improvement = now;
            }
            if (gbest != 0 && p.restart_interval > 0.0 && now - last_improvement >= p.restart_interval &&
                now - last_restart >= p.restart_interval) {
                rs.elite = best_rep;
                std::string line;
                if (restart_population(b, 0, best, gbest, gconf, rs, now, line) > 0) say(line);
                last_restart = now;
            }
            if (pending && now - last_save >= p.save_interval) {
                if (checkpoint) checkpoint(best.data(), n, user);
                pending = false;
                last_save = now;
            }
            if (now - last_progress >= 2.0 && gbest != 0) {
                say(fmt("[t=%gs] moves=%llu best score=%lld conflicts=%lld", now, (unsigned long long)res[0].moves,
                        (long long)gbest, (long long)gconf));
                last_progress = now;
            }
        }
        b.collect(res, best.data(), true);
        const double search_s = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        // the final best W: rescored and checked exactly on the device
        // (tensor cores), or on the host above the shared-memory orders
        int64_t fin_score = 0, fin_conf = 0;
        bool fin_exact = false;
        if (!b.vstats_valid.empty() && b.vstats_valid[0]) {
            fin_score = b.vstats[0].score;
            fin_conf = b.vstats[0].conflicts;
            fin_exact = b.vstats[0].exact == 1;
        } else {
            const CpuState fin = CpuState::from_entries(n, w, best);
            fin_score = fin.score();
            fin_conf = fin.conflicts();
            fin_exact = fin.verify_weighing();
        }
        if (fin_score != res[0].score || fin_conf != res[0].conflicts)
            throw std::runtime_error("CUDA final best snapshot score mismatch");
        const uint64_t moves = res[0].moves, evals = res[0].cand_evals;
        say(fmt("done moves=%llu candidate_evaluations=%llu seconds=%g moves_per_sec=%g "
                "candidate_evaluations_per_sec=%g restarted_replicas=%llu",
                (unsigned long long)moves, (unsigned long long)evals, search_s,
                search_s > 0 ? moves / search_s : 0.0, search_s > 0 ? evals / search_s : 0.0,
                (unsigned long long)rs.restarted));
        out->score = res[0].score;
        out->conflicts = res[0].conflicts;
        out->replicas = replicas;
        out->solved = res[0].score == 0;
        out->verified = out->solved ? (fin_exact ? 1 : 0) : 0;
        out->best_replica = res[0].best_replica;
        out->moves = moves;
        out->candidate_evaluations = evals;
        out->restarted_replicas = rs.restarted;
        out->iterations = res[0].iters;
        out->initialization_seconds = init_s;
        out->search_seconds = search_s;
        out->time_to_solution_seconds = solve_s;
        if (best_out) std::memcpy(best_out, best.data(), best.size());
        if (out->solved && !out->verified) return fail(XW_ERR_INTERNAL, "score reached zero but exact verification failed");
        return XW_OK;
    })
}

}  // extern "C"
