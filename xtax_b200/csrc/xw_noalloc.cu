// xw_noalloc.cu -- annealing without any device allocation.
//
// For callers that cannot call cudaMalloc: a host whose device memory is
// owned by its own pool allocator (a framework's caching allocator, a
// plugin host with a fixed budget), code that must not add the implicit
// device synchronisation of cudaMalloc/cudaFree to a latency-sensitive
// loop.  xw_anneal_noalloc runs the same anneal kernel as the batch engine,
// with every scratch structure (the job record, the replica records that
// hold each replica's working W, best W and minority lists, the work list
// and the per-round work counters) in one file-scope device array of
// XW_NOALLOC_SCRATCH_BYTES.  The caller passes the start states and
// receives the best states and scores in its own device buffers.
//
// Costs and rules:
//  * every GPU that loads this library holds the array
//    (XW_NOALLOC_SCRATCH_BYTES, 4 MiB) until the process exits;
//  * the first call on a device, with that device current, resolves the
//    array's device address with cudaGetSymbolAddress and raises the
//    kernel's shared-memory limit; make that first call before any stream
//    capture;
//  * all calls share the array and each rewrites it from the call's inputs,
//    so calls whose work overlaps on the GPU (different streams, or other
//    threads) race; serialise them.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>

#include "../../include/xw.h"
#include "xw_device.cuh"
#include "xw_host_internal.h"
#include "xw_kernels.h"

namespace xw {

namespace {

static __device__ __align__(256) unsigned char g_noalloc_scratch[XW_NOALLOC_SCRATCH_BYTES];

constexpr int kMaxDevices = 64;
std::mutex g_setup_mu;
unsigned char* g_scratch_ptr[kMaxDevices] = {};

struct NoallocLayout {
    size_t off_job, off_counters, off_rec_off, off_items, off_ladder, off_records, record_bytes, total;
    int max_rounds;
};

size_t align256(size_t v) { return (v + 255) & ~size_t(255); }

NoallocLayout noalloc_layout(int n, int m, int replicas, int rounds) {
    NoallocLayout L;
    L.max_rounds = rounds;
    L.off_job = 0;
    L.off_counters = align256(sizeof(XwJob));
    L.off_rec_off = align256(L.off_counters + sizeof(uint32_t) * (size_t)rounds);
    L.off_items = align256(L.off_rec_off + sizeof(uint64_t) * (size_t)replicas);
    L.off_ladder = align256(L.off_items + sizeof(uint32_t) * (size_t)replicas);
    L.off_records = align256(L.off_ladder + sizeof(double) * (size_t)replicas);
    const size_t nn = xw_pad16((uint32_t)(n * n));
    L.record_bytes = (128 + 2 * nn + xw_pad16((uint32_t)(n * m)) + 127) & ~size_t(127);
    L.total = L.off_records + L.record_bytes * (size_t)replicas;
    return L;
}

// Fills the job record, the ladder and every replica record from the
// caller's start states.  One block; thread 0 writes the job and ladder.
__global__ void noalloc_init_kernel(unsigned char* scratch, XwJob job, NoallocLayout L, const int8_t* starts,
                                    double bottom, double ratio, uint64_t obj_sq, uint64_t obj_par,
                                    int forced_objective) {
    XwJob* J = reinterpret_cast<XwJob*>(scratch + L.off_job);
    double* ladder = reinterpret_cast<double*>(scratch + L.off_ladder);
    uint64_t* rec_off = reinterpret_cast<uint64_t*>(scratch + L.off_rec_off);
    uint32_t* items = reinterpret_cast<uint32_t*>(scratch + L.off_items);
    const int R = job.replicas, n = job.n;
    if (threadIdx.x == 0) {
        *J = job;
        double t = bottom;
        for (int r = 0; r < R; ++r) {  // geometric ladder, same products as the host
            ladder[r] = t;
            t = __dmul_rn(t, ratio);
        }
    }
    __syncthreads();
    for (int r = threadIdx.x; r < R; r += blockDim.x) {
        const size_t off = L.off_records + (size_t)r * L.record_bytes;
        rec_off[r] = off;
        items[r] = (uint32_t)r;
        RepHeader* H = reinterpret_cast<RepHeader*>(scratch + off);
        memset(H, 0, sizeof(RepHeader));
        // no score yet (the kernel computes it from W when it loads the
        // replica): a replica the kernel refuses cannot read as solved
        H->score = H->best_score = INT32_MAX;
        H->conflicts = H->best_conflicts = INT32_MAX;
        H->job = 0;
        H->stream = (uint32_t)r;
        H->temperature = ladder[r];
        H->reheat_temperature = ladder[r];
        H->rung = r;
        if (forced_objective >= 0) {
            H->obj_kind = forced_objective;
        } else {
            // the reference's per-replica objective mix (xweigh_cuda.cu:969-981)
            const uint32_t h = (uint32_t)r * 0x9e3779b9u + 0x85ebca6bu;
            H->obj_kind = (uint64_t)h < obj_sq ? 1 : (uint64_t)h < obj_par ? 2 : 0;
        }
        const int8_t* src = starts + (size_t)r * n * n;
        int8_t* w = reinterpret_cast<int8_t*>(scratch + off + job.off_w);
        int8_t* b = reinterpret_cast<int8_t*>(scratch + off + job.off_best);
        for (int i = 0; i < n * n; ++i) {
            w[i] = src[i];
            b[i] = src[i];
        }
    }
}

// Copies each replica's best W and {best score, best conflicts, score,
// moves} into the caller's buffers.  A replica the kernel flagged (a start
// row whose weight is not w, a failed self-check) reports best score -1 and
// best conflicts -err instead, so that it cannot read as solved.
__global__ void noalloc_output_kernel(const unsigned char* scratch, NoallocLayout L, int n, int R, int8_t* best,
                                      int64_t* stats, uint32_t off_best) {
    const int r = blockIdx.x;
    if (r >= R) return;
    const size_t off = L.off_records + (size_t)r * L.record_bytes;
    const RepHeader* H = reinterpret_cast<const RepHeader*>(scratch + off);
    const int8_t* src = reinterpret_cast<const int8_t*>(scratch + off + off_best);
    for (int i = threadIdx.x; i < n * n; i += blockDim.x) best[(size_t)r * n * n + i] = src[i];
    if (threadIdx.x == 0) {
        const bool bad = H->err != 0;
        stats[4 * r + 0] = bad ? -1 : H->best_score;
        stats[4 * r + 1] = bad ? -(int64_t)H->err : H->best_conflicts;
        stats[4 * r + 2] = bad ? -1 : H->score;
        stats[4 * r + 3] = (int64_t)H->moves;
    }
}

int32_t nfail(int32_t code, const std::string& msg) {
    set_last_error(msg);
    return code;
}

uint64_t coin(double p) {
    if (!(p > 0.0)) return 0;
    if (p >= 1.0) return 4294967296ull;
    return (uint64_t)std::ceil(p * 4294967296.0);
}
}  // namespace
}  // namespace xw

using namespace xw;

extern "C" int32_t xw_anneal_noalloc(int32_t n, int32_t w, const xw_params* p, int32_t replicas, uint64_t iters,
                                     const int8_t* starts, int8_t* best, int64_t* stats, void* stream_handle) {
    if (!p || !starts || !best || !stats) return nfail(XW_ERR_INVALID, "xw_anneal_noalloc: null argument");
    {
        const std::string e = validate(n, w, *p);
        if (!e.empty()) return nfail(XW_ERR_INVALID, e);
    }
    if (n > XW_MAX_ORDER_SHARED)
        return nfail(XW_ERR_CAPACITY, "xw_anneal_noalloc: order above the shared-memory kernel's maximum of 256");
    if (replicas < 1) return nfail(XW_ERR_INVALID, "xw_anneal_noalloc: replica count must be positive");
    if (iters < 1) return nfail(XW_ERR_INVALID, "xw_anneal_noalloc: iterations must be positive");
    if (!(p->t_init > 0.0))
        return nfail(XW_ERR_INVALID, "xw_anneal_noalloc: t_init must be positive (no host calibration here)");
    if (p->tempering && replicas > XW_MAX_RUNGS)
        return nfail(XW_ERR_INVALID, "xw_anneal_noalloc: a tempering ladder has at most 256 rungs");
    const int m = n - w < w ? n - w : w;
    const uint64_t per = p->tempering ? (uint64_t)p->exchange_interval : (uint64_t)p->moves_per_launch;
    const uint64_t rounds64 = (iters + per - 1) / per;
    if (rounds64 > 4096) return nfail(XW_ERR_CAPACITY, "xw_anneal_noalloc: more than 4096 launch rounds");
    const int rounds = (int)rounds64;
    const NoallocLayout L = noalloc_layout(n, m, replicas, rounds);
    if (L.total > XW_NOALLOC_SCRATCH_BYTES) {
        char msg[256];
        std::snprintf(msg, sizeof msg,
                      "xw_anneal_noalloc: %d replicas of W(%d,%d) need %zu bytes of scratch; the static "
                      "scratch holds %d bytes",
                      replicas, n, w, L.total, XW_NOALLOC_SCRATCH_BYTES);
        return nfail(XW_ERR_CAPACITY, msg);
    }
    cudaStream_t stream = static_cast<cudaStream_t>(stream_handle);
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return nfail(XW_ERR_CUDA, std::string("cudaGetDevice failed: ") + cudaGetErrorString(e));
    if (dev < 0 || dev >= kMaxDevices) return nfail(XW_ERR_INVALID, "xw_anneal_noalloc: device ordinal too large");

    const bool job_general = needs_general_kernel(*p);
    const int opl = anneal_opl(n);
    const uint32_t slot = anneal_slot_bytes(n, m, opl);
    const int wpb = p->warps_per_block > 0 ? p->warps_per_block : 4;
    const void* fn = anneal_kernel_fn(opl, job_general);
    unsigned char* scratch = nullptr;
    {
        std::lock_guard<std::mutex> lock(g_setup_mu);
        if (!g_scratch_ptr[dev]) {
            // set-up, once per device: the array's device address (its host
            // name is only a stand-in), then the kernel's shared-memory limit
            void* ptr = nullptr;
            e = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
            if (e != cudaSuccess)
                return nfail(XW_ERR_CUDA, std::string("cudaGetSymbolAddress failed: ") + cudaGetErrorString(e));
            g_scratch_ptr[dev] = static_cast<unsigned char*>(ptr);
        }
        scratch = g_scratch_ptr[dev];
    }
    // the kernel's shared-memory limit goes to the device's opt-in maximum,
    // as every other launcher of it sets it, so that no call lowers the
    // limit a batch or server launch of a larger order relies on
    int optin = 0;
    e = cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    if (e == cudaSuccess && (size_t)wpb * slot > (size_t)optin)
        return nfail(XW_ERR_CAPACITY, "xw_anneal_noalloc: the replicas' shared memory exceeds the device's limit");
    cudaFuncAttributes attr{};
    if (e == cudaSuccess) e = cudaFuncGetAttributes(&attr, fn);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, optin - (int)attr.sharedSizeBytes);
    if (e != cudaSuccess) return nfail(XW_ERR_CAPACITY, std::string("cudaFuncSetAttribute failed: ") + cudaGetErrorString(e));
    int per_sm = 0, sms = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, 32 * wpb, (size_t)wpb * slot);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess || per_sm < 1)
        return nfail(XW_ERR_CAPACITY, "xw_anneal_noalloc: the anneal kernel does not fit on this device");
    const int blocks = std::max(1, std::min((replicas + wpb - 1) / wpb, per_sm * sms));

    // the job record, as the batch engine builds it
    XwJob job;
    std::memset(&job, 0, sizeof job);
    job.n = n;
    job.w = w;
    job.m = m;
    job.sparse = w <= n - w;
    job.tempering = p->tempering != 0;
    job.move_set = p->move_set;
    job.candidate_samples = p->candidate_samples;
    job.target_samples = p->target_samples;
    job.moves_per_cool = p->moves_per_cool;
    job.stuck_threshold = p->stuck_threshold;
    job.objective = p->objective;
    job.general = needs_general_kernel(*p) ? 1 : 0;
    job.replicas = replicas;
    const uint32_t base = (uint32_t)p->seed;
    const uint64_t key = ((uint64_t)base << 32) ^ p->seed ^ 0xd1b54a32d192ed03ull;
    job.key0 = (uint32_t)key;
    job.key1 = (uint32_t)(key >> 32);
    const uint32_t nn = xw_pad16((uint32_t)(n * n));
    job.off_w = 128;
    job.off_best = 128 + nn;
    job.off_mino = 128 + 2 * nn;
    job.record_bytes = (uint32_t)L.record_bytes;
    job.thr_greedy = coin(p->greedy_fraction);
    job.thr_target = coin(p->target_fraction);
    job.thr_double = p->move_set == 0 ? coin(p->double_sign_fraction) : 0;
    job.thr_sign = coin(p->sign_fraction);
    job.thr_swsign = coin(p->switch_sign_fraction);
    job.t_min = p->t_min;
    job.cooling = p->cooling;
    job.reheat = p->reheat;
    job.ladder_off = 0;
    const double bottom = std::min(p->t_min, p->t_init);
    const double ratio = replicas > 1 ? std::pow(p->t_init / std::max(bottom, 1.0e-12), 1.0 / (double)(replicas - 1))
                                      : 1.0;
    // objective-mix thresholds on the hash: choice < f  <=>  h < f*2^32
    const double f1 = p->squared_objective_fraction, f2 = p->squared_objective_fraction + p->parity_objective_fraction;
    const uint64_t obj_sq = coin(f1), obj_par = coin(f2);

    noalloc_init_kernel<<<1, 256, 0, stream>>>(scratch, job, L, starts, bottom, ratio, obj_sq, obj_par, p->objective);
    e = cudaGetLastError();
    if (e != cudaSuccess) return nfail(XW_ERR_CUDA, std::string("noalloc init launch failed: ") + cudaGetErrorString(e));
    // work counters start at zero every call
    e = cudaMemsetAsync(scratch + L.off_counters, 0, sizeof(uint32_t) * (size_t)rounds, stream);
    if (e != cudaSuccess) return nfail(XW_ERR_CUDA, std::string("cudaMemsetAsync failed: ") + cudaGetErrorString(e));
    uint64_t left = iters;
    for (int k = 0; k < rounds; ++k) {
        AnnealArgs a;
        a.jobs = reinterpret_cast<XwJob*>(scratch + L.off_job);
        a.arena = scratch;
        a.rec_off = reinterpret_cast<const uint64_t*>(scratch + L.off_rec_off);
        a.items = reinterpret_cast<const uint32_t*>(scratch + L.off_items);
        a.n_items = (uint32_t)replicas;
        a.slot_bytes = slot;
        a.counter = reinterpret_cast<uint32_t*>(scratch + L.off_counters) + k;
        a.iters = std::min(left, per);
        a.stop_on_solve = p->stop_on_solve;
        a.one_zero = 0;
        left -= a.iters;
        e = launch_anneal(a, opl, job_general, wpb, blocks, stream);
        if (e != cudaSuccess) return nfail(XW_ERR_CUDA, std::string("anneal launch failed: ") + cudaGetErrorString(e));
        if (job.tempering) {
            e = launch_exchange(a.jobs, 1, scratch, a.rec_off, reinterpret_cast<const double*>(scratch + L.off_ladder),
                                p->stop_on_solve, stream);
            if (e != cudaSuccess)
                return nfail(XW_ERR_CUDA, std::string("exchange launch failed: ") + cudaGetErrorString(e));
        }
    }
    noalloc_output_kernel<<<replicas, 128, 0, stream>>>(scratch, L, n, replicas, best, stats, job.off_best);
    e = cudaGetLastError();
    if (e != cudaSuccess) return nfail(XW_ERR_CUDA, std::string("noalloc output launch failed: ") + cudaGetErrorString(e));
    return XW_OK;
}
