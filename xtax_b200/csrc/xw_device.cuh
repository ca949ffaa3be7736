// xw_device.cuh -- device-side building blocks shared by the annealing and
// rescoring kernels: the Philox4x32-10 counter-based generator, the draw
// layout, the deterministic acceptance exponential and the job / replica
// record layouts in HBM.
#pragma once

#include <cstdint>

#include "xw_layout.h"

namespace xw {

// Philox4x32-10 (Salmon, Moraes, Dror, Shaw, SC'11): ten rounds of
// (hi0,lo0)=M0*c0, (hi1,lo1)=M1*c2, c'=(hi1^c1^k0, lo1, hi0^c3^k1, lo0),
// with the key bumped by the Weyl constants between rounds.
__device__ __forceinline__ uint4 philox4x32_10(uint4 c, uint32_t k0, uint32_t k1) {
#pragma unroll
    for (int r = 0; r < 10; ++r) {
        const uint32_t lo0 = 0xD2511F53u * c.x;
        const uint32_t hi0 = __umulhi(0xD2511F53u, c.x);
        const uint32_t lo1 = 0xCD9E8D57u * c.z;
        const uint32_t hi1 = __umulhi(0xCD9E8D57u, c.z);
        c = make_uint4(hi1 ^ c.y ^ k0, lo1, hi0 ^ c.w ^ k1, lo0);
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
    return c;
}

__device__ __forceinline__ uint32_t pick(uint4 v, int j) {
    return j == 0 ? v.x : j == 1 ? v.y : j == 2 ? v.z : v.w;
}

// Draw layout (identical in the oracle): word j of
// Philox(ctr = {slot, it_lo, it_hi, stream}, key).  slot 0 is the move-level
// block, slot 1 + 128*c + b is block b of candidate c; retries of a rejected
// index draw set slot bits 24..31 to the retry number.
__device__ __forceinline__ uint32_t cand_slot(int c, int b) {
    return 1u + 128u * (uint32_t)c + (uint32_t)b;
}

__device__ __forceinline__ uint4 draw_block(uint32_t slot, uint64_t it, uint32_t stream,
                                            uint32_t k0, uint32_t k1) {
    return philox4x32_10(make_uint4(slot, (uint32_t)it, (uint32_t)(it >> 32), stream), k0, k1);
}

// Lemire multiply-shift index in [0,count) from a 32-bit word; a word in the
// rejection zone (probability < count/2^32) is replaced by the same word of
// the retry counters.
__device__ __forceinline__ bool lemire_ok(uint32_t v, uint32_t count, uint32_t& out) {
    const uint64_t prod = (uint64_t)v * count;
    const uint32_t low = (uint32_t)prod;
    out = (uint32_t)(prod >> 32);
    return low >= count || low >= (0u - count) % count;
}

static __device__ __noinline__ uint32_t lemire_retry(uint32_t slot, uint64_t it, uint32_t stream,
                                              uint32_t k0, uint32_t k1, int j, uint32_t count) {
    uint32_t out = 0;
#pragma unroll 1
    for (uint32_t retry = 1; retry <= 255; ++retry) {
        const uint4 b = draw_block((slot & 0x00ffffffu) | (retry << 24), it, stream, k0, k1);
        const uint32_t v = pick(b, j);
        if (lemire_ok(v, count, out) || retry == 255) return out;
    }
    return out;
}

// The rare branch of an index draw (low word below count): the threshold
// test that needs an integer remainder, then retries.  Out of line so the
// common path of every index draw is a multiply and a compare.
static __device__ __noinline__ uint32_t lemire_edge(uint32_t v, uint32_t slot, uint64_t it, uint32_t stream,
                                             uint32_t k0, uint32_t k1, int j, uint32_t count) {
    uint32_t out;
    if (lemire_ok(v, count, out)) return out;
    return lemire_retry(slot, it, stream, k0, k1, j, count);
}

// Index in [0,count) from word v of (slot, j): Lemire's multiply-shift with
// the rejection handled by lemire_edge.
__device__ __forceinline__ uint32_t draw_index(uint32_t v, uint32_t count, uint32_t slot, uint64_t it,
                                               uint32_t stream, uint32_t k0, uint32_t k1, int j) {
    const uint64_t prod = (uint64_t)v * count;
    if ((uint32_t)prod >= count) return (uint32_t)(prod >> 32);
    return lemire_edge(v, slot, it, stream, k0, k1, j, count);
}

// exp(x) for x <= 0 by Cody-Waite reduction and a degree-14 Taylor
// polynomial, every step an explicitly rounded IEEE operation so that the
// CPU oracle (same operations, -ffp-contract=off) produces the same bits.
__device__ __forceinline__ double acceptance_exp(double x) {
    if (x >= 0.0) return 1.0;
    if (!(x > -40.0)) return (x > -745.0) ? 0x1p-60 : 0.0;
    const double k = rint(__dmul_rn(x, 0x1.71547652b82fep+0));
    double r = __fma_rn(-k, 0x1.62e42fee00000p-1, x);
    r = __fma_rn(-k, 0x1.a39ef35793c76p-33, r);
    double p = 0x1.93974a8c07c9dp-37;
    p = __fma_rn(p, r, 0x1.6124613a86d09p-33);
    p = __fma_rn(p, r, 0x1.1eed8eff8d898p-29);
    p = __fma_rn(p, r, 0x1.ae64567f544e4p-26);
    p = __fma_rn(p, r, 0x1.27e4fb7789f5cp-22);
    p = __fma_rn(p, r, 0x1.71de3a556c734p-19);
    p = __fma_rn(p, r, 0x1.a01a01a01a01ap-16);
    p = __fma_rn(p, r, 0x1.a01a01a01a01ap-13);
    p = __fma_rn(p, r, 0x1.6c16c16c16c17p-10);
    p = __fma_rn(p, r, 0x1.1111111111111p-7);
    p = __fma_rn(p, r, 0x1.5555555555555p-5);
    p = __fma_rn(p, r, 0x1.5555555555555p-3);
    p = __fma_rn(p, r, 0x1.0000000000000p-1);
    p = __fma_rn(p, r, 1.0);
    p = __fma_rn(p, r, 1.0);
    const double scale = __longlong_as_double((long long)(1023 + (int)k) << 52);
    return __dmul_rn(p, scale);
}

// Chunked launches: chunk c of a replica starts once chunk c-1 has released
// the replica's record.  Items are taken in chunk-major order by resident
// warps, so the chunk waited for is always running or done and the wait
// ends; how long it lasts is at most that chunk's own run time, which can be
// long when the queue runs ahead of a slow replica (a mixed batch, or
// replicas that finished early).  So the wait is bounded by elapsed device
// time (%globaltimer; kChunkWaitNs unless the launch sets its own limit),
// with an iteration cap behind it.  A chunk that gives up flags the replica
// (XW_ERR_CHUNK), runs nothing, and publishes the count with kChunkPoison
// set: the count is raised with an atomic maximum, so the predecessor that
// is still running cannot clear the mark when it finishes, and every later
// chunk of the replica sees it and skips too instead of running beside that
// predecessor on the same record.
constexpr uint64_t kChunkWaitNs = 30ull * 1000000000ull;
constexpr uint32_t kChunkSpinLimit = 1u << 28;
constexpr uint32_t kChunkPoison = 0x80000000u;

// The replica's chunk count once it reaches `want` (kChunkPoison set when a
// chunk before gave up), or 0 when the wait ran out.
static __device__ __noinline__ uint32_t wait_chunk(const uint32_t* flag, uint32_t want, uint64_t limit_ns) {
    uint32_t v = 0;
    uint64_t t0, t;
    if (limit_ns == 0) limit_ns = kChunkWaitNs;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t0));
#pragma unroll 1
    for (uint32_t spin = 0; spin < kChunkSpinLimit; ++spin) {
        asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(flag) : "memory");
        if (v >= want) return v;
        __nanosleep(256);
        asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
        if (t - t0 > limit_ns) return 0;
    }
    return 0;
}

// Every lane's record writes are made visible device-wide before lane 0
// publishes the chunk count (a release-ordered atomic maximum, so that a
// poisoned count stays poisoned).  `gm`: the lanes that own the replica.
__device__ __forceinline__ void release_chunk(uint32_t* flag, uint32_t value, int lane, unsigned gm = 0xffffffffu) {
    __threadfence();
    __syncwarp(gm);
    if (lane == 0) asm volatile("red.release.gpu.global.max.u32 [%0], %1;" ::"l"(flag), "r"(value) : "memory");
}

// One chunk of a chunked launch: chunk_begin waits for the replica's
// previous chunk and says whether this one runs (false: flag the replica,
// skip); chunk_end publishes this chunk's count, poisoned when it did not
// run.  Every lane of the replica's lane group `gm` calls both.  (The chunk
// body is called between them by the kernel itself: wrapping it in a lambda
// raised the lean kernel's spills from 40 to 412 bytes a thread and made the
// W(26,25) tempering batch 9% slower on B200.)
__device__ __forceinline__ bool chunk_begin(const uint32_t* done, uint32_t c, uint64_t limit_ns, uint32_t* err,
                                            int lane, unsigned gm) {
    bool ok = true;
    if (c > 0) {
        const uint32_t seen = wait_chunk(done, c, limit_ns);
        ok = __all_sync(gm, seen != 0 && !(seen & kChunkPoison));
    }
    __syncwarp(gm);
    if (!ok && lane == 0) atomicOr(err, XW_ERR_CHUNK);
    return ok;
}

__device__ __forceinline__ void chunk_end(uint32_t* done, uint32_t c, bool ran, int lane, unsigned gm) {
    release_chunk(done, ran ? c + 1 : (kChunkPoison | (c + 1)), lane, gm);
}

// Metropolis test u*2^-32 < exp(-delta/T), delta > 0.
__device__ __forceinline__ bool metropolis_accept(int64_t delta, double temperature, uint32_t u) {
    const double t = temperature > 1.0e-12 ? temperature : 1.0e-12;
    const double x = __ddiv_rn(-(double)delta, t);
    return __dmul_rn((double)u, 0x1p-32) < acceptance_exp(x);
}

}  // namespace xw
