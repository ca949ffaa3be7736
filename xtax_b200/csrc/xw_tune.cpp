// xw_tune.cpp -- launch-shape autotuner for the anneal kernel.
//
// The shape of a launch class has two tunables: replicas per warp (1, or 2
// for orders up to 16, where a half-warp covers a replica's rows) and warps
// per CTA (1..16), which sets how many warps share an SM's shared memory and
// how the persistent scheduler's CTAs tile the SMs.  xw_autotune() (C ABI)
// times short trial runs of each class of a batch at every shape that fits
// and records the fastest per (class kind, shared-bytes-per-slot class);
// classes of at most one replica per SM also try the latency mode (a CTA of
// 2..16 warps per replica speculating that many iterations at a time);
// tuned_shape() reads that table, which persists in a small text cache file
// (XW_TUNE_CACHE, default ~/.cache/xw_tune.txt).  Without an entry: 4 warps
// per CTA, and two replicas per warp for the orders up to 16.
#include <cuda_runtime.h>

#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <filesystem>
#include <mutex>
#include <string>
#include <vector>

#include "xw_host_internal.h"

namespace xw {

namespace {

struct Entry {
    int kind;
    uint32_t slot_lo, slot_hi;  // slot-byte class [lo, hi)
    int wpb;
    int rpw;
};

std::mutex g_mu;
std::vector<Entry> g_table;
bool g_loaded = false;

std::string cache_path() {
    if (const char* p = std::getenv("XW_TUNE_CACHE")) return p;
    const char* home = std::getenv("HOME");
    return std::string(home ? home : "/tmp") + "/.cache/xw_tune.txt";
}

// lines "kind slot_lo slot_hi wpb [rpw]"; a missing rpw reads as 1
void load_locked() {
    if (g_loaded) return;
    g_loaded = true;
    FILE* f = std::fopen(cache_path().c_str(), "r");
    if (!f) return;
    char line[256];
    while (std::fgets(line, sizeof line, f)) {
        Entry e{};
        e.rpw = 1;
        const int got = std::sscanf(line, "%d %u %u %d %d", &e.kind, &e.slot_lo, &e.slot_hi, &e.wpb, &e.rpw);
        if (got < 4 || e.wpb < 1 || e.wpb > 16 || e.rpw < 1 || e.rpw > 2) continue;
        if (e.rpw == 2 && e.kind != kTunePairKind) e.rpw = 1;
        g_table.push_back(e);
    }
    std::fclose(f);
}

void save_locked() {
    const std::filesystem::path path(cache_path());
    std::error_code ec;
    if (path.has_parent_path()) std::filesystem::create_directories(path.parent_path(), ec);
    FILE* f = std::fopen(path.c_str(), "w");
    if (!f) return;
    for (const Entry& e : g_table)
        std::fprintf(f, "%d %u %u %d %d\n", e.kind, e.slot_lo, e.slot_hi, e.wpb, e.rpw);
    std::fclose(f);
}

// slot-byte classes are powers of two
void slot_class(uint32_t slot, uint32_t& lo, uint32_t& hi) {
    lo = 256;
    while (lo * 2 <= slot) lo *= 2;
    hi = lo * 2;
}

int env_int(const char* name, int lo, int hi) {
    const char* env = std::getenv(name);
    if (!env || !*env) return 0;
    const int v = std::atoi(env);
    return v >= lo && v <= hi ? v : 0;
}

}  // namespace

int tune_kind(int n, int candidate_samples) {
    if (n <= 16 && candidate_samples <= 16) return kTunePairKind;
    return anneal_opl(n);
}

TunedShape tuned_shape(int kind, uint32_t slot_bytes, int device) {
    (void)device;
    // untuned: one replica per warp for the orders up to 16 too (a full
    // B200, 4096 replicas of W(14,13): 0.863 G iterations/s at one replica
    // per warp against 0.797 G at two); the autotuner may pick two
    TunedShape s{4, 1};
    {
        std::lock_guard<std::mutex> lock(g_mu);
        load_locked();
        for (const Entry& e : g_table)
            if (e.kind == kind && slot_bytes >= e.slot_lo && slot_bytes < e.slot_hi) {
                s = TunedShape{e.wpb, e.rpw};
                break;
            }
    }
    if (const int v = env_int("XW_WARPS_PER_BLOCK", 1, 16)) s.wpb = v;
    if (const int v = env_int("XW_REPLICAS_PER_WARP", 1, 2)) s.rpw = v;
    if (kind != kTunePairKind) s.rpw = 1;
    return s;
}

int tuned_warps_per_replica(uint32_t slot_bytes, int device) {
    (void)device;
    // untuned default: 64 warps, a cluster of four CTAs (W(12,11) single
    // searches on B200, per search: 1.81 / 3.17 M moves/s at 8 / 16 warps
    // on one SM, 5.02 M at 32 on two); the host falls back to 32 or 16
    // where a class has more replicas than a quarter or half of the SMs
    int k = 64;
    {
        std::lock_guard<std::mutex> lock(g_mu);
        load_locked();
        for (const Entry& e : g_table)
            if (e.kind == kTuneLatencyKind && slot_bytes >= e.slot_lo && slot_bytes < e.slot_hi) {
                k = e.wpb;
                break;
            }
    }
    if (const int v = env_int("XW_WARPS_PER_REPLICA", 1, 64)) k = v;
    return k;
}

int tuned_warps_per_block(int opl, uint32_t slot_bytes, int device) {
    return tuned_shape(opl, slot_bytes, device).wpb;
}

void record_tuned(int kind, uint32_t slot_bytes, int wpb, int rpw) {
    std::lock_guard<std::mutex> lock(g_mu);
    load_locked();
    uint32_t lo, hi;
    slot_class(slot_bytes, lo, hi);
    for (Entry& e : g_table)
        if (e.kind == kind && e.slot_lo == lo) {
            e.wpb = wpb;
            e.rpw = rpw;
            save_locked();
            return;
        }
    g_table.push_back(Entry{kind, lo, hi, wpb, rpw});
    save_locked();
}

}  // namespace xw
