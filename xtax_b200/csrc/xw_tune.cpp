// xw_tune.cpp -- launch-shape autotuner for the anneal kernel.
//
// The tunable is the number of replica warps per CTA (1..16): it sets how
// many warps share an SM's shared memory and how the persistent scheduler's
// CTAs tile the SMs.  xw_autotune() (C ABI) times short trial runs of a
// synthetic population for each candidate shape and records the fastest per
// (rows per lane, shared-bytes-per-warp class); tuned_warps_per_block()
// reads that table, which persists in a small text cache file (XW_TUNE_CACHE,
// default ~/.cache/xw_tune.txt).  Without an entry 4 warps per CTA are used.
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
    int opl;
    uint32_t slot_lo, slot_hi;  // slot-byte class [lo, hi)
    int wpb;
};

std::mutex g_mu;
std::vector<Entry> g_table;
bool g_loaded = false;

std::string cache_path() {
    if (const char* p = std::getenv("XW_TUNE_CACHE")) return p;
    const char* home = std::getenv("HOME");
    return std::string(home ? home : "/tmp") + "/.cache/xw_tune.txt";
}

void load_locked() {
    if (g_loaded) return;
    g_loaded = true;
    FILE* f = std::fopen(cache_path().c_str(), "r");
    if (!f) return;
    Entry e;
    while (std::fscanf(f, "%d %u %u %d", &e.opl, &e.slot_lo, &e.slot_hi, &e.wpb) == 4)
        if (e.wpb >= 1 && e.wpb <= 16) g_table.push_back(e);
    std::fclose(f);
}

void save_locked() {
    const std::filesystem::path path(cache_path());
    std::error_code ec;
    if (path.has_parent_path()) std::filesystem::create_directories(path.parent_path(), ec);
    FILE* f = std::fopen(path.c_str(), "w");
    if (!f) return;
    for (const Entry& e : g_table) std::fprintf(f, "%d %u %u %d\n", e.opl, e.slot_lo, e.slot_hi, e.wpb);
    std::fclose(f);
}

// slot-byte classes are powers of two
void slot_class(uint32_t slot, uint32_t& lo, uint32_t& hi) {
    lo = 256;
    while (lo * 2 <= slot) lo *= 2;
    hi = lo * 2;
}

}  // namespace

int tuned_warps_per_block(int opl, uint32_t slot_bytes, int device) {
    (void)device;
    if (const char* env = std::getenv("XW_WARPS_PER_BLOCK")) {
        const int v = std::atoi(env);
        if (v >= 1 && v <= 16) return v;
    }
    std::lock_guard<std::mutex> lock(g_mu);
    load_locked();
    for (const Entry& e : g_table)
        if (e.opl == opl && slot_bytes >= e.slot_lo && slot_bytes < e.slot_hi) return e.wpb;
    return 4;
}

void record_tuned(int opl, uint32_t slot_bytes, int wpb) {
    std::lock_guard<std::mutex> lock(g_mu);
    load_locked();
    uint32_t lo, hi;
    slot_class(slot_bytes, lo, hi);
    for (Entry& e : g_table)
        if (e.opl == opl && e.slot_lo == lo) {
            e.wpb = wpb;
            save_locked();
            return;
        }
    g_table.push_back(Entry{opl, lo, hi, wpb});
    save_locked();
}

}  // namespace xw
