// xw_cli.cpp -- the command lines of libxw: xweigh_cuda, a drop-in for
// src/xweigh_cuda_main.cpp of flinty-mathematics/xtax, and (built with
// XW_CLI_CPU) xweigh, a drop-in for src/xweigh_main.cpp, the CPU annealer.
//
// Same positional arguments, options, defaults, validation messages,
// existence checks (impossibility_reason), Sylvester short-circuit, output
// lines, CSV writes and exit codes.  The parser is this file's own; where
// the reference's parser library reports an argument error it prints the
// same message and exits with the same code (105 validation, 106 missing
// argument, 109 unexpected argument), followed by
// "Run with --help for more information.".
#include <algorithm>
#include <atomic>
#include <cctype>
#include <chrono>
#include <cerrno>
#include <climits>
#include <cmath>
#include <csignal>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <functional>
#include <map>
#include <random>
#include <string>
#include <sys/stat.h>
#include <unistd.h>
#include <vector>

#include "../../include/xw.h"

namespace {

std::atomic<bool> g_interrupted{false};
std::atomic<bool> g_stop_once{false};
const char k_interrupt_msg[] = "\n[interrupt received, finishing and writing the best result so far...]\n";

// stop_signal.hpp:52-89: the first Ctrl-C sets the stop flag and prints one
// acknowledgement; later ones are swallowed so the best result is written
void on_interrupt(int) {
    if (!g_stop_once.exchange(true)) {
        g_interrupted.store(true);
        xw_request_stop();
        const ssize_t r = write(STDERR_FILENO, k_interrupt_msg, sizeof(k_interrupt_msg) - 1);
        (void)r;
    }
}

struct ArgError {
    int code;
    std::string message;
};

bool parse_int(const std::string& s, long long& out) {
    if (s.empty()) return false;
    errno = 0;
    char* end = nullptr;
    const long long v = std::strtoll(s.c_str(), &end, 10);
    if (errno != 0 || *end != '\0') return false;
    out = v;
    return true;
}

bool parse_uint64(const std::string& s, uint64_t& out) {
    if (s.empty() || s[0] == '-') return false;
    errno = 0;
    char* end = nullptr;
    const unsigned long long v = std::strtoull(s.c_str(), &end, 10);
    if (errno != 0 || *end != '\0') return false;
    out = v;
    return true;
}

bool parse_double(const std::string& s, double& out) {
    if (s.empty()) return false;
    errno = 0;
    char* end = nullptr;
    const double v = std::strtod(s.c_str(), &end);
    if (errno != 0 || *end != '\0') return false;
    out = v;
    return true;
}

struct Option {
    std::vector<std::string> names;
    std::string help;
    std::function<void(const std::string&)> set;
    bool flag = false;   // takes no value (set is called with "")
};

bool file_exists(const std::string& p) {
    struct stat st;
    return stat(p.c_str(), &st) == 0 && S_ISREG(st.st_mode);
}

bool is_power_of_two(int v) { return v > 0 && (v & (v - 1)) == 0; }

void print_matrix(const std::vector<int8_t>& W, int n) {
    for (int r = 0; r < n; ++r) {
        for (int c = 0; c < n; ++c) {
            std::printf("%d", (int)W[(size_t)c * n + r]);
            if (c + 1 < n) std::putchar(',');
        }
        std::putchar('\n');
    }
}

// finish, xweigh_cuda_main.cpp:119-146
bool finish(const std::vector<int8_t>& W, int n, int w, const std::string& output) {
    const int flags = xw_verify(n, w, W.data());
    int64_t st[4];
    xw_score(n, w, W.data(), st);
    if (!(flags & 1)) {
        std::fprintf(stderr, "Error: internal support invariant failed\n");
        return false;
    }
    const bool solved = st[0] == 0;
    if (solved && !(flags & 2)) {
        std::fprintf(stderr, "Error: score reached zero but exact verification failed\n");
        return false;
    }
    std::printf("Final best score: %lld conflicts=%lld\n", (long long)st[0], (long long)st[1]);
    if (solved)
        std::printf("Found W(%d,%d); exact verification passed\n", n, w);
    else
        std::printf("No weighing matrix found; wrote the best fixed-weight candidate to %s\n", output.c_str());
    if (g_interrupted.load()) std::printf("[interrupted] best candidate written before exit\n");
    if (n <= 20) {
        std::printf("W:\n");
        print_matrix(W, n);
    }
    return true;
}

// valid_params, xweigh_cuda_main.cpp:54-117
std::string valid_params(const xw_params& p) {
    if (p.device < 0) return "--device must be nonnegative";
    if (p.replicas < 0) return "--replicas must be nonnegative";
    if (p.moves_per_launch < 1) return "--moves-per-launch must be positive";
    if (p.max_seconds < 0.0) return "--max-seconds must be nonnegative";
    if (p.save_interval < 0.0) return "--save-interval must be nonnegative";
    if (p.sign_fraction < 0.0 || p.sign_fraction > 1.0) return "--sign-fraction must be in [0, 1]";
    if (p.double_sign_fraction < 0.0 || p.double_sign_fraction > 1.0) return "--double-sign-fraction must be in [0, 1]";
    if (p.switch_sign_fraction < 0.0 || p.switch_sign_fraction > 1.0) return "--switch-sign-fraction must be in [0, 1]";
    if (p.squared_objective_fraction < 0.0 || p.squared_objective_fraction > 1.0)
        return "--squared-objective-fraction must be in [0, 1]";
    if (p.parity_objective_fraction < 0.0 || p.parity_objective_fraction > 1.0)
        return "--parity-objective-fraction must be in [0, 1]";
    if (p.squared_objective_fraction + p.parity_objective_fraction > 1.0)
        return "alternate objective fractions must sum to at most 1";
    if (p.greedy_fraction < 0.0 || p.greedy_fraction > 1.0) return "--greedy-fraction must be in [0, 1]";
    if (p.target_fraction < 0.0 || p.target_fraction > 1.0) return "--target-fraction must be in [0, 1]";
    if (p.candidate_samples < 1 || p.candidate_samples > XW_MAX_CANDIDATE_SAMPLES)
        return "--candidate-samples must be in [1, " + std::to_string(XW_MAX_CANDIDATE_SAMPLES) + "]";
    if (p.target_samples < 1 || p.target_samples > XW_MAX_TARGET_SAMPLES)
        return "--target-samples must be in [1, " + std::to_string(XW_MAX_TARGET_SAMPLES) + "]";
    if (p.t_init < 0.0) return "--t-init must be nonnegative";
    if (p.t_min <= 0.0) return "--t-min must be positive";
    if (p.cooling <= 0.0 || p.cooling >= 1.0) return "--cooling must be in (0, 1)";
    if (p.moves_per_cool < 1) return "--moves-per-cool must be positive";
    if (p.stuck_threshold < 1) return "--stuck-threshold must be positive";
    if (p.reheat <= 0.0) return "--reheat must be positive";
    if (p.restart_interval < 0.0) return "--restart-interval must be nonnegative";
    if (p.restart_fraction <= 0.0 || p.restart_fraction > 1.0) return "--restart-fraction must be in (0, 1]";
    if (p.restart_kick_min < 0) return "--restart-kick-min must be nonnegative";
    if (p.restart_kick_max < p.restart_kick_min) return "--restart-kick-max must be at least --restart-kick-min";
    if (p.exchange_interval < 1) return "--exchange-interval must be positive";
    if (p.objective < -1 || p.objective > 2) return "--objective must be -1, 0, 1 or 2";
    if (p.move_set < 0 || p.move_set > 1) return "--move-set must be 0 or 1";
    if (p.start_kind < 0 || p.start_kind > 1) return "--start-kind must be 0 or 1";
    return {};
}

struct CliState {
    std::string output = "best_W.csv";
};

// The shared parser: options by name (--name value, --name=value, flags),
// then the positionals n and w.  False after printing --help.
bool parse_args(int argc, char** argv, std::vector<Option>& opts, const char* title, long long& order,
                long long& weight) {
    std::vector<std::string> positional;
    bool have_n = false, have_w = false;
    std::map<std::string, Option*> by_name;
    for (auto& o : opts)
        for (auto& nm : o.names) by_name[nm] = &o;

    std::vector<std::string> extras;
    for (int i = 1; i < argc; ++i) {
        std::string a = argv[i];
        if (a == "-h" || a == "--help") {
            std::printf("%s\nUsage: %s [OPTIONS] n w\n\n"
                        "Positionals:\n  n INT:INT in [1 - 32767] REQUIRED\n                              Matrix order n\n"
                        "  w INT:INT in [1 - 32767] REQUIRED\n                              Matrix weight w\n\nOptions:\n"
                        "  -h,--help                   Print this help message and exit\n",
                        title, argv[0]);
            for (auto& o : opts) {
                std::string names;
                for (auto& nm : o.names) names += (names.empty() ? "" : ",") + nm;
                std::printf("  %-27s %s\n", names.c_str(), o.help.c_str());
            }
            return false;
        }
        if (a.size() > 1 && a[0] == '-' && !(a.size() > 1 && (std::isdigit((unsigned char)a[1]) || a[1] == '.'))) {
            std::string name = a, value;
            bool inline_value = false;
            const size_t eq = a.find('=');
            if (a.rfind("--", 0) == 0 && eq != std::string::npos) {
                name = a.substr(0, eq);
                value = a.substr(eq + 1);
                inline_value = true;
            }
            auto it = by_name.find(name);
            if (it == by_name.end()) {
                extras.push_back(a);
                continue;
            }
            if (it->second->flag) {
                if (inline_value) throw ArgError{107, name + ": flag does not take a value"};
            } else if (!inline_value) {
                if (i + 1 >= argc) throw ArgError{106, name + " requires 1 argument(s) but received 0"};
                value = argv[++i];
            }
            it->second->set(value);
            continue;
        }
        if (positional.size() < 2) positional.push_back(a);
        else extras.push_back(a);
    }
    // positionals n then w, each checked against CLI::Range(1, MAX_ORDER)
    for (size_t k = 0; k < positional.size(); ++k) {
        const std::string& v = positional[k];
        long long x;
        const char* nm = k == 0 ? "n" : "w";
        if (!parse_int(v, x) || x < 1 || x > 32767)
            throw ArgError{105, std::string(nm) + ": Value " + v + " not in range [1 - 32767]"};
        (k == 0 ? order : weight) = x;
        (k == 0 ? have_n : have_w) = true;
    }
    if (!extras.empty()) {
        // reported last-seen first
        std::string msg = extras.size() == 1 ? "The following argument was not expected:"
                                             : "The following arguments were not expected:";
        for (auto it = extras.rbegin(); it != extras.rend(); ++it) msg += " " + *it;
        throw ArgError{109, msg};
    }
    if (!have_n) throw ArgError{106, "n is required"};
    if (!have_w) throw ArgError{106, "w is required"};
    return true;

}



void log_line(const char* line, void*) {
    std::printf("%s\n", line);
    std::fflush(stdout);
}

void checkpoint(const int8_t* best, int32_t n, void* user) {
    const CliState* st = static_cast<const CliState*>(user);
    if (xw_write_csv(st->output.c_str(), n, best) != XW_OK)
        std::fprintf(stderr, "Warning: %s\n", xw_last_error());
}

[[maybe_unused]] int run(int argc, char** argv) {
    xw_params p;
    xw_params_default(&p);
    CliState state;
    std::string start_file;
    long long order = 0, weight = 0;

    std::vector<Option> opts;
    auto add = [&](std::vector<std::string> names, std::string help, std::function<void(const std::string&)> set) {
        opts.push_back(Option{std::move(names), std::move(help), std::move(set), false});
    };
    auto conv_err = [](const std::string& name, const std::string& v) {
        return ArgError{107, name + ": Value " + v + " could not be converted"};
    };
    auto int_opt = [&](const std::string& name, int32_t* dst) {
        return [=](const std::string& v) {
            long long x;
            if (!parse_int(v, x) || x < INT32_MIN || x > INT32_MAX) throw conv_err(name, v);
            *dst = (int32_t)x;
        };
    };
    auto dbl_opt = [&](const std::string& name, double* dst) {
        return [=](const std::string& v) {
            double x;
            if (!parse_double(v, x)) throw conv_err(name, v);
            *dst = x;
        };
    };
    auto u64_opt = [&](const std::string& name, uint64_t* dst) {
        return [=](const std::string& v) {
            uint64_t x;
            if (!parse_uint64(v, x)) throw conv_err(name, v);
            *dst = x;
        };
    };

    // xweigh_cuda_main.cpp:159-231
    add({"-o", "--out"}, "Output CSV for the best matrix", [&](const std::string& v) { state.output = v; });
    add({"--start"}, "Start every replica from a complete fixed-weight ternary CSV", [&](const std::string& v) {
        if (!file_exists(v)) throw ArgError{105, "--start: File does not exist: " + v};
        start_file = v;
    });
    add({"--device"}, "CUDA device ordinal", int_opt("--device", &p.device));
    add({"--replicas"}, "Independent GPU replicas (0 = occupancy-based)", int_opt("--replicas", &p.replicas));
    add({"--moves-per-launch"}, "Annealing iterations per replica between host checkpoints",
        int_opt("--moves-per-launch", &p.moves_per_launch));
    add({"--seed"}, "Base RNG seed (0 = random_device)", u64_opt("--seed", &p.seed));
    add({"--max-seconds"}, "Wall-clock search budget (0 = until solved or interrupted)",
        dbl_opt("--max-seconds", &p.max_seconds));
    add({"--save-interval"}, "Minimum seconds between best-matrix writes", dbl_opt("--save-interval", &p.save_interval));
    add({"--sign-fraction"}, "Probability of proposing a sign flip", dbl_opt("--sign-fraction", &p.sign_fraction));
    add({"--double-sign-fraction"}, "Probability of first proposing an atomic double sign flip",
        dbl_opt("--double-sign-fraction", &p.double_sign_fraction));
    add({"--switch-sign-fraction"}, "Probability of flipping each sign in a support switch",
        dbl_opt("--switch-sign-fraction", &p.switch_sign_fraction));
    add({"--squared-objective-fraction"}, "Fraction of replicas guided by squared Gram residual",
        dbl_opt("--squared-objective-fraction", &p.squared_objective_fraction));
    add({"--parity-objective-fraction"}, "Fraction of replicas minimizing odd support intersections",
        dbl_opt("--parity-objective-fraction", &p.parity_objective_fraction));
    add({"--greedy-fraction"}, "Probability of selecting the best sampled move",
        dbl_opt("--greedy-fraction", &p.greedy_fraction));
    add({"--candidate-samples"}, "Candidate count for a sampled greedy move",
        int_opt("--candidate-samples", &p.candidate_samples));
    add({"--target-fraction"}, "Probability of targeting a high-residual row",
        dbl_opt("--target-fraction", &p.target_fraction));
    add({"--target-samples"}, "Tournament size for high-residual row selection",
        int_opt("--target-samples", &p.target_samples));
    add({"--t-init"}, "Initial temperature (0 = auto-calibrate)", dbl_opt("--t-init", &p.t_init));
    add({"--t-min"}, "Minimum temperature", dbl_opt("--t-min", &p.t_min));
    add({"--cooling"}, "Geometric cooling factor", dbl_opt("--cooling", &p.cooling));
    add({"--moves-per-cool"}, "Moves between cooling steps", int_opt("--moves-per-cool", &p.moves_per_cool));
    add({"--stuck-threshold"}, "Moves without improvement before reheating",
        int_opt("--stuck-threshold", &p.stuck_threshold));
    add({"--reheat"}, "Fraction of initial temperature restored when stuck", dbl_opt("--reheat", &p.reheat));
    add({"--restart-interval"}, "Seconds without a global improvement before elite restarts (0 disables)",
        dbl_opt("--restart-interval", &p.restart_interval));
    add({"--restart-fraction"}, "Fraction of non-elite replicas restarted from the global best",
        dbl_opt("--restart-fraction", &p.restart_fraction));
    add({"--restart-kick-min"}, "Minimum legal perturbation moves after an elite restart",
        int_opt("--restart-kick-min", &p.restart_kick_min));
    add({"--restart-kick-max"}, "Maximum legal perturbation moves after an elite restart",
        int_opt("--restart-kick-max", &p.restart_kick_max));
    // extensions of this implementation
    add({"--max-moves"}, "Total move budget over all replicas (0 = none)", u64_opt("--max-moves", &p.max_moves));
    add({"--tempering"}, "1: replicas form one parallel-tempering ladder t-min..t-init", int_opt("--tempering", &p.tempering));
    add({"--exchange-interval"}, "Iterations between tempering exchanges",
        int_opt("--exchange-interval", &p.exchange_interval));
    add({"--objective"}, "-1 reference per-replica mix, 0 L1, 1 squared Gram residual, 2 parity",
        int_opt("--objective", &p.objective));
    add({"--move-set"}, "0 flip/switch/double flip, 1 flip/within-row swap", int_opt("--move-set", &p.move_set));
    add({"--start-kind"}, "0 regular random start, 1 row-only random start", int_opt("--start-kind", &p.start_kind));
    add({"--warps-per-block"}, "Replica warps per CTA (0 = autotuned)", int_opt("--warps-per-block", &p.warps_per_block));

    if (!parse_args(argc, argv, opts, "xweigh_cuda shared-memory weighing-matrix annealer", order, weight))
        return 0;
    const int n = (int)order, w = (int)weight;
    if (w > n) {
        std::fprintf(stderr, "Error: w must not exceed n\n");
        return 1;
    }
    const std::string err = valid_params(p);
    if (!err.empty()) {
        std::fprintf(stderr, "Error: %s\n", err.c_str());
        return 1;
    }
    const std::string impossible = xw_impossibility_reason(n, w);
    if (!impossible.empty()) {
        std::fprintf(stderr, "Error: W(%d,%d) cannot exist: %s\n", n, w, impossible.c_str());
        return 1;
    }

    std::vector<int8_t> start;
    if (!start_file.empty()) {
        start.resize((size_t)n * n);
        if (xw_read_csv(start_file.c_str(), n, w, start.data()) != XW_OK) {
            std::fprintf(stderr, "Error: %s\n", xw_last_error());
            return 1;
        }
        int64_t st[4];
        xw_score(n, w, start.data(), st);
        std::printf("[start] loaded %s score=%lld conflicts=%lld\n", start_file.c_str(), (long long)st[0],
                    (long long)st[1]);
        if (st[0] == 0) {
            if (xw_write_csv(state.output.c_str(), n, start.data()) != XW_OK) {
                std::fprintf(stderr, "Error: %s\n", xw_last_error());
                return 1;
            }
            return finish(start, n, w, state.output) ? 0 : 1;
        }
    }
    // Sylvester short-circuit, xweigh_cuda_main.cpp:270-277
    if (start.empty() && is_power_of_two(w) && n % w == 0) {
        std::vector<int8_t> best((size_t)n * n);
        xw_sylvester(n, w, best.data());
        std::printf("[construct] using direct sum of Sylvester blocks\n");
        if (xw_write_csv(state.output.c_str(), n, best.data()) != XW_OK) {
            std::fprintf(stderr, "Error: %s\n", xw_last_error());
            return 1;
        }
        return finish(best, n, w, state.output) ? 0 : 1;
    }
    if (p.seed == 0) p.seed = (uint64_t)std::random_device{}();
    std::fflush(stdout);
    xw_result res;
    std::vector<int8_t> best((size_t)n * n);
    const int rc = xw_run(n, w, &p, start.empty() ? nullptr : start.data(), log_line, checkpoint, &state, &res,
                          best.data());
    if (rc != XW_OK) {
        std::fprintf(stderr, "Error: %s\n", xw_last_error());
        return 1;
    }
    if (xw_write_csv(state.output.c_str(), n, best.data()) != XW_OK) {
        std::fprintf(stderr, "Error: %s\n", xw_last_error());
        return 1;
    }
    return finish(best, n, w, state.output) ? 0 : 1;
}

// valid_params, xweigh_main.cpp:54-88
std::string valid_cpu_params(const xw_cpu_params& p) {
    if (p.threads < 1) return "--threads must be positive";
    if (p.max_seconds < 0.0) return "--max-seconds must be nonnegative";
    if (p.save_interval < 0.0) return "--save-interval must be nonnegative";
    if (p.sign_fraction < 0.0 || p.sign_fraction > 1.0) return "--sign-fraction must be in [0, 1]";
    if (p.greedy_fraction < 0.0 || p.greedy_fraction > 1.0) return "--greedy-fraction must be in [0, 1]";
    if (p.target_fraction < 0.0 || p.target_fraction > 1.0) return "--target-fraction must be in [0, 1]";
    if (p.candidate_samples < 1) return "--candidate-samples must be positive";
    if (p.target_samples < 1) return "--target-samples must be positive";
    if (p.exchange_interval < 1) return "--exchange-interval must be positive";
    if (p.t_init < 0.0) return "--t-init must be nonnegative";
    if (p.t_min <= 0.0) return "--t-min must be positive";
    if (p.cooling <= 0.0 || p.cooling >= 1.0) return "--cooling must be in (0, 1)";
    if (p.moves_per_cool < 1) return "--moves-per-cool must be positive";
    if (p.stuck_threshold < 1) return "--stuck-threshold must be positive";
    if (p.reheat <= 0.0) return "--reheat must be positive";
    if (p.reseed_factor < 1.0) return "--reseed-factor must be at least 1";
    return {};
}

// The xweigh command line (xweigh_main.cpp:88-270) over xw_cpu_run.
[[maybe_unused]] int run_cpu(int argc, char** argv) {
    xw_cpu_params p;
    xw_cpu_params_default(&p);
    CliState state;
    std::string start_file;
    long long order = 0, weight = 0;
    std::vector<Option> opts;
    auto add = [&](std::vector<std::string> names, std::string help, std::function<void(const std::string&)> set,
                   bool flag = false) {
        opts.push_back(Option{std::move(names), std::move(help), std::move(set), flag});
    };
    auto conv_err = [](const std::string& name, const std::string& v) {
        return ArgError{107, name + ": Value " + v + " could not be converted"};
    };
    auto int_opt = [&](const std::string& name, int32_t* dst) {
        return [=](const std::string& v) {
            long long x;
            if (!parse_int(v, x) || x < INT32_MIN || x > INT32_MAX) throw conv_err(name, v);
            *dst = (int32_t)x;
        };
    };
    auto dbl_opt = [&](const std::string& name, double* dst) {
        return [=](const std::string& v) {
            double x;
            if (!parse_double(v, x)) throw conv_err(name, v);
            *dst = x;
        };
    };
    add({"-o", "--out"}, "Output CSV for the best matrix", [&](const std::string& v) { state.output = v; });
    add({"--start"}, "Start from a complete fixed-weight ternary CSV", [&](const std::string& v) {
        if (!file_exists(v)) throw ArgError{105, "--start: File does not exist: " + v};
        start_file = v;
    });
    add({"-t", "--threads"}, "Number of worker threads (default: physical cores)", int_opt("--threads", &p.threads));
    // physical and logical processors count alike on this host, and workers
    // are not pinned: both switches are accepted for the reference's scripts
    add({"--use-hyperthreads"}, "Default to all logical processors (ignored with --threads)",
        [&](const std::string&) {}, true);
    add({"--no-pin"}, "Do not pin workers to physical cores on Windows", [&](const std::string&) {}, true);
    add({"--seed"}, "Base RNG seed (0 = random_device)", [&](const std::string& v) {
        uint64_t x;
        if (!parse_uint64(v, x)) throw conv_err("--seed", v);
        p.seed = x;
    });
    add({"--max-seconds"}, "Wall-clock search budget (0 = until solved or interrupted)",
        dbl_opt("--max-seconds", &p.max_seconds));
    add({"--save-interval"}, "Minimum seconds between best-matrix writes", dbl_opt("--save-interval", &p.save_interval));
    add({"--sign-fraction"}, "Probability of proposing a sign flip instead of a support switch",
        dbl_opt("--sign-fraction", &p.sign_fraction));
    add({"--greedy-fraction"}, "Probability of selecting the best of sampled candidate moves",
        dbl_opt("--greedy-fraction", &p.greedy_fraction));
    add({"--candidate-samples"}, "Candidate count for a sampled greedy move",
        int_opt("--candidate-samples", &p.candidate_samples));
    add({"--target-fraction"}, "Probability of targeting a high-residual row",
        dbl_opt("--target-fraction", &p.target_fraction));
    add({"--target-samples"}, "Tournament size for high-residual row selection",
        int_opt("--target-samples", &p.target_samples));
    add({"--tempering"}, "Parallel tempering for two or more workers", [&](const std::string&) { p.tempering = 1; },
        true);
    add({"--no-tempering"}, "Independent annealing workers", [&](const std::string&) { p.tempering = 0; }, true);
    add({"--exchange-interval"}, "Approximate moves per worker between replica exchanges",
        int_opt("--exchange-interval", &p.exchange_interval));
    add({"--t-init"}, "Initial temperature (0 = auto-calibrate)", dbl_opt("--t-init", &p.t_init));
    add({"--t-min"}, "Minimum temperature", dbl_opt("--t-min", &p.t_min));
    add({"--cooling"}, "Single-worker geometric cooling factor", dbl_opt("--cooling", &p.cooling));
    add({"--moves-per-cool"}, "Single-worker moves between cooling steps",
        int_opt("--moves-per-cool", &p.moves_per_cool));
    add({"--stuck-threshold"}, "Single-worker moves without improvement before reheating",
        int_opt("--stuck-threshold", &p.stuck_threshold));
    add({"--reheat"}, "Fraction of initial temperature restored when stuck", dbl_opt("--reheat", &p.reheat));
    add({"--reseed-factor"}, "Reseed from the best when this factor behind it",
        dbl_opt("--reseed-factor", &p.reseed_factor));
    if (!parse_args(argc, argv, opts, "xweigh unrestricted weighing-matrix annealer", order, weight)) return 0;

    const int n = (int)order, w = (int)weight;
    if (w > n) {
        std::fprintf(stderr, "Error: w must not exceed n\n");
        return 1;
    }
    const std::string err = valid_cpu_params(p);
    if (!err.empty()) {
        std::fprintf(stderr, "Error: %s\n", err.c_str());
        return 1;
    }
    const std::string impossible = xw_impossibility_reason(n, w);
    if (!impossible.empty()) {
        std::fprintf(stderr, "Error: W(%d,%d) cannot exist: %s\n", n, w, impossible.c_str());
        return 1;
    }
    if (n > XW_MAX_ORDER_CUDA) {
        std::fprintf(stderr, "Error: orders above %d are outside this build\n", XW_MAX_ORDER_CUDA);
        return 1;
    }
    if (p.seed == 0) p.seed = (uint64_t)std::random_device{}();
    const auto t_init0 = std::chrono::steady_clock::now();
    std::vector<int8_t> start((size_t)n * n);
    const bool loaded = !start_file.empty();
    const bool sylvester = !loaded && is_power_of_two(w) && n % w == 0;
    if (loaded) {
        if (xw_read_csv(start_file.c_str(), n, w, start.data()) != XW_OK) {
            std::fprintf(stderr, "Error: %s\n", xw_last_error());
            return 1;
        }
    } else if (sylvester) {
        xw_sylvester(n, w, start.data());
    } else if (xw_random_start(n, w, (uint32_t)p.seed, start.data()) != XW_OK) {
        std::fprintf(stderr, "Error: %s\n", xw_last_error());
        return 1;
    }
    const double init_s = std::chrono::duration<double>(std::chrono::steady_clock::now() - t_init0).count();
    // a reference worker's state: W twice, int16 Gram, int64 residuals,
    // u16 minority lists (xweigh_anneal.hpp:185-190)
    const int m = std::min(w, n - w);
    const double worker_bytes = (double)n * n * 4 + 8.0 * n + 2.0 * n * m;
    std::printf("[init] seconds=%g worker_mib=%g total_worker_mib=%g\n", init_s, worker_bytes / 1048576.0,
                worker_bytes * p.threads / 1048576.0);
    int64_t st[4];
    xw_score(n, w, start.data(), st);
    if (loaded)
        std::printf("[start] loaded %s score=%lld conflicts=%lld\n", start_file.c_str(), (long long)st[0],
                    (long long)st[1]);
    else if (sylvester)
        std::printf("[construct] using direct sum of Sylvester blocks\n");
    std::vector<int8_t> best = start;
    if (st[0] != 0) {
        std::fflush(stdout);
        xw_cpu_result res;
        const int rc = xw_cpu_run(n, w, &p, start.data(), log_line, checkpoint, &state, &res, best.data());
        if (rc != XW_OK) {
            std::fprintf(stderr, "Error: %s\n", xw_last_error());
            return 1;
        }
    }
    if (xw_write_csv(state.output.c_str(), n, best.data()) != XW_OK) {
        std::fprintf(stderr, "Error: %s\n", xw_last_error());
        return 1;
    }
    return finish(best, n, w, state.output) ? 0 : 1;
}

}  // namespace

int main(int argc, char** argv) {
    std::signal(SIGINT, on_interrupt);
    try {
#ifdef XW_CLI_CPU
        return run_cpu(argc, argv);
#else
        return run(argc, argv);
#endif
    } catch (const ArgError& e) {
        std::fprintf(stderr, "%s\nRun with --help for more information.\n", e.message.c_str());
        return e.code;
    } catch (const std::bad_alloc&) {
        std::fprintf(stderr, "Error: insufficient host memory\n");
    } catch (const std::exception& e) {
        std::fprintf(stderr, "Error: %s\n", e.what());
    }
    return 1;
}
