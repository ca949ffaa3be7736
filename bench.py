"""Benchmark: moves/sec of the uniform tempering population, W(26,25).

Workload (one "step"): 128 independent W(26,25) searches x 32-rung
geometric tempering ladder (T 0.1 .. 6, exchange every 10^4 iterations),
4096 replicas, 10^9 moves (244141 iterations per replica), each replica
starting from the reference's seeded regular random start.  Seeds are
per instance, so every step is the same computation (the population is
reset on the device between steps).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

One JSON line on rank 0.  `value` is device-timed moves/sec with the start
states resident in HBM; `e2e` is the same metric through the C ABI's
whole-batch call (xw_batch_solve) with host buffers, host<->device copies
inside the timed region.  `--impl reference` times the reference's own
CPU engine (oracle/_ref/xweigh, all host threads) on the same (n, w) and
tempering setup.  N > 1: one process per GPU, each running its own 128
instances (weak scaling, no collective on the data path).
"""
import argparse
import dataclasses
import json
import os
import re
import statistics
import subprocess
import sys
import tempfile
import threading
import time

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, REPO)

N_ORDER, W_WEIGHT = 26, 25
INSTANCES, RUNGS = 128, 32
TOTAL_MOVES = 10 ** 9
EXCHANGE = 10_000
T_MIN, T_MAX = 0.1, 6.0
ITERS = -(-TOTAL_MOVES // (INSTANCES * RUNGS))   # 244141 iterations per replica
REF_XWEIGH = os.path.join(REPO, "oracle", "_ref", "xweigh")
REF_XWEIGH_CUDA = os.path.join(REPO, "oracle", "_ref", "xweigh_cuda")
METRIC = "moves/sec (uniform W(26,25) tempering population)"
WORKLOAD = (f"W({N_ORDER},{W_WEIGHT}): {INSTANCES} instances x {RUNGS}-rung tempering ladder "
            f"T {T_MIN}..{T_MAX}, exchange every {EXCHANGE} moves, {TOTAL_MOVES:.0e} moves per step")


def log(*a):
    print(*a, file=sys.stderr, flush=True)


def dist_info():
    return int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")), \
        int(os.environ.get("LOCAL_RANK", "0"))


# ---------------------------------------------------------------- reference CPU
def run_reference_cpu(seconds, threads, seed=1):
    """The reference xweigh on `threads` host threads for `seconds`; returns
    (moves, seconds) from its `done moves=... seconds=...` line
    (xweigh_anneal.hpp:1263-1265)."""
    with tempfile.TemporaryDirectory() as td:
        out = subprocess.run(
            [REF_XWEIGH, str(N_ORDER), str(W_WEIGHT), "-t", str(threads), "--seed", str(seed),
             "--max-seconds", str(seconds), "--t-init", str(T_MAX), "--t-min", str(T_MIN),
             "--exchange-interval", str(EXCHANGE), "-o", os.path.join(td, "w.csv")],
            capture_output=True, text=True, timeout=seconds * 4 + 60)
    m = re.search(r"done moves=(\d+) seconds=([0-9.e+-]+)", out.stdout)
    if not m:
        raise RuntimeError("reference xweigh gave no done line: " + out.stdout[-300:] + out.stderr[-300:])
    return int(m.group(1)), float(m.group(2))


def run_reference_cuda(seconds, seed=1, n=N_ORDER, w=W_WEIGHT, replicas=INSTANCES * RUNGS):
    """The reference xweigh_cuda (the plain kernel, one instance per launch)
    on the same shape: by default 4096 replicas of W(26,25)."""
    with tempfile.TemporaryDirectory() as td:
        out = subprocess.run(
            [REF_XWEIGH_CUDA, str(n), str(w), "--replicas", str(replicas),
             "--t-init", str(T_MAX), "--t-min", str(T_MIN), "--seed", str(seed), "--max-seconds", str(seconds),
             "--restart-interval", "0", "-o", os.path.join(td, "w.csv")],
            capture_output=True, text=True, timeout=seconds * 4 + 120)
    m = re.search(r"done moves=(\d+) .*?seconds=([0-9.e+-]+) moves_per_sec=([0-9.e+-]+)", out.stdout)
    if not m:
        raise RuntimeError("reference xweigh_cuda gave no done line: " + out.stdout[-300:] + out.stderr[-300:])
    return int(m.group(1)), float(m.group(2))


def reference_arm(args):
    rank, world, _ = dist_info()
    if rank != 0:
        return
    if not os.path.exists(REF_XWEIGH):
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/xweigh was not built"}))
        return
    threads = os.cpu_count() or 1
    sample = args.ref_seconds
    for _ in range(args.warmup):
        run_reference_cpu(max(1.0, sample / 4), threads)
    moves = secs = 0
    for k in range(args.steps):
        mv, s = run_reference_cpu(sample, threads, seed=1 + k)
        moves += mv
        secs += s
    value = moves / secs
    line = {
        "metric": METRIC, "value": value, "unit": "moves/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": secs * 1e3 / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "int32", "data": "synthetic",
        "impl": "reference",
        "config": {"workload": f"W({N_ORDER},{W_WEIGHT}): one reference xweigh search, parallel tempering "
                               f"with one rung per host thread ({threads} rungs, T {T_MIN}..{T_MAX}, exchange "
                               f"every {EXCHANGE} moves per thread), {sample:g} s of search per step",
                   "engine": "reference xweigh CPU, parallel tempering over threads",
                   "threads": threads, "sample_seconds_per_step": sample,
                   "compared_with": WORKLOAD},
        "cpu_baseline": {"value": value, "unit": "moves/s", "cores": threads, "kind": "reference",
                         "sample": f"xweigh {N_ORDER} {W_WEIGHT} -t {threads} --max-seconds {sample} per step"},
        "e2e": {"value": value, "unit": "moves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------- clocks
class ClockSampler:
    """nvidia-smi clocks and throttle reasons, sampled during the timed region."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.QUERY}", "--format=csv,noheader",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
        return self

    def __exit__(self, *exc):
        self.rows = []
        if self.proc is None:
            return
        self.proc.terminate()
        try:
            out, _ = self.proc.communicate(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
            out, _ = self.proc.communicate()
        for line in out.splitlines():
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 9:
                self.rows.append(parts)

    def summary(self):
        rows = getattr(self, "rows", [])
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}

        def mhz(s):
            m = re.match(r"([0-9.]+)", s)
            return float(m.group(1)) if m else None

        sm = [mhz(r[1]) for r in rows if mhz(r[1])]
        mx = [mhz(r[2]) for r in rows if mhz(r[2])]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower().startswith("active")})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


# ---------------------------------------------------------------- ours
def reduce_over_ranks(world, device, max_vals, sum_vals):
    """(max over ranks of max_vals, sum over ranks of sum_vals): the whole-job
    time is the slowest rank's, the work is every rank's.  Every rank calls
    it at the same point; world 1 needs no process group."""
    if world == 1:
        return list(max_vals), list(sum_vals)
    import torch
    import torch.distributed as dist
    mx = torch.tensor(list(max_vals), dtype=torch.float64, device=device)
    sm = torch.tensor(list(sum_vals), dtype=torch.float64, device=device)
    dist.all_reduce(mx, op=dist.ReduceOp.MAX)
    dist.all_reduce(sm, op=dist.ReduceOp.SUM)
    return mx.tolist(), sm.tolist()


def make_jobs(rank):
    """Rank r's shard: its own INSTANCES searches, seeds disjoint across ranks
    (independent searches, so no data crosses GPUs)."""
    return [{"n": N_ORDER, "w": W_WEIGHT, "seed": 1 + rank * INSTANCES + i, "replicas": RUNGS}
            for i in range(INSTANCES)]


def make_params():
    import xtax_b200 as X
    # tempering on the L1 score for every rung (no alternate objectives),
    # reference move mix otherwise; replicas keep running after a solve so
    # every step does the same 10^9 moves
    return X.Params(tempering=1, exchange_interval=EXCHANGE, t_min=T_MIN, t_init=T_MAX,
                    squared_objective_fraction=0.0, parity_objective_fraction=0.0, stop_on_solve=0)


def algorithmic_smem_bytes(cand_evals, two_row_evals, accepted_rows, n=N_ORDER, g=4):
    """Shared-memory bytes the moves need at minimum, from the move
    statistics the kernel counts: each evaluated candidate reads, per row it
    changes (one, or two for the counted two-row candidates), (n-1) Gram
    entries of g bytes and (n-1) W entries; each row an accepted move
    changes writes 2(n-1) Gram entries (the row and its mirror column)."""
    reads = (cand_evals + two_row_evals) * (n - 1) * (g + 1)
    writes = accepted_rows * 2 * (n - 1) * g
    return reads + writes


def ours(args):
    import torch
    import xtax_b200 as X

    rank, world, local = dist_info()
    torch.cuda.set_device(local)
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=600))
    p = make_params()
    p.device = local
    jobs = make_jobs(rank)
    t_build = time.time()
    batch = X.Batch(jobs, p)
    log(f"[bench] rank {rank}: batch built in {time.time() - t_build:.1f}s shape={batch.shape()}")
    # a dedicated stream: the library launches on it and the CUDA events
    # below are recorded on it (the legacy default stream has handle 0,
    # which the library would read as "use your own stream")
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    batch.set_stream(stream.cuda_stream)
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device="cuda")  # > 126 MB L2

    iters = args.iters

    def step(timed):
        batch.reset()
        if timed:
            batch.run_timed(iters)
        else:
            batch.run(iters)

    for _ in range(args.warmup):
        step(False)
    torch.cuda.synchronize()

    def barrier():
        if world > 1:
            torch.distributed.barrier()

    step_ms, launch_ms = [], []
    moves = evals = evals2 = acc = acc_rows = 0
    barrier()
    torch.cuda.synchronize()
    with ClockSampler(local) as clk:
        for k in range(args.steps):
            flush.fill_(k & 0xff)
            start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            start.record(stream)
            step(True)
            stop.record(stream)
            stop.synchronize()
            step_ms.append(start.elapsed_time(stop))
            launch_ms.extend(batch.launch_times())
            res = batch.results()
            moves += sum(r.moves for r, _ in res)
            evals += sum(r.candidate_evaluations for r, _ in res)
            evals2 += sum(r.two_row_evaluations for r, _ in res)
            acc += sum(r.accepted_moves for r, _ in res)
            acc_rows += sum(r.accepted_rows for r, _ in res)
    torch.cuda.synchronize()
    barrier()
    total_ms = sum(step_ms)
    (total_ms,), (moves, evals, evals2, acc, acc_rows) = reduce_over_ranks(
        world, "cuda", [total_ms], [float(moves), float(evals), float(evals2), float(acc), float(acc_rows)])
    value = moves / (total_ms / 1e3)

    # end to end: the C ABI whole-batch call with host buffers
    starts = None
    e2e_value = None
    h2d, d2h = batch.transfer_bytes()
    launch_shape = list(batch.shape())
    launch_classes = batch.classes()
    # the device-resident batch is done: its device memory returns to the
    # library's pool, where the end-to-end call's batch finds it
    torch.cuda.synchronize()
    batch.close()
    if args.e2e_steps > 0:
        import numpy as np
        starts = np.concatenate([X.random_start(N_ORDER, W_WEIGHT, (j["seed"] + r * 0x9e3779b9) & 0xffffffff)
                                 for j in jobs for r in range(RUNGS)])
        pinned = torch.from_numpy(starts).pin_memory()
        host = pinned.numpy()
        e2e_moves = 0
        # one untimed call first, as the device-timed steps have their warm-up
        X.batch_solve(jobs, p, starts=host, iters=iters)
        torch.cuda.synchronize()
        barrier()
        t0 = time.perf_counter()
        for _ in range(args.e2e_steps):
            res, best = X.batch_solve(jobs, p, starts=host, iters=iters)
            e2e_moves += sum(r.moves for r in res)
        torch.cuda.synchronize()
        e2e_s = time.perf_counter() - t0
        (e2e_s,), (e2e_moves,) = reduce_over_ranks(world, "cuda", [e2e_s], [float(e2e_moves)])
        e2e_value = e2e_moves / e2e_s

    clocks = clk.summary()
    if world > 1:
        torch.distributed.destroy_process_group()
    if rank != 0:
        return

    anneal_launches = [ms for ms in launch_ms if ms > 0]
    avg_launch_ms = statistics.mean(anneal_launches)
    nl = max(1, len(anneal_launches)) * world
    alg_bytes = algorithmic_smem_bytes(evals / nl, evals2 / nl, acc_rows / nl)
    sm_mhz = clocks.get("sm_mhz") or 1965.0
    smem_peak = 148 * 128 * sm_mhz * 1e6 / 1e9   # GB/s, nominal: 128 B/clk/SM
    achieved = alg_bytes / (avg_launch_ms / 1e3) / 1e9
    prof = load_profile_figure("traffic_bytes_per_launch")
    issue = load_profile_figure("issue_active_pct")
    # instruction issue: the profiled warp instructions per replica iteration
    # times the iterations per second, against one warp instruction per
    # scheduler per cycle (148 SMs x 4 schedulers x median SM clock)
    inst_per_iter = load_profile_figure("warp_instructions_per_iteration")
    iters_per_launch = args.steps * INSTANCES * RUNGS * iters / max(1, len(anneal_launches))
    issue_rate = inst_per_iter * iters_per_launch / (avg_launch_ms / 1e3) if inst_per_iter else None
    issue_peak = 148 * 4 * sm_mhz * 1e6
    line = {
        "metric": METRIC, "value": value, "unit": "moves/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "int32", "data": "synthetic",
        "config": {"workload": WORKLOAD, "replicas_per_gpu": INSTANCES * RUNGS,
                   "iterations_per_replica": iters, "l2": "flushed between steps (256 MiB write)",
                   "launch_shape": launch_shape, "launch_classes": launch_classes,
                   "parallelism": f"instances x{world} GPUs"},
        "gpu_launches": args.steps * (2 * (-(-iters // EXCHANGE)) + 1),
        "roofline": {"bound": "smem", "achieved": achieved, "peak": smem_peak, "unit": "GB/s",
                     "frac": achieved / smem_peak, "traffic": int(prof) if prof else None,
                     "issue_active_pct_ncu": issue,
                     "issue_frac": issue_rate / issue_peak if issue_rate else None,
                     "warp_instructions_per_iteration_ncu": inst_per_iter,
                     "move_statistics": {"candidate_evaluations": evals, "two_row_evaluations": evals2,
                                         "accepted_moves": acc, "accepted_rows": acc_rows, "moves": moves,
                                         "acceptance": acc / moves if moves else None},
                     "kernel": "anneal_kernel", "avg_launch_ms": avg_launch_ms,
                     "peak_source": "nominal 128 B/clk/SM x 148 SMs x median SM clock (no measured shared-memory peak)"},
        "clocks": clocks,
    }
    if e2e_value is not None:
        line["e2e"] = {"value": e2e_value, "unit": "moves/s", "h2d_bytes_per_step": h2d,
                       "d2h_bytes_per_step": d2h, "steps": args.e2e_steps}
    if args.cpu_seconds > 0 and os.path.exists(REF_XWEIGH):
        threads = os.cpu_count() or 1
        mv, s = run_reference_cpu(args.cpu_seconds, threads)
        line["cpu_baseline"] = {"value": mv / s, "unit": "moves/s", "cores": threads, "kind": "reference",
                                "sample": f"reference xweigh {N_ORDER} {W_WEIGHT} -t {threads} tempering, "
                                          f"{args.cpu_seconds:g} s wall"}
    if args.plain_seconds > 0 and os.path.exists(REF_XWEIGH_CUDA):
        try:
            mv, s = run_reference_cuda(args.plain_seconds)
            line["plain_kernel"] = {"impl": "reference xweigh_cuda (sm_100a build)", "value": mv / s,
                                    "unit": "moves/s", "replicas": INSTANCES * RUNGS,
                                    "sample_seconds": args.plain_seconds}
        except Exception as e:  # noqa: BLE001 - report, do not fail the bench
            line["plain_kernel"] = {"unavailable": str(e)[:200]}
    if args.rescore:
        line["rescore"] = rescore_bench(torch, X, [int(v) for v in args.rescore_orders.split(",")])
    if args.c1:
        line["single_replica"] = c1_bench(X, args.c1_ref_seconds)
    if args.uneven_iters > 0:
        line["uneven"] = uneven_bench(X, args.uneven_iters)
    if args.large_iters > 0:
        line["large_order"] = large_bench(X, args.large_iters, args.large_ref_seconds)
    if args.serve_requests > 0:
        line["serving"] = serving_bench(X, args.serve_requests, args.serve_plain, args.serve_quantum,
                                        args.serve_reference, args.serve_reference_cap, args.serve_light,
                                        args.serve_light_rate)
    print(json.dumps(line), flush=True)


REF_HARNESS = os.path.join(REPO, "oracle", "_ref", "ref_harness")


def rescore_bench(torch, X, orders=(32, 64, 96, 128)):
    """Batched exact W W^T (tcgen05 kind::i8): 65536 fixed-degree ternary
    matrices per order n (32, 64, 96, 128 by default), w = n/2, resident in
    HBM.  HBM-bound: n^2 bytes in and 16 bytes out per matrix."""
    import ctypes as C
    peaks = {}
    try:
        with open(os.path.join(REPO, "MEASURED_PEAKS.json")) as f:
            peaks = json.load(f)
    except (OSError, ValueError):
        pass
    hbm = peaks.get("hbm_gbs", 6650.0)
    out = {"matrices_per_order": 65536, "peak_source": "MEASURED_PEAKS.json hbm_gbs" if peaks else "fallback 6.65 TB/s",
           "orders": {}}
    count = 65536
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device="cuda")
    stream = torch.cuda.current_stream()
    for n in orders:
        w = n // 2
        gen = torch.Generator(device="cuda").manual_seed(n)
        W = torch.zeros((count, n, n), dtype=torch.int8, device="cuda")
        for c0 in range(0, count, 4096):
            keys = torch.rand((4096, n, n), device="cuda", generator=gen)
            idx = keys.argsort(dim=2)[:, :, :w]
            signs = (torch.randint(0, 2, (4096, n, w), device="cuda", generator=gen) * 2 - 1).to(torch.int8)
            W[c0:c0 + 4096].scatter_(2, idx, signs)
            del keys, idx, signs
        stats = torch.zeros((count, 4), dtype=torch.int32, device="cuda")

        def launch():
            rc = X.lib().xw_rescore_device(C.c_void_p(W.data_ptr()), count, n, w, C.c_void_p(stats.data_ptr()),
                                           None, 0, C.c_void_p(stream.cuda_stream))
            if rc != X.XW_OK:
                raise RuntimeError(X.lib().xw_last_error().decode())

        for _ in range(3):
            launch()
        torch.cuda.synchronize()
        times = []
        for _ in range(10):
            flush.fill_(1)
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            launch()
            b.record(stream)
            b.synchronize()
            times.append(a.elapsed_time(b))
        if X.lib().xw_rescore_status() != X.XW_OK:
            raise RuntimeError("rescore pipeline wait expired")
        ms = statistics.median(times)
        alg_bytes = count * (n * n + 16)
        gbs = alg_bytes / (ms / 1e3) / 1e9
        entry = {"ms": ms, "matrices_per_sec": count / (ms / 1e3),
                 "roofline": {"bound": "hbm", "achieved": gbs, "peak": hbm, "unit": "GB/s", "frac": gbs / hbm,
                              "algorithmic_bytes": alg_bytes},
                 "tensor_ops": 2 * n ** 3 * count}
        if os.path.exists(REF_HARNESS):
            threads = os.cpu_count() or 1
            sample = 16384 if n <= 64 else 4096
            r = subprocess.run([REF_HARNESS, "rescore_bench", str(n), str(w), str(sample), str(threads)],
                               capture_output=True, text=True, timeout=600)
            try:
                ref = json.loads(r.stdout.strip().splitlines()[-1])
                entry["cpu_baseline"] = {"value": ref["matrices_per_sec"], "unit": "matrices/s", "cores": threads,
                                         "kind": "reference",
                                         "sample": f"{sample} matrices: State::from_entries + verify_weighing"}
            except (ValueError, IndexError, KeyError):
                pass
        out["orders"][str(n)] = entry
        del W, stats
    return out


# ---------------------------------------------------------------- single replicas (C1)
C1_SEEDS = 32
C1_MOVES = 10 ** 6


def c1_bench(X, ref_seconds):
    """W(12,11), one replica per search, 32 seeds: row-only fixed-degree
    starts, the squared objective, sign flips and within-row swaps, geometric
    cooling 4 -> 0.05 over 1e6 moves (500 moves per step), no reheat; each
    search stops at its solve or its 1e6 moves.  All 32 run in one launch per
    round.  Beside it, the reference's CPU xweigh, one thread, on the same
    order and schedule (its own move set and L1 objective: the closest run the
    reference offers)."""
    import numpy as np
    cooling = (0.05 / 4.0) ** (1.0 / 2000.0)
    p = X.Params(t_init=4.0, t_min=0.05, cooling=cooling, moves_per_cool=500, stuck_threshold=2_000_000_000,
                 objective=1, move_set=1, start_kind=1, stop_on_solve=2, moves_per_launch=100_000,
                 max_moves=C1_MOVES)
    jobs = [{"n": 12, "w": 11, "seed": k, "replicas": 1} for k in range(1, C1_SEEDS + 1)]

    def searches(params):
        b = X.Batch(jobs, params)
        classes = b.classes()
        b.run_timed(C1_MOVES)
        b.synchronize()
        ms = sum(b.launch_times())
        res = b.results()
        b.close()
        moves = sum(r.moves for r, _ in res)
        solved = [r for r, _ in res if r.solved]
        return {"moves": moves, "ms": ms, "moves_per_sec": moves / (ms / 1e3),
                "moves_per_sec_per_search": moves / (ms / 1e3) / C1_SEEDS,
                "solved": len(solved), "searches": C1_SEEDS,
                "median_solve_iteration": float(np.median([r.solved_iteration for r in solved])) if solved else None,
                "launch_classes": classes}

    out = {"workload": f"W(12,11) x {C1_SEEDS} seeds, 1 replica each, squared objective, flips + within-row "
                       f"swaps, cooling 4 -> 0.05 over {C1_MOVES:.0e} moves",
           "device": searches(p)}
    # the same searches one warp per replica (no latency mode)
    out["device_one_warp"] = searches(dataclasses.replace(p, warps_per_replica=1))
    # the same schedule with the reference's moves, L1 objective and regular
    # starts: the solve rate of the move set, on the device
    out["device_reference_moves"] = searches(dataclasses.replace(p, objective=0, move_set=0, start_kind=0))
    if ref_seconds > 0 and os.path.exists(REF_XWEIGH):
        mv = secs = 0.0
        ok = runs = 0
        t_end = time.perf_counter() + ref_seconds
        seed = 1
        while time.perf_counter() < t_end:
            with tempfile.TemporaryDirectory() as td:
                r = subprocess.run([REF_XWEIGH, "12", "11", "-t", "1", "--seed", str(seed), "--t-init", "4",
                                    "--t-min", "0.05", "--cooling", repr(cooling), "--moves-per-cool", "500",
                                    "--stuck-threshold", "2000000000", "--max-seconds", "2",
                                    "-o", os.path.join(td, "w.csv")], capture_output=True, text=True, timeout=60)
            m = re.search(r"done moves=(\d+) seconds=([0-9.e+-]+)", r.stdout)
            if m:
                mv += int(m.group(1))
                secs += float(m.group(2))
                runs += 1
                ok += "exact verification passed" in r.stdout
            seed += 1
        out["reference_cpu_1thread"] = {"moves_per_sec": mv / secs if secs else None, "runs": runs, "solved": ok,
                                        "max_seconds_per_run": 2}
    return out


# ---------------------------------------------------------------- orders beyond shared memory
LARGE_N, LARGE_W, LARGE_R = 276, 275, 2368


def large_bench(X, iters, ref_seconds):
    """W(276,275) with 2368 replicas and the reference's defaults otherwise
    (t_init 6, t_min 0.1, cooling and reheat, no restarts).  276 is about the
    largest order whose state the reference's kernel holds in one CTA's
    shared memory; here it runs on the large-order kernel in its default
    form (bit planes in shared memory, the Gram matrix in HBM, 8 warps per
    SM) and in its two others (the Gram matrix and masks in HBM, 16 warps
    per SM; bit planes with every Gram entry recomputed).  Beside it the
    reference's xweigh_cuda on the same order and replica count."""
    p = X.Params(stop_on_solve=0, t_init=6.0, t_min=0.1, moves_per_launch=1000,
                 squared_objective_fraction=0.0, parity_objective_fraction=0.0)

    def form(which):
        # XW_LARGE_PLANES selects the kernel's form when the batch is built
        old = os.environ.get("XW_LARGE_PLANES")
        os.environ["XW_LARGE_PLANES"] = str(which)
        try:
            b = X.Batch([{"n": LARGE_N, "w": LARGE_W, "seed": 1, "replicas": LARGE_R}], p)
        finally:
            if old is None:
                del os.environ["XW_LARGE_PLANES"]
            else:
                os.environ["XW_LARGE_PLANES"] = old
        (cls,) = b.classes()
        b.run(1000)          # the first launch builds each replica's arena (Gram matrix, or planes and residuals)
        b.synchronize()
        r0 = b.results()[0][0]
        b.run_timed(iters)
        b.synchronize()
        ms = sum(b.launch_times())
        r = b.results()[0][0]
        b.close()
        moves = r.moves - r0.moves
        return {"moves": moves, "ms": ms, "moves_per_sec": moves / (ms / 1e3), "error": r.error,
                "candidate_evaluations": r.candidate_evaluations - r0.candidate_evaluations,
                "two_row_evaluations": r.two_row_evaluations - r0.two_row_evaluations,
                "accepted_moves": r.accepted_moves - r0.accepted_moves,
                "launch_class": cls,
                "kernel": "anneal_large_kernel, " + {1: "Gram matrix in HBM",
                                                     2: "bit planes in shared memory, Gram entries recomputed",
                                                     3: "bit planes in shared memory, Gram matrix in HBM"}[cls["large"]]}

    out = {"workload": f"W({LARGE_N},{LARGE_W}) x {LARGE_R} replicas, cooling from T 6 (t_min 0.1), L1 objective, "
                       f"the reference's moves, {iters} iterations per replica",
           "device": form(2), "device_stored_gram": form(0), "device_bit_planes": form(1)}
    if ref_seconds > 0 and os.path.exists(REF_XWEIGH_CUDA):
        try:
            mv, secs = run_reference_cuda(ref_seconds, n=LARGE_N, w=LARGE_W, replicas=LARGE_R)
            out["reference_xweigh_cuda"] = {"moves_per_sec": mv / secs, "sample_seconds": ref_seconds,
                                            "impl": "reference xweigh_cuda (sm_100a build), shared-memory state"}
        except Exception as e:  # noqa: BLE001 - report, do not fail the bench
            out["reference_xweigh_cuda"] = {"unavailable": str(e)[:200]}
    return out


# ---------------------------------------------------------------- uneven batch (C3)
UNEVEN = ((14, 13), (18, 17), (20, 19), (24, 23), (30, 29))
UNEVEN_INSTANCES, UNEVEN_RUNGS = 64, 16


def uneven_bench(X, iters):
    """1024 replicas each of W(14,13), W(18,17), W(20,19), W(24,23) and
    W(30,29) (64 instances x 16-rung tempering ladder per order) in one
    persistent launch per round, at the autotuned warps per CTA, against
    the same searches run as five launches, one order at a time."""
    import numpy as np
    p = X.Params(tempering=1, exchange_interval=EXCHANGE, t_min=T_MIN, t_init=T_MAX,
                 squared_objective_fraction=0.0, parity_objective_fraction=0.0, stop_on_solve=0)
    jobs = [{"n": n, "w": w, "seed": 7000 + 100 * i + k, "replicas": UNEVEN_RUNGS}
            for i, (n, w) in enumerate(UNEVEN) for k in range(UNEVEN_INSTANCES)]
    wpb, tune_ms = X.autotune(jobs, p, iters=5000)

    def timed(js, steps=3):
        b = X.Batch(js, p)
        timed.classes = b.classes()
        b.reset()
        b.run(iters)           # warm-up (builds the CUDA graph)
        b.synchronize()
        ms = []
        for _ in range(steps):
            b.reset()
            b.run(iters)
            b.synchronize()
            ms.append(sum(b.launch_times()))
        moves = sum(r.moves for r, _ in b.results())
        shape = b.shape()
        b.close()
        return moves, float(np.median(ms)), shape

    moves, ms, shape = timed(jobs)
    out = {"workload": f"{len(UNEVEN)} orders x {UNEVEN_INSTANCES} instances x {UNEVEN_RUNGS}-rung ladder "
                       f"T {T_MIN}..{T_MAX}, exchange every {EXCHANGE}, {iters} iterations per replica",
           "autotuned_warps_per_block": wpb, "autotune_trial_ms": tune_ms, "launch_shape": list(shape),
           "launch_classes": timed.classes,
           "batched": {"moves": moves, "ms": ms, "moves_per_sec": moves / (ms / 1e3)}}
    pm = pms = 0.0
    for (n, w) in UNEVEN:
        m, t, _ = timed([j for j in jobs if j["n"] == n], steps=1)
        pm += m
        pms += t
    out["one_order_per_launch"] = {"moves": pm, "ms": pms, "moves_per_sec": pm / (pms / 1e3)}
    return out


# ---------------------------------------------------------------- serving (C5)
SERVE_ORDERS = (12, 14, 18, 20, 24, 26, 30)
SERVE_RATE = 200.0
SERVE_REPLICAS = 256
SERVE_BUDGET = 10 ** 8


def serving_stream(count, seed=5, rate=SERVE_RATE):
    """The mixed request stream: Poisson arrivals at `rate` requests/s
    (seeded exponential gaps; 200/s is the workload's); 70% W(n, n-1) with
    n uniform in SERVE_ORDERS, 30% W(n, 4) with n uniform in 16..64; request
    k has seed 1000 + k."""
    import numpy as np
    rng = np.random.default_rng(seed)
    out, t = [], 0.0
    for k in range(count):
        t += rng.exponential(1.0 / rate)
        if rng.random() < 0.7:
            n = int(rng.choice(SERVE_ORDERS))
            w = n - 1
        else:
            n, w = int(rng.integers(16, 65)), 4
        out.append((t, n, w, 1000 + k))
    return out


def serve_stream(X, reqs, **cfg):
    """Submit `reqs` at their arrival times to a server, wait for all, and
    summarise time-to-exact (submission to first exact solution) and moves/s.
    Requests answered by Sylvester blocks (w a power of two dividing n) are
    counted apart and left out of both figures."""
    import numpy as np
    with X.Server(**cfg) as srv:
        t0 = time.perf_counter()
        ids = []
        for (ta, n, w, seed) in reqs:
            d = ta - (time.perf_counter() - t0)
            if d > 0:
                time.sleep(d)
            ids.append(srv.submit(n, w, seed, replicas=SERVE_REPLICAS, max_moves=SERVE_BUDGET))
        res = [srv.wait(i)[0] for i in ids]
        wall = time.perf_counter() - t0
        st = srv.stats()
    searched = [r for r in res if not r.sylvester]
    solved = [r for r in searched if r.solved]
    tte = np.array([r.time_to_solution_seconds for r in solved]) if solved else np.array([-1.0])
    moves = sum(r.moves for r in searched)
    failed = [r for r in res if r.state != X.REQ_DONE]
    per_request = [(bool(r.sylvester), bool(r.solved), r.time_to_solution_seconds) for r in res]
    return per_request, {
        "requests": len(reqs), "searched": len(searched), "sylvester": len(res) - len(searched),
        "solved": len(solved), "censored_at_budget": len(searched) - len(solved), "failed": len(failed),
        "all_solutions_verified": all(r.verified for r in solved),
        "time_to_exact_s": {"p50": float(np.percentile(tte, 50)), "p99": float(np.percentile(tte, 99)),
                            "mean": float(tte.mean())},
        "moves": moves, "wall_s": wall, "moves_per_sec": moves / wall,
        "device_s": st.device_seconds, "rounds": st.rounds,
        "config": {"quantum_iters": st.quantum_iters, "schedule": ["all", "least_attained"][st.schedule],
                   "max_active_replicas": st.max_active_replicas,
                   "max_resident_replicas": st.max_resident_replicas},
    }


def serve_reference_plain(reqs, cap_seconds):
    """The reference's plain kernel on the stream's first requests, one
    xweigh_cuda process per request (its one-instance-per-launch mode), 256
    replicas, at most `cap_seconds` of search each (it has no move budget),
    replayed live: each request arrives at its own time, waits while the
    process of an earlier one holds the GPU, and its time-to-exact runs from
    its arrival to the moment the process prints its `new best score=0`
    line (read as it is printed).  Requests the reference answers with
    Sylvester blocks are counted apart."""
    import numpy as np
    tte, moves, busy, solved, syl = [], 0, 0.0, 0, 0
    t0 = time.perf_counter()
    for (ta, n, w, seed) in reqs:
        wait = ta - (time.perf_counter() - t0)
        if wait > 0:
            time.sleep(wait)
        with tempfile.TemporaryDirectory() as td:
            ts = time.perf_counter()
            proc = subprocess.Popen(
                [REF_XWEIGH_CUDA, str(n), str(w), "--replicas", str(SERVE_REPLICAS), "--seed", str(seed),
                 "--max-seconds", str(cap_seconds), "--restart-interval", "0", "-o", os.path.join(td, "w.csv")],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True, bufsize=1)
            t_solve, lines = None, []
            for line in proc.stdout:
                lines.append(line)
                if t_solve is None and " new best score=0 " in line:
                    t_solve = time.perf_counter()
            proc.wait(timeout=cap_seconds * 4 + 120)
            busy += time.perf_counter() - ts
        out_text = "".join(lines)
        m = re.search(r"done moves=(\d+) ", out_text)
        moves += int(m.group(1)) if m else 0
        if t_solve is not None:
            solved += 1
            tte.append(t_solve - t0 - ta)
        elif "[construct] using direct sum of Sylvester blocks" in out_text:
            syl += 1
    t = np.array(tte) if tte else np.array([-1.0])
    return {"requests": len(reqs), "sylvester": syl, "solved": solved, "cap_seconds_per_request": cap_seconds,
            "time_to_exact_s": {"p50": float(np.percentile(t, 50)), "p99": float(np.percentile(t, 99))},
            "moves": moves, "busy_s": busy, "moves_per_sec": moves / busy if busy > 0 else 0.0,
            "arrivals": "live (real-time arrivals, one process at a time)",
            "impl": "reference xweigh_cuda (sm_100a build), one process per request"}


def tte_summary(per_request):
    """p50/p99 time-to-exact over the searched (not Sylvester) requests that solved."""
    import numpy as np
    t = np.array([x for syl, ok, x in per_request if ok and not syl] or [-1.0])
    return {"p50": float(np.percentile(t, 50)), "p99": float(np.percentile(t, 99)),
            "solved": int(sum(1 for syl, ok, _ in per_request if ok and not syl)),
            "searched": int(sum(1 for syl, _, _ in per_request if not syl))}


def serving_bench(X, count, plain_count, quantum, ref_count=0, ref_cap=3.0, light_count=0, light_rate=10.0):
    """The serving workload: the request stream through the continuous-
    batching server, and its first `plain_count` requests both served and
    one request at a time (resident cap of one request: the plain
    one-instance-per-launch mode), same kernel and budgets."""
    reqs = serving_stream(count)
    out = {"workload": f"{count} requests, Poisson {SERVE_RATE:g}/s; 70% W(n,n-1) n in {list(SERVE_ORDERS)}, "
                       f"30% W(n,4) n in 16..64; {SERVE_REPLICAS} replicas and a {SERVE_BUDGET:.0e}-move budget "
                       f"per request; time-to-exact from submission, Sylvester short-circuits excluded",
           "served": serve_stream(X, reqs, quantum_iters=quantum)[1]}
    per_pre = None
    if plain_count > 0:
        pre = reqs[:plain_count]
        out["prefix_requests"] = len(pre)
        per_pre, out["served_prefix"] = serve_stream(X, pre, quantum_iters=quantum)
        out["plain_prefix"] = serve_stream(X, pre, quantum_iters=quantum, schedule=X.SCHED_ALL,
                                           max_resident_replicas=SERVE_REPLICAS)[1]
    if light_count > 0:
        # the same mix at a rate the device keeps up with: time-to-exact is
        # then the engine's, not the queue's
        light = serving_stream(light_count, seed=9, rate=light_rate)
        out["unsaturated"] = dict(serve_stream(X, light, quantum_iters=quantum)[1], rate_per_s=light_rate)
    if ref_count > 0 and os.path.exists(REF_XWEIGH_CUDA):
        try:
            out["plain_reference"] = serve_reference_plain(reqs[:ref_count], ref_cap)
            if per_pre is not None and len(per_pre) >= ref_count:
                # the same first requests, served (from the prefix run)
                out["served_first_requests"] = dict(tte_summary(per_pre[:ref_count]), requests=ref_count)
        except Exception as e:  # noqa: BLE001 - report, do not fail the bench
            out["plain_reference"] = {"unavailable": str(e)[:200]}
    return out


def load_profile_figure(name):
    """A figure (`name = value`) of the committed ncu summary of this
    workload's anneal kernel, if any: DRAM bytes (read + write) per launch,
    issue-slot utilisation."""
    path = os.path.join(REPO, "profiles", "anneal_kernel_w26_tempering.md")
    try:
        with open(path) as f:
            m = re.search(name + r"\s*=\s*([0-9.]+)", f.read())
        return float(m.group(1)) if m else None
    except OSError:
        return None


def free_port():
    import socket
    with socket.socket(socket.AF_INET, socket.SOCK_STREAM) as sk:
        sk.bind(("127.0.0.1", 0))
        return sk.getsockname()[1]


def spawn_ranks(gpus):
    """`--gpus N` without a launcher: start N ranks of this script under
    torch.distributed.run on this node (one process per GPU) and return its
    exit status.  Under torchrun (WORLD_SIZE set) nothing is spawned."""
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", f"--nproc-per-node={gpus}",
           "--master-addr", "127.0.0.1", "--master-port", str(free_port()), os.path.abspath(__file__)] + sys.argv[1:]
    log(f"[bench] starting {gpus} ranks: {' '.join(cmd)}")
    return subprocess.call(cmd)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--e2e-steps", type=int, default=3)
    ap.add_argument("--cpu-seconds", type=float, default=10.0)
    ap.add_argument("--plain-seconds", type=float, default=8.0)
    ap.add_argument("--ref-seconds", type=float, default=10.0)
    ap.add_argument("--iters", type=int, default=ITERS, help="iterations per replica per step (profiling cases)")
    ap.add_argument("--rescore", type=int, default=1, help="also time the batched tensor-core rescoring")
    ap.add_argument("--rescore-orders", default="32,64,96,128", help="orders of that section (multiples of 32)")
    ap.add_argument("--c1", type=int, default=1, help="also time single-replica W(12,11) searches")
    ap.add_argument("--c1-ref-seconds", type=float, default=8.0,
                    help="wall seconds of single-thread reference runs beside them")
    ap.add_argument("--uneven-iters", type=int, default=20000,
                    help="iterations per replica of the uneven-orders batch (0: none)")
    ap.add_argument("--large-iters", type=int, default=4000,
                    help="iterations per replica of the W(276,275) large-order section (0: none)")
    ap.add_argument("--large-ref-seconds", type=float, default=6.0,
                    help="seconds of the reference's xweigh_cuda on that order")
    ap.add_argument("--serve-requests", type=int, default=400, help="requests of the serving stream (0: none)")
    ap.add_argument("--serve-plain", type=int, default=60,
                    help="prefix of the stream also run one request at a time")
    ap.add_argument("--serve-quantum", type=int, default=2000, help="iterations per replica per server round")
    ap.add_argument("--serve-reference", type=int, default=60,
                    help="requests of the stream also run by the reference's xweigh_cuda, one process each, "
                         "arriving live")
    ap.add_argument("--serve-reference-cap", type=float, default=2.0,
                    help="search seconds per request for the reference's xweigh_cuda")
    ap.add_argument("--serve-light", type=int, default=100,
                    help="requests of the same mix at an unsaturating rate (0: none)")
    ap.add_argument("--serve-light-rate", type=float, default=10.0, help="arrivals per second of that stream")
    args = ap.parse_args()
    if args.gpus > 1 and "WORLD_SIZE" not in os.environ:
        sys.exit(spawn_ranks(args.gpus))
    if args.warmup < 3:
        log("[bench] warmup raised to 3")
        args.warmup = 3
    if args.impl == "reference":
        reference_arm(args)
    else:
        ours(args)


if __name__ == "__main__":
    main()
