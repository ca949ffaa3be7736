"""xtax_b200 -- B200-native weighing-matrix population annealer.

Python view of the C ABI in include/xw.h (library: xtax_b200/libxw.so).
The names follow the reference's xweigh_cuda interface
(src/xweigh_cuda.hpp of flinty-mathematics/xtax): ``Params`` mirrors
``xweigh_cuda::Params``, ``query_device`` and ``run_annealer`` mirror the
functions of the same names, and ``RunResult`` mirrors ``RunResult``.
Errors raise ``XwError`` with the library's message, as the reference's
``std::runtime_error``s carry theirs.

There is no CPU fallback: every call goes through the CUDA library, and
importing this package fails loudly when libxw.so is missing.
"""
import ctypes as C
import os
from dataclasses import dataclass, field, fields
from typing import List, Optional

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libxw.so")
HEADER = os.path.join(os.path.dirname(_HERE), "include", "xw.h")

XW_OK, XW_ERR_INVALID, XW_ERR_CUDA, XW_ERR_CAPACITY, XW_ERR_INTERNAL = 0, 1, 2, 3, 4
XW_ERR_NOT_FOUND, XW_ERR_TIMEOUT, XW_ERR_IO = 5, 6, 7
# device error bits of a replica (xw_replica_state.error)
XW_DEVERR_SCORE, XW_DEVERR_MINORITY, XW_DEVERR_KERNEL, XW_DEVERR_CHUNK = 1, 2, 4, 8
MAX_ORDER_CUDA = 1024      # largest order the device path anneals
MAX_ORDER_SHARED = 256     # largest order whose replica state sits in shared memory (and served orders)
MAX_CANDIDATE_SAMPLES = 32
MAX_TARGET_SAMPLES = 64


class XwError(RuntimeError):
    def __init__(self, code, message):
        super().__init__(message)
        self.code = code


class _Params(C.Structure):
    _fields_ = [("device", C.c_int32), ("replicas", C.c_int32), ("moves_per_launch", C.c_int32),
                ("seed", C.c_uint64), ("max_seconds", C.c_double), ("save_interval", C.c_double),
                ("sign_fraction", C.c_double), ("double_sign_fraction", C.c_double),
                ("switch_sign_fraction", C.c_double), ("squared_objective_fraction", C.c_double),
                ("parity_objective_fraction", C.c_double), ("greedy_fraction", C.c_double),
                ("candidate_samples", C.c_int32), ("target_fraction", C.c_double),
                ("target_samples", C.c_int32), ("t_init", C.c_double), ("t_min", C.c_double),
                ("cooling", C.c_double), ("moves_per_cool", C.c_int32),
                ("stuck_threshold", C.c_int32), ("reheat", C.c_double),
                ("restart_interval", C.c_double), ("restart_fraction", C.c_double),
                ("restart_kick_min", C.c_int32), ("restart_kick_max", C.c_int32),
                ("max_moves", C.c_uint64), ("tempering", C.c_int32),
                ("exchange_interval", C.c_int32), ("objective", C.c_int32),
                ("move_set", C.c_int32), ("start_kind", C.c_int32), ("stop_on_solve", C.c_int32),
                ("warps_per_block", C.c_int32), ("replicas_per_warp", C.c_int32),
                ("warps_per_replica", C.c_int32), ("restart_kicks", C.c_int32)]


class _DeviceInfo(C.Structure):
    _fields_ = [("name", C.c_char * 256), ("ordinal", C.c_int32), ("compute_major", C.c_int32),
                ("compute_minor", C.c_int32), ("multiprocessors", C.c_int32),
                ("global_memory", C.c_uint64), ("max_shared_memory_per_block", C.c_uint64)]


class _Result(C.Structure):
    _fields_ = [("score", C.c_int64), ("conflicts", C.c_int64), ("replicas", C.c_int32),
                ("solved", C.c_int32), ("verified", C.c_int32), ("best_replica", C.c_int32),
                ("moves", C.c_uint64), ("candidate_evaluations", C.c_uint64),
                ("restarted_replicas", C.c_uint64), ("iterations", C.c_uint64),
                ("initialization_seconds", C.c_double), ("search_seconds", C.c_double),
                ("time_to_solution_seconds", C.c_double), ("device", _DeviceInfo)]


class JobSpec(C.Structure):
    """One search W(n,w) of a batch (xw_job_spec)."""
    _fields_ = [("n", C.c_int32), ("w", C.c_int32), ("seed", C.c_uint64), ("replicas", C.c_int32),
                ("reserved", C.c_int32), ("max_moves", C.c_uint64)]


class JobResult(C.Structure):
    _fields_ = [("score", C.c_int64), ("conflicts", C.c_int64), ("best_replica", C.c_int32),
                ("solved", C.c_int32), ("verified", C.c_int32), ("error", C.c_int32),
                ("moves", C.c_uint64), ("candidate_evaluations", C.c_uint64),
                ("iterations", C.c_uint64), ("solved_iteration", C.c_uint64),
                ("time_to_solution_seconds", C.c_double), ("accepted_moves", C.c_uint64),
                ("accepted_rows", C.c_uint64), ("two_row_evaluations", C.c_uint64)]


class ReplicaState(C.Structure):
    _fields_ = [("iterations", C.c_uint64), ("moves", C.c_uint64),
                ("candidate_evaluations", C.c_uint64), ("score", C.c_int64),
                ("conflicts", C.c_int64), ("best_score", C.c_int64),
                ("best_conflicts", C.c_int64), ("objective_total", C.c_int64),
                ("temperature", C.c_double), ("reheat_temperature", C.c_double),
                ("moves_since_improvement", C.c_int32), ("cooling_counter", C.c_int32),
                ("rung", C.c_int32), ("objective_kind", C.c_int32), ("status", C.c_uint32),
                ("error", C.c_uint32), ("accepted_moves", C.c_uint32), ("accepted_rows", C.c_uint32),
                ("two_row_evaluations", C.c_uint32), ("reserved", C.c_uint32)]


class LaunchClass(C.Structure):
    """xw_launch_class: one launch of a batch's round and its shape."""
    _fields_ = [("min_order", C.c_int32), ("max_order", C.c_int32), ("large", C.c_int32),
                ("rows_per_lane", C.c_int32), ("replicas_per_warp", C.c_int32),
                ("warps_per_block", C.c_int32), ("blocks", C.c_int32), ("slot_bytes", C.c_int32),
                ("chunks", C.c_int32), ("replicas", C.c_int32), ("general", C.c_int32),
                ("warps_per_replica", C.c_int32)]


class CpuParams(C.Structure):
    """xw_cpu_params: xweigh::Params of the CPU annealer."""
    _fields_ = [("threads", C.c_int32), ("tempering", C.c_int32), ("seed", C.c_uint64),
                ("max_seconds", C.c_double), ("save_interval", C.c_double), ("sign_fraction", C.c_double),
                ("greedy_fraction", C.c_double), ("candidate_samples", C.c_int32),
                ("target_fraction", C.c_double), ("target_samples", C.c_int32),
                ("exchange_interval", C.c_int32), ("t_init", C.c_double), ("t_min", C.c_double),
                ("cooling", C.c_double), ("moves_per_cool", C.c_int32), ("stuck_threshold", C.c_int32),
                ("reheat", C.c_double), ("reseed_factor", C.c_double)]


class CpuResult(C.Structure):
    _fields_ = [("score", C.c_int64), ("conflicts", C.c_int64), ("solved", C.c_int32), ("verified", C.c_int32),
                ("moves", C.c_uint64), ("seconds", C.c_double), ("t_init", C.c_double), ("threads", C.c_int32),
                ("reserved", C.c_int32)]


class ServerConfig(C.Structure):
    """xw_server_config: the serving loop's device, round length and capacities."""
    _fields_ = [("device", C.c_int32), ("quantum_iters", C.c_int32), ("max_requests", C.c_int32),
                ("max_resident_replicas", C.c_int32), ("max_replica_ids", C.c_int32),
                ("warps_per_block", C.c_int32), ("prep_threads", C.c_int32),
                ("sylvester_shortcut", C.c_int32), ("arena_bytes", C.c_uint64),
                ("schedule", C.c_int32), ("max_active_replicas", C.c_int32),
                ("replicas_per_warp", C.c_int32), ("reserved", C.c_int32 * 5)]


class _Request(C.Structure):
    _fields_ = [("n", C.c_int32), ("w", C.c_int32), ("seed", C.c_uint64), ("replicas", C.c_int32),
                ("reserved", C.c_int32), ("max_moves", C.c_uint64), ("params", C.POINTER(_Params)),
                ("starts", C.POINTER(C.c_int8))]


class RequestResult(C.Structure):
    """xw_request_result: state, outcome and timing of one served request."""
    _fields_ = [("state", C.c_int32), ("status", C.c_int32), ("n", C.c_int32), ("w", C.c_int32),
                ("replicas", C.c_int32), ("solved", C.c_int32), ("verified", C.c_int32),
                ("sylvester", C.c_int32), ("best_replica", C.c_int32), ("reserved", C.c_int32),
                ("score", C.c_int64), ("conflicts", C.c_int64), ("moves", C.c_uint64),
                ("candidate_evaluations", C.c_uint64), ("iterations", C.c_uint64),
                ("solved_iteration", C.c_uint64), ("submit_seconds", C.c_double),
                ("admit_seconds", C.c_double), ("finish_seconds", C.c_double),
                ("time_to_solution_seconds", C.c_double), ("t_init", C.c_double),
                ("error", C.c_char * 192)]


class ServerStats(C.Structure):
    _fields_ = [("submitted", C.c_uint64), ("admitted", C.c_uint64), ("finished", C.c_uint64),
                ("solved", C.c_uint64), ("cancelled", C.c_uint64), ("failed", C.c_uint64),
                ("sylvester", C.c_uint64), ("queued", C.c_uint64), ("running", C.c_uint64),
                ("resident_replicas", C.c_uint64), ("rounds", C.c_uint64), ("moves", C.c_uint64),
                ("device_seconds", C.c_double), ("busy_seconds", C.c_double),
                ("arena_bytes", C.c_uint64), ("arena_bytes_used", C.c_uint64),
                ("quantum_iters", C.c_int32), ("max_resident_replicas", C.c_int32),
                ("schedule", C.c_int32), ("max_active_replicas", C.c_int32)]


REQ_QUEUED, REQ_RUNNING, REQ_DONE, REQ_CANCELLED, REQ_FAILED = 0, 1, 2, 3, 4
SCHED_ALL, SCHED_LEAST_ATTAINED = 0, 1

class EscapeMove(C.Structure):
    """xw_escape_move: a support switch out of an elite state with its deltas."""
    _fields_ = [("row1", C.c_int32), ("row2", C.c_int32), ("col1", C.c_int32), ("col2", C.c_int32),
                ("new1", C.c_int32), ("new2", C.c_int32), ("score_delta", C.c_int64),
                ("conflict_delta", C.c_int64)]


LOG_FN = C.CFUNCTYPE(None, C.c_char_p, C.c_void_p)
CHECKPOINT_FN = C.CFUNCTYPE(None, C.POINTER(C.c_int8), C.c_int32, C.c_void_p)

_lib = None


def lib():
    """The loaded libxw.so (raises if the library was not built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: build it with `make -C xtax_b200/csrc`")
        L = C.CDLL(LIB_PATH)
        P = C.POINTER
        i32, u32, u64, i8 = C.c_int32, C.c_uint32, C.c_uint64, C.c_int8
        sig = {
            "xw_params_default": (None, [P(_Params)]),
            "xw_last_error": (C.c_char_p, []),
            "xw_validate_params": (i32, [i32, i32, P(_Params)]),
            "xw_query_device": (i32, [i32, P(_DeviceInfo)]),
            "xw_run": (i32, [i32, i32, P(_Params), P(i8), LOG_FN, CHECKPOINT_FN, C.c_void_p,
                             P(_Result), P(i8)]),
            "xw_request_stop": (None, []),
            "xw_clear_stop": (None, []),
            "xw_random_start": (i32, [i32, i32, u32, P(i8)]),
            "xw_row_start": (i32, [i32, i32, u64, u32, P(i8)]),
            "xw_sylvester": (i32, [i32, i32, P(i8)]),
            "xw_score": (i32, [i32, i32, P(i8), P(C.c_int64)]),
            "xw_verify": (i32, [i32, i32, P(i8)]),
            "xw_read_csv": (i32, [C.c_char_p, i32, i32, P(i8)]),
            "xw_write_csv": (i32, [C.c_char_p, i32, P(i8)]),
            "xw_impossibility_reason": (C.c_char_p, [i32, i32]),
            "xw_calibrate": (C.c_double, [i32, i32, P(i8), P(_Params), u32]),
            "xw_batch_create": (i32, [P(JobSpec), i32, P(_Params), P(i8), P(C.c_void_p)]),
            "xw_batch_set_stream": (i32, [C.c_void_p, C.c_void_p]),
            "xw_batch_reset": (i32, [C.c_void_p]),
            "xw_batch_run": (i32, [C.c_void_p, u64]),
            "xw_batch_run_timed": (i32, [C.c_void_p, u64]),
            "xw_batch_synchronize": (i32, [C.c_void_p]),
            "xw_batch_launch_times": (i32, [C.c_void_p, P(C.c_float), i32, P(i32)]),
            "xw_batch_results": (i32, [C.c_void_p, P(JobResult), P(i8)]),
            "xw_batch_read_replica": (i32, [C.c_void_p, i32, i32, P(ReplicaState), P(i8), P(i8),
                                            P(C.c_uint8)]),
            "xw_batch_shape": (i32, [C.c_void_p, P(i32), P(i32), P(i32)]),
            "xw_batch_classes": (i32, [C.c_void_p, P(LaunchClass), i32, P(i32)]),
            "xw_cpu_params_default": (None, [P(CpuParams)]),
            "xw_cpu_run": (i32, [i32, i32, P(CpuParams), P(i8), LOG_FN, CHECKPOINT_FN, C.c_void_p, P(CpuResult),
                                 P(i8)]),
            "xw_batch_restart": (i32, [C.c_void_p, i32, P(i32)]),
            "xw_batch_bytes": (i32, [C.c_void_p, P(u64), P(u64)]),
            "xw_batch_destroy": (None, [C.c_void_p]),
            "xw_batch_solve": (i32, [P(JobSpec), i32, P(_Params), P(i8), u64, P(JobResult), P(i8)]),
            "xw_anneal_noalloc": (i32, [i32, i32, P(_Params), i32, u64, C.c_void_p, C.c_void_p,
                                        C.c_void_p, C.c_void_p]),
            "xw_rescore": (i32, [P(i8), C.c_int64, i32, i32, P(i32), P(i32)]),
            "xw_rescore_device": (i32, [C.c_void_p, C.c_int64, i32, i32, C.c_void_p, C.c_void_p, i32,
                                        C.c_void_p]),
            "xw_rescore_status": (i32, []),
            "xw_autotune": (i32, [P(JobSpec), i32, P(_Params), u64, P(i32), P(C.c_float)]),
            "xw_batch_save": (i32, [C.c_void_p, C.c_char_p]),
            "xw_batch_load": (i32, [C.c_char_p, P(_Params), P(C.c_void_p)]),
            "xw_escape_scan": (i32, [i32, i32, P(i8), i32, P(EscapeMove), P(i32)]),
            "xw_server_config_default": (None, [P(ServerConfig)]),
            "xw_server_create": (i32, [P(ServerConfig), P(C.c_void_p)]),
            "xw_submit": (i32, [C.c_void_p, P(_Request), P(u64)]),
            "xw_poll": (i32, [C.c_void_p, u64, P(RequestResult), P(i8)]),
            "xw_wait": (i32, [C.c_void_p, u64, C.c_double, P(RequestResult), P(i8)]),
            "xw_cancel": (i32, [C.c_void_p, u64]),
            "xw_checkpoint": (i32, [C.c_void_p, u64, C.c_double, P(RequestResult), P(i8)]),
            "xw_request_save": (i32, [C.c_void_p, u64, C.c_char_p, C.c_double]),
            "xw_submit_snapshot": (i32, [C.c_void_p, C.c_char_p, P(u64)]),
            "xw_release": (i32, [C.c_void_p, u64]),
            "xw_server_get_stats": (i32, [C.c_void_p, P(ServerStats)]),
            "xw_server_destroy": (None, [C.c_void_p]),
        }
        for name, (res, args) in sig.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def _check(rc):
    if rc != XW_OK:
        raise XwError(rc, lib().xw_last_error().decode())


def _i8(a):
    return a.ctypes.data_as(C.POINTER(C.c_int8))


# ---- the reference interface -------------------------------------------------

@dataclass
class Params:
    """xweigh_cuda::Params (xweigh_cuda.hpp:14-44) plus extensions."""
    device: int = 0
    replicas: int = 0
    moves_per_launch: int = 4096
    seed: int = 0
    max_seconds: float = 0.0
    save_interval: float = 2.0
    output: str = "best_W.csv"
    sign_fraction: float = 0.5
    double_sign_fraction: float = 0.25
    switch_sign_fraction: float = 0.5
    squared_objective_fraction: float = 0.25
    parity_objective_fraction: float = 0.25
    greedy_fraction: float = 0.5
    candidate_samples: int = 4
    target_fraction: float = 0.7
    target_samples: int = 8
    t_init: float = 0.0
    t_min: float = 0.25
    cooling: float = 0.999
    moves_per_cool: int = 500
    stuck_threshold: int = 50000
    reheat: float = 1.0
    restart_interval: float = 5.0
    restart_fraction: float = 0.25
    restart_kick_min: int = 2
    restart_kick_max: int = 64
    max_moves: int = 0
    tempering: int = 0
    exchange_interval: int = 10000
    objective: int = -1
    move_set: int = 0
    start_kind: int = 0
    stop_on_solve: int = 1
    warps_per_block: int = 0
    replicas_per_warp: int = 0
    warps_per_replica: int = 0
    restart_kicks: int = 0

    def to_c(self):
        p = _Params()
        lib().xw_params_default(C.byref(p))
        for f in fields(self):
            if f.name != "output":
                setattr(p, f.name, getattr(self, f.name))
        return p


@dataclass
class DeviceInfo:
    name: str
    ordinal: int
    compute_major: int
    compute_minor: int
    multiprocessors: int
    global_memory: int
    max_shared_memory_per_block: int


@dataclass
class State:
    """The best matrix of a run: column-major int8 entries (State::entries)."""
    order: int
    weight: int
    entries: np.ndarray
    score: int
    conflicts: int

    def solved(self):
        return self.score == 0

    def matrix(self):
        """Row-major n x n view."""
        return self.entries.reshape(self.order, self.order).T.copy()


@dataclass
class RunResult:
    """xweigh_cuda::RunResult (xweigh_cuda.hpp:56-65) plus solve metadata."""
    best: State
    device: DeviceInfo
    replicas: int = 0
    moves: int = 0
    candidate_evaluations: int = 0
    restarted_replicas: int = 0
    initialization_seconds: float = 0.0
    search_seconds: float = 0.0
    solved: bool = False
    verified: bool = False
    time_to_solution_seconds: float = -1.0
    log: List[str] = field(default_factory=list)


def _device_info(d):
    return DeviceInfo(d.name.decode(), d.ordinal, d.compute_major, d.compute_minor,
                      d.multiprocessors, d.global_memory, d.max_shared_memory_per_block)


def query_device(ordinal: int = 0) -> DeviceInfo:
    """xweigh_cuda::query_device (xweigh_cuda.cu:1382-1417)."""
    d = _DeviceInfo()
    _check(lib().xw_query_device(ordinal, C.byref(d)))
    return _device_info(d)


def validate_params(order: int, weight: int, params: Params):
    _check(lib().xw_validate_params(order, weight, C.byref(params.to_c())))


def run_annealer(order: int, weight: int, params: Params,
                 initial_state: Optional[np.ndarray] = None, echo=False) -> RunResult:
    """xweigh_cuda::run_annealer (xweigh_cuda.cu:1419-2436)."""
    lines = []

    def on_log(line, _user):
        s = line.decode()
        lines.append(s)
        if echo:
            print(s, flush=True)

    log_cb = LOG_FN(on_log)
    ck_cb = CHECKPOINT_FN(lambda *_: None)
    res = _Result()
    best = np.zeros(order * order, dtype=np.int8)
    start = None
    if initial_state is not None:
        start = np.ascontiguousarray(initial_state, dtype=np.int8).reshape(-1)
    rc = lib().xw_run(order, weight, C.byref(params.to_c()), _i8(start) if start is not None else None,
                      log_cb, ck_cb, None, C.byref(res), _i8(best))
    _check(rc)
    return RunResult(State(order, weight, best, res.score, res.conflicts), _device_info(res.device),
                     res.replicas, res.moves, res.candidate_evaluations, res.restarted_replicas,
                     res.initialization_seconds, res.search_seconds, bool(res.solved),
                     bool(res.verified), res.time_to_solution_seconds, lines)


# ---- host helpers ----------------------------------------------------------------

def random_start(n, w, seed):
    out = np.zeros(n * n, dtype=np.int8)
    _check(lib().xw_random_start(n, w, seed & 0xffffffff, _i8(out)))
    return out


def row_start(n, w, seed, replica):
    out = np.zeros(n * n, dtype=np.int8)
    _check(lib().xw_row_start(n, w, seed, replica, _i8(out)))
    return out


def sylvester(n, w):
    out = np.zeros(n * n, dtype=np.int8)
    _check(lib().xw_sylvester(n, w, _i8(out)))
    return out


def score(n, w, W):
    W = np.ascontiguousarray(W, dtype=np.int8)
    st = np.zeros(4, dtype=np.int64)
    _check(lib().xw_score(n, w, _i8(W), st.ctypes.data_as(C.POINTER(C.c_int64))))
    return st


def verify(n, w, W):
    W = np.ascontiguousarray(W, dtype=np.int8)
    return lib().xw_verify(n, w, _i8(W))


def rescore(W_rowmajor, n, w, gram=False):
    """Batched exact W W^T (xw_rescore): W_rowmajor is (count, n, n) int8.
    Returns stats (count, 4) int32 {score, conflicts, squared, exact} and,
    with gram=True, G (count, n, n) int32."""
    W = np.ascontiguousarray(W_rowmajor, dtype=np.int8)
    count = W.size // (n * n)
    stats = np.zeros((count, 4), dtype=np.int32)
    G = np.zeros((count, n, n), dtype=np.int32) if gram else None
    _check(lib().xw_rescore(_i8(W), count, n, w, stats.ctypes.data_as(C.POINTER(C.c_int32)),
                            G.ctypes.data_as(C.POINTER(C.c_int32)) if gram else None))
    return (stats, G) if gram else stats


def impossibility_reason(n, w):
    return lib().xw_impossibility_reason(n, w).decode()


def philox_key(seed):
    """Philox key of a job: the reference's curand seed derivation
    (xweigh_cuda.cu:1724-1727) split into two 32-bit words."""
    base = seed & 0xffffffff
    k = ((base << 32) ^ seed ^ 0xd1b54a32d192ed03) & 0xffffffffffffffff
    return k & 0xffffffff, k >> 32


# ---- batches -------------------------------------------------------------------

class Batch:
    """A population of independent searches resident on one device."""

    def __init__(self, jobs, params: Params, starts: Optional[np.ndarray] = None):
        self.specs = (JobSpec * len(jobs))()
        for i, j in enumerate(jobs):
            s = self.specs[i]
            s.n, s.w, s.seed, s.replicas = j["n"], j["w"], j.get("seed", 1), j["replicas"]
            s.max_moves = j.get("max_moves", 0)
        self.jobs = [dict(j) for j in jobs]
        self.params = params
        h = C.c_void_p()
        st = None
        if starts is not None:
            st = np.ascontiguousarray(starts, dtype=np.int8).reshape(-1)
        _check(lib().xw_batch_create(self.specs, len(jobs), C.byref(params.to_c()),
                                     _i8(st) if st is not None else None, C.byref(h)))
        self.h = h

    def close(self):
        if getattr(self, "h", None):
            lib().xw_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()

    def save(self, path):
        """xw_batch_save: exact population snapshot (atomic write)."""
        _check(lib().xw_batch_save(self.h, os.fspath(path).encode()))

    @classmethod
    def load(cls, path, jobs, params: Optional[Params] = None):
        """xw_batch_load: a batch that continues from a snapshot.  `jobs` are
        the saved batch's job dicts (for result shapes); `params` (optional)
        replaces the run-time settings."""
        self = cls.__new__(cls)
        self.jobs = [dict(j) for j in jobs]
        self.params = params
        h = C.c_void_p()
        pc = params.to_c() if params is not None else None
        _check(lib().xw_batch_load(os.fspath(path).encode(), C.byref(pc) if pc is not None else None, C.byref(h)))
        self.h = h
        return self

    def set_stream(self, stream_ptr):
        _check(lib().xw_batch_set_stream(self.h, C.c_void_p(stream_ptr)))

    def reset(self):
        _check(lib().xw_batch_reset(self.h))

    def run(self, iters):
        _check(lib().xw_batch_run(self.h, iters))

    def run_timed(self, iters):
        _check(lib().xw_batch_run_timed(self.h, iters))

    def synchronize(self):
        _check(lib().xw_batch_synchronize(self.h))

    def launch_times(self):
        cap = 4096
        ms = (C.c_float * cap)()
        cnt = C.c_int32()
        _check(lib().xw_batch_launch_times(self.h, ms, cap, C.byref(cnt)))
        return [ms[i] for i in range(min(cnt.value, cap))]

    def shape(self):
        a, b, c = C.c_int32(), C.c_int32(), C.c_int32()
        _check(lib().xw_batch_shape(self.h, C.byref(a), C.byref(b), C.byref(c)))
        return a.value, b.value, c.value

    def restart(self, job=0):
        """xw_batch_restart: one elite restart of `job`; returns the number of
        replicas restarted."""
        n = C.c_int32()
        _check(lib().xw_batch_restart(self.h, job, C.byref(n)))
        return n.value

    def classes(self):
        """The launches of a round, one dict per launch class (xw_batch_classes)."""
        arr = (LaunchClass * 16)()
        n = C.c_int32()
        _check(lib().xw_batch_classes(self.h, arr, 16, C.byref(n)))
        return [{f: getattr(arr[i], f) for f, _ in LaunchClass._fields_} for i in range(min(n.value, 16))]

    def transfer_bytes(self):
        """(host-to-device bytes at creation, device-to-host bytes per results())"""
        a, b = C.c_uint64(), C.c_uint64()
        _check(lib().xw_batch_bytes(self.h, C.byref(a), C.byref(b)))
        return a.value, b.value

    def results(self):
        res = (JobResult * len(self.jobs))()
        total = sum(j["n"] * j["n"] for j in self.jobs)
        best = np.zeros(total, dtype=np.int8)
        _check(lib().xw_batch_results(self.h, res, _i8(best)))
        out, off = [], 0
        for j, r in zip(self.jobs, res):
            nn = j["n"] * j["n"]
            out.append((r, best[off:off + nn].copy()))
            off += nn
        return out

    def replica(self, job, r):
        n, w = self.jobs[job]["n"], self.jobs[job]["w"]
        m = min(w, n - w)
        st = ReplicaState()
        W = np.zeros(n * n, dtype=np.int8)
        B = np.zeros(n * n, dtype=np.int8)
        # minority lists are u8 up to the shared-memory orders, u16 above
        M = np.zeros(max(n * m, 1), dtype=np.uint8 if n <= MAX_ORDER_SHARED else np.uint16)
        _check(lib().xw_batch_read_replica(self.h, job, r, C.byref(st), _i8(W), _i8(B),
                                           M.ctypes.data_as(C.POINTER(C.c_uint8))))
        return st, W, B, M[: n * m]


def _specs(jobs):
    specs = (JobSpec * len(jobs))()
    for i, j in enumerate(jobs):
        specs[i].n, specs[i].w, specs[i].seed, specs[i].replicas = j["n"], j["w"], j.get("seed", 1), j["replicas"]
        specs[i].max_moves = j.get("max_moves", 0)
    return specs


def batch_solve(jobs, params: Params, starts=None, iters=0):
    """xw_batch_solve: upload, run, read back through host buffers."""
    specs = _specs(jobs)
    res = (JobResult * len(jobs))()
    best = np.zeros(sum(j["n"] * j["n"] for j in jobs), dtype=np.int8)
    st = None if starts is None else np.ascontiguousarray(starts, dtype=np.int8).reshape(-1)
    _check(lib().xw_batch_solve(specs, len(jobs), C.byref(params.to_c()),
                                _i8(st) if st is not None else None, iters, res, _i8(best)))
    return list(res), best


class Server:
    """A continuous-batching request loop on one device (xw_server_*).

    ``submit`` queues one W(n,w) search and returns its id; ``wait`` and
    ``poll`` return ``(RequestResult, W)`` with W the column-major int8 best
    matrix once the request has finished (else None)."""

    def __init__(self, device=0, **config):
        cfg = ServerConfig()
        lib().xw_server_config_default(C.byref(cfg))
        cfg.device = device
        for k, v in config.items():
            setattr(cfg, k, v)
        h = C.c_void_p()
        _check(lib().xw_server_create(C.byref(cfg), C.byref(h)))
        self.h = h
        self._orders = {}

    def submit(self, n, w, seed, replicas=256, max_moves=0, params: Optional[Params] = None, starts=None):
        r = _Request()
        r.n, r.w, r.seed, r.replicas, r.max_moves = n, w, seed, replicas, max_moves
        pc = params.to_c() if params is not None else None
        r.params = C.pointer(pc) if pc is not None else None
        st = None
        if starts is not None:
            st = np.ascontiguousarray(starts, dtype=np.int8).reshape(-1)
            if st.size != replicas * n * n:
                raise ValueError("starts must hold replicas*n*n entries")
            r.starts = _i8(st)
        rid = C.c_uint64()
        _check(lib().xw_submit(self.h, C.byref(r), C.byref(rid)))
        self._orders[rid.value] = n
        return rid.value

    def _out(self, rid, res, W):
        return res, (W if res.state >= REQ_DONE else None)

    def poll(self, rid):
        res = RequestResult()
        n = self._orders.get(rid, MAX_ORDER_SHARED)
        W = np.zeros(n * n, dtype=np.int8)
        _check(lib().xw_poll(self.h, rid, C.byref(res), _i8(W)))
        return self._out(rid, res, W)

    def wait(self, rid, timeout=-1.0):
        res = RequestResult()
        n = self._orders.get(rid, MAX_ORDER_SHARED)
        W = np.zeros(n * n, dtype=np.int8)
        _check(lib().xw_wait(self.h, rid, float(timeout), C.byref(res), _i8(W)))
        return self._out(rid, res, W)

    def checkpoint(self, rid, timeout=-1.0):
        """xw_checkpoint: (result, best W so far) at the end of the request's
        next round; a finished request's final result and W."""
        res = RequestResult()
        n = self._orders.get(rid, MAX_ORDER_SHARED)
        W = np.zeros(n * n, dtype=np.int8)
        _check(lib().xw_checkpoint(self.h, rid, float(timeout), C.byref(res), _i8(W)))
        return res, W

    def save(self, rid, path, timeout=-1.0):
        """xw_request_save: exact snapshot of a running request's population."""
        _check(lib().xw_request_save(self.h, rid, os.fspath(path).encode(), float(timeout)))

    def submit_snapshot(self, path):
        """xw_submit_snapshot: continue a one-job snapshot as a new request."""
        rid = C.c_uint64()
        _check(lib().xw_submit_snapshot(self.h, os.fspath(path).encode(), C.byref(rid)))
        res = RequestResult()
        _check(lib().xw_poll(self.h, rid.value, C.byref(res), None))
        self._orders[rid.value] = res.n
        return rid.value

    def cancel(self, rid):
        _check(lib().xw_cancel(self.h, rid))

    def release(self, rid):
        _check(lib().xw_release(self.h, rid))
        self._orders.pop(rid, None)

    def stats(self):
        st = ServerStats()
        _check(lib().xw_server_get_stats(self.h, C.byref(st)))
        return st

    def close(self):
        if getattr(self, "h", None):
            lib().xw_server_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:  # noqa: BLE001 - interpreter shutdown
            pass


def autotune(jobs, params: Params, iters=2000):
    """xw_autotune: the fastest warps per CTA for this batch shape, recorded
    in the tuning cache; returns (warps_per_block, device ms)."""
    specs = _specs(jobs)
    wpb, ms = C.c_int32(), C.c_float()
    _check(lib().xw_autotune(specs, len(jobs), C.byref(params.to_c()), iters, C.byref(wpb), C.byref(ms)))
    return wpb.value, ms.value


def cpu_run(n, w, start=None, log=None, **params):
    """xw_cpu_run: the CPU annealer (the reference's xweigh engine) with
    xweigh::Params fields as keywords; returns (CpuResult, best W
    column-major)."""
    p = CpuParams()
    lib().xw_cpu_params_default(C.byref(p))
    for k, v in params.items():
        setattr(p, k, v)
    best = np.zeros(n * n, dtype=np.int8)
    st = None if start is None else np.ascontiguousarray(start, dtype=np.int8).reshape(-1)
    lines = []
    cb = LOG_FN(lambda line, _u: (log or lines.append)(line.decode()))
    res = CpuResult()
    _check(lib().xw_cpu_run(n, w, C.byref(p), None if st is None else _i8(st), cb, CHECKPOINT_FN(0), None,
                            C.byref(res), _i8(best)))
    return res, best


def escape_scan(n, w, W_colmajor, limit):
    """xw_escape_scan: the `limit` best support switches out of W, as tuples
    (row1, row2, col1, col2, new1, new2, score_delta, conflict_delta)."""
    W = np.ascontiguousarray(W_colmajor, dtype=np.int8).reshape(-1)
    out = (EscapeMove * max(limit, 1))()
    cnt = C.c_int32()
    _check(lib().xw_escape_scan(n, w, _i8(W), limit, out, C.byref(cnt)))
    return [(m.row1, m.row2, m.col1, m.col2, m.new1, m.new2, m.score_delta, m.conflict_delta)
            for m in out[:cnt.value]]


def header_symbols(path=HEADER):
    """Function names declared in the public C header."""
    import re
    text = open(path).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(xw_[a-z0-9_]+)\s*\(", text)) - {"xw_log_fn", "xw_checkpoint_fn"})
