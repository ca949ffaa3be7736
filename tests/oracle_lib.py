"""ctypes view of oracle/liboracle.so, the CPU checker the tests compare with.

Test infrastructure: only tests/, __graft_entry__.smoke() and bench.py's
cpu_baseline leg use this module.
"""
import ctypes as C
import os

import numpy as np

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB_PATH = os.path.join(REPO, "oracle", "liboracle.so")


class RefParams(C.Structure):
    _fields_ = [("sign_fraction", C.c_double), ("greedy_fraction", C.c_double),
                ("target_fraction", C.c_double), ("candidate_samples", C.c_int32),
                ("target_samples", C.c_int32), ("t_init", C.c_double), ("t_min", C.c_double),
                ("cooling", C.c_double), ("reheat", C.c_double), ("reseed_factor", C.c_double),
                ("moves_per_cool", C.c_int32), ("stuck_threshold", C.c_int32)]


class WalkResult(C.Structure):
    _fields_ = [("moves", C.c_int64), ("accepted", C.c_int64), ("score", C.c_int64),
                ("conflicts", C.c_int64), ("best_score", C.c_int64),
                ("best_conflicts", C.c_int64), ("initial_temperature", C.c_double),
                ("temperature", C.c_double), ("worker_seed", C.c_uint32),
                ("hash", C.c_uint64)]


class Job(C.Structure):
    _fields_ = [("n", C.c_int32), ("w", C.c_int32), ("tempering", C.c_int32),
                ("move_set", C.c_int32), ("candidate_samples", C.c_int32),
                ("target_samples", C.c_int32), ("moves_per_cool", C.c_int32),
                ("stuck_threshold", C.c_int32), ("key0", C.c_uint32), ("key1", C.c_uint32),
                ("objective", C.c_int32), ("pad_", C.c_int32),
                ("greedy_fraction", C.c_double), ("target_fraction", C.c_double),
                ("double_sign_fraction", C.c_double), ("sign_fraction", C.c_double),
                ("switch_sign_fraction", C.c_double),
                ("squared_objective_fraction", C.c_double),
                ("parity_objective_fraction", C.c_double),
                ("t_min", C.c_double), ("cooling", C.c_double), ("reheat", C.c_double)]


class RepScalars(C.Structure):
    _fields_ = [("it", C.c_uint64), ("moves", C.c_uint64), ("cand_evals", C.c_uint64),
                ("score", C.c_int64), ("conflicts", C.c_int64), ("obj_total", C.c_int64),
                ("best_score", C.c_int64), ("best_conflicts", C.c_int64),
                ("temperature", C.c_double), ("reheat_temperature", C.c_double),
                ("msi", C.c_int32), ("cool_ctr", C.c_int32), ("rung", C.c_int32),
                ("obj_kind", C.c_int32)]


_lib = None


def lib():
    global _lib
    if _lib is None:
        L = C.CDLL(LIB_PATH)
        P = C.POINTER
        L.xwo_philox4x32_10.argtypes = [P(C.c_uint32), P(C.c_uint32), P(C.c_uint32)]
        L.xwo_mt_stream.argtypes = [C.c_uint32, C.c_int, P(C.c_uint32)]
        L.xwo_mt_uniform_stream.argtypes = [C.c_uint32, C.c_uint32, C.c_int, P(C.c_uint32)]
        L.xwo_mt_canonical_stream.argtypes = [C.c_uint32, C.c_int, P(C.c_double)]
        L.xwo_exp.argtypes = [C.c_double]
        L.xwo_exp.restype = C.c_double
        L.xwo_random_start.argtypes = [C.c_int, C.c_int, C.c_uint32, P(C.c_int8)]
        L.xwo_sylvester.argtypes = [C.c_int, C.c_int, P(C.c_int8)]
        L.xwo_row_start.argtypes = [C.c_int, C.c_int, C.c_uint32, C.c_uint32, C.c_uint32, P(C.c_int8)]
        L.xwo_rescore.argtypes = [C.c_int, C.c_int, P(C.c_int8), P(C.c_int64), P(C.c_int64), P(C.c_int64)]
        L.xwo_verify.argtypes = [C.c_int, C.c_int, P(C.c_int8)]
        L.xwo_verify.restype = C.c_int
        L.xwo_ref_params_default.argtypes = [P(RefParams)]
        L.xwo_calibrate.argtypes = [C.c_int, C.c_int, C.c_uint32, P(RefParams)]
        L.xwo_calibrate.restype = C.c_double
        L.xwo_ref_walk.argtypes = [C.c_int, C.c_int, C.c_uint32, C.c_int64, P(RefParams),
                                   P(WalkResult), P(C.c_int8), P(C.c_int8), P(C.c_int8)]
        L.xwo_rep_create.argtypes = [P(Job), C.c_uint32, P(C.c_int8), C.c_double, C.c_int32]
        L.xwo_rep_create.restype = C.c_void_p
        L.xwo_rep_destroy.argtypes = [C.c_void_p]
        L.xwo_rep_run.argtypes = [C.c_void_p, C.c_int64, C.c_int]
        L.xwo_rep_run.restype = C.c_int64
        L.xwo_rep_get.argtypes = [C.c_void_p, P(RepScalars), P(C.c_int8), P(C.c_int8),
                                  P(C.c_uint16), P(C.c_int32), P(C.c_int32)]
        L.xwo_rep_set_temperature.argtypes = [C.c_void_p, C.c_double, C.c_int32]
        L.xwo_rep_check.argtypes = [C.c_void_p]
        L.xwo_rep_check.restype = C.c_int
        L.xwo_exchange.argtypes = [P(Job), P(C.c_void_p), C.c_int, P(C.c_double), C.c_uint64]
        L.xwo_exchange.restype = C.c_int
        L.xwo_kick.argtypes = [C.c_int, C.c_int, P(C.c_int8), P(C.c_int32), C.c_uint32, C.c_uint32, C.c_uint64,
                               C.c_uint32, C.c_uint32, C.c_int, C.c_uint64, P(C.c_int8)]
        _lib = L
    return _lib


def ptr(a, ctype):
    return a.ctypes.data_as(C.POINTER(ctype))


def philox(ctr, key):
    c = np.array(ctr, dtype=np.uint32)
    k = np.array(key, dtype=np.uint32)
    o = np.zeros(4, dtype=np.uint32)
    lib().xwo_philox4x32_10(ptr(c, C.c_uint32), ptr(k, C.c_uint32), ptr(o, C.c_uint32))
    return [int(x) for x in o]


def random_start(n, w, seed):
    W = np.zeros(n * n, dtype=np.int8)
    lib().xwo_random_start(n, w, seed & 0xffffffff, ptr(W, C.c_int8))
    return W


def row_start(n, w, key0, key1, stream):
    W = np.zeros(n * n, dtype=np.int8)
    lib().xwo_row_start(n, w, key0, key1, stream, ptr(W, C.c_int8))
    return W


def sylvester(n, w):
    W = np.zeros(n * n, dtype=np.int8)
    lib().xwo_sylvester(n, w, ptr(W, C.c_int8))
    return W


def rescore(n, w, W):
    W = np.ascontiguousarray(W, dtype=np.int8)
    st = np.zeros(4, dtype=np.int64)
    G = np.zeros(n * n, dtype=np.int64)
    res = np.zeros(n, dtype=np.int64)
    lib().xwo_rescore(n, w, ptr(W, C.c_int8), ptr(st, C.c_int64), ptr(G, C.c_int64),
                      ptr(res, C.c_int64))
    return st, G.reshape(n, n), res


def verify(n, w, W):
    W = np.ascontiguousarray(W, dtype=np.int8)
    return lib().xwo_verify(n, w, ptr(W, C.c_int8))


def ref_params(**kw):
    p = RefParams()
    lib().xwo_ref_params_default(C.byref(p))
    for k, v in kw.items():
        setattr(p, k, v)
    return p


def ref_walk(n, w, seed, max_moves, **kw):
    p = ref_params(**kw)
    r = WalkResult()
    s = np.zeros(n * n, dtype=np.int8)
    f = np.zeros(n * n, dtype=np.int8)
    b = np.zeros(n * n, dtype=np.int8)
    lib().xwo_ref_walk(n, w, seed, max_moves, C.byref(p), C.byref(r), ptr(s, C.c_int8),
                       ptr(f, C.c_int8), ptr(b, C.c_int8))
    return r, s, f, b


def make_job(n, w, **kw):
    """Device-algorithm job with the reference xweigh_cuda defaults
    (xweigh_cuda.hpp:14-44)."""
    j = Job()
    j.n, j.w = n, w
    j.tempering = 0
    j.move_set = 0
    j.candidate_samples = 4
    j.target_samples = 8
    j.moves_per_cool = 500
    j.stuck_threshold = 50000
    j.key0, j.key1 = 0x12345678, 0x9abcdef0
    j.objective = -1
    j.greedy_fraction = 0.5
    j.target_fraction = 0.7
    j.double_sign_fraction = 0.25
    j.sign_fraction = 0.5
    j.switch_sign_fraction = 0.5
    j.squared_objective_fraction = 0.25
    j.parity_objective_fraction = 0.25
    j.t_min = 0.25
    j.cooling = 0.999
    j.reheat = 1.0
    for k, v in kw.items():
        setattr(j, k, v)
    return j


class Replica:
    def __init__(self, job, index, W0, t0, rung=0):
        self.job = job
        self.n = job.n
        self.w = job.w
        W0 = np.ascontiguousarray(W0, dtype=np.int8)
        self.h = lib().xwo_rep_create(C.byref(job), index, ptr(W0, C.c_int8), t0, rung)
        if not self.h:
            raise ValueError("bad replica start")

    def __del__(self):
        if getattr(self, "h", None):
            lib().xwo_rep_destroy(self.h)
            self.h = None

    def run(self, iters, stop_on_solve=True):
        return lib().xwo_rep_run(self.h, iters, 1 if stop_on_solve else 0)

    def set_temperature(self, t, rung):
        lib().xwo_rep_set_temperature(self.h, t, rung)

    def check(self):
        return lib().xwo_rep_check(self.h)

    def get(self):
        n = self.n
        m = min(self.w, n - self.w)
        s = RepScalars()
        W = np.zeros(n * n, dtype=np.int8)
        B = np.zeros(n * n, dtype=np.int8)
        M = np.zeros(max(n * m, 1), dtype=np.uint16)
        G = np.zeros(n * n, dtype=np.int32)
        R = np.zeros(n, dtype=np.int32)
        lib().xwo_rep_get(self.h, C.byref(s), ptr(W, C.c_int8), ptr(B, C.c_int8),
                          ptr(M, C.c_uint16), ptr(G, C.c_int32), ptr(R, C.c_int32))
        return s, W, B, M[: n * m], G.reshape(n, n), R


def exchange(job, reps, ladder, rnd):
    arr = (C.c_void_p * len(reps))(*[r.h for r in reps])
    lad = np.ascontiguousarray(ladder, dtype=np.float64)
    return lib().xwo_exchange(C.byref(job), arr, len(reps), ptr(lad, C.c_double), rnd)


def kick(n, w, E, esc, key0, key1, rnd, replica, index, steps, thr_sign):
    """The device kick of an elite restart (restart mode 1) of replica
    `replica`, the index-th restarted in round `rnd`, from elite E
    (column-major); esc = (row1, row2, col1, col2, new1, new2) or None."""
    E = np.ascontiguousarray(E, dtype=np.int8).reshape(-1)
    K = np.zeros(n * n, dtype=np.int8)
    e = None if esc is None else np.ascontiguousarray(esc[:6], dtype=np.int32)
    lib().xwo_kick(n, w, ptr(E, C.c_int8), None if e is None else ptr(e, C.c_int32), key0, key1, rnd, replica,
                   index, steps, thr_sign, ptr(K, C.c_int8))
    return K
