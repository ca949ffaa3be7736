"""The allocation-free entry point, xw_anneal_noalloc, against the batch engine.

xw_anneal_noalloc serves callers that cannot call cudaMalloc (device memory
owned by their own pool allocator or a fixed budget; loops that cannot take
the device synchronisation cudaMalloc/cudaFree imply).  It keeps its scratch
in a static device array instead.  Here it is called through the C ABI with
device buffers the test owns, twice in a row on the same inputs, and each
call's outputs must equal the existing batch entry point's: every replica's
best state and its best score, best conflicts, score and move count.  The
work is integer, so the tolerance is zero.  Two more cases: a start state
the kernel refuses must not read as solved, and a call must leave the
anneal kernel's shared-memory limit where a batch of a larger slot needs it.
The file is collected last only so that a run stopping at its first failure
has run every other test first; each test here stands alone.
"""
import ctypes as C

import numpy as np
import pytest

import xtax_b200 as X

pytestmark = pytest.mark.gpu


def _run_noalloc(torch, n, w, p, R, iters, d_starts, d_best, d_stats):
    rc = X.lib().xw_anneal_noalloc(n, w, C.byref(p.to_c()), R, iters, C.c_void_p(d_starts.data_ptr()),
                                   C.c_void_p(d_best.data_ptr()), C.c_void_p(d_stats.data_ptr()), None)
    assert rc == X.XW_OK, X.lib().xw_last_error().decode()
    torch.cuda.synchronize()
    return d_best.cpu().numpy().reshape(R, n * n), d_stats.cpu().numpy().reshape(R, 4)


@pytest.mark.parametrize("n,w,R,iters,kw", [
    (26, 25, 64, 3000, dict(t_init=4.0, moves_per_launch=1000)),
    (16, 4, 32, 2000, dict(t_init=2.0, tempering=1, exchange_interval=500, t_min=0.1)),
])
def test_noalloc_matches_batch_engine_on_two_calls(n, w, R, iters, kw):
    torch = pytest.importorskip("torch")
    seed = 4242 + n
    p = X.Params(seed=seed, stop_on_solve=0, **kw)
    starts = np.concatenate([X.random_start(n, w, (seed + r * 0x9e3779b9) & 0xffffffff) for r in range(R)])

    batch = X.Batch([{"n": n, "w": w, "seed": seed, "replicas": R}], p, starts=starts)
    batch.run(iters)
    batch.synchronize()
    ref_best, ref_stats = [], []
    for r in range(R):
        st, _, B, _ = batch.replica(0, r)
        ref_best.append(B)
        ref_stats.append((st.best_score, st.best_conflicts, st.score, st.moves))
    batch.close()

    dev = torch.device("cuda:0")
    d_starts = torch.from_numpy(starts).to(dev)
    d_best = torch.zeros(R * n * n, dtype=torch.int8, device=dev)
    d_stats = torch.zeros(R * 4, dtype=torch.int64, device=dev)
    for _ in range(2):
        d_best.fill_(0)
        d_stats.fill_(-1)
        torch.cuda.synchronize()
        best, stats = _run_noalloc(torch, n, w, p, R, iters, d_starts, d_best, d_stats)
        for r in range(R):
            assert (best[r] == ref_best[r]).all(), r
            assert tuple(int(x) for x in stats[r]) == ref_stats[r], r


def test_noalloc_rejects_requests_beyond_its_scratch():
    torch = pytest.importorskip("torch")
    dev = torch.device("cuda:0")
    n, w = 64, 4
    R = 2000   # 2000 records of W(64,4) need about 17 MB
    buf = torch.zeros(16, dtype=torch.int8, device=dev)
    stats = torch.zeros(4, dtype=torch.int64, device=dev)
    p = X.Params(seed=1, t_init=2.0)
    rc = X.lib().xw_anneal_noalloc(n, w, C.byref(p.to_c()), R, 1000, C.c_void_p(buf.data_ptr()),
                                   C.c_void_p(buf.data_ptr()), C.c_void_p(stats.data_ptr()), None)
    assert rc == X.XW_ERR_CAPACITY
    assert "static scratch holds 4194304 bytes" in X.lib().xw_last_error().decode()
    p0 = X.Params(seed=1, t_init=0.0)
    rc = X.lib().xw_anneal_noalloc(n, w, C.byref(p0.to_c()), 4, 1000, C.c_void_p(buf.data_ptr()),
                                   C.c_void_p(buf.data_ptr()), C.c_void_p(stats.data_ptr()), None)
    assert rc == X.XW_ERR_INVALID


def test_noalloc_refused_start_reports_an_error_not_a_solve():
    torch = pytest.importorskip("torch")
    n, w, R = 12, 11, 4
    starts = np.concatenate([X.random_start(n, w, 99 + r) for r in range(R)]).reshape(R, n, n).copy()
    # replica 2: column-major W, so row 0's entries are starts[2][:, 0];
    # one more zero gives that row weight w - 1
    col = int(np.flatnonzero(starts[2][:, 0])[0])
    starts[2][col, 0] = 0
    dev = torch.device("cuda:0")
    d_starts = torch.from_numpy(starts.reshape(-1)).to(dev)
    d_best = torch.zeros(R * n * n, dtype=torch.int8, device=dev)
    d_stats = torch.zeros(R * 4, dtype=torch.int64, device=dev)
    p = X.Params(seed=5, t_init=2.0, moves_per_launch=500, stop_on_solve=0)
    _, stats = _run_noalloc(torch, n, w, p, R, 1000, d_starts, d_best, d_stats)
    assert tuple(int(x) for x in stats[2][:3]) == (-1, -2, -1)   # XW_ERR_MINORITY = 2
    for r in (0, 1, 3):
        assert stats[r][0] >= 0 and stats[r][2] >= 0


def test_noalloc_call_leaves_a_larger_batch_launchable():
    torch = pytest.importorskip("torch")
    # the batch's CTA holds 16 warp slots of W(30,29); the noalloc call runs
    # the same kernel with four slots of W(12,11) in between
    jobs = [{"n": 30, "w": 29, "seed": 11 + k, "replicas": 16} for k in range(4)]
    p = X.Params(seed=11, t_init=3.0, moves_per_launch=1000, stop_on_solve=0, warps_per_block=16,
                 warps_per_replica=1, squared_objective_fraction=0.0, parity_objective_fraction=0.0)

    def run(with_noalloc):
        b = X.Batch(jobs, p)
        if with_noalloc:
            n, w, R = 12, 11, 4
            q = X.Params(seed=3, t_init=2.0, moves_per_launch=500, stop_on_solve=0, warps_per_block=4,
                         squared_objective_fraction=0.0, parity_objective_fraction=0.0)
            st = np.concatenate([X.random_start(n, w, 7 + r) for r in range(R)])
            dev = torch.device("cuda:0")
            _run_noalloc(torch, n, w, q, R, 1000, torch.from_numpy(st).to(dev),
                         torch.zeros(R * n * n, dtype=torch.int8, device=dev),
                         torch.zeros(R * 4, dtype=torch.int64, device=dev))
        b.run(2000)
        b.synchronize()
        out = [(r.score, r.moves, r.error) for r, _ in b.results()]
        b.close()
        return out

    plain = run(False)
    assert all(e == 0 for _, _, e in plain)
    assert run(True) == plain
