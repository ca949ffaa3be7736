"""Chunked launches: more replicas than resident warps.

A batch whose replicas outnumber the device's resident warps splits each
replica's iterations per launch into consecutive chunks, scheduled
chunk-major (a chunk waits for its replica's previous one), so that the last
wave of a launch is not part-filled.  Each replica still runs its iterations
in order, so every replica state is identical whatever the chunk count
(XW_CHUNKS forces one), and the oracle replays them.
"""
import pytest

import oracle_lib as O
import xtax_b200 as X
from test_gpu_parity import compare, oracle_job, start_of

pytestmark = pytest.mark.gpu


def run_states(monkeypatch, chunks, jobs, p, iters):
    if chunks is None:
        monkeypatch.delenv("XW_CHUNKS", raising=False)
    else:
        monkeypatch.setenv("XW_CHUNKS", str(chunks))
    b = X.Batch(jobs, p)
    b.run(iters)
    b.synchronize()
    states = []
    for j, jb in enumerate(jobs):
        for r in range(jb["replicas"]):
            st, W, B, M = b.replica(j, r)
            assert st.error == 0
            states.append((st.iterations, st.moves, st.candidate_evaluations, st.score, st.conflicts,
                           st.best_score, st.best_conflicts, st.objective_total, st.temperature, st.rung,
                           W.tobytes(), B.tobytes(), M.tobytes()))
    results = [(r.score, r.conflicts, r.best_replica, r.moves) for r, _ in b.results()]
    b.close()
    return states, results


@pytest.mark.parametrize("tempering", [0, 1])
def test_chunked_launches_leave_every_replica_unchanged(monkeypatch, tempering):
    # 3600 replicas: more than the 2368 resident warps of a B200 for these orders
    jobs = [{"n": 12, "w": 11, "seed": 40 + k, "replicas": 16} for k in range(150)] + \
           [{"n": 14, "w": 7, "seed": 900 + k, "replicas": 16} for k in range(75)]
    if tempering:
        p = X.Params(stop_on_solve=0, tempering=1, exchange_interval=400, t_min=0.1, t_init=6.0,
                     squared_objective_fraction=0.0, parity_objective_fraction=0.0)
    else:
        p = X.Params(stop_on_solve=0, t_init=4.0, moves_per_launch=400, stuck_threshold=300, moves_per_cool=40)
    base = run_states(monkeypatch, 1, jobs, p, 1200)
    assert run_states(monkeypatch, None, jobs, p, 1200) == base     # the batch's own choice
    assert run_states(monkeypatch, 5, jobs, p, 1200) == base


def test_chunked_launch_matches_oracle(monkeypatch):
    monkeypatch.setenv("XW_CHUNKS", "4")
    n, w, R, iters = 13, 9, 3000, 900
    p = X.Params(stop_on_solve=0, t_init=4.0, moves_per_launch=300)
    seed = 4321
    b = X.Batch([{"n": n, "w": w, "seed": seed, "replicas": R}], p)
    temps = {r: b.replica(0, r)[0].reheat_temperature for r in (0, 1, 1777, R - 1)}
    b.run(iters)
    b.synchronize()
    job = oracle_job(n, w, seed, p)
    for r, t in temps.items():
        rep = O.Replica(job, r, start_of(n, w, seed, r, p), t, r)
        rep.run(iters, stop_on_solve=False)
        compare(b, 0, r, rep)
    b.close()


def test_chunked_large_order_launches_leave_every_replica_unchanged(monkeypatch):
    # the HBM-resident kernel (orders above 256): its Gram arena and lazy best
    # copies carry over between a replica's chunks
    jobs = [{"n": 260, "w": 259, "seed": 71, "replicas": 24}, {"n": 300, "w": 20, "seed": 72, "replicas": 16}]
    p = X.Params(stop_on_solve=0, t_init=8.0, moves_per_launch=30)
    base = run_states(monkeypatch, 1, jobs, p, 90)
    assert run_states(monkeypatch, 3, jobs, p, 90) == base


def test_a_chunk_waits_out_a_long_predecessor(monkeypatch):
    """One replica in two chunks: a second warp takes the second chunk at
    once and waits for the whole first chunk (over a second here, at the
    largest order).  The wait is bounded by device time, not by a short spin
    count, so the replica ends unflagged and as the unchunked run."""
    jobs = [{"n": 1024, "w": 1023, "seed": 5, "replicas": 1}]
    p = X.Params(stop_on_solve=0, t_init=8.0, moves_per_launch=60000)
    base = run_states(monkeypatch, 1, jobs, p, 60000)
    assert run_states(monkeypatch, 2, jobs, p, 60000) == base


def test_a_chunk_wait_that_runs_out_flags_the_replica_and_skips_its_later_chunks(monkeypatch):
    """The wait of a chunk for its replica's previous chunk is bounded by
    device time.  With the bound cut to 2 ms (XW_CHUNK_WAIT_NS) and a first
    chunk of 10^5 iterations (a few tenths of a second for one warp), the
    second chunk's wait runs out: it flags the replica, runs nothing, and
    marks the replica's chunk count so that the third chunk skips as well
    instead of running beside the first on the same record.  The first
    chunk runs to its end, so the replica holds exactly its iterations, and
    the next batch (default bound) runs normally."""
    jobs = [{"n": 26, "w": 25, "seed": 17, "replicas": 1}]
    p = X.Params(stop_on_solve=0, t_init=4.0, moves_per_launch=300000, warps_per_replica=1,
                 squared_objective_fraction=0.0, parity_objective_fraction=0.0)
    monkeypatch.setenv("XW_CHUNKS", "3")
    monkeypatch.setenv("XW_CHUNK_WAIT_NS", "2000000")
    b = X.Batch(jobs, p)
    b.run(300000)
    b.synchronize()
    st = b.replica(0, 0)[0]
    assert st.error == X.XW_DEVERR_CHUNK
    assert st.iterations == 100000
    assert b.results()[0][0].error == X.XW_DEVERR_CHUNK
    b.close()
    monkeypatch.delenv("XW_CHUNK_WAIT_NS")
    monkeypatch.setenv("XW_CHUNKS", "1")
    base, _ = run_states(monkeypatch, 1, jobs, p, 30000)
    assert run_states(monkeypatch, 3, jobs, p, 30000)[0] == base


def test_served_requests_end_the_same_in_chunked_rounds(monkeypatch):
    """The serving loop's class launches run chunked when a class has more
    replicas than resident warps; forcing chunks on small requests shows that
    a served request's outcome does not depend on them."""
    from test_gpu_server import outcome, req, serve
    reqs = [req(12, 11, 4242, 8, 200000), req(16, 4, 77, 16, 5000), req(26, 25, 9, 32, 4000)]
    monkeypatch.setenv("XW_CHUNKS", "1")
    base, _ = serve(reqs)
    monkeypatch.setenv("XW_CHUNKS", "3")
    chunked, _ = serve(reqs)
    assert [outcome(r, W) for r, W in chunked] == [outcome(r, W) for r, W in base]
