"""Parity of the CUDA annealer with the oracle, through the C ABI.

Every replica of a device run is replayed by the CPU oracle from the same
start, key and temperature; after K iterations the whole replica state must
be identical: W, best W, minority lists, iteration and move counters,
scores, objective totals, temperature and counters.  Integer work, so the
bar is bit-exact.  Tempering runs also replay the device's exchange sweeps.
"""
import numpy as np
import pytest

import oracle_lib as O
import xtax_b200 as X

pytestmark = pytest.mark.gpu


def oracle_job(n, w, seed, p: X.Params):
    k0, k1 = X.philox_key(seed)
    return O.make_job(n, w, tempering=p.tempering, move_set=p.move_set,
                      candidate_samples=p.candidate_samples, target_samples=p.target_samples,
                      moves_per_cool=p.moves_per_cool, stuck_threshold=p.stuck_threshold,
                      key0=k0, key1=k1, objective=p.objective,
                      greedy_fraction=p.greedy_fraction, target_fraction=p.target_fraction,
                      double_sign_fraction=p.double_sign_fraction, sign_fraction=p.sign_fraction,
                      switch_sign_fraction=p.switch_sign_fraction,
                      squared_objective_fraction=p.squared_objective_fraction,
                      parity_objective_fraction=p.parity_objective_fraction,
                      t_min=p.t_min, cooling=p.cooling, reheat=p.reheat)


def start_of(n, w, seed, r, p):
    if p.start_kind == 1:
        k0, k1 = X.philox_key(seed)
        return O.row_start(n, w, k0, k1, r)
    return O.random_start(n, w, (seed + r * 0x9e3779b9) & 0xffffffff)


def compare(batch, job_index, r, rep):
    st, W, B, M = batch.replica(job_index, r)
    s, oW, oB, oM, _, _ = rep.get()
    assert st.error == 0
    ctx = f"job {job_index} replica {r}"
    assert st.iterations == s.it, ctx
    assert st.moves == s.moves, ctx
    assert st.candidate_evaluations == s.cand_evals, ctx
    assert (st.score, st.conflicts) == (s.score, s.conflicts), ctx
    assert (st.best_score, st.best_conflicts) == (s.best_score, s.best_conflicts), ctx
    assert st.objective_total == s.obj_total, ctx
    assert st.temperature == s.temperature, ctx
    assert st.moves_since_improvement == s.msi and st.cooling_counter == s.cool_ctr, ctx
    assert st.rung == s.rung, ctx
    assert (W == oW).all(), ctx
    assert (B == oB).all(), ctx
    assert (M == oM).all(), ctx


CASES = [
    # n, w, replicas, iterations, params
    (12, 11, 6, 3000, dict(t_init=4.0, moves_per_launch=1000, stuck_threshold=700, moves_per_cool=50)),
    (16, 4, 6, 2500, dict(t_init=3.0, moves_per_launch=1250, double_sign_fraction=0.4)),
    (20, 10, 5, 2000, dict(t_init=5.0, moves_per_launch=2000)),
    (13, 9, 5, 2000, dict(t_init=4.0, moves_per_launch=700, target_samples=12, candidate_samples=7)),
    (26, 25, 4, 2000, dict(t_init=6.0, moves_per_launch=1000, target_samples=3)),
    (40, 39, 3, 800, dict(t_init=6.0, moves_per_launch=400)),
    (64, 4, 3, 800, dict(t_init=2.0, moves_per_launch=800)),
    (70, 30, 2, 300, dict(t_init=8.0, moves_per_launch=300)),
    (12, 11, 4, 2000, dict(t_init=4.0, moves_per_launch=1000, move_set=1, start_kind=1,
                           objective=1, sign_fraction=0.3)),
    (16, 4, 4, 1500, dict(t_init=2.0, moves_per_launch=500, move_set=1, start_kind=1, objective=0)),
    (30, 29, 3, 1200, dict(t_init=6.0, moves_per_launch=600, objective=2)),
    # edge cases: the largest order (four rows per lane), w = n (no zeros:
    # flips only), w = 1 (one nonzero per row), an odd order
    (128, 64, 2, 120, dict(t_init=8.0, moves_per_launch=60)),
    (128, 127, 2, 120, dict(t_init=8.0, moves_per_launch=120)),
    (8, 8, 4, 1500, dict(t_init=3.0, moves_per_launch=500)),
    (9, 1, 3, 800, dict(t_init=1.0, moves_per_launch=400)),
    (21, 16, 3, 900, dict(t_init=5.0, moves_per_launch=300)),
    # orders above 128: eight rows per lane, int16 Gram, 256-bit row masks
    (160, 159, 2, 60, dict(t_init=8.0, moves_per_launch=30)),
    (200, 20, 2, 60, dict(t_init=6.0, moves_per_launch=60)),
    (256, 255, 1, 40, dict(t_init=8.0, moves_per_launch=20)),
    (256, 4, 2, 50, dict(t_init=2.0, moves_per_launch=50, move_set=1, start_kind=1)),
]


@pytest.mark.parametrize("wpr", [1, 0], ids=["one_warp", "latency_mode"])
@pytest.mark.parametrize("n,w,R,iters,kw", CASES, ids=lambda v: str(v) if not isinstance(v, dict) else "")
def test_cooling_population_matches_oracle(n, w, R, iters, kw, wpr):
    # wpr 0: a population this small runs in the latency mode (orders up to
    # 32: a CTA of warps per replica speculating iterations); 1: one warp
    # per replica
    if wpr == 0 and n > 32:
        pytest.skip("the latency mode covers orders up to 32")
    p = X.Params(stop_on_solve=0, warps_per_replica=wpr, **kw)
    seed = 1000 + n * 7 + w
    batch = X.Batch([{"n": n, "w": w, "seed": seed, "replicas": R}], p)
    assert all((c["warps_per_replica"] > 1) == (wpr == 0) for c in batch.classes())
    temps = [batch.replica(0, r)[0].reheat_temperature for r in range(R)]
    batch.run(iters)
    batch.synchronize()
    job = oracle_job(n, w, seed, p)
    for r in range(R):
        rep = O.Replica(job, r, start_of(n, w, seed, r, p), temps[r], r)
        rep.run(iters, stop_on_solve=False)
        assert rep.check() == 0
        compare(batch, 0, r, rep)
    batch.close()


@pytest.mark.parametrize("wpr", [1, 0], ids=["one_warp", "latency_mode"])
@pytest.mark.parametrize("n,w,R,interval,rounds", [(12, 11, 8, 300, 4), (26, 25, 6, 500, 3), (16, 4, 5, 250, 4)])
def test_tempering_matches_oracle(n, w, R, interval, rounds, wpr):
    p = X.Params(stop_on_solve=0, tempering=1, exchange_interval=interval, t_min=0.1, t_init=6.0,
                 squared_objective_fraction=0.0, parity_objective_fraction=0.0, warps_per_replica=wpr)
    seed = 77 + n
    batch = X.Batch([{"n": n, "w": w, "seed": seed, "replicas": R},
                     {"n": n, "w": w, "seed": seed + 1, "replicas": R}], p)
    batch.run(interval * rounds)
    batch.synchronize()
    bottom, top = 0.1, 6.0
    ratio = (top / bottom) ** (1.0 / (R - 1))
    ladder, t = [], bottom
    for _ in range(R):
        ladder.append(t)
        t *= ratio
    for jidx, s in enumerate([seed, seed + 1]):
        job = oracle_job(n, w, s, p)
        reps = [O.Replica(job, r, start_of(n, w, s, r, p), ladder[r], r) for r in range(R)]
        for k in range(rounds):
            for rep in reps:
                rep.run(interval, stop_on_solve=False)
            O.exchange(job, reps, ladder, k)
        for r, rep in enumerate(reps):
            compare(batch, jidx, r, rep)
    batch.close()


def test_mixed_orders_in_one_launch_match_oracle():
    # replicas of different (n, w) share one persistent launch per class
    p = X.Params(stop_on_solve=0, t_init=4.0, moves_per_launch=600)
    jobs = [{"n": 14, "w": 13, "seed": 5, "replicas": 3}, {"n": 24, "w": 23, "seed": 6, "replicas": 2},
            {"n": 18, "w": 9, "seed": 7, "replicas": 2}, {"n": 33, "w": 32, "seed": 8, "replicas": 2}]
    batch = X.Batch(jobs, p)
    temps = [[batch.replica(j, r)[0].reheat_temperature for r in range(jb["replicas"])]
             for j, jb in enumerate(jobs)]
    batch.run(1800)
    batch.synchronize()
    for j, jb in enumerate(jobs):
        job = oracle_job(jb["n"], jb["w"], jb["seed"], p)
        for r in range(jb["replicas"]):
            rep = O.Replica(job, r, start_of(jb["n"], jb["w"], jb["seed"], r, p), temps[j][r], r)
            rep.run(1800, stop_on_solve=False)
            compare(batch, j, r, rep)
    batch.close()


@pytest.mark.parametrize("extra", [None, {"n": 9, "w": 1, "seed": 12, "replicas": 2}],
                         ids=["one_zero_only", "with_sparse_rows"])
def test_one_zero_class_and_a_mixed_class_match_oracle(extra):
    """A class whose jobs all have one zero per row (w = n - 1) runs the
    kernel with the minority size and side as constants; a class that also
    holds another shape (W(9,1): one nonzero per row) runs the lean kernel
    for any shape.  Either way every replica replays on the oracle (a
    replica given the wrong kernel would carry an error flag instead)."""
    p = X.Params(stop_on_solve=0, t_init=5.0, moves_per_launch=700, warps_per_replica=1)
    jobs = [{"n": 20, "w": 19, "seed": 11, "replicas": 3}, {"n": 31, "w": 30, "seed": 13, "replicas": 2}]
    if extra:
        jobs.append(extra)
    batch = X.Batch(jobs, p)
    assert all(c["warps_per_replica"] == 1 and c["rows_per_lane"] == 1 for c in batch.classes())
    temps = [[batch.replica(j, r)[0].reheat_temperature for r in range(jb["replicas"])]
             for j, jb in enumerate(jobs)]
    batch.run(1400)
    batch.synchronize()
    for j, jb in enumerate(jobs):
        job = oracle_job(jb["n"], jb["w"], jb["seed"], p)
        for r in range(jb["replicas"]):
            rep = O.Replica(job, r, start_of(jb["n"], jb["w"], jb["seed"], r, p), temps[j][r], r)
            rep.run(1400, stop_on_solve=False)
            compare(batch, j, r, rep)
    batch.close()


SMALL_CASES = [c for c in CASES if c[0] <= 16]


@pytest.mark.parametrize("rpw", [1, 2])
@pytest.mark.parametrize("n,w,R,iters,kw", SMALL_CASES, ids=lambda v: str(v) if not isinstance(v, dict) else "")
def test_orders_up_to_16_match_oracle_at_one_and_two_replicas_per_warp(n, w, R, iters, kw, rpw):
    # two replicas per warp: each half-warp owns a replica; an odd count
    # leaves one half of the last warp without one
    R = R + 1
    p = X.Params(stop_on_solve=0, replicas_per_warp=rpw, warps_per_replica=1, **kw)
    seed = 3000 + n * 7 + w
    batch = X.Batch([{"n": n, "w": w, "seed": seed, "replicas": R}], p)
    assert all(c["replicas_per_warp"] == rpw for c in batch.classes())
    temps = [batch.replica(0, r)[0].reheat_temperature for r in range(R)]
    batch.run(iters)
    batch.synchronize()
    job = oracle_job(n, w, seed, p)
    for r in range(R):
        rep = O.Replica(job, r, start_of(n, w, seed, r, p), temps[r], r)
        rep.run(iters, stop_on_solve=False)
        compare(batch, 0, r, rep)
    batch.close()


def test_replicas_per_warp_leaves_every_replica_unchanged():
    # a mixed batch at one and at two replicas per warp (orders up to 16
    # share warps two by two), tempering and cooling jobs, 900 replicas
    jobs = [{"n": 12, "w": 11, "seed": 60 + k, "replicas": 16} for k in range(30)] + \
           [{"n": 16, "w": 4, "seed": 160 + k, "replicas": 16} for k in range(20)] + \
           [{"n": 15, "w": 9, "seed": 260 + k, "replicas": 5} for k in range(12)]
    out = []
    for rpw in (1, 2):
        p = X.Params(stop_on_solve=0, tempering=1, exchange_interval=300, t_min=0.1, t_init=6.0,
                     replicas_per_warp=rpw, squared_objective_fraction=0.0, parity_objective_fraction=0.0)
        b = X.Batch(jobs, p)
        b.run(900)
        b.synchronize()
        states = []
        for j, jb in enumerate(jobs):
            for r in range(jb["replicas"]):
                st, W, B, M = b.replica(j, r)
                assert st.error == 0
                states.append((st.iterations, st.moves, st.score, st.best_score, st.objective_total,
                               st.temperature, st.rung, W.tobytes(), B.tobytes(), M.tobytes()))
        b.close()
        out.append(states)
    assert out[0] == out[1]


def test_orders_of_several_classes_in_one_round_match_oracle():
    # a batch whose orders span the rows-per-lane classes runs one launch
    # per class side by side in each round (eight rows per lane with the
    # int16 Gram and 256-bit masks for the order above 128, one row per
    # lane for 26, two for 40)
    p = X.Params(stop_on_solve=0, t_init=5.0, moves_per_launch=100)
    jobs = [{"n": 150, "w": 149, "seed": 21, "replicas": 1}, {"n": 26, "w": 25, "seed": 22, "replicas": 2},
            {"n": 40, "w": 4, "seed": 23, "replicas": 2}]
    batch = X.Batch(jobs, p)
    temps = [[batch.replica(j, r)[0].reheat_temperature for r in range(jb["replicas"])]
             for j, jb in enumerate(jobs)]
    batch.run(200)
    batch.synchronize()
    for j, jb in enumerate(jobs):
        job = oracle_job(jb["n"], jb["w"], jb["seed"], p)
        for r in range(jb["replicas"]):
            rep = O.Replica(job, r, start_of(jb["n"], jb["w"], jb["seed"], r, p), temps[j][r], r)
            rep.run(200, stop_on_solve=False)
            compare(batch, j, r, rep)
    batch.close()


@pytest.mark.parametrize("wpr", [2, 4, 8, 16, 32, 64])
@pytest.mark.parametrize("stop", [0, 2])
def test_latency_mode_ends_every_replica_as_one_warp(wpr, stop):
    # every warps-per-replica count and both deterministic stop rules (run
    # on, or stop at the replica's own solve): replicas end identical to the
    # one-warp kernel's, counters and best states included; W(12,11) solves
    # within the budget for some seeds, so stop rule 2 ends replicas early
    jobs = [{"n": 12, "w": 11, "seed": 900 + k, "replicas": 3} for k in range(6)] + \
           [{"n": 30, "w": 29, "seed": 950, "replicas": 2}, {"n": 15, "w": 5, "seed": 951, "replicas": 3}]
    out = []
    for k in (1, wpr):
        p = X.Params(stop_on_solve=stop, t_init=3.0, moves_per_launch=2500, warps_per_replica=k,
                     stuck_threshold=900, moves_per_cool=60, max_moves=3 * 9000)
        b = X.Batch(jobs, p)
        b.run(9000)
        b.synchronize()
        states = []
        for j, jb in enumerate(jobs):
            for r in range(jb["replicas"]):
                st, W, B, M = b.replica(j, r)
                assert st.error == 0
                states.append((st.iterations, st.moves, st.candidate_evaluations, st.score, st.best_score,
                               st.objective_total, st.temperature, st.moves_since_improvement,
                               st.cooling_counter, W.tobytes(), B.tobytes(), M.tobytes()))
        res = [(r.score, r.conflicts, r.best_replica, r.moves, r.solved, r.solved_iteration) for r, _ in b.results()]
        b.close()
        out.append((states, res))
    assert out[0] == out[1]


@pytest.mark.parametrize("wpr", [32, 64])
def test_latency_cluster_with_the_job_stop_rule(wpr):
    """Stop rule 1 (every replica of a job stops soon after any solve) on
    clusters of two and four CTAs per replica: the job's solved flag, which
    other replicas set while the launch runs, reaches every CTA of a cluster
    as one value, so they stop together; every replica ends without an
    error, and the solved jobs report a verified solution."""
    jobs = [{"n": 12, "w": 11, "seed": 900 + k, "replicas": 3} for k in range(8)]
    p = X.Params(stop_on_solve=1, t_init=3.0, moves_per_launch=2500, warps_per_replica=wpr,
                 stuck_threshold=900, moves_per_cool=60, max_moves=3 * 20000)
    b = X.Batch(jobs, p)
    assert all(c["warps_per_replica"] == wpr for c in b.classes())
    b.run(20000)
    b.synchronize()
    for j, jb in enumerate(jobs):
        for r in range(jb["replicas"]):
            assert b.replica(j, r)[0].error == 0
    res = b.results()
    b.close()
    assert any(r.solved for r, _ in res)
    for r, W in res:
        if r.solved:
            assert r.verified and X.verify(12, 11, W) == 3
