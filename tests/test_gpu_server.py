"""The continuous-batching server (xw_server_*, xw_submit/xw_wait/...).

A served request's replicas follow exactly the trajectories the oracle
replays (each stops at its own solve, the request ends at the end of the
round in which its first replica solved), so the reported first solution,
its iteration and every counter are the same when the request runs alone
and when it shares rounds with other requests.  Integer work: bit-exact.
"""
import time

import numpy as np
import pytest

import oracle_lib as O
import xtax_b200 as X

from test_gpu_parity import oracle_job, start_of

pytestmark = pytest.mark.gpu

BASE = dict(t_init=4.0, stuck_threshold=700, moves_per_cool=50)


def serve(reqs, **cfg):
    cfg.setdefault("quantum_iters", 500)
    with X.Server(**cfg) as s:
        ids = [s.submit(**r) for r in reqs]
        out = [s.wait(i, timeout=300) for i in ids]
        stats = s.stats()
    return out, stats


def outcome(res, W):
    return (res.state, res.status, res.solved, res.verified, res.sylvester, res.best_replica, res.score,
            res.conflicts, res.moves, res.candidate_evaluations, res.iterations, res.solved_iteration,
            W.tobytes())


def ladder(R, t_min, t_init):
    bottom = min(t_min, t_init)
    ratio = (t_init / max(bottom, 1e-12)) ** (1.0 / (R - 1)) if R > 1 else 1.0
    out, t = [], bottom
    for _ in range(R):
        out.append(t)
        t *= ratio
    return out


def req(n, w, seed, R, iters, **kw):
    return dict(n=n, w=w, seed=seed, replicas=R, max_moves=R * iters, params=X.Params(**{**BASE, **kw}))


def test_served_request_matches_oracle_replay():
    n, w, seed, R = 12, 11, 4242, 8
    (res, W), = serve([req(n, w, seed, R, 200000)])[0]
    assert res.state == X.REQ_DONE and res.status == X.XW_OK
    assert res.solved and res.verified
    p = X.Params(**BASE)
    job = oracle_job(n, w, seed, p)
    temps = ladder(R, p.t_min, p.t_init)
    moves = evals = 0
    solves = []
    for r in range(R):
        rep = O.Replica(job, r, start_of(n, w, seed, r, p), temps[r], r)
        rep.run(res.iterations, stop_on_solve=True)
        s, _, B, _, _, _ = rep.get()
        moves += s.moves
        evals += s.cand_evals
        if s.best_score == 0:
            solves.append((s.it - 1, r, B))
    assert (moves, evals) == (res.moves, res.candidate_evaluations)
    first = min(solves, key=lambda t: (t[0], t[1]))
    assert res.solved_iteration == first[0]
    assert res.best_replica == first[1]
    assert (W == first[2]).all()
    # the request ended in the round of its first solve
    assert first[0] < res.iterations <= (first[0] // 500 + 1) * 500


@pytest.mark.parametrize("schedule", [X.SCHED_LEAST_ATTAINED, X.SCHED_ALL])
def test_request_alone_equals_request_in_mix(schedule):
    target = req(12, 11, 4242, 16, 200000)
    budget = req(26, 25, 99, 32, 3000)                       # runs out of budget
    wide = req(34, 4, 5, 24, 4000, t_init=2.0)               # n > 32: the two-rows-per-lane launch
    others = [req(14, 13, 11, 24, 4000), req(18, 9, 12, 16, 3000), req(20, 19, 13, 32, 2500),
              req(30, 29, 14, 20, 2000, objective=2), req(16, 4, 15, 8, 5000)]
    (alone_t,), _ = serve([target])
    (alone_b,), _ = serve([budget])
    (alone_w,), _ = serve([wide])
    mix, st = serve(others[:2] + [target] + others[2:4] + [wide, budget] + others[4:], schedule=schedule,
                    max_active_replicas=64)
    assert alone_t[0].solved and alone_t[0].verified
    assert not alone_b[0].solved and alone_b[0].iterations == 3000
    assert outcome(*alone_t) == outcome(*mix[2])
    assert outcome(*alone_w) == outcome(*mix[5])
    assert outcome(*alone_b) == outcome(*mix[6])
    assert st.finished == len(mix) and st.failed == 0
    for res, W in mix:
        assert res.state == X.REQ_DONE
        if res.solved:
            assert res.verified and X.verify(res.n, res.w, W) == 3


def test_served_outcomes_do_not_depend_on_replicas_per_warp():
    """Orders up to 16 served one and two replicas per warp (the untuned
    server runs one) reach the same outcomes, move for move."""
    reqs = [req(12, 11, 4242, 16, 200000), req(14, 13, 11, 24, 4000), req(16, 4, 15, 8, 5000),
            req(13, 9, 21, 9, 3000, objective=1, move_set=1)]
    one, _ = serve(reqs, replicas_per_warp=1)
    two, _ = serve(reqs, replicas_per_warp=2)
    assert [outcome(*o) for o in one] == [outcome(*o) for o in two]
    assert one[0][0].solved and one[0][0].verified


def test_round_length_does_not_change_the_first_solution():
    r = req(12, 11, 777, 12, 200000)
    (a,), _ = serve([r], quantum_iters=250)
    (b,), _ = serve([r], quantum_iters=1000)
    assert a[0].solved and b[0].solved
    assert (a[0].solved_iteration, a[0].best_replica) == (b[0].solved_iteration, b[0].best_replica)
    assert (a[1] == b[1]).all()


def test_tempering_request_alone_equals_mix():
    t = dict(n=14, w=13, seed=31, replicas=16, max_moves=16 * 4000,
             params=X.Params(tempering=1, exchange_interval=1000, t_min=0.1, t_init=6.0,
                             squared_objective_fraction=0.0, parity_objective_fraction=0.0))
    (alone,), _ = serve([t])
    mix, _ = serve([req(20, 19, 3, 32, 4000), t, req(12, 11, 4, 8, 4000)])
    assert outcome(*alone) == outcome(*mix[1])


def test_tempering_request_matches_oracle():
    n, w, seed, R, E = 12, 11, 53, 6, 1000
    p = X.Params(tempering=1, exchange_interval=E, t_min=0.1, t_init=6.0,
                 squared_objective_fraction=0.0, parity_objective_fraction=0.0)
    (res, W), = serve([dict(n=n, w=w, seed=seed, replicas=R, max_moves=R * 3000, params=p)])[0]
    job = oracle_job(n, w, seed, p)
    lad = ladder(R, p.t_min, p.t_init)
    reps = [O.Replica(job, r, start_of(n, w, seed, r, p), lad[r], r) for r in range(R)]
    it, rnd = 0, 0
    while it < res.iterations:
        step = min(E, res.iterations - it)
        for rep in reps:
            rep.run(step, stop_on_solve=True)
        it += step
        if it % E == 0 and not any(rep.get()[0].best_score == 0 for rep in reps):
            O.exchange(job, reps, lad, rnd)
            rnd += 1
    got = [rep.get() for rep in reps]
    assert sum(g[0].moves for g in got) == res.moves
    if res.solved:
        first = min((g[0].it - 1, r) for r, g in enumerate(got) if g[0].best_score == 0)
        assert (res.solved_iteration, res.best_replica) == first
    else:
        best = min((g[0].best_score, g[0].best_conflicts, r) for r, g in enumerate(got))
        assert (res.score, res.conflicts, res.best_replica) == best
    assert (W == got[res.best_replica][2]).all()


def test_sylvester_short_circuit_and_rejections():
    with X.Server(quantum_iters=500) as s:
        i = s.submit(16, 4, 1, replicas=32, max_moves=10 ** 6)
        res, W = s.wait(i, timeout=60)
        assert res.state == X.REQ_DONE and res.sylvester and res.solved and res.verified
        assert res.moves == 0 and X.verify(16, 4, W) == 3
        with pytest.raises(X.XwError) as e:
            s.submit(7, 3, 1)                                  # odd order needs a square weight
        assert e.value.code == X.XW_ERR_INVALID
        with pytest.raises(X.XwError) as e:
            s.submit(12, 11, 1, replicas=0)
        assert e.value.code == X.XW_ERR_INVALID
        with pytest.raises(X.XwError) as e:
            s.submit(12, 11, 1, replicas=8, params=X.Params(tempering=1, exchange_interval=750))
        assert e.value.code == X.XW_ERR_INVALID               # not a multiple of the round
        with pytest.raises(X.XwError) as e:
            s.poll(123456)
        assert e.value.code == X.XW_ERR_NOT_FOUND


def test_cancel_and_time_limit():
    with X.Server(quantum_iters=500) as s:
        hard = s.submit(62, 61, 5, replicas=64)               # no budget: runs until cancelled
        time.sleep(0.5)
        res, _ = s.poll(hard)
        assert res.state in (X.REQ_QUEUED, X.REQ_RUNNING)
        with pytest.raises(X.XwError) as e:
            s.wait(hard, timeout=0.05)
        assert e.value.code == X.XW_ERR_TIMEOUT
        s.cancel(hard)
        res, W = s.wait(hard, timeout=60)
        assert res.state == X.REQ_CANCELLED and res.moves > 0
        assert X.score(62, 61, W)[0] == res.score
        timed = s.submit(62, 61, 6, replicas=64, params=X.Params(max_seconds=0.3))
        res, _ = s.wait(timed, timeout=60)
        assert res.state == X.REQ_DONE and res.finish_seconds - res.admit_seconds >= 0.3
        s.release(timed)
        with pytest.raises(X.XwError):
            s.poll(timed)
        st = s.stats()
        assert st.cancelled == 1 and st.running == 0 and st.resident_replicas == 0


def test_least_attained_schedule_runs_one_request_per_round_at_capacity():
    reqs = [req(30, 29, 40 + k, 256, 2000) for k in range(3)]   # no solve within 2000 iterations: 4 rounds each
    out, st = serve(reqs, max_active_replicas=256)
    assert all(r.state == X.REQ_DONE and r.iterations == 2000 for r, _ in out)
    assert st.rounds == 12 and st.schedule == X.SCHED_LEAST_ATTAINED


def test_checkpoint_of_a_running_request_reports_its_best_so_far():
    """xw_checkpoint: the best W of a running request at the end of its next
    round, with that W's own score; later checkpoints never get worse."""
    n, w = 30, 29
    with X.Server(quantum_iters=500) as s:
        rid = s.submit(**req(n, w, 77, 64, 10 ** 6))
        r1, W1 = s.checkpoint(rid, timeout=120)
        assert r1.state == X.REQ_RUNNING and r1.iterations >= 500
        st = X.score(n, w, W1)
        assert (st[0], st[1]) == (r1.score, r1.conflicts)
        r2, W2 = s.checkpoint(rid, timeout=120)
        assert r2.iterations > r1.iterations
        assert (r2.score, r2.conflicts) <= (r1.score, r1.conflicts)
        st = X.score(n, w, W2)
        assert (st[0], st[1]) == (r2.score, r2.conflicts)
        s.cancel(rid)
        res, _ = s.wait(rid, timeout=120)
        assert res.state == X.REQ_CANCELLED


@pytest.mark.parametrize("tempering", [0, 1])
def test_request_snapshot_resumes_move_for_move(tmp_path, tempering):
    """xw_request_save + xw_submit_snapshot: a request saved after a few
    rounds, cancelled, and resumed in another server ends exactly as the
    same request run without interruption (rounds of the same length from
    the same iteration counts)."""
    kw = dict(tempering=1, exchange_interval=1000, t_min=0.1, t_init=6.0) if tempering else {}
    r = req(30, 29, 91, 32, 12000, **kw)
    (ref, Wref), = serve([r], quantum_iters=500)[0]
    path = tmp_path / "request.xwpop"
    with X.Server(quantum_iters=500) as s:
        rid = s.submit(**r)
        for _ in range(3):
            s.checkpoint(rid, timeout=120)
        s.save(rid, path, timeout=120)
        s.cancel(rid)
        s.wait(rid, timeout=120)
    with X.Server(quantum_iters=500) as s:
        rid = s.submit_snapshot(path)
        res, W = s.wait(rid, timeout=300)
    assert res.state == X.REQ_DONE and res.status == X.XW_OK
    assert (res.best_replica, res.score, res.conflicts, res.moves, res.candidate_evaluations, res.iterations) == \
        (ref.best_replica, ref.score, ref.conflicts, ref.moves, ref.candidate_evaluations, ref.iterations)
    assert (W == Wref).all()
    # the same snapshot also resumes as a batch
    b = X.Batch.load(path, [{"n": 30, "w": 29, "replicas": 32}])
    b.run(500)
    b.synchronize()
    (jr, _), = b.results()
    assert jr.error == 0
    b.close()


def test_saving_a_finished_request_is_refused(tmp_path):
    with X.Server(quantum_iters=500) as s:
        rid = s.submit(**req(12, 11, 5, 8, 200000))
        s.wait(rid, timeout=120)
        with pytest.raises(X.XwError):
            s.save(rid, tmp_path / "late.xwpop", timeout=10)


def test_retired_requests_are_verified_on_the_device_as_on_the_host():
    """Every retiring request's W is rescored on the device (tensor cores
    for orders padded to 32..128, zero padding past n) in one batch per
    round; the returned score, conflicts and exact flag must agree with the
    host's int64 check (xw_score / xw_verify) for solved and unsolved
    requests alike, across orders of every padded size."""
    reqs = [req(12, 11, 31, 8, 200000), req(14, 13, 32, 8, 200000), req(20, 19, 33, 8, 3000),
            req(36, 4, 34, 8, 200000), req(40, 39, 35, 4, 2000), req(70, 4, 36, 4, 200000),
            req(100, 99, 37, 2, 300), req(26, 25, 38, 16, 4000), req(150, 149, 39, 2, 100)]
    out, _ = serve(reqs)
    states = [(r["n"], r["w"], res.state, res.status, res.error.decode()) for (res, _), r in zip(out, reqs)]
    for (res, W), r in zip(out, reqs):
        n, w = r["n"], r["w"]
        assert res.state == X.REQ_DONE and res.status == X.XW_OK, states
        host = X.score(n, w, W)
        assert (res.score, res.conflicts) == (host[0], host[1]), (n, w)
        assert bool(res.verified) == (bool(res.solved) and X.verify(n, w, W) == 3), (n, w)
        if res.solved:
            assert res.verified and res.score == 0, (n, w)
