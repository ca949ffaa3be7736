"""Full-size properties of the CUDA annealer (sizes the oracle cannot replay).

Size-independent checks at the benchmark's shape: every replica's tracked
score equals a full recompute of its W, every reported best W has the
reported score, every solution verifies W W^T = wI exactly in int64, and no
replica fails its device self-check (the kernel rebuilds the Gram from W at
every launch and compares with the tracked score).
"""
import numpy as np
import pytest

import oracle_lib as O
import xtax_b200 as X

pytestmark = pytest.mark.gpu


def test_tempering_population_at_benchmark_shape_is_consistent():
    # 128 instances x 32 rungs of W(26,25), the uniform population's shape
    p = X.Params(tempering=1, exchange_interval=1000, t_min=0.1, t_init=6.0,
                 squared_objective_fraction=0.0, parity_objective_fraction=0.0)
    jobs = [{"n": 26, "w": 25, "seed": 1 + i, "replicas": 32} for i in range(128)]
    b = X.Batch(jobs, p)
    b.run(3000)
    b.synchronize()
    res = b.results()
    rng = np.random.default_rng(0)
    for j in rng.choice(128, 8, replace=False):
        r_best, best = res[j]
        assert r_best.error == 0
        st = O.rescore(26, 25, best)[0]
        assert int(st[0]) == r_best.score and int(st[1]) == r_best.conflicts
        rungs = set()
        for r in rng.choice(32, 4, replace=False):
            s, W, B, M = b.replica(int(j), int(r))
            assert s.error == 0 and s.iterations == 3000
            assert int(O.rescore(26, 25, W)[0][0]) == s.score
            assert int(O.rescore(26, 25, B)[0][0]) == s.best_score
            rungs.add(s.rung)
        assert all(0 <= x < 32 for x in rungs)
    b.close()


def test_solutions_verify_exactly():
    p = X.Params(t_init=4.0, moves_per_launch=2000)
    jobs = [{"n": 10, "w": 9, "seed": 3, "replicas": 64}, {"n": 12, "w": 11, "seed": 4, "replicas": 256},
            {"n": 16, "w": 4, "seed": 5, "replicas": 64}, {"n": 7, "w": 4, "seed": 6, "replicas": 64}]
    res, best = X.batch_solve(jobs, p, iters=200000)
    off = 0
    for jb, r in zip(jobs, res):
        n, w = jb["n"], jb["w"]
        W = best[off:off + n * n]
        off += n * n
        assert r.error == 0
        st = O.rescore(n, w, W)[0]
        assert int(st[0]) == r.score
        if r.solved:
            assert r.verified == 1
            assert O.verify(n, w, W) == 3
    assert sum(r.solved for r in res) >= 2


def test_run_annealer_drop_in_solves_small_order():
    r = X.run_annealer(10, 9, X.Params(seed=11, replicas=256, max_seconds=20.0))
    assert r.solved and r.verified
    assert O.verify(10, 9, r.best.entries) == 3
    assert any(line.startswith("done moves=") for line in r.log)
    assert any(line.startswith("[cuda] device=") for line in r.log)


def test_cli_drop_in_solves_and_writes_csv(tmp_path):
    import os
    import subprocess
    cli = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "xtax_b200", "bin", "xweigh_cuda")
    out = tmp_path / "w.csv"
    r = subprocess.run([cli, "12", "11", "--seed", "7", "--replicas", "512", "--max-seconds", "60", "-o", str(out)],
                       capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    lines = r.stdout.splitlines()
    assert lines[0].startswith("[cuda] device=") and any(l.startswith("done moves=") for l in lines)
    assert "Found W(12,11); exact verification passed" in r.stdout
    rows = [list(map(int, l.split(","))) for l in out.read_text().splitlines()]
    W = np.array(rows, dtype=np.int8).T.reshape(-1)   # column-major
    assert O.verify(12, 11, W) == 3


def test_elite_restarts_keep_replicas_consistent():
    # a stagnating search (hard order, short restart interval): restarted
    # replicas are loaded back by the kernel, which rebuilds their Gram and
    # checks the scores written for them (a mismatch fails the run)
    p = X.Params(seed=3, replicas=64, moves_per_launch=500, max_seconds=1.5, restart_interval=0.05,
                 restart_fraction=0.5)
    r = X.run_annealer(30, 29, p)
    restarts = [line for line in r.log if line.startswith("[restart] seconds=")]
    assert restarts and r.restarted_replicas >= 32 * len(restarts) // 2
    assert r.restarted_replicas == sum(int(l.split("replicas=")[1].split()[0]) for l in restarts)
    done = [line for line in r.log if line.startswith("done moves=")][0]
    assert f"restarted_replicas={r.restarted_replicas}" in done
    assert X.score(30, 29, r.best.entries)[0] == r.best.score


def test_snapshot_resume_is_bit_exact(tmp_path):
    # K iterations, save, load into a new batch, L more == K + L in one batch
    p = X.Params(tempering=1, exchange_interval=500, t_min=0.1, t_init=6.0, stop_on_solve=0,
                 squared_objective_fraction=0.0, parity_objective_fraction=0.0)
    jobs = [{"n": 14, "w": 13, "seed": 3, "replicas": 8}, {"n": 20, "w": 19, "seed": 4, "replicas": 8},
            {"n": 40, "w": 4, "seed": 5, "replicas": 6}]
    ref = X.Batch(jobs, p)
    ref.run(2000)
    ref.synchronize()
    a = X.Batch(jobs, p)
    a.run(1000)
    a.synchronize()
    a.save(tmp_path / "pop.bin")
    a.close()
    b = X.Batch.load(tmp_path / "pop.bin", jobs)
    b.run(1000)
    b.synchronize()
    for j, jb in enumerate(jobs):
        for r in range(jb["replicas"]):
            s1, W1, B1, M1 = ref.replica(j, r)
            s2, W2, B2, M2 = b.replica(j, r)
            assert (s1.iterations, s1.moves, s1.score, s1.best_score, s1.temperature, s1.rung) == \
                   (s2.iterations, s2.moves, s2.score, s2.best_score, s2.temperature, s2.rung)
            assert (W1 == W2).all() and (B1 == B2).all() and (M1 == M2).all()
    # reset() of a loaded batch returns to the snapshot
    b.reset()
    b.run(1000)
    b.synchronize()
    assert [r.moves for r, _ in b.results()] == [r.moves for r, _ in ref.results()]
    ref.close()
    b.close()


def escape_brute_force(n, w, W):
    """Every support switch out of W in scan order (r1 < r2, c1, c2, new1,
    new2 ascending) with its exact deltas, from a full int64 recompute of the
    two changed Gram rows."""
    M = W.reshape(n, n).T.astype(np.int64)          # row-major
    G = M @ M.T
    out = []
    for r1 in range(n):
        for r2 in range(r1 + 1, n):
            for c1 in range(n):
                if M[r1, c1] == 0 or M[r2, c1] != 0:
                    continue
                for c2 in range(n):
                    if M[r2, c2] == 0 or M[r1, c2] != 0:
                        continue
                    for nv1 in (-1, 1):
                        for nv2 in (-1, 1):
                            N = M.copy()
                            N[r1, c1] = 0
                            N[r2, c2] = 0
                            N[r1, c2] = nv1
                            N[r2, c1] = nv2
                            ds = dc = 0
                            for o in range(n):
                                if o in (r1, r2):
                                    continue
                                for r in (r1, r2):
                                    old, new = G[r, o], N[r] @ N[o]
                                    ds += int(abs(new)) - int(abs(old))
                                    dc += int(new != 0) - int(old != 0)
                            out.append((r1, r2, c1, c2, nv1, nv2, int(ds), int(dc)))
    return out


@pytest.mark.parametrize("n,w,limit", [(8, 7, 12), (10, 5, 40), (12, 3, 1000), (9, 4, 7), (12, 11, 5)])
def test_device_escape_scan_matches_brute_force(n, w, limit):
    W = O.random_start(n, w, 100 + n * w)
    got = X.escape_scan(n, w, W, limit)
    ref = escape_brute_force(n, w, W)
    ref = sorted(enumerate(ref), key=lambda t: (t[1][6], t[1][7], t[0]))[:limit]
    assert got == [r for _, r in ref]
