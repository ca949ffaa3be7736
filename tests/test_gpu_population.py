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
