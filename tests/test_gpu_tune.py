"""The launch-shape autotuner (xw_autotune) and shape independence.

A batch of uneven orders is tuned over warps per CTA; the winner is recorded
in the tuning cache and used by later batches with warps_per_block = 0.  The
shape changes only scheduling: every replica's trajectory, and so every
result, is the same at every shape.
"""
import pytest

import xtax_b200 as X

pytestmark = pytest.mark.gpu

JOBS = [{"n": n, "w": n - 1, "seed": 5 + 10 * n + k, "replicas": 16} for n in (14, 18, 30) for k in range(8)]


def params(**kw):
    return X.Params(tempering=1, exchange_interval=500, t_min=0.1, t_init=6.0, stop_on_solve=0,
                    squared_objective_fraction=0.0, parity_objective_fraction=0.0, **kw)


def test_autotune_records_and_applies_the_fastest_shape(tmp_path, monkeypatch):
    monkeypatch.setenv("XW_TUNE_CACHE", str(tmp_path / "tune.txt"))
    monkeypatch.delenv("XW_WARPS_PER_BLOCK", raising=False)
    wpb, ms = X.autotune(JOBS, params(), iters=500)
    assert wpb in (1, 2, 4, 8, 16) and ms > 0
    # cache lines: kind (rows per lane), slot-byte class, warps per CTA,
    # replicas per warp
    rows = [tuple(int(v) for v in line.split()) for line in (tmp_path / "tune.txt").read_text().splitlines()]
    assert any(kind == 1 and w == wpb and rpw == 1 for kind, _, _, w, rpw in rows)
    b = X.Batch(JOBS, params(warps_per_block=0))
    assert b.shape()[0] == wpb
    b.close()


def test_results_do_not_depend_on_the_launch_shape():
    out = []
    for wpb in (1, 3, 8):
        b = X.Batch(JOBS, params(warps_per_block=wpb))
        assert b.shape()[0] == wpb
        b.run(1500)
        b.synchronize()
        out.append([(r.score, r.conflicts, r.best_replica, r.moves, r.candidate_evaluations, W.tobytes())
                    for r, W in b.results()])
        b.close()
    assert out[0] == out[1] == out[2]
