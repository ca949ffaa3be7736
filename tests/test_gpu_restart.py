"""Elite restarts with the kicks on the device (restart mode 1).

The reference kicks the elite's copies on the host with mt19937 after
reading the population back (xweigh_cuda.cu:2089-2193).  In mode 1 one CTA
per restarted replica rewrites its record in place from the elite's best W:
the escape move, row kicks or random moves from a Philox stream per (job,
restart round, replica).  The oracle restates the kick; every restarted
record must hold exactly the oracle's kicked W, its minority lists in column
order, its exact scores, the better of it and the elite as best, and the
reheat temperature.  The next launch's load self-check then accepts it.
"""
import math

import numpy as np
import pytest

import oracle_lib as O
import xtax_b200 as X

pytestmark = pytest.mark.gpu


def coin(p):
    return 0 if p <= 0 else (1 << 32) if p >= 1 else math.ceil(p * 4294967296.0)


def minority_lists(n, w, K):
    m = min(w, n - w)
    sparse = w <= n - w
    out = []
    for r in range(n):
        cols = [c for c in range(n) if (K[c * n + r] != 0) == sparse]
        out.extend(cols[:m])
    return np.array(out, dtype=np.int64)


@pytest.mark.parametrize("n,w,R,kw", [
    (18, 9, 12, dict()),
    (26, 25, 9, dict(sign_fraction=0.3)),
    (12, 12, 6, dict()),                       # w = n: flips only
    (40, 20, 7, dict(restart_kick_max=120)),   # two rows per lane
    (270, 269, 3, dict(moves_per_launch=50)),  # above 256: the state in HBM, u16 minority lists
])
def test_device_kicks_match_the_oracle(n, w, R, kw):
    seed = 500 + n
    iters = kw.pop("moves_per_launch", 1500)
    p = X.Params(seed=seed, stop_on_solve=0, t_init=3.0, moves_per_launch=iters, restart_kicks=1,
                 restart_fraction=0.5, restart_kick_min=2, warps_per_replica=1, **kw)
    b = X.Batch([{"n": n, "w": w, "seed": seed, "replicas": R}], p)
    b.run(iters)
    b.synchronize()
    k0, k1 = X.philox_key(seed)
    cursor = 0
    for rnd in range(2):
        (res, best), = b.results()
        elite, gbest, gconf = res.best_replica, res.score, res.conflicts
        count = min(max(math.ceil(p.restart_fraction * (R - 1)), 1), R - 1)
        esc = X.escape_scan(n, w, best, max(count * 4, 1))
        pool = min(len(esc), max(count * 4, 1))
        selected, scanned = [], 0
        while len(selected) < count and scanned < 2 * R:
            r = (cursor + scanned) % R
            scanned += 1
            if r != elite:
                selected.append(r)
        cursor = (cursor + scanned) % R
        reheat_t = {r: b.replica(0, r)[0].reheat_temperature for r in selected}
        assert b.restart(0) == count
        for idx, r in enumerate(selected):
            steps = p.restart_kick_min + (idx * (p.restart_kick_max - p.restart_kick_min) // (count - 1)
                                          if count > 1 else 0)
            e = esc[(idx + rnd * count) % pool] if pool else None
            K = O.kick(n, w, best, e, k0, k1, rnd, r, idx, steps, coin(p.sign_fraction))
            assert O.verify(n, w, K) >= 1   # still fixed-weight rows and columns
            st, W, B, M = b.replica(0, r)
            ctx = (rnd, idx, r)
            assert (W == K).all(), ctx
            sc, _, _ = O.rescore(n, w, K)
            assert (st.score, st.conflicts) == (sc[0], sc[1]), ctx
            better = (sc[0], sc[1]) < (gbest, gconf)
            assert (B == (K if better else best)).all(), ctx
            assert (st.best_score, st.best_conflicts) == ((sc[0], sc[1]) if better else (gbest, gconf)), ctx
            assert (M.astype(np.int64) == minority_lists(n, w, K)).all(), ctx
            assert st.temperature == max(p.t_min, reheat_t[r] * p.reheat), ctx
            assert (st.moves_since_improvement, st.cooling_counter) == (0, 0), ctx
        # the next launch loads the rewritten records and checks their scores
        b.run(iters)
        b.synchronize()
        assert all(b.replica(0, r)[0].error == 0 for r in range(R))
    b.close()


def test_host_and_device_kick_restarts_in_the_drop_in_run():
    # the drop-in run's stagnation restarts in both modes keep every replica
    # consistent (a replica that failed its load self-check would fail the run)
    for mode in (0, 1):
        p = X.Params(seed=3, replicas=64, moves_per_launch=500, max_seconds=1.0, restart_interval=0.05,
                     restart_fraction=0.5, restart_kicks=mode)
        r = X.run_annealer(30, 29, p)
        restarts = [line for line in r.log if line.startswith("[restart] seconds=")]
        assert restarts and r.restarted_replicas > 0
