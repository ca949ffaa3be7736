"""The oracle pinned against the reference's own outputs (tests/golden/).

CPU only.  Each fixture was produced by running flinty-mathematics/xtax code
(see tests/golden/make_golden.py); the oracle must reproduce it bit for bit.
"""
import ctypes as C
import json
import math
import os

import numpy as np
import pytest

import oracle_lib as O

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def gold(name):
    with open(os.path.join(GOLD, name)) as f:
        return json.load(f)


def test_mt19937_standard_value():
    # [rand.predef]: the 10000th output of a default-seeded mt19937 is 4123659995
    out = np.zeros(10000, dtype=np.uint32)
    O.lib().xwo_mt_stream(5489, 10000, O.ptr(out, C.c_uint32))
    assert int(out[-1]) == 4123659995


def test_philox_known_answers():
    # Known-answer vectors of Philox4x32-10 published with the Random123
    # library (Salmon et al., SC'11).
    assert O.philox([0, 0, 0, 0], [0, 0]) == [0x6627e8d5, 0xe169c58d, 0xbc57ac4c, 0x9b00dbd8]
    assert O.philox([0xffffffff] * 4, [0xffffffff] * 2) == [0x408f276d, 0x41c83b0e, 0xa20bc7c6, 0x6d5451fd]
    assert O.philox([0x243f6a88, 0x85a308d3, 0x13198a2e, 0x03707344], [0xa4093822, 0x299f31d0]) == \
        [0xd16cfe09, 0x94fdcceb, 0x5001e420, 0x24126ea1]


def test_exp_accuracy():
    xs = np.concatenate([-np.linspace(0, 39.9, 4001), -np.logspace(-12, 1.6, 500)])
    for x in xs:
        e = O.lib().xwo_exp(float(x))
        ref = math.exp(float(x))
        assert abs(e - ref) <= 4e-16 * ref, (x, e, ref)
    assert O.lib().xwo_exp(-50.0) > 0 and O.lib().xwo_exp(-50.0) < 2.0 ** -32
    assert O.lib().xwo_exp(-800.0) == 0.0
    assert O.lib().xwo_exp(0.0) == 1.0


@pytest.mark.parametrize("case", gold("starts.json"), ids=lambda c: f"W{c['n']}_{c['w']}_s{c['seed']}")
def test_random_start_matches_reference(case):
    n, w = case["n"], case["w"]
    W = O.random_start(n, w, case["seed"])
    assert W.tolist() == case["entries"]
    st, _, _ = O.rescore(n, w, W)
    assert int(st[0]) == case["score"] and int(st[1]) == case["conflicts"]
    assert O.verify(n, w, W) & 1 == case["support_ok"]


@pytest.mark.parametrize("case", gold("sylvester.json"), ids=lambda c: f"S{c['n']}_{c['w']}")
def test_sylvester_matches_reference(case):
    n, w = case["n"], case["w"]
    W = O.sylvester(n, w)
    assert W.tolist() == case["entries"]
    flags = O.verify(n, w, W)
    assert (flags & 1) == case["support_ok"] and ((flags >> 1) & 1) == case["weighing_ok"]


def _replay_moves(case):
    n, w = case["n"], case["w"]
    W = np.array(case["start"], dtype=np.int8)
    out = np.zeros(4, dtype=np.int64)
    for mv in case["moves"]:
        kind, r1, r2, c1, c2, a, b, ds, dc, score, conf = mv
        if case["cmd"] == "moves":
            if kind == 0:
                k, v1, v2 = 0, 0, 0
            else:
                k, v1, v2 = 1, int(W[c1 * n + r1]), int(W[c2 * n + r2])
        else:
            k, v1, v2 = (2, 0, 0) if kind == 2 else (1, a, b)
        bad = O.lib().xwo_move_eval(n, w, O.ptr(W, C.c_int8), k, r1, r2, c1, c2, v1, v2, 1,
                                   O.ptr(out, C.c_int64))
        assert bad == 0
        assert (int(out[0]), int(out[1])) == (ds, dc), mv
        st, _, _ = O.rescore(n, w, W)
        assert (int(st[0]), int(st[1])) == (score, conf)
    assert W.tolist() == case["final"]


@pytest.mark.parametrize("case", gold("moves.json"), ids=lambda c: f"W{c['n']}_{c['w']}")
def test_move_deltas_match_reference(case):
    _replay_moves(case)


@pytest.mark.parametrize("case", gold("compound.json"), ids=lambda c: f"W{c['n']}_{c['w']}")
def test_compound_move_deltas_match_reference_decomposition(case):
    _replay_moves(case)


@pytest.mark.parametrize("case", gold("calibrate.json"), ids=lambda c: f"W{c['n']}_{c['w']}")
def test_calibration_matches_reference(case):
    n, w = case["n"], case["w"]
    p = O.ref_params()
    t = O.lib().xwo_calibrate(n, w, case["seed"], C.byref(p))
    assert t == case["t"]


@pytest.mark.parametrize("case", gold("walks.json"),
                         ids=lambda c: f"W{c['n']}_{c['w']}_s{c['seed']}")
def test_reference_walk_matches(case):
    r, s, f, b = O.ref_walk(case["n"], case["w"], case["seed"], case["max_moves"],
                            t_init=case["t_init_arg"], t_min=case["t_min"],
                            cooling=case["cooling"], moves_per_cool=case["moves_per_cool"],
                            stuck_threshold=case["stuck_threshold"])
    assert r.initial_temperature == case["initial_temperature"]
    assert r.worker_seed == case["worker_seed"]
    assert r.moves == case["moves"]
    assert r.accepted == case["accepted"]
    assert f"{r.hash:016x}" == case["hash"]
    assert (r.score, r.conflicts) == (case["score"], case["conflicts"])
    assert (r.best_score, r.best_conflicts) == (case["best_score"], case["best_conflicts"])
    assert r.temperature == case["temperature"]
    assert s.tolist() == case["start"] and f.tolist() == case["final"] and b.tolist() == case["best"]


@pytest.mark.parametrize("case", gold("cli_runs.json"), ids=lambda c: f"seed{c['seed']}")
def test_reference_cli_solve_reproduced(case):
    # the reference xweigh CLI with one thread is deterministic once it solves
    r, _, f, _ = O.ref_walk(case["n"], case["w"], case["seed"], 10 ** 9)
    assert r.score == 0
    assert r.moves == case["moves"]
    assert f.tolist() == case["final"]
    assert O.verify(case["n"], case["w"], f) == 3


def test_device_replica_incremental_state_consistent():
    # device-mode moves keep G, residuals, minority lists and scores equal to
    # a full recompute for every move kind and objective
    for n, w, ms in [(12, 11, 0), (16, 4, 0), (20, 10, 0), (13, 9, 0), (12, 11, 1), (16, 4, 1)]:
        job = O.make_job(n, w, move_set=ms, double_sign_fraction=0.4)
        for idx in range(6):
            W0 = O.random_start(n, w, 100 + idx) if ms == 0 else O.row_start(n, w, 7, 9, idx)
            rep = O.Replica(job, idx, W0, 3.0)
            for _ in range(20):
                rep.run(50, stop_on_solve=False)
                assert rep.check() == 0


def test_row_start_rows_have_weight_w():
    for n, w in [(12, 11), (16, 4), (30, 29)]:
        W = O.row_start(n, w, 1, 2, 3).reshape(n, n)  # [col][row]
        assert (np.count_nonzero(W, axis=0) == w).all()
        assert set(np.unique(W).tolist()) <= {-1, 0, 1}
