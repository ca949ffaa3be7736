"""The CPU annealer and its xweigh command line against the reference's own.

tests/golden/cpu_cli.json holds the reference xweigh's output (built from
its sources here) for option errors, existence checks, the Sylvester
construction and one-thread runs that solve.  A one-thread run is
deterministic for a seed: the drop-in must retrace it move for move (same
move count in the done line, same start line, same final W and closing
lines); only the timed "new best" lines, which the reference throttles by
wall clock, may differ.  Multi-thread runs (parallel tempering, not
deterministic) must solve and verify.
"""
import json
import os
import subprocess

import numpy as np
import pytest

import xtax_b200 as X

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CLI = os.path.join(REPO, "xtax_b200", "bin", "xweigh")
with open(os.path.join(REPO, "tests", "golden", "cpu_cli.json")) as f:
    GOLD = json.load(f)


@pytest.mark.parametrize("case", GOLD["errors"], ids=lambda c: " ".join(c["args"]))
def test_errors_match_reference(case, tmp_path):
    r = subprocess.run([CLI] + case["args"] + ["-o", str(tmp_path / "o.csv")], capture_output=True, text=True,
                       timeout=60)
    assert (r.returncode, r.stdout, r.stderr) == (case["returncode"], case["stdout"], case["stderr"])


@pytest.mark.parametrize("case", GOLD["sylvester"], ids=lambda c: " ".join(c["args"]))
def test_sylvester_matches_reference(case, tmp_path):
    out = tmp_path / "o.csv"
    r = subprocess.run([CLI] + case["args"] + ["-o", str(out)], capture_output=True, text=True, timeout=60)
    assert r.returncode == case["returncode"]
    assert [l for l in r.stdout.splitlines() if not l.startswith("[init]")] == case["stdout_lines"]
    assert out.read_text() == case["csv"]


@pytest.mark.parametrize("case", GOLD["runs"], ids=lambda c: f"W({c['n']},{c['w']}) seed {c['seed']}")
def test_one_thread_run_retraces_reference(case, tmp_path):
    out = tmp_path / "o.csv"
    r = subprocess.run([CLI, str(case["n"]), str(case["w"]), "-t", "1", "--seed", str(case["seed"]), "-o", str(out)]
                       + case["extra"], capture_output=True, text=True, timeout=600)
    assert r.returncode == case["returncode"], r.stderr
    lines = r.stdout.splitlines()
    done = [l for l in lines if l.startswith("done moves=")][0]
    assert int(done.split()[1].split("=")[1]) == case["moves"]
    assert [l for l in lines if l.startswith("[t=0s] start")][0] == case["start_line"]
    assert out.read_text() == case["csv"]
    assert [l for l in lines if l.startswith(("Final", "Found", "No weighing", "W:"))
            or (l and l[0] in "-01" and "," in l)] == case["final_lines"]


def test_tempering_run_solves_and_verifies(tmp_path):
    out = tmp_path / "o.csv"
    r = subprocess.run([CLI, "12", "11", "-t", "4", "--seed", "9", "--max-seconds", "60", "-o", str(out)],
                       capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stderr
    assert "(parallel tempering)" in r.stdout
    assert "Found W(12,11); exact verification passed" in r.stdout


def test_c_abi_run():
    # xw_cpu_run through ctypes: the same result as the command line
    case = GOLD["runs"][0]
    res, W = X.cpu_run(case["n"], case["w"], threads=1, seed=case["seed"])
    assert res.solved and res.verified and res.moves == case["moves"]
    rows = [list(map(int, l.split(","))) for l in case["csv"].splitlines()]
    assert (W.reshape(case["n"], case["n"]).T == np.array(rows, dtype=np.int8)).all()
