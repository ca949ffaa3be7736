"""The drop-in xweigh_cuda CLI against the reference CLI's own outputs.

tests/golden/cuda_cli.json holds the reference xweigh_cuda's stdout, stderr,
exit code and output CSV for every path that needs no GPU: option
validation, existence checks, the Sylvester construction and argument
errors.  The drop-in must reproduce them byte for byte.
"""
import json
import os
import subprocess

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CLI = os.path.join(REPO, "xtax_b200", "bin", "xweigh_cuda")
GOLD = os.path.join(REPO, "tests", "golden", "cuda_cli.json")

with open(GOLD) as f:
    CASES = json.load(f)


@pytest.mark.parametrize("case", CASES, ids=lambda c: " ".join(c["args"]))
def test_cli_matches_reference(case, tmp_path):
    out = tmp_path / "best.csv"
    r = subprocess.run([CLI] + case["args"] + ["-o", str(out)], capture_output=True, text=True, timeout=60,
                       cwd=tmp_path)
    assert r.returncode == case["returncode"], (r.stdout, r.stderr)
    assert r.stdout == case["stdout"]
    assert r.stderr == case["stderr"]
    csv = out.read_text() if out.exists() else None
    assert csv == case["csv"]


def test_cli_start_file_already_solved(tmp_path):
    # a solved --start is written back and reported without device work
    src = os.path.join(REPO, "tests", "golden", "csv", "ok_10_9.csv")
    out = tmp_path / "o.csv"
    r = subprocess.run([CLI, "10", "9", "--start", src, "-o", str(out)], capture_output=True, text=True,
                       timeout=60)
    assert r.returncode == 0, r.stderr
    assert r.stdout.startswith(f"[start] loaded {src} score=0 conflicts=0\nFinal best score: 0 conflicts=0\n"
                               "Found W(10,9); exact verification passed\nW:\n")
    assert out.read_text() == open(src).read()


def test_cli_bad_start_file_reports_reference_message(tmp_path):
    src = os.path.join(REPO, "tests", "golden", "csv", "bad_weight.csv")
    r = subprocess.run([CLI, "10", "9", "--start", src, "-o", str(tmp_path / "o.csv")], capture_output=True,
                       text=True, timeout=60)
    assert r.returncode == 1
    assert r.stderr == "Error: start matrix row 1 has weight 10, expected 9\n"


def test_cli_help():
    r = subprocess.run([CLI, "--help"], capture_output=True, text=True, timeout=60)
    assert r.returncode == 0
    assert "--double-sign-fraction" in r.stdout and "--restart-kick-max" in r.stdout
