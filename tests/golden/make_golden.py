"""Regenerate the golden fixtures from the reference's own code.

Run in a container that has the reference tree (read-only) after
`make -C oracle` has built oracle/_ref/ from it:

    python tests/golden/make_golden.py            (every fixture)
    python tests/golden/make_golden.py cpu_cli    (cpu_cli.json alone)

Every fixture here comes from executing flinty-mathematics/xtax code:
oracle/_ref/ref_harness (a driver around src/xweigh_anneal.hpp),
oracle/_ref/xweigh (src/xweigh_main.cpp) and oracle/_ref/xweigh_cuda
(src/xweigh_cuda_main.cpp, only its paths that need no GPU).  Tests read
the committed JSON files; nothing at test time needs the reference tree.
"""
import json
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
REF = os.path.join(REPO, "oracle", "_ref")
HARNESS = os.path.join(REF, "ref_harness")


def harness(*args):
    out = subprocess.run([HARNESS] + [str(a) for a in args], check=True,
                         capture_output=True, text=True).stdout
    return [json.loads(line) for line in out.splitlines() if line.strip()]


def dump(name, obj):
    with open(os.path.join(HERE, name), "w") as f:
        json.dump(obj, f, separators=(",", ":"))
        f.write("\n")
    print("wrote", name)


def starts():
    cases = [(12, 11, 1), (12, 11, 2), (10, 9, 2), (16, 4, 1), (26, 25, 1),
             (30, 29, 3), (20, 10, 5), (7, 4, 1), (13, 9, 2), (64, 4, 7),
             (64, 32, 11), (14, 13, 99), (18, 17, 1234567), (24, 23, 4294967295)]
    return [harness("start", n, w, s)[0] for n, w, s in cases]


def moves():
    cases = [(12, 11, 3, 300), (16, 4, 4, 300), (20, 10, 5, 300), (26, 25, 6, 200),
             (13, 9, 7, 200), (64, 4, 8, 150)]
    return [harness("moves", n, w, s, k)[0] for n, w, s, k in cases]


def compound():
    cases = [(12, 11, 3, 200), (16, 4, 4, 200), (20, 10, 5, 200), (26, 25, 6, 150)]
    return [harness("compound", n, w, s, k)[0] for n, w, s, k in cases]


def walks():
    cases = [
        # n w seed max_moves t_init t_min cooling moves_per_cool stuck
        (10, 9, 2, 10**8, 0, 0.25, 0.999, 500, 50000),     # solves at 42303 moves
        (12, 11, 1, 200000, 0, 0.25, 0.999, 500, 50000),
        (12, 11, 5, 300000, 4.0, 0.05, 0.997811, 500, 2000),  # reheat + reseed paths
        (16, 4, 3, 200000, 0, 0.25, 0.999, 500, 50000),
        (26, 25, 1, 100000, 6.0, 0.1, 0.99, 100, 5000),
        (20, 10, 9, 100000, 0, 0.25, 0.999, 500, 3000),
    ]
    return [harness("walk", *c)[0] for c in cases]


def calibrate():
    cases = [(12, 11, 1), (26, 25, 7), (16, 4, 2), (30, 29, 3)]
    return [harness("calibrate", n, w, s)[0] for n, w, s in cases]


def sylvester():
    cases = [(16, 4), (8, 8), (12, 4), (32, 16), (4, 4), (6, 2), (64, 4)]
    return [harness("sylvester", n, w)[0] for n, w in cases]


CSV_CASES = {
    "ok_10_9.csv": None,  # filled from a solved run below
    "short_row.csv": "1,1,1\n",
    "nonternary.csv": None,
    "empty_entry.csv": None,
    "bad_weight.csv": None,
    "bad_column.csv": None,
    "too_many_rows.csv": None,
    "extra_entry.csv": None,
}


def csv_fixtures(solved_w):
    n, w = 10, 9
    rows = [[solved_w[c * n + r] for c in range(n)] for r in range(n)]

    def text(rs):
        return "".join(",".join(str(v) for v in row) + "\n" for row in rs)

    files = {}
    files["ok_10_9.csv"] = text(rows)
    files["short_row.csv"] = text(rows[:3]) + "1,1,1\n" + text(rows[4:])
    bad = [list(r) for r in rows]; bad[2][3] = 2
    files["nonternary.csv"] = text(bad)
    e = text(rows).splitlines(); e[1] = e[1].replace(",", ", ,", 1)
    files["empty_entry.csv"] = "\n".join(e) + "\n"
    bw = [list(r) for r in rows]
    z = bw[0].index(0); bw[0][z] = 1
    files["bad_weight.csv"] = text(bw)
    # swap a zero and a nonzero between two rows' positions in one column only
    bc = [list(r) for r in rows]
    z0 = bc[0].index(0)
    nz = next(c for c in range(n) if c != z0 and bc[0][c] != 0)
    bc[0][z0], bc[0][nz] = bc[0][nz], 0
    files["bad_column.csv"] = text(bc)
    files["too_many_rows.csv"] = text(rows) + text(rows[:1])
    ex = text(rows).splitlines(); ex[4] = ex[4] + ",0"
    files["extra_entry.csv"] = "\n".join(ex) + "\n"
    files["spaces_ok.csv"] = "".join(" " + " , ".join(str(v) for v in row) + " \r\n" for row in rows)
    out = []
    for name, body in sorted(files.items()):
        path = os.path.join(HERE, "csv", name)
        with open(path, "w", newline="") as f:
            f.write(body)
        rec = harness("csv", n, w, path)[0]
        rec["path"] = "csv/" + name
        out.append(rec)
    return out


def cli_runs():
    """Reference CPU xweigh runs that solve: deterministic for one thread."""
    res = []
    for seed in (1, 2, 3):
        outp = f"/tmp/xw_golden_{seed}.csv"
        r = subprocess.run([os.path.join(REF, "xweigh"), "10", "9", "-t", "1",
                            "--seed", str(seed), "-o", outp],
                           capture_output=True, text=True, timeout=600)
        done = [l for l in r.stdout.splitlines() if l.startswith("done moves=")][0]
        moves = int(done.split()[1].split("=")[1])
        W = []
        rows = [list(map(int, l.split(","))) for l in open(outp).read().splitlines()]
        for c in range(10):
            for rr in range(10):
                W.append(rows[rr][c])
        res.append({"n": 10, "w": 9, "seed": seed, "moves": moves, "returncode": r.returncode,
                    "final": W, "final_lines": [l for l in r.stdout.splitlines()
                                                 if l.startswith(("Final", "Found", "No weighing"))]})
    return res


def cuda_cli_nogpu():
    """Paths of the reference xweigh_cuda CLI that run without a GPU:
    option validation, existence checks, the Sylvester construction and
    argument parsing errors."""
    cases = [
        ["10", "9", "--sign-fraction", "2"],
        ["10", "9", "--candidate-samples", "33"],
        ["10", "9", "--target-samples", "0"],
        ["10", "9", "--cooling", "1"],
        ["10", "9", "--t-min", "0"],
        ["10", "9", "--squared-objective-fraction", "0.6", "--parity-objective-fraction", "0.6"],
        ["10", "9", "--restart-kick-min", "5", "--restart-kick-max", "4"],
        ["10", "9", "--restart-fraction", "0"],
        ["10", "9", "--moves-per-launch", "0"],
        ["10", "9", "--replicas", "-1"],
        ["10", "9", "--device", "-1"],
        ["9", "10"],
        ["6", "6"],
        ["7", "5"],
        ["11", "9"],
        ["14", "7"],
        ["16", "4"],
        ["8", "8"],
        ["32", "16"],
        ["12", "4"],
        ["10"],
        ["10", "9", "--bogus", "3"],
        ["abc", "9"],
        ["40000", "9"],
        ["10", "9", "--start", "/nonexistent/start.csv"],
    ]
    out = []
    for args in cases:
        outp = "/tmp/xw_golden_cuda_cli.csv"
        if os.path.exists(outp):
            os.remove(outp)
        r = subprocess.run([os.path.join(REF, "xweigh_cuda")] + args + ["-o", outp],
                           capture_output=True, text=True, timeout=60)
        csv_text = open(outp).read() if os.path.exists(outp) else None
        out.append({"args": args, "returncode": r.returncode, "stdout": r.stdout,
                    "stderr": r.stderr, "csv": csv_text})
    return out


def cpu_cli():
    """The reference CPU xweigh CLI: option validation, existence checks,
    the Sylvester construction and argument errors (no timing in their
    output), and one-thread runs that solve, whose trajectories are
    deterministic: the final W, the move count of the done line, the start
    line and the closing lines."""
    errors = [
        ["10", "9", "--sign-fraction", "2"],
        ["10", "9", "--threads", "0"],
        ["10", "9", "--candidate-samples", "0"],
        ["10", "9", "--target-samples", "0"],
        ["10", "9", "--cooling", "1"],
        ["10", "9", "--t-min", "0"],
        ["10", "9", "--reseed-factor", "0.5"],
        ["10", "9", "--exchange-interval", "0"],
        ["9", "10"],
        ["6", "6"],
        ["7", "5"],
        ["14", "7"],
        ["10"],
        ["10", "9", "--bogus", "3"],
        ["abc", "9"],
    ]
    out = {"errors": [], "sylvester": [], "runs": []}
    for args in errors:
        r = subprocess.run([os.path.join(REF, "xweigh")] + args + ["-o", "/tmp/xw_golden_cpu.csv"],
                           capture_output=True, text=True, timeout=60)
        out["errors"].append({"args": args, "returncode": r.returncode, "stdout": r.stdout, "stderr": r.stderr})
    for args in (["16", "4"], ["8", "8"], ["12", "4", "-t", "2"]):
        outp = "/tmp/xw_golden_cpu_syl.csv"
        r = subprocess.run([os.path.join(REF, "xweigh")] + args + ["-o", outp], capture_output=True, text=True,
                           timeout=60)
        lines = [l for l in r.stdout.splitlines() if not l.startswith("[init]")]
        out["sylvester"].append({"args": args, "returncode": r.returncode, "stdout_lines": lines,
                                 "csv": open(outp).read()})
    for n, w, seed, extra in [(10, 9, 4, []), (10, 9, 5, []), (10, 9, 6, ["--no-tempering"]),
                              (12, 11, 2, []), (10, 9, 7, ["--t-init", "3", "--sign-fraction", "0.3"])]:
        outp = "/tmp/xw_golden_cpu_run.csv"
        r = subprocess.run([os.path.join(REF, "xweigh"), str(n), str(w), "-t", "1", "--seed", str(seed),
                            "-o", outp] + extra, capture_output=True, text=True, timeout=600)
        lines = r.stdout.splitlines()
        done = [l for l in lines if l.startswith("done moves=")][0]
        start = [l for l in lines if l.startswith("[t=0s] start")][0]
        out["runs"].append({"n": n, "w": w, "seed": seed, "extra": extra, "returncode": r.returncode,
                            "moves": int(done.split()[1].split("=")[1]), "start_line": start,
                            "csv": open(outp).read(),
                            "final_lines": [l for l in lines if l.startswith(("Final", "Found", "No weighing", "W:"))
                                            or (l and l[0] in "-01" and "," in l)]})
    return out


def main():
    if not os.path.exists(HARNESS):
        sys.exit("build oracle/_ref first: make -C oracle")
    if sys.argv[1:] == ["cpu_cli"]:
        dump("cpu_cli.json", cpu_cli())
        return
    dump("starts.json", starts())
    dump("moves.json", moves())
    dump("compound.json", compound())
    dump("calibrate.json", calibrate())
    dump("sylvester.json", sylvester())
    w = walks()
    dump("walks.json", w)
    solved = harness("walk", 10, 9, 2, 10**8, 0, 0.25, 0.999, 500, 50000)[0]["final"]
    dump("csv.json", csv_fixtures(solved))
    dump("cli_runs.json", cli_runs())
    dump("cuda_cli.json", cuda_cli_nogpu())
    dump("cpu_cli.json", cpu_cli())


if __name__ == "__main__":
    main()
