"""Generates tests/golden/ref_counts.json: exhaustive counts made by the reference's OWN
new_strategy search (include/emp_strategy.h and the headers it includes), compiled
unmodified from the reference tree into oracle/_ref/ by ``make -C oracle ref`` with the
project-written stand-ins of oracle/ref_shim/ for its missing external libraries.

    python tests/golden/make_ref_counts.py --reference /path/to/reference [--jobs N] [--big]

The reference refuses a puzzle with identical pieces unless it was built with
HANDLE_IDENTICAL_PIECES, and the other way round (include/emp_piece_db.h:876-891); each
puzzle runs with the matching build.  Every record holds the puzzle (CSV), the position
order, the node and solution counts, the SHA-256 of the results.bin the reference wrote,
and how many identical-mask writes fell outside a bitfield (the reference's
include/emp_piece_db.h:874-875 can index another kind's piece; the stand-in bitfield
drops such a write and counts it).  Cases:

  examples     the reference's doc/example puzzles, row-major and spiral
  config0      5x5, 3 border / 5 interior colours, seeds 0..3 (row-major)
  random       the 24 random 3x3..6x6 puzzles of tests/test_bt_gpu.py (same draws)
  quirk        random small puzzles whose identical masks clear other pieces' bits or
               write outside a bitfield
  batch        instances of the 4096-instance mixed batch with small trees
  resume       set_initial_state (the --initial_situation parameter) from mid-board
               situations of random puzzles: the search resumes there and runs to its end
  8x8 (--big)  whole counts of 8x8 workload seeds (--big-seeds)

The JSON is committed; the tests never run the reference.
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import hashlib
import json
import os
import random
import re
import subprocess
import sys
import tempfile
import time

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from edge_matching_puzzle_b200.puzzle import Puzzle, generate, mixed_batch  # noqa: E402
from oracle.oracle import OraclePuzzle  # noqa: E402

OUT = os.path.join(HERE, "ref_counts.json")
REF_BIN = os.path.join(ROOT, "oracle", "_ref")


def run_reference(case):
    """Runs one case through the matching reference build; returns the case with counts."""
    pz = Puzzle.from_csv(case["csv"])
    build = "identical" if OraclePuzzle(pz.width, pz.height, pz.colors).has_identical else "plain"
    with tempfile.TemporaryDirectory() as d:
        src = os.path.join(d, "puzzle.txt")
        with open(src, "w") as f:
            f.write(case["csv"])
        strategy = case["order"]
        if strategy not in ("basic", "spiral"):
            raise ValueError(strategy)
        res = os.path.join(d, "results.bin")
        t0 = time.time()
        cmd = [os.path.join(REF_BIN, "emp_ref_strategy_" + build), src, strategy, res]
        if case.get("initial_situation"):
            cmd.append(case["initial_situation"])
        p = subprocess.run(cmd, capture_output=True, text=True, cwd=d)
        secs = time.time() - t0
        out = p.stdout
        if p.returncode != 0:
            raise RuntimeError(f"{case['name']}: reference exited {p.returncode}: {out[-500:]} {p.stderr[-500:]}")
        with open(res, "rb") as f:
            digest = hashlib.sha256(f.read()).hexdigest()
    grab = lambda pat: int(re.search(pat, out).group(1))  # noqa: E731
    rec = dict(case)
    rec.update(build=build, nodes=grab(r"Total situations explored : (\d+)"), solutions=grab(r"Nb solutions : (\d+)"),
               out_of_range_writes=grab(r"identical-mask writes outside a bitfield : (\d+)"),
               results_sha256=digest, new_max_lines=len(re.findall(r"^New max : ", out, re.M)),
               ref_seconds=round(secs, 2))
    return rec


def small_random_cases():
    """The draws of tests/test_bt_gpu.py::test_random_small_puzzles."""
    cases = []
    for seed in range(24):
        rng = random.Random(1000 + seed)
        while True:
            w, h = rng.randint(3, 6), rng.randint(3, 6)
            pz = generate(w, h, rng.randint(1, 3), rng.randint(2, 5), rng.randint(0, 1 << 30))
            if OraclePuzzle(w, h, pz.colors).estimate(2000) < 3e6:
                break
        cases.append(dict(name=f"random_{seed}", group="random", csv=pz.to_csv(), order="basic"))
    return cases


def quirk_cases(count=24):
    """Small puzzles with few colours, so that half-symmetric pieces make the reference's
    identical masks clear other pieces' bits (cross-kind twins), some of them outside the
    bitfield."""
    cases = []
    rng = random.Random(77)
    tries = 0
    while len(cases) < count and tries < 20000:
        tries += 1
        w, h = rng.randint(4, 6), rng.randint(4, 6)
        pz = generate(w, h, rng.randint(1, 2), rng.randint(1, 3), rng.randint(0, 1 << 30))
        op = OraclePuzzle(w, h, pz.colors)
        if not op.has_identical or not cross_kind_twins(pz) or op.estimate(2000) > 2e6:
            continue
        cases.append(dict(name=f"quirk_{len(cases)}", group="quirk", csv=pz.to_csv(),
                          order="basic" if len(cases) % 3 else "spiral"))
    # Long 3-wide boards: a border piece's twin index then lies past the centre kind's
    # bitfield storage, so the reference writes outside it.
    found = 0
    while found < 6 and tries < 40000:
        tries += 1
        h = rng.randint(18, 30)
        pz = generate(3, h, rng.randint(1, 2), 1, rng.randint(0, 1 << 30))
        op = OraclePuzzle(3, h, pz.colors)
        if not op.has_identical or not cross_kind_twins(pz) or op.estimate(2000) > 2e6:
            continue
        case = dict(name=f"quirk_long_{found}", group="quirk", csv=pz.to_csv(), order="basic")
        if run_reference(case)["out_of_range_writes"]:
            cases.append(case)
            found += 1
    return cases


def cross_kind_twins(pz):
    """True when two pieces of different kinds compare equal under the reference's
    emp_piece::compare_to (include/emp_piece.h:193-220): a half-symmetric piece compares
    only two of its sides."""
    def sim(c):
        if c[0] == c[2] and c[1] == c[3]:
            return 2 if c[0] == c[1] else 1
        return 0

    def compare(a, b, o):
        inc = 1 << sim(a)
        i = 0
        while i <= 3 and a[i] == b[(i + o) & 3]:
            i += inc
        return i > 3

    kinds = [sum(1 for x in c if x == 0) for c in pz.colors]
    for i, a in enumerate(pz.colors):
        for j in range(i):
            b = pz.colors[j]
            if kinds[i] != kinds[j] and any(compare(a, b, o) for o in range(0, 4, 1 << sim(b))):
                return True
    return False


def batch_cases(limit_nodes=3e6, count=400):
    counts = json.load(open(os.path.join(HERE, "batch_counts.json")))
    small = [r for r in counts["records"] if r["nodes"] <= limit_nodes]
    small.sort(key=lambda r: r["instance"])
    step = max(1, len(small) // count)
    chosen = {r["instance"] for r in small[::step][:count]}
    puzzles = mixed_batch()
    return [dict(name=f"batch_{i}", group="batch", csv=puzzles[i].to_csv(), order="basic", batch_index=i)
            for i in sorted(chosen)]


def resume_cases(count=12):
    """Mid-board situations reached by the plain search: the first solution's path cut at
    several depths (the situation string lists the pieces placed at the levels before the
    cut, in the reference's board format)."""
    from edge_matching_puzzle_b200.puzzle import board_string, spiral_order
    cases = []
    rng = random.Random(5)
    while len(cases) < count:
        w, h = rng.randint(4, 6), rng.randint(4, 6)
        pz = generate(w, h, rng.randint(1, 3), rng.randint(2, 5), rng.randint(0, 1 << 30))
        op = OraclePuzzle(w, h, pz.colors)
        if op.estimate(2000) > 3e6:
            continue
        spiral = len(cases) % 2 == 1
        order = spiral_order(w, h) if spiral else list(range(w * h))
        r, _ = op.run(order=order)
        if not r.solutions:
            continue
        board = list(r.first_board)[: w * h]
        cut = rng.randint(2, w * h - 2)
        keep = set(order[:cut])
        cells = [board[p] if p in keep else -1 for p in range(w * h)]
        cases.append(dict(name=f"resume_{len(cases)}", group="resume", csv=pz.to_csv(),
                          order="spiral" if spiral else "basic", initial_situation=board_string(w, h, cells),
                          resume_depth=cut))
    return cases


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", required=True, help="root of the reference project (read-only)")
    ap.add_argument("--jobs", type=int, default=os.cpu_count() or 1)
    ap.add_argument("--big", action="store_true", help="also count whole 8x8 workload seeds")
    ap.add_argument("--big-seeds", default="4,12,1",
                    help="comma-separated 8x8 workload seeds for --big (the reference's search is single-threaded: "
                         "2.9e7 placements/s per core, so a seed of 2e11 placements takes about two hours)")
    a = ap.parse_args()
    subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "ref", "REF=" + a.reference], check=True)
    cases = []
    for name in ("3_3", "4_4", "5_5", "5_5_bis"):
        with open(os.path.join(a.reference, "doc", "example", name + ".txt")) as f:
            csv = f.read()
        for order in ("basic", "spiral"):
            cases.append(dict(name=f"example_{name}_{order}", group="examples", csv=csv, order=order))
    for seed in range(4):
        cases.append(dict(name=f"config0_{seed}", group="config0", csv=generate(5, 5, 3, 5, seed).to_csv(),
                          order="basic", seed=seed))
    cases += small_random_cases()
    cases += quirk_cases()
    cases += batch_cases()
    cases += resume_cases()
    if a.big:
        for seed in (int(x) for x in a.big_seeds.split(",")):
            cases.append(dict(name=f"8x8_{seed}", group="8x8", csv=generate(8, 8, 4, 8, seed).to_csv(),
                              order="basic", seed=seed))
    records = []
    with cf.ProcessPoolExecutor(a.jobs) as ex:
        for rec in ex.map(run_reference, cases):
            records.append(rec)
            print(rec["name"], rec["build"], rec["nodes"], rec["solutions"], rec["out_of_range_writes"], flush=True)
    data = {"source": "oracle/_ref: the reference's emp_strategy built from its own sources with oracle/ref_shim",
            "records": records}
    with open(OUT, "w") as f:
        json.dump(data, f, indent=1)


if __name__ == "__main__":
    main()
