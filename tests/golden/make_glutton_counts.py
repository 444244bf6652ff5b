"""Generates tests/golden/glutton_16x16.json: the CPU oracle's glutton max search
(restatement of include/CUDA_glutton_max.h, pinned on the reference's
tests/CUDA_glutton_max_* boards) on the 16x16 workload puzzle (5 border / 17 interior
colours, seed 7), bounded by a push budget.

    python tests/golden/make_glutton_counts.py [--push-budget 3]

The oracle evaluates about 6.5e3 trials per second here, so each of the first pushes of
the 16x16 search takes minutes; the GPU test (tests/test_gm_gpu.py) compares the GPU
search with this file instead of running the oracle.  The oracle's trial count is the
reference's own unit of work (one evaluation per candidate of its in-place sweeps plus
one per committed push).
"""
from __future__ import annotations

import argparse
import json
import os
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from edge_matching_puzzle_b200.puzzle import generate  # noqa: E402
from oracle.oracle import OraclePuzzle  # noqa: E402


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--push-budget", type=int, default=3)
    a = ap.parse_args()
    pz = generate(16, 16, 5, 17, 7)
    op = OraclePuzzle(16, 16, pz.colors)
    records = []
    for pb in range(1, a.push_budget + 1):
        t0 = time.time()
        r = op.glutton(push_budget=pb)
        records.append(dict(push_budget=pb, status=r.status, placements=r.placements, max_level=r.max_level,
                            level=r.level, pushes=r.pushes, pops=r.pops, levels_evaluated=r.levels_evaluated,
                            played=list(r.played)[: r.level], max_played=list(r.max_played)[: r.max_level],
                            cpu_seconds=round(time.time() - t0, 1)))
        print(json.dumps({k: v for k, v in records[-1].items() if k not in ("played", "max_played")}), flush=True)
    with open(os.path.join(HERE, "glutton_16x16.json"), "w") as f:
        json.dump({"puzzle": "generate(16, 16, 5, 17, 7)", "records": records}, f, indent=1)


if __name__ == "__main__":
    main()
