"""Generates tests/golden/config_counts.json: exhaustive row-major counts computed by the
CPU oracle (the restatement of the reference's emp_strategy, pinned on the reference's own
golden vectors) for seeded puzzles of the project's workloads.

    python tests/golden/make_config_counts.py [--threads N] [--seeds 4,3,1] [--config 8x8]

Each record holds the per-seed solution count and node count of the whole search
(emp_strategy::specific_run semantics: position 0 keeps its first candidate) plus the
number of depth-12 prefixes.  Records are appended as they finish, so the script can be
stopped and resumed.
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

OUT = os.path.join(HERE, "config_counts.json")
WORKLOADS = {
    "5x5": dict(width=5, height=5, border=3, interior=5),
    "8x8": dict(width=8, height=8, border=4, interior=8),
}


def load():
    if os.path.exists(OUT):
        with open(OUT) as f:
            return json.load(f)
    return {"generator": "edge_matching_puzzle_b200.puzzle.generate", "records": []}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--threads", type=int, default=os.cpu_count() or 1)
    ap.add_argument("--seeds", default="0")
    ap.add_argument("--config", default="5x5")
    ap.add_argument("--depth", type=int, default=12)
    a = ap.parse_args()
    cfg = WORKLOADS[a.config]
    data = load()
    done = {(r["config"], r["seed"]) for r in data["records"]}
    for seed in [int(s) for s in a.seeds.split(",")]:
        if (a.config, seed) in done:
            continue
        pz = generate(cfg["width"], cfg["height"], cfg["border"], cfg["interior"], seed)
        op = OraclePuzzle(pz.width, pz.height, pz.colors)
        depth = min(a.depth, pz.nb_pieces)
        t0 = time.time()
        count, nodes_lo, sols_lo, pref = op.expand(depth, max_prefixes=1 << 62)
        nodes_hi, sols_hi = op.subtrees_parallel(pref, depth, 0, count, a.threads)
        rec = dict(config=a.config, seed=seed, width=pz.width, height=pz.height, border_colors=cfg["border"],
                   interior_colors=cfg["interior"], order="row-major", identical=op.has_identical,
                   split_depth=depth, prefixes=count, nodes=nodes_lo + nodes_hi, solutions=sols_lo + sols_hi,
                   cpu_seconds=round(time.time() - t0, 1), threads=a.threads)
        data["records"].append(rec)
        with open(OUT + ".tmp", "w") as f:
            json.dump(data, f, indent=1)
        os.replace(OUT + ".tmp", OUT)
        print(json.dumps(rec), flush=True)


if __name__ == "__main__":
    main()
