"""Generates tests/golden/batch_counts.json: exhaustive row-major counts, by the CPU
oracle, of the instances of the batched workload (puzzle.mixed_batch(4096), splitmix64
stream seed 2) that the oracle can finish here.

    python tests/golden/make_batch_counts.py [--processes N] [--estimate-limit 1e10]

Instances whose estimated tree (the oracle's Knuth estimator, 300 probes) is below the
estimate limit are counted, smallest first, each with a node limit of three times that
limit.  Only complete counts are recorded.  Records are appended as instances finish,
so the script can be stopped and resumed.
"""
from __future__ import annotations

import argparse
import json
import multiprocessing as mp
import os
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

OUT = os.path.join(HERE, "batch_counts.json")


def _count(job):
    index, width, height, colors, node_limit = job
    from oracle.oracle import OraclePuzzle
    t0 = time.time()
    r, _ = OraclePuzzle(width, height, colors).run(node_limit=node_limit)
    return index, width, int(r.nodes), int(r.solutions), int(r.status), time.time() - t0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--processes", type=int, default=max(1, (os.cpu_count() or 2) - 1))
    ap.add_argument("--estimate-limit", type=float, default=1e10)
    args = ap.parse_args()
    from edge_matching_puzzle_b200.puzzle import mixed_batch
    from oracle.oracle import OraclePuzzle
    batch = mixed_batch(4096)
    data = {"generator": "edge_matching_puzzle_b200.puzzle.mixed_batch(4096, seed=2)", "order": "row-major",
            "estimate_limit": args.estimate_limit, "records": []}
    if os.path.exists(OUT):
        with open(OUT) as f:
            data = json.load(f)
    done = {r["instance"] for r in data["records"]}
    jobs = []
    for i, pz in enumerate(batch):
        if i in done:
            continue
        est = OraclePuzzle(pz.width, pz.height, pz.colors).estimate(300, seed=1)
        if est < args.estimate_limit:
            jobs.append((est, (i, pz.width, pz.height, pz.colors, int(3 * args.estimate_limit))))
    jobs.sort(key=lambda j: j[0])
    ctx = mp.get_context("spawn")
    with ctx.Pool(args.processes) as pool:
        for k, (i, side, nodes, sols, status, sec) in enumerate(pool.imap_unordered(_count, [j[1] for j in jobs])):
            if status == 0:
                data["records"].append({"instance": i, "side": side, "nodes": nodes, "solutions": sols})
            if k % 10 == 0 or k == len(jobs) - 1:
                data["records"].sort(key=lambda r: r["instance"])
                with open(OUT, "w") as f:
                    json.dump(data, f, indent=0)
                print(f"{k + 1}/{len(jobs)} instances, last {sec:.1f}s", flush=True)
    data["records"].sort(key=lambda r: r["instance"])
    with open(OUT, "w") as f:
        json.dump(data, f, indent=0)


if __name__ == "__main__":
    main()
