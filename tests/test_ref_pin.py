"""The oracle against the reference's OWN search (CPU, no GPU).

tests/golden/ref_counts.json holds the counts that the reference's emp_strategy
(include/emp_strategy.h, include/emp_position_strategy.h, include/emp_piece_db.h, built
unmodified into oracle/_ref/ with the project's stand-ins for its missing libraries) gave
on: the reference examples, the config-0 puzzles, the 24 random puzzles of the GPU tests,
puzzles whose identical-piece masks clear other pieces' bits or fall outside a bitfield,
400 instances of the mixed batch, resumed searches (--initial_situation) and 14 whole
8x8 workload seeds (all the CPU can count but seed 5).  Every one
of them has identical pieces except the reference examples, so this pins the
HANDLE_IDENTICAL_PIECES path that every workload puzzle takes.  The GPU suite compares
the CUDA path with the same file (tests/test_bt_gpu.py).
"""
from __future__ import annotations

import hashlib
import json
import os

import pytest

from edge_matching_puzzle_b200.puzzle import (Puzzle, parse_board_string, row_major_order, situation_transitions,
                                              spiral_order)
from oracle.oracle import OraclePuzzle

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
with open(os.path.join(ROOT, "tests", "golden", "ref_counts.json")) as _f:
    RECORDS = json.load(_f)["records"]


def order_of(rec, pz):
    return spiral_order(pz.width, pz.height) if rec["order"] == "spiral" else row_major_order(pz.width, pz.height)


def test_identical_piece_path_is_covered():
    identical = [r for r in RECORDS if r["build"] == "identical"]
    assert len(identical) >= 300
    assert any(r["out_of_range_writes"] for r in RECORDS)
    assert {r["group"] for r in identical} >= {"config0", "random", "quirk", "batch", "resume"}


@pytest.mark.parametrize("rec", [r for r in RECORDS if r["group"] not in ("resume", "8x8")], ids=lambda r: r["name"])
def test_oracle_equals_reference(rec, tmp_path):
    pz = Puzzle.from_csv(rec["csv"])
    op = OraclePuzzle(pz.width, pz.height, pz.colors)
    assert op.has_identical == (rec["build"] == "identical")
    res = str(tmp_path / "results.bin")
    r, _ = op.run(order=order_of(rec, pz), results_bin=res)
    assert (r.nodes, r.solutions) == (rec["nodes"], rec["solutions"])
    with open(res, "rb") as f:
        assert hashlib.sha256(f.read()).hexdigest() == rec["results_sha256"]


@pytest.mark.parametrize("rec", [r for r in RECORDS if r["group"] == "resume"], ids=lambda r: r["name"])
def test_oracle_resume_equals_reference(rec, tmp_path):
    pz = Puzzle.from_csv(rec["csv"])
    op = OraclePuzzle(pz.width, pz.height, pz.colors)
    order = order_of(rec, pz)
    trans = situation_transitions(pz, order, parse_board_string(pz.width, pz.height, rec["initial_situation"]))
    assert len(trans) == rec["resume_depth"]
    res = str(tmp_path / "results.bin")
    r = op.resume(trans, order=order, results_bin=res)
    assert (r.nodes, r.solutions) == (rec["nodes"], rec["solutions"])
    with open(res, "rb") as f:
        assert hashlib.sha256(f.read()).hexdigest() == rec["results_sha256"]


def test_8x8_workload_seeds_equal_reference():
    """Whole 8x8 workload seeds (4 border / 8 interior colours) counted by the reference's
    own search: equal to the CPU oracle's counts in tests/golden/config_counts.json, which
    the GPU suite checks the CUDA path against (test_8x8_full_count_against_cpu_golden).
    The oracle needs minutes per seed, so this compares the two files."""
    with open(os.path.join(ROOT, "tests", "golden", "config_counts.json")) as f:
        oracle = {r["seed"]: (r["nodes"], r["solutions"]) for r in json.load(f)["records"] if r["config"] == "8x8"}
    recs = [r for r in RECORDS if r["group"] == "8x8"]
    assert len(recs) >= 14
    for rec in recs:
        assert rec["build"] == "identical"
        assert (rec["nodes"], rec["solutions"]) == oracle[rec["seed"]], rec["name"]
