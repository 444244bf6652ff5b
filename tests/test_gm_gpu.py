"""GPU parity of the glutton max search against the CPU oracle (restatement of
include/CUDA_glutton_max.h, pinned on the reference's tests/CUDA_glutton_max_* boards).

The search trajectory (every push and pop, the final and best boards) must be
identical; the number of candidate trials is not compared, because the GPU runs the
validity fixpoint as passes over a fixed level instead of the reference's in-place
sweep (same fixpoint, different number of evaluations)."""
from __future__ import annotations

import random

import pytest

from edge_matching_puzzle_b200 import native
from edge_matching_puzzle_b200.puzzle import Puzzle, board_string, generate
from oracle.oracle import OraclePuzzle

pytestmark = pytest.mark.gpu


def _boards(pz, r):
    cells = [-1] * pz.nb_pieces
    for level in range(r.level if r.status == 0 else 0):
        pi = r.played[level]
        cells[pi & 0xFF] = (((pi >> 8) & 0xFF) << 2) | (pi >> 16)
    best = [-1] * pz.nb_pieces
    for level in range(r.max_level):
        pi = r.max_played[level]
        if pi != 0xFFFFFFFF:
            best[pi & 0xFF] = (((pi >> 8) & 0xFF) << 2) | (pi >> 16)
    return cells, best


@pytest.mark.parametrize("name", ["3_3", "4_4", "5_5"])
def test_reference_glutton_boards(reference_vectors, name):
    pz = Puzzle.from_csv(reference_vectors["puzzles"][name])
    r = native.glutton_max(native.NativePuzzle(pz.width, pz.height, pz.colors), timeout_ms=60000)
    assert r.status == 0
    assert board_string(pz.width, pz.height, list(r.final_board)) == reference_vectors["glutton_max"][name][-1]


def _compare(pz, push_budget=0, blocks=0):
    want = OraclePuzzle(pz.width, pz.height, pz.colors).glutton(push_budget=push_budget)
    got = native.glutton_max(native.NativePuzzle(pz.width, pz.height, pz.colors), push_budget=push_budget,
                             timeout_ms=60000, blocks=blocks)
    assert (got.status, got.max_level, got.pushes, got.pops, got.levels) == \
        (want.status, want.max_level, want.pushes, want.pops, want.levels_evaluated)
    cells, best = _boards(pz, want)
    if want.status == 0:
        assert list(got.final_board)[: pz.nb_pieces] == [c & 0xFFFFFFFF for c in cells]
    assert [c if c != 0xFFFFFFFF else -1 for c in list(got.best_board)[: pz.nb_pieces]] == best


# blocks: 1 = one block, 0 = one block per SM (the trials of each pass shared over the grid)
@pytest.mark.parametrize("blocks", [1, 0])
@pytest.mark.parametrize("seed", range(12))
def test_random_puzzles_full_search(seed, blocks):
    rng = random.Random(500 + seed)
    w, h = rng.randint(3, 5), rng.randint(3, 5)
    _compare(generate(w, h, rng.randint(2, 3), rng.randint(3, 6), seed), blocks=blocks)


@pytest.mark.parametrize("blocks", [1, 0])
@pytest.mark.parametrize("seed,budget", [(0, 10), (1, 40), (2, 100)])
def test_push_budget_trajectory(seed, budget, blocks):
    """Bounded searches on larger puzzles stop at the same point with the same best board."""
    _compare(generate(8, 8, 4, 8, seed), push_budget=budget, blocks=blocks)


def test_grid_and_single_block_agree_on_16x16():
    """The first levels of the 16x16 search: the multi-block search takes the single
    block's trajectory (same pushes, pops, boards and trial count)."""
    pz = generate(16, 16, 5, 17, 7)
    h = native.NativePuzzle(16, 16, pz.colors)
    one = native.glutton_max(h, push_budget=40, timeout_ms=120000, blocks=1)
    grid = native.glutton_max(h, push_budget=40, timeout_ms=120000, blocks=0)
    for f in ("status", "max_level", "level", "pushes", "pops", "levels", "passes", "trials"):
        assert getattr(one, f) == getattr(grid, f), f
    assert list(one.best_board) == list(grid.best_board)
    assert list(one.final_board) == list(grid.final_board)


def test_placement_budget_stops_the_search():
    """A placement budget (trial evaluations + pushes) stops the search at a level start."""
    import ctypes
    pz = generate(5, 5, 3, 5, 11)
    h = native.NativePuzzle(5, 5, pz.colors)
    full = native.glutton_max(h, timeout_ms=60000)
    budget = (full.trials + full.pushes) // 2
    cfg = native.GmConfig()
    cfg.device = -1
    cfg.timeout_ms = 60000
    cfg.placement_budget = budget
    r = native.GmResult()
    st = native.load().emp_glutton_max(h.handle, ctypes.byref(cfg), ctypes.byref(r))
    assert st == native.EMP_INCOMPLETE and r.status == 1
    assert r.trials + r.pushes >= budget
    assert r.levels < full.levels


def test_16x16_first_pushes_against_oracle():
    """The 16x16 workload puzzle (5 border / 17 interior colours, seed 7) at its own size:
    the first pushes of the GPU search, one block and the whole grid, take the oracle's
    trajectory (tests/golden/glutton_16x16.json, made by make_glutton_counts.py: the
    oracle needs minutes per push at this size)."""
    import json
    import os
    with open(os.path.join(os.path.dirname(__file__), "golden", "glutton_16x16.json")) as f:
        recs = json.load(f)["records"]
    pz = generate(16, 16, 5, 17, 7)
    h = native.NativePuzzle(16, 16, pz.colors)
    for rec in recs:
        for blocks in (1, 0):
            got = native.glutton_max(h, push_budget=rec["push_budget"], timeout_ms=120000, blocks=blocks)
            assert (got.status, got.max_level, got.level, got.pushes, got.pops, got.levels) == \
                (rec["status"], rec["max_level"], rec["level"], rec["pushes"], rec["pops"], rec["levels_evaluated"])
            cells = [-1] * 256
            for pi in rec["played"]:
                cells[pi & 0xFF] = (((pi >> 8) & 0xFF) << 2) | (pi >> 16)
            assert [c if c != 0xFFFFFFFF else -1 for c in list(got.final_board)[:256]] == cells
