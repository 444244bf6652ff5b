"""The CPU oracle reproduces every golden vector the reference ships for this path.

These pins are what makes the oracle a trustworthy checker of the CUDA kernels:
  * tests/new_strategy_{3_3,4_4,5_5}: node and solution counts, the full "New max" trace
    and the results.bin dump, byte for byte (spiral order);
  * tests/CUDA_glutton_max_{3_3,4_4,5_5}: final boards of the glutton max search;
  * tests_CUDA/backtracker_{3_3,4_4,5_5}: first solution in row-major order.
"""
from __future__ import annotations

import base64
import os
import tempfile

import pytest

from edge_matching_puzzle_b200.puzzle import Puzzle, board_string, spiral_order
from oracle.oracle import OraclePuzzle


def _oracle(reference_vectors, name):
    pz = Puzzle.from_csv(reference_vectors["puzzles"][name])
    return pz, OraclePuzzle(pz.width, pz.height, pz.colors)


@pytest.mark.parametrize("name", ["3_3", "4_4", "5_5"])
def test_new_strategy_spiral_golden(reference_vectors, name):
    pz, op = _oracle(reference_vectors, name)
    gold = reference_vectors["new_strategy"][name]
    with tempfile.TemporaryDirectory() as d:
        path = os.path.join(d, "results.bin")
        r, log = op.run(order=spiral_order(pz.width, pz.height), results_bin=path, with_log=True)
        with open(path, "rb") as f:
            assert f.read() == base64.b64decode(gold["results_bin_b64"])
    lines = log.split("\n") + [f"Total situations explored : {r.nodes}", f"Nb solutions : {r.solutions}"]
    # the reference harness matches expected lines in order
    i = 0
    for line in lines:
        if i < len(gold["expected_stdout"]) and line == gold["expected_stdout"][i]:
            i += 1
    assert i == len(gold["expected_stdout"])


@pytest.mark.parametrize("name,nodes,solutions", [("3_3", 37, 2), ("4_4", 3284, 12), ("5_5", 37938, 1)])
def test_new_strategy_counts(reference_vectors, name, nodes, solutions):
    pz, op = _oracle(reference_vectors, name)
    r, _ = op.run(order=spiral_order(pz.width, pz.height))
    assert (r.nodes, r.solutions) == (nodes, solutions)


@pytest.mark.parametrize("name", ["3_3", "4_4", "5_5"])
def test_glutton_golden(reference_vectors, name):
    pz, op = _oracle(reference_vectors, name)
    r = op.glutton()
    assert r.status == 0
    cells = [-1] * pz.nb_pieces
    for level in range(pz.nb_pieces):
        pi = r.played[level]
        cells[pi & 0xFF] = (((pi >> 8) & 0xFF) << 2) | (pi >> 16)
    assert board_string(pz.width, pz.height, cells) == reference_vectors["glutton_max"][name][-1]


@pytest.mark.parametrize("name", ["3_3", "4_4", "5_5"])
def test_backtracker_first_solution_golden(reference_vectors, name):
    pz, op = _oracle(reference_vectors, name)
    r, _ = op.run()
    assert board_string(pz.width, pz.height, list(r.first_board)) == reference_vectors["backtracker_first_solution"][name]


def test_split_counts_equal_whole_run(reference_vectors):
    """Expansion to depth d plus every subtree equals the whole search (row-major)."""
    pz, op = _oracle(reference_vectors, "5_5_bis")
    whole, _ = op.run()
    for depth in (1, 3, 7, 12, 24):
        count, nlo, slo, pref = op.expand(depth, max_prefixes=1 << 20)
        nhi, shi = op.subtrees_parallel(pref, depth, 0, count, 2)
        assert (nlo + nhi, slo + shi) == (whole.nodes, whole.solutions)


@pytest.mark.parametrize("name", ["3_3", "4_4", "5_5"])
def test_variable_space_search_golden(reference_vectors, name):
    """The reference's variable-space CUDA_backtracker, restated (op_vs_trace): its
    selection lines for 3x3 and its first solutions (tests_CUDA/backtracker_*)."""
    pz = Puzzle.from_csv(reference_vectors["puzzles"][name])
    events, board = OraclePuzzle(pz.width, pz.height, pz.colors).vs_trace(max_events=1 << 16)
    assert board is not None
    assert board_string(pz.width, pz.height, board) == reference_vectors["backtracker_first_solution"][name]
    want = reference_vectors["backtracker_trace"][name]
    if want:
        got = [f"Thread {l} : selected variable {v} at step {s}" for l, v, s in events]
        assert got == want
