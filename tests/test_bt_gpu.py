"""GPU parity of the exhaustive backtracker against the CPU oracle (bit-exact counts).

The CUDA path is reached through the C ABI (libemp_b200.so); the oracle is the judge.
"""
from __future__ import annotations

import random

import pytest

from edge_matching_puzzle_b200 import native
from edge_matching_puzzle_b200.puzzle import Puzzle, board_string, generate, row_major_order, spiral_order
from oracle.oracle import OraclePuzzle

pytestmark = pytest.mark.gpu


def _check(pz: Puzzle, order=None, depths=(None,), **kw):
    op = OraclePuzzle(pz.width, pz.height, pz.colors)
    want, _ = op.run(order=order)
    npz = native.NativePuzzle(pz.width, pz.height, pz.colors, order=order)
    for d in depths:
        r = native.bt_count(npz, split_depth=d or 0, **kw)
        assert r.status == native.EMP_OK
        assert (r.nodes, r.solutions) == (want.nodes, want.solutions), (d, r.nodes, want.nodes)
        if want.solutions:
            assert r.has_first_solution
            assert list(r.first_solution)[: pz.nb_pieces] == list(want.first_board)[: pz.nb_pieces]
        else:
            assert not r.has_first_solution
    return want


@pytest.mark.parametrize("name", ["3_3", "4_4", "5_5", "5_5_bis"])
def test_reference_examples_row_major(reference_vectors, name):
    pz = Puzzle.from_csv(reference_vectors["puzzles"][name])
    _check(pz, depths=(1, 2, 4, pz.nb_pieces - 1))


@pytest.mark.parametrize("name", ["3_3", "4_4", "5_5"])
def test_reference_examples_spiral(reference_vectors, name):
    """The spiral order reproduces the reference's golden counts 37/3284/37938."""
    pz = Puzzle.from_csv(reference_vectors["puzzles"][name])
    want = _check(pz, order=spiral_order(pz.width, pz.height), depths=(1, 3, pz.nb_pieces - 1))
    assert (want.nodes, want.solutions) == {"3_3": (37, 2), "4_4": (3284, 12), "5_5": (37938, 1)}[name]


def test_backtracker_first_solution_golden(reference_vectors):
    for name in ("3_3", "4_4", "5_5"):
        pz = Puzzle.from_csv(reference_vectors["puzzles"][name])
        r = native.bt_count(native.NativePuzzle(pz.width, pz.height, pz.colors), stop_at_first=1)
        board = board_string(pz.width, pz.height, list(r.first_solution))
        assert board == reference_vectors["backtracker_first_solution"][name]


@pytest.mark.parametrize("seed", [0, 1, 2, 3])
def test_config0_counts(config_counts, seed):
    rec = [r for r in config_counts["records"] if r["config"] == "5x5" and r["seed"] == seed][0]
    pz = generate(5, 5, 3, 5, seed)
    r = native.bt_count(native.NativePuzzle(5, 5, pz.colors), split_depth=12)
    assert (r.nodes, r.solutions) == (rec["nodes"], rec["solutions"])
    assert r.has_first_solution


@pytest.mark.parametrize("seed", range(24))
def test_random_small_puzzles(seed):
    """Mixed shapes and colour counts, including puzzles whose identical-piece masks
    clear unrelated candidates (half-symmetric pieces), against the oracle."""
    rng = random.Random(1000 + seed)
    while True:  # draw until the tree is small enough for the oracle (a few seconds)
        w, h = rng.randint(3, 6), rng.randint(3, 6)
        pz = generate(w, h, rng.randint(1, 3), rng.randint(2, 5), rng.randint(0, 1 << 30))
        if OraclePuzzle(w, h, pz.colors).estimate(2000) < 3e6:
            break
    _check(pz, depths=(1, min(5, w * h - 1), w * h - 1), split_budget=rng.choice([0, 256]),
           table_placement=seed % 2)  # shared-memory tables and global-memory tables


def test_batch_of_small_puzzles_one_launch():
    """Many small puzzles in one plan (tables read from global memory), per-puzzle parity."""
    rng = random.Random(77)
    puzzles = []
    while len(puzzles) < 24:
        n = rng.randint(4, 5)
        pz = generate(n, n, rng.randint(2, 3), rng.randint(3, 5), rng.randint(0, 1 << 30))
        if OraclePuzzle(n, n, pz.colors).estimate(1000) < 1e6:
            puzzles.append(pz)
    handles = [native.NativePuzzle(p.width, p.height, p.colors) for p in puzzles]
    res = native.bt_count_batch(handles, split_depth=3, split_budget=128)
    for pz, r in zip(puzzles, res):
        want, _ = OraclePuzzle(pz.width, pz.height, pz.colors).run()
        assert (r.nodes, r.solutions) == (want.nodes, want.solutions)
        if want.solutions:
            assert list(r.first_solution)[: pz.nb_pieces] == list(want.first_board)[: pz.nb_pieces]


def test_quirky_identical_masks_present():
    """At least one workload puzzle exercises identical masks with extra clears."""
    found = 0
    for seed in range(16):
        pz = generate(8, 8, 4, 8, seed)
        found += native.NativePuzzle(8, 8, pz.colors).info().identical_masks_with_extra > 0
    assert found >= 1


def test_8x8_subtree_parity_sample():  # noqa: D103
    """Per-subtree node and solution counts of an 8x8 workload puzzle against the oracle."""
    pz = generate(8, 8, 4, 8, 5)  # seed with identical masks that clear extra candidates
    npz = native.NativePuzzle(8, 8, pz.colors)
    assert npz.info().identical_masks_with_extra > 0
    op = OraclePuzzle(8, 8, pz.colors)
    depth = 18
    plan = native.BtPlan([npz], split_depth=depth, keep_subtree_counts=1, split_budget=512, timeout_ms=60000,
                         table_placement=1)
    total = plan.subtrees()
    count, _, _, _ = op.expand(depth)
    assert total == count
    sample = 1500
    stride = max(1, total // sample)
    plan.select(7, stride, sample)
    plan.run()
    res = plan.results()[0]
    nodes, sols = plan.subtree_counts(sample)
    for i in range(0, sample, 7):
        prefix = plan.subtree_prefix(i, depth)
        want_n, want_s, st = op.subtree(prefix)
        assert (nodes[i], sols[i]) == (want_n, want_s), i
    assert res.nodes == sum(nodes) and res.solutions == sum(sols)


def test_8x8_largest_seed_subtree_sample():
    """Seed 13, the largest workload tree (1.5e13 placements, beyond a CPU count here):
    per-subtree counts of a spread-out sample of its depth-12 subtrees against the oracle."""
    pz = generate(8, 8, 4, 8, 13)
    npz = native.NativePuzzle(8, 8, pz.colors)
    op = OraclePuzzle(8, 8, pz.colors)
    depth = 12
    plan = native.BtPlan([npz], split_depth=depth, keep_subtree_counts=1, timeout_ms=120000)
    total = plan.subtrees()
    count, _, _, _ = op.expand(depth, max_prefixes=1 << 40)
    assert total == count
    sample = 600
    stride = total // sample
    plan.select(3, stride, sample)
    plan.run()
    res = plan.results()[0]
    assert res.status == native.EMP_OK
    nodes, sols = plan.subtree_counts(sample)
    for i in range(0, sample, 10):
        prefix = plan.subtree_prefix(i, depth)
        want_n, want_s, _ = op.subtree(prefix)
        assert (nodes[i], sols[i]) == (want_n, want_s), i
    assert res.nodes == sum(nodes) and res.solutions == sum(sols)


@pytest.mark.parametrize("rank", range(5))
def test_8x8_full_count_against_cpu_golden(config_counts, rank):
    """Whole exhaustive count of an 8x8 workload seed (the five smallest trees, 3.8e9 to
    4.8e10 placements) equals the CPU oracle's count."""
    recs = sorted((r for r in config_counts["records"] if r["config"] == "8x8"), key=lambda r: r["nodes"])
    rec = recs[rank]
    pz = generate(8, 8, 4, 8, rec["seed"])
    r = native.bt_count(native.NativePuzzle(8, 8, pz.colors), split_depth=12, timeout_ms=60000)
    assert r.status == native.EMP_OK
    assert (r.nodes, r.solutions) == (rec["nodes"], rec["solutions"])


def test_split_depth_invariance():
    pz = generate(6, 6, 3, 4, 11)
    npz = native.NativePuzzle(6, 6, pz.colors)
    got = {d: (lambda r: (r.nodes, r.solutions))(native.bt_count(npz, split_depth=d)) for d in (1, 6, 12, 20, 35)}
    assert len(set(got.values())) == 1


@pytest.mark.parametrize("budget", [64, 1024, 1 << 20])
def test_split_budget_invariance(budget):
    """Handing work back between rounds (small budgets: many rounds) changes nothing."""
    pz = generate(6, 6, 3, 4, 5)
    want = _check(pz, depths=(6,), split_budget=budget)
    r = native.bt_count(native.NativePuzzle(6, 6, pz.colors), split_depth=6, split_budget=budget)
    assert r.nodes == want.nodes
    if budget == 64:
        assert r.rounds > 1


def test_timeout_stops_kernel():
    pz = generate(8, 8, 4, 8, 13)  # the largest tree of the workload
    npz = native.NativePuzzle(8, 8, pz.colors)
    import ctypes
    cfg = native.bt_config(split_depth=12, timeout_ms=200)
    r = native.BtResult()
    st = native.load().emp_bt_count(npz.handle, ctypes.byref(cfg), ctypes.byref(r))
    assert st == native.EMP_INCOMPLETE
    assert r.kernel_ms < 5000


def test_stop_at_any_solution(config_counts):
    """stop_at_any ends the run at the first solution any thread finds: a solution board,
    a device time to it, fewer placements than the whole count.  A puzzle without
    solutions is counted completely."""
    recs = {r["seed"]: r for r in config_counts["records"] if r["config"] == "8x8"}
    pz = generate(8, 8, 4, 8, 4)  # one solution
    npz = native.NativePuzzle(8, 8, pz.colors)
    full = native.bt_count(npz, split_depth=12)
    r = native.bt_count(npz, split_depth=12, stop_at_any=1)
    assert r.has_first_solution and r.first_found_us > 0
    assert list(r.first_solution) == list(full.first_solution)
    assert r.nodes < recs[4]["nodes"]
    pz0 = generate(8, 8, 4, 8, 12)  # no solution
    r0 = native.bt_count(native.NativePuzzle(8, 8, pz0.colors), split_depth=12, stop_at_any=1)
    assert r0.first_found_us == 0 and not r0.has_first_solution
    assert (r0.nodes, r0.solutions) == (recs[12]["nodes"], 0)
    assert r0.status == native.EMP_OK


def _results_bin(pz, order, solutions, total):
    """The reference's solution file from (node_index, board) pairs."""
    import struct
    n = pz.width * pz.height
    out = struct.pack("<4I", 1, pz.width, pz.height, 1)
    for pos in order:
        out += struct.pack("<2I", pos % pz.width, pos // pz.width)
    field = (n - 1).bit_length() + 2
    words = (n * field + 63) // 64
    for node_index, board in solutions:
        v = 0
        for i, pos in enumerate(order):
            v |= board[pos] << (i * field)
        out += v.to_bytes(8 * words, "little") + struct.pack("<Q", node_index)
    return out + struct.pack("<Q", total)


@pytest.mark.parametrize("seed", range(8))
def test_solution_dump_matches_oracle_results_bin(tmp_path, seed):
    """emp_bt_solutions: every solution with the node index of the sequential search,
    byte-identical to the oracle's results.bin (row-major and spiral orders)."""
    rng = random.Random(7000 + seed)
    while True:
        w, h = rng.randint(3, 5), rng.randint(3, 5)
        pz = generate(w, h, rng.randint(1, 3), rng.randint(2, 4), rng.randint(0, 1 << 30))
        op = OraclePuzzle(w, h, pz.colors)
        if op.estimate(1000) < 2e6:
            break
    orders = [row_major_order(w, h)]
    if sorted(spiral_order(w, h)) == list(range(w * h)):  # the spiral walk covers boards with w >= h
        orders.append(spiral_order(w, h))
    for order in orders:
        path = str(tmp_path / "oracle.bin")
        want, _ = op.run(order=order, results_bin=path)
        npz = native.NativePuzzle(w, h, pz.colors, order=order)
        found, sols, res = native.bt_solutions(npz, capacity=1 << 16, split_depth=min(4, w * h - 2))
        assert found == want.solutions and res.nodes == want.nodes
        assert _results_bin(pz, order, sols, res.nodes) == open(path, "rb").read()
