"""GPU parity of the exhaustive backtracker against the CPU oracle (bit-exact counts).

The CUDA path is reached through the C ABI (libemp_b200.so); the oracle is the checker.
"""
from __future__ import annotations

import hashlib
import json
import os
import random

import pytest

from edge_matching_puzzle_b200 import native
from edge_matching_puzzle_b200.puzzle import Puzzle, board_string, generate, row_major_order, spiral_order
from oracle.oracle import OraclePuzzle

pytestmark = pytest.mark.gpu

with open(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "ref_counts.json")) as _f:
    REF_RECORDS = json.load(_f)["records"]


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


CPU_COUNTED_8X8 = [0, 1, 2, 3, 4, 5, 6, 7, 8, 9, 10, 11, 12, 14, 15]


@pytest.mark.parametrize("seed", CPU_COUNTED_8X8)
def test_8x8_full_count_against_cpu_golden(config_counts, seed):
    """Whole exhaustive count of every 8x8 workload seed the CPU could count (all but
    seed 13, 1.5e13 placements: see test_8x8_largest_seed_subtree_sample) equals the
    CPU oracle's count: 3.8e9 to 1.27e12 placements per seed, 2.6e12 in all."""
    rec = [r for r in config_counts["records"] if r["config"] == "8x8" and r["seed"] == seed][0]
    pz = generate(8, 8, 4, 8, seed)
    r = native.bt_count(native.NativePuzzle(8, 8, pz.colors), split_depth=12, timeout_ms=240000)
    assert r.status == native.EMP_OK
    assert (r.nodes, r.solutions) == (rec["nodes"], rec["solutions"])
    assert bool(r.has_first_solution) == (rec["solutions"] > 0)


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


def _ref_order(rec, pz):
    return spiral_order(pz.width, pz.height) if rec["order"] == "spiral" else row_major_order(pz.width, pz.height)


@pytest.mark.parametrize("group", ["examples", "config0", "random", "quirk", "batch"])
def test_counts_equal_reference_build(group):
    """Counts of the puzzles that the reference's own emp_strategy counted (built from
    its sources into oracle/_ref; tests/golden/ref_counts.json): identical-piece masks,
    cross-kind twin masks, masks written outside a bitfield, row-major and spiral."""
    recs = [r for r in REF_RECORDS if r["group"] == group]
    assert recs
    for rec in recs:
        pz = Puzzle.from_csv(rec["csv"])
        npz = native.NativePuzzle(pz.width, pz.height, pz.colors, order=_ref_order(rec, pz))
        r = native.bt_count(npz, split_depth=min(6, pz.nb_pieces - 1))
        assert r.status == native.EMP_OK
        assert (r.nodes, r.solutions) == (rec["nodes"], rec["solutions"]), rec["name"]


@pytest.mark.parametrize("group", ["examples", "config0", "quirk"])
def test_results_bin_equals_reference_build(group):
    """Every solution of the GPU solution dump, written as results.bin, has the SHA-256
    of the file the reference's own build wrote."""
    for rec in [r for r in REF_RECORDS if r["group"] == group and r["solutions"] <= 4096]:
        pz = Puzzle.from_csv(rec["csv"])
        order = _ref_order(rec, pz)
        npz = native.NativePuzzle(pz.width, pz.height, pz.colors, order=order)
        found, sols, res = native.bt_solutions(npz, capacity=4096, split_depth=min(4, pz.nb_pieces - 2))
        assert found == rec["solutions"] and res.nodes == rec["nodes"], rec["name"]
        digest = hashlib.sha256(_results_bin(pz, order, sols, res.nodes)).hexdigest()
        assert digest == rec["results_sha256"], rec["name"]


def test_solution_dump_capacity_keeps_reference_order(reference_vectors, tmp_path):
    """With fewer slots than solutions, emp_bt_solutions returns the FIRST solutions in
    the reference's order (the 4x4 example has 12), not the first ones to arrive."""
    pz = Puzzle.from_csv(reference_vectors["puzzles"]["4_4"])
    order = spiral_order(4, 4)
    npz = native.NativePuzzle(4, 4, pz.colors, order=order)
    found_all, all_sols, res = native.bt_solutions(npz, capacity=64, split_depth=3)
    assert found_all == 12
    want_path = str(tmp_path / "oracle.bin")
    want, _ = OraclePuzzle(4, 4, pz.colors).run(order=order, results_bin=want_path)
    assert _results_bin(pz, order, all_sols, res.nodes) == open(want_path, "rb").read()
    for cap in (1, 5, 11):
        found, sols, _ = native.bt_solutions(npz, capacity=cap, split_depth=3)
        assert found == 12 and len(sols) == cap
        assert sols == all_sols[:cap]
    assert all_sols[0][0] == want.first_solution_nodes
    assert all_sols[0][1][:16] == list(want.first_board)[:16]


def test_lost_first_solution_record_is_reported():
    """A first-solution record whose lock wait runs out is reported as EMP_FIRST_LOST
    (exact counts, no board), not as a run without a first solution.  The test holds
    every record's lock from the start (a lock nothing releases) with a 1 us bound."""
    import ctypes
    pz = generate(5, 5, 3, 5, 0)
    want, _ = OraclePuzzle(5, 5, pz.colors).run()
    npz = native.NativePuzzle(5, 5, pz.colors)
    cfg = native.bt_config(split_depth=6, hold_first_lock=1, first_lock_wait_us=1)
    r = native.BtResult()
    st = native.load().emp_bt_count(npz.handle, ctypes.byref(cfg), ctypes.byref(r))
    assert st == native.EMP_FIRST_LOST and r.status == native.EMP_FIRST_LOST
    assert not r.has_first_solution
    assert (r.nodes, r.solutions) == (want.nodes, want.solutions)
    ok = native.bt_count(npz, split_depth=6)
    assert ok.status == native.EMP_OK and ok.has_first_solution


def test_resume_equals_reference_build():
    """emp_bt_resume (--initial_situation) against the reference's own set_initial_state +
    specific_run on mid-board situations, row-major and spiral."""
    from edge_matching_puzzle_b200.puzzle import parse_board_string, situation_transitions
    recs = [r for r in REF_RECORDS if r["group"] == "resume"]
    assert recs
    for rec in recs:
        pz = Puzzle.from_csv(rec["csv"])
        order = _ref_order(rec, pz)
        trans = situation_transitions(pz, order, parse_board_string(pz.width, pz.height, rec["initial_situation"]))
        npz = native.NativePuzzle(pz.width, pz.height, pz.colors, order=order)
        for budget in (0, 64):  # work handed between threads, or not
            r = native.bt_resume(npz, trans, split_budget=budget)
            assert r.status == native.EMP_OK
            assert (r.nodes, r.solutions) == (rec["nodes"], rec["solutions"]), rec["name"]


def test_resume_rejects_unreachable_situation():
    pz = generate(5, 5, 3, 5, 0)
    npz = native.NativePuzzle(5, 5, pz.colors)
    with pytest.raises(native.EmpError):
        native.bt_resume(npz, [0, 0, 0])  # the same corner twice


def test_resume_solutions_results_bin_equals_reference_build():
    """new_strategy with --initial_situation: the resumed search's results.bin (solutions
    with the resumed search's node indices) has the SHA-256 of the reference's file."""
    from edge_matching_puzzle_b200.puzzle import parse_board_string, situation_transitions
    for rec in [r for r in REF_RECORDS if r["group"] == "resume" and r["solutions"] <= 4096]:
        pz = Puzzle.from_csv(rec["csv"])
        order = _ref_order(rec, pz)
        trans = situation_transitions(pz, order, parse_board_string(pz.width, pz.height, rec["initial_situation"]))
        npz = native.NativePuzzle(pz.width, pz.height, pz.colors, order=order)
        found, sols, res = native.bt_resume_solutions(npz, trans, capacity=4096)
        assert found == rec["solutions"] and res.nodes == rec["nodes"], rec["name"]
        assert hashlib.sha256(_results_bin(pz, order, sols, res.nodes)).hexdigest() == rec["results_sha256"], rec["name"]


@pytest.mark.parametrize("placement", [1, 2, 3, 4])
def test_stack_placements_equal_reference_build(placement):
    """Every placement of the DFS stack (shared 32-bit, shared 16-bit, global, one DFS per
    warp) gives the reference build's counts, with work handed back (small split budget)."""
    recs = [r for r in REF_RECORDS if r["group"] in ("config0", "random", "quirk")]
    for rec in recs:
        pz = Puzzle.from_csv(rec["csv"])
        npz = native.NativePuzzle(pz.width, pz.height, pz.colors, order=_ref_order(rec, pz))
        for tp in (1, 2):  # tables in global, then shared memory
            r = native.bt_count(npz, split_depth=min(4, pz.nb_pieces - 1), split_budget=64,
                                stack_placement=placement, table_placement=tp)
            assert r.status == native.EMP_OK
            assert (r.nodes, r.solutions) == (rec["nodes"], rec["solutions"]), (rec["name"], tp)


@pytest.mark.parametrize("name", ["3_3", "4_4", "5_5"])
def test_variable_space_debug_mode(reference_vectors, name):
    """emp_bt_variable_space: the reference's own CUDA_backtracker search on the GPU, its
    selection lines for 3x3 (tests_CUDA/backtracker_3_3) and first solutions, and every
    selection equal to the oracle's restatement."""
    pz = Puzzle.from_csv(reference_vectors["puzzles"][name])
    events, board, st = native.bt_variable_space(native.NativePuzzle(pz.width, pz.height, pz.colors),
                                                 capacity=1 << 16)
    assert st == native.EMP_OK and board is not None
    assert board_string(pz.width, pz.height, board) == reference_vectors["backtracker_first_solution"][name]
    want_events, want_board = OraclePuzzle(pz.width, pz.height, pz.colors).vs_trace(max_events=1 << 16)
    assert events == want_events and board == want_board
    if reference_vectors["backtracker_trace"][name]:
        assert [f"Thread {l} : selected variable {v} at step {s}" for l, v, s in events] == \
            reference_vectors["backtracker_trace"][name]


def test_warp_mode_resume_and_solutions_equal_reference_build():
    """One DFS per warp (stack_placement 4): resumed counts and the resumed search's
    results.bin equal the reference build's, with and without work handed back."""
    from edge_matching_puzzle_b200.puzzle import parse_board_string, situation_transitions
    for rec in [r for r in REF_RECORDS if r["group"] == "resume"]:
        pz = Puzzle.from_csv(rec["csv"])
        order = _ref_order(rec, pz)
        trans = situation_transitions(pz, order, parse_board_string(pz.width, pz.height, rec["initial_situation"]))
        npz = native.NativePuzzle(pz.width, pz.height, pz.colors, order=order)
        for budget in (0, 64):
            r = native.bt_resume(npz, trans, split_budget=budget, stack_placement=4)
            assert r.status == native.EMP_OK
            assert (r.nodes, r.solutions) == (rec["nodes"], rec["solutions"]), rec["name"]
        if rec["solutions"] <= 4096:
            found, sols, res = native.bt_resume_solutions(npz, trans, capacity=4096, stack_placement=4)
            assert found == rec["solutions"] and res.nodes == rec["nodes"], rec["name"]
            assert hashlib.sha256(_results_bin(pz, order, sols, res.nodes)).hexdigest() == \
                rec["results_sha256"], rec["name"]


@pytest.mark.parametrize("seed", [4, 12])
def test_warp_mode_8x8_full_count(config_counts, seed):
    """One DFS per warp on whole 8x8 workload counts (3.8e9 and 1.9e10 placements), with
    the first solution, against the CPU oracle's counts."""
    rec = [r for r in config_counts["records"] if r["config"] == "8x8" and r["seed"] == seed][0]
    pz = generate(8, 8, 4, 8, seed)
    h = native.NativePuzzle(8, 8, pz.colors)
    r = native.bt_count(h, split_depth=12, stack_placement=4, timeout_ms=240000)
    assert r.status == native.EMP_OK
    assert (r.nodes, r.solutions) == (rec["nodes"], rec["solutions"])
    ref = native.bt_count(h, split_depth=12)
    assert bool(r.has_first_solution) == (rec["solutions"] > 0)
    assert list(r.first_solution)[:64] == list(ref.first_solution)[:64]
