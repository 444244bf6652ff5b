"""Batched runs of the exhaustive backtracker: one CUDA graph per run (device-side round
loop), per-puzzle split depths for mixed sizes, per-puzzle completeness under a
deadline, and the autotuner.  Counts are checked against the CPU oracle."""
from __future__ import annotations

import ctypes
import random

import pytest

from edge_matching_puzzle_b200 import native
from edge_matching_puzzle_b200.puzzle import generate, mixed_batch
from oracle.oracle import OraclePuzzle

pytestmark = pytest.mark.gpu


def _oracle_counts(pz):
    want, _ = OraclePuzzle(pz.width, pz.height, pz.colors).run()
    return want.nodes, want.solutions


def _small_mixed(count, seed, limit=2e5):
    rng = random.Random(seed)
    out = []
    while len(out) < count:
        side = rng.randint(3, 6)
        pz = generate(side, side, rng.randint(2, 4), rng.randint(3, 7), rng.randint(0, 1 << 30))
        if OraclePuzzle(side, side, pz.colors).estimate(500) < limit:
            out.append(pz)
    return out


@pytest.mark.parametrize("budget", [64, 2048])
def test_graph_run_matches_host_loop(budget):
    """The same plan run by the host round loop and as one graph launch: same counts; the
    graph is relaunched, and rebuilt after a new selection."""
    pz = generate(6, 6, 3, 4, 5)
    want = _oracle_counts(pz)
    h = native.NativePuzzle(6, 6, pz.colors)
    host = native.BtPlan([h], split_depth=6, split_budget=budget)
    host.run()
    r0 = host.results()[0]
    graph = native.BtPlan([h], split_depth=6, split_budget=budget, use_graph=1)
    for _ in range(2):
        graph.run()
        r1 = graph.results()[0]
        assert (r1.nodes, r1.solutions) == (r0.nodes, r0.solutions) == want
        assert r1.status == native.EMP_OK
        if budget == 64:
            assert r1.rounds > 1
    n = graph.subtrees()
    count = (n - 1 + 2) // 3
    for plan in (graph, host):
        plan.select(1, 3, count)
        plan.run()
    assert (graph.results()[0].nodes, graph.results()[0].solutions) == \
        (host.results()[0].nodes, host.results()[0].solutions)
    host.close()
    graph.close()


@pytest.mark.parametrize("target", [1, 16, 256])
def test_per_puzzle_split_depths_match_oracle(target):
    """Mixed sizes in one graph launch, each puzzle split at its own depth."""
    puzzles = _small_mixed(48, 900 + target)
    handles = [native.NativePuzzle(p.width, p.height, p.colors) for p in puzzles]
    res = native.bt_count_batch(handles, split_subtrees=target, split_budget=256, use_graph=1)
    for pz, r in zip(puzzles, res):
        assert (r.nodes, r.solutions) == _oracle_counts(pz)
        assert r.status == native.EMP_OK
        assert 1 <= r.split_depth <= pz.nb_pieces - 1
        if target == 1:
            assert r.split_depth == 1


def test_per_puzzle_depth_limit():
    puzzles = _small_mixed(8, 31)
    handles = [native.NativePuzzle(p.width, p.height, p.colors) for p in puzzles]
    res = native.bt_count_batch(handles, split_subtrees=1 << 30, split_depth=5)
    for pz, r in zip(puzzles, res):
        assert r.split_depth <= 5
        assert (r.nodes, r.solutions) == _oracle_counts(pz)


@pytest.mark.parametrize("use_graph", [0, 1])
def test_deadline_marks_only_unfinished_puzzles(use_graph):
    """A batch holding 9x9 puzzles far too large to finish and small ones: under a
    deadline, the large ones are flagged incomplete, the small ones are exact."""
    small = _small_mixed(12, 4242)
    big = [generate(9, 9, 3, 4, s) for s in (1, 2)]
    puzzles = small[:6] + big[:1] + small[6:] + big[1:]
    handles = [native.NativePuzzle(p.width, p.height, p.colors) for p in puzzles]
    cfg = native.bt_config(split_subtrees=512, timeout_ms=400, use_graph=use_graph)
    res = (native.BtResult * len(handles))()
    arr = (ctypes.c_void_p * len(handles))(*[h.handle for h in handles])
    st = native.load().emp_bt_count_batch(arr, len(handles), ctypes.byref(cfg), res)
    assert st == native.EMP_INCOMPLETE
    for pz, r in zip(puzzles, res):
        if pz.width == 9:
            assert r.status == native.EMP_INCOMPLETE
            assert r.nodes > 0
        else:
            assert r.status == native.EMP_OK
            assert (r.nodes, r.solutions) == _oracle_counts(pz)
    assert res[0].kernel_ms < 5000


def test_autotune_picks_a_runnable_configuration():
    puzzles = _small_mixed(16, 77, limit=1e6)
    handles = [native.NativePuzzle(p.width, p.height, p.colors) for p in puzzles]
    tune = native.bt_autotune(handles, trial_ms=100, use_graph=1, table_placement=1)
    assert tune.trials >= 8
    assert tune.best_rate >= tune.default_rate > 0
    best = native.config_dict(tune.best)

    res = native.bt_count_batch(handles, **best)
    for pz, r in zip(puzzles, res):
        assert (r.nodes, r.solutions) == _oracle_counts(pz)


def test_mixed_batch_sample_against_oracle():
    """The first 512 instances of the batched workload (sides 4..9) under a deadline:
    every instance with a small tree finishes, and every finished instance that the
    oracle can count quickly is exact."""
    batch = mixed_batch(512)
    handles = [native.NativePuzzle(p.width, p.height, p.colors) for p in batch]
    res = native.bt_count_batch(handles, split_subtrees=1024, timeout_ms=3000, use_graph=1, table_placement=1)
    checked = 0
    for pz, r in zip(batch, res):
        est = OraclePuzzle(pz.width, pz.height, pz.colors).estimate(300)
        if est < 2e4:
            assert r.status == native.EMP_OK
        if r.status == native.EMP_OK and est < 1e6:
            assert (r.nodes, r.solutions) == _oracle_counts(pz)
            checked += 1
    assert checked > 200


def test_full_batch_against_cpu_counts():
    """All 4096 instances of the batched workload in one graph launch with a deadline:
    every instance the GPU finishes and the CPU oracle counted (tests/golden/
    batch_counts.json, made by make_batch_counts.py) has exactly the oracle's counts, and
    every small instance of side 6 or less is finished.  Subtrees are queued by piece
    count, so those come first; a 7x7 instance can wait behind the huge subtrees of
    other 7x7 instances until the deadline, which is correct (it is flagged)."""
    import json
    import os
    with open(os.path.join(os.path.dirname(__file__), "golden", "batch_counts.json")) as f:
        golden = {r["instance"]: (r["nodes"], r["solutions"]) for r in json.load(f)["records"]}
    batch = mixed_batch(4096)
    handles = [native.NativePuzzle(p.width, p.height, p.colors) for p in batch]
    res = native.bt_count_batch(handles, split_subtrees=1024, timeout_ms=4000, use_graph=1, table_placement=1)
    checked = 0
    golden7 = finished7 = 0
    for i, r in enumerate(res):
        assert r.status in (native.EMP_OK, native.EMP_INCOMPLETE), (i, r.status)
        if r.status == native.EMP_OK and i in golden:
            assert (r.nodes, r.solutions) == golden[i], i
            checked += 1
        if i in golden and golden[i][0] < 20000 and batch[i].width <= 6:
            assert r.status == native.EMP_OK, i
        if i in golden and batch[i].width == 7:
            golden7 += 1
            finished7 += r.status == native.EMP_OK
    assert checked >= 1500
    # 7x7 instances queue behind 4x4..6x6 ones and share the GPU with the 8x8 and 9x9
    # subtrees that threads take once the 7x7 ones are handed out; 60 to 83 of the 430
    # CPU-countable ones finished within the 4 s on a B200 with the default global stack.
    # A scheduling change that starves them fails here
    assert golden7 >= 100 and finished7 >= golden7 // 10, (finished7, golden7)
