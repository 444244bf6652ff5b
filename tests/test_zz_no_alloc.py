"""emp_glutton_max_noalloc against emp_glutton_max.

The no-allocation entry point runs the glutton max search in a fixed device array
compiled into the library.  Its results must equal those of emp_glutton_max (which
allocates fresh buffers each call) on consecutive calls, including a call that follows
a larger puzzle's call and so starts with that puzzle's leftovers in the array.

The file is named to be collected last: it must pass both alone, in a fresh process
where its first call does the one-time set-up, and after every other test."""
from __future__ import annotations

import pytest

from edge_matching_puzzle_b200 import native
from edge_matching_puzzle_b200.puzzle import generate

pytestmark = pytest.mark.gpu

FIELDS = ("status", "max_level", "level", "trials", "pushes", "pops", "passes", "levels")


def _same(a, b):
    for f in FIELDS:
        assert getattr(a, f) == getattr(b, f), f
    assert list(a.best_board) == list(b.best_board)
    assert list(a.final_board) == list(b.final_board)


def _pair(pz, push_budget):
    handle = native.NativePuzzle(pz.width, pz.height, pz.colors)
    want = native.glutton_max(handle, push_budget=push_budget, timeout_ms=60000)
    got = native.glutton_max_noalloc(handle, push_budget=push_budget, timeout_ms=60000)
    _same(got, want)
    return got


# (width, height, border colours, interior colours, seed, push budget); run in this
# order so that each smaller puzzle follows a larger one's leftovers in the array
CASES = [
    (16, 16, 5, 17, 7, 300),   # 256 pieces: the largest puzzle the array holds
    (5, 5, 3, 5, 11, 0),       # full search
    (8, 8, 4, 8, 3, 150),
    (4, 4, 2, 4, 2, 0),
]


def test_noalloc_matches_allocating_search_on_consecutive_calls():
    for w, h, b, i, seed, budget in CASES:
        _pair(generate(w, h, b, i, seed), budget)


def test_noalloc_repeated_call_same_result():
    handle_pz = generate(8, 8, 4, 8, 3)
    handle = native.NativePuzzle(handle_pz.width, handle_pz.height, handle_pz.colors)
    first = native.glutton_max_noalloc(handle, push_budget=120, timeout_ms=60000)
    second = native.glutton_max_noalloc(handle, push_budget=120, timeout_ms=60000)
    _same(first, second)
    _same(first, native.glutton_max(handle, push_budget=120, timeout_ms=60000))


def test_noalloc_leaves_free_device_memory_unchanged():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device visible to torch")
    pz = generate(6, 6, 3, 6, 5)
    handle = native.NativePuzzle(pz.width, pz.height, pz.colors)
    native.glutton_max_noalloc(handle, push_budget=200)           # set-up on this device
    before = torch.cuda.mem_get_info()[0]
    for _ in range(3):
        native.glutton_max_noalloc(handle, push_budget=200)
    assert torch.cuda.mem_get_info()[0] == before
