"""Learned value ordering on the GPU: features, tensor-core inference, training
gradients, training and ordered plans.

- Features are compared exactly with the oracle's restatement.
- Gradients of the f32 CUDA kernels are compared with the float64 oracle: relative
  tolerance 1e-3, absolute 1e-5 x the largest gradient.
- Tensor-core scores (BF16 operands, FP32 accumulation) are compared with a PyTorch
  fp32 reference of the same network: |difference| <= 0.03 (1 + max |score|), the
  rounding of 512 + 256 BF16 products.
- Ordered plans must give the plain order's exhaustive counts exactly."""
from __future__ import annotations

import numpy as np
import pytest

from edge_matching_puzzle_b200 import native
from edge_matching_puzzle_b200.puzzle import generate, row_major_order
from oracle import mlp_oracle
from oracle.oracle import OraclePuzzle

pytestmark = pytest.mark.gpu


def _members(op):
    return [[op.piece_of(k, i) for i in range(op.nb_kind(k))] for k in range(3)]


def _sample_rows(pz, depth, count, seed):
    """(prefix, candidate) pairs taken from the oracle's expansion of the puzzle."""
    op = OraclePuzzle(pz.width, pz.height, pz.colors)
    n_pref, _, _, pref = op.expand(depth, max_prefixes=1 << 40)
    rng = np.random.default_rng(seed)
    rows = []
    for i in rng.choice(n_pref, size=min(count, n_pref), replace=False):
        p = [int(v) for v in pref[i * depth:(i + 1) * depth]]
        l = int(rng.integers(1, depth))
        rows.append((p[:l], p[l]))
    return op, rows


@pytest.mark.parametrize("shape", [(5, 5, 3, 5, 3), (6, 6, 3, 4, 11), (8, 8, 4, 8, 2)])
def test_features_match_oracle(shape):
    w, h, b, i, seed = shape
    pz = generate(w, h, b, i, seed)
    op, rows = _sample_rows(pz, min(10, w * h - 1), 200, seed)
    got = native.mlp_features(native.NativePuzzle(w, h, pz.colors), [r[0] for r in rows], [r[1] for r in rows])
    order = row_major_order(w, h)
    members = _members(op)
    for k, (prefix, t) in enumerate(rows):
        want = mlp_oracle.features(w, h, pz.colors, order, members, prefix, t)
        assert np.array_equal(got[k], want), (k, prefix, t, np.nonzero(got[k])[0], np.nonzero(want)[0])


def test_loss_gradient_matches_fp64_oracle():
    m = native.Mlp(seed=5)
    rng = np.random.default_rng(0)
    x = (rng.random((96, 512)) < 0.05).astype(np.float32)
    y = (rng.random(96) < 0.3).astype(np.float32)
    w = rng.uniform(0.5, 2.0, 96).astype(np.float32)
    loss, g = m.loss_grad(x, y, w)
    want_loss, want_g = mlp_oracle.loss_grad(m.params(), x, y, w)
    assert abs(loss - want_loss) <= 1e-5 * (1 + abs(want_loss))
    np.testing.assert_allclose(g, want_g, rtol=1e-3, atol=1e-5 * np.max(np.abs(want_g)))


@pytest.mark.parametrize("rows", [1, 127, 129, 40000])
def test_tensor_core_scores_match_fp32_reference(rows):
    torch = pytest.importorskip("torch")
    m = native.Mlp(seed=7)
    rng = np.random.default_rng(rows)
    x = (rng.random((rows, 512)) < 0.04).astype(np.float32)
    p = torch.from_numpy(m.params())
    w1 = p[:256 * 512].reshape(256, 512)
    o = 256 * 512
    b1 = p[o:o + 256]; o += 256
    w2 = p[o:o + 256 * 256].reshape(256, 256); o += 256 * 256
    b2 = p[o:o + 256]; o += 256
    w3 = p[o:o + 256]; o += 256
    b3 = p[o]
    xt = torch.from_numpy(x)
    ref = (torch.relu(torch.relu(xt @ w1.T + b1) @ w2.T + b2) @ w3 + b3).numpy()
    tc = m.score(x)
    f32 = m.score_f32(x)
    np.testing.assert_allclose(f32, ref, rtol=1e-4, atol=1e-4)
    assert np.max(np.abs(tc - ref)) <= 0.03 * (1 + np.max(np.abs(ref)))


def _solved(count, seed0):
    """Small puzzles and their first solutions found by the GPU search."""
    pzs, handles, boards = [], [], []
    s = seed0
    while len(pzs) < count:
        pz = generate(6, 6, 3, 4, s)
        s += 1
        h = native.NativePuzzle(6, 6, pz.colors)
        r = native.bt_count(h, split_depth=6, stop_at_any=1)
        if r.has_first_solution:
            pzs.append(pz)
            handles.append(h)
            boards.append(list(r.first_solution))
    return pzs, handles, boards


def test_training_lowers_the_loss():
    _, handles, boards = _solved(24, 3000)
    m = native.Mlp(seed=11)
    rep = m.train(handles, boards, epochs=15, batch=512, learning_rate=2e-3)
    assert rep.puzzles == 24 and rep.positives > 0 and rep.samples > rep.positives
    assert rep.last_loss < rep.first_loss


def test_ordered_plan_keeps_the_exhaustive_counts():
    _, handles, boards = _solved(16, 4000)
    m = native.Mlp(seed=3)
    m.train(handles, boards, epochs=5, batch=512)
    for seed in (21, 22):
        pz = generate(7, 7, 3, 6, seed)  # about 3e10 placements each
        h = native.NativePuzzle(7, 7, pz.colors)
        plain = native.BtPlan([h], split_depth=8)
        plain.run()
        want = plain.results()[0]
        ordered = native.BtPlan([h], split_depth=8)
        ordered.order(m)
        ordered.run()
        got = ordered.results()[0]
        assert (got.nodes, got.solutions) == (want.nodes, want.solutions)
        # the queue really changed
        n = plain.subtrees()
        first = [tuple(ordered.subtree_prefix(i, 8)) for i in range(min(n, 16))]
        plain_first = [tuple(plain.subtree_prefix(i, 8)) for i in range(min(n, 16))]
        assert sorted(first) != first or first != plain_first
        plain.close()
        ordered.close()


def test_ordered_plan_stops_at_a_solution():
    _, handles, boards = _solved(16, 5000)
    m = native.Mlp(seed=3)
    m.train(handles, boards, epochs=5, batch=512)
    pz = generate(8, 8, 4, 8, 4)  # one solution
    h = native.NativePuzzle(8, 8, pz.colors)
    plan = native.BtPlan([h], split_depth=12, stop_at_any=1)
    plan.order(m)
    plan.run()
    r = plan.results()[0]
    assert r.has_first_solution and r.first_found_us > 0
    full = native.bt_count(h, split_depth=12)
    assert list(r.first_solution) == list(full.first_solution)
    plan.close()
