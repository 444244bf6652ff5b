"""The float64 oracle of the scoring network checks itself: its gradient equals
central finite differences of its loss (CPU only)."""
from __future__ import annotations

import numpy as np

from oracle import mlp_oracle


def test_oracle_gradient_matches_finite_differences():
    rng = np.random.default_rng(1)
    p = rng.normal(0, 0.05, mlp_oracle.PARAMS)
    x = (rng.random((12, 512)) < 0.08).astype(np.float64)
    y = (rng.random(12) < 0.4).astype(np.float64)
    w = rng.uniform(0.5, 2.0, 12)
    _, g = mlp_oracle.loss_grad(p, x, y, w)
    idx = list(rng.choice(mlp_oracle.PARAMS, size=40, replace=False)) + [mlp_oracle.PARAMS - 1]
    eps = 1e-6
    for i in idx:
        q = p.copy()
        q[i] += eps
        lp, _ = mlp_oracle.loss_grad(q, x, y, w)
        q[i] -= 2 * eps
        lm, _ = mlp_oracle.loss_grad(q, x, y, w)
        fd = (lp - lm) / (2 * eps)
        assert abs(fd - g[i]) <= 1e-6 + 1e-4 * abs(fd), (i, fd, g[i])


def test_oracle_features_are_one_hot_blocks():
    from edge_matching_puzzle_b200.puzzle import generate, row_major_order
    from oracle.oracle import OraclePuzzle
    pz = generate(5, 5, 3, 5, 3)
    op = OraclePuzzle(5, 5, pz.colors)
    members = [[op.piece_of(k, i) for i in range(op.nb_kind(k))] for k in range(3)]
    n, _, _, pref = op.expand(6, max_prefixes=1 << 20)
    p = [int(v) for v in pref[:6]]
    f = mlp_oracle.features(5, 5, pz.colors, row_major_order(5, 5), members, p[:5], p[5])
    assert set(np.unique(f)) <= {0.0, 1.0}
    for s in range(4):
        assert f[32 * s:32 * s + 32].sum() == 1 and f[128 + 3 * s:131 + 3 * s].sum() == 1
    assert f[204:220].sum() == 1 and f[220:236].sum() == 1 and f[255] == 1
