"""CPU oracle of the learned value ordering -- TEST INFRASTRUCTURE ONLY.

A numpy restatement, in float64, of what the CUDA library computes for the
candidate-scoring network (edge_matching_puzzle_b200/csrc/emp_mlp.cu): the 512
features of a candidate placement, the network's forward pass and the gradient of its
weighted logistic loss.  The reference project has no learned component, so there is
no reference code to follow here; the tests use this file to check the CUDA kernels
(features exactly, scores and gradients within the tolerances the tests state).
Only tests/ may import it.
"""
from __future__ import annotations

from typing import Sequence, Tuple

import numpy as np

INPUTS, HIDDEN = 512, 256
PARAMS = HIDDEN * INPUTS + HIDDEN + HIDDEN * HIDDEN + HIDDEN + HIDDEN + 1


def split_params(p: np.ndarray):
    p = np.asarray(p, dtype=np.float64)
    o = 0
    w1 = p[o:o + HIDDEN * INPUTS].reshape(HIDDEN, INPUTS)
    o += HIDDEN * INPUTS
    b1 = p[o:o + HIDDEN]
    o += HIDDEN
    w2 = p[o:o + HIDDEN * HIDDEN].reshape(HIDDEN, HIDDEN)
    o += HIDDEN * HIDDEN
    b2 = p[o:o + HIDDEN]
    o += HIDDEN
    w3 = p[o:o + HIDDEN]
    o += HIDDEN
    b3 = p[o]
    return w1, b1, w2, b2, w3, b3


def forward(p: np.ndarray, x: np.ndarray):
    w1, b1, w2, b2, w3, b3 = split_params(p)
    x = np.asarray(x, dtype=np.float64)
    h1 = np.maximum(x @ w1.T + b1, 0.0)
    h2 = np.maximum(h1 @ w2.T + b2, 0.0)
    return h2 @ w3 + b3, h1, h2


def loss_grad(p: np.ndarray, x: np.ndarray, y: np.ndarray, w: np.ndarray) -> Tuple[float, np.ndarray]:
    """Mean weighted logistic loss sum w (softplus(s) - y s) / sum w and its gradient
    with respect to the parameters (same order as the library's parameter array)."""
    x = np.asarray(x, dtype=np.float64)
    y = np.asarray(y, dtype=np.float64)
    w = np.asarray(w, dtype=np.float64)
    w1, b1, w2, b2, w3, b3 = split_params(p)
    s, h1, h2 = forward(p, x)
    sp = np.logaddexp(0.0, s)
    loss = float(np.sum(w * (sp - y * s)) / np.sum(w))
    ds = w * (1.0 / (1.0 + np.exp(-s)) - y) / np.sum(w)
    dw3 = h2.T @ ds
    db3 = ds.sum()
    dh2 = np.outer(ds, w3) * (h2 > 0)
    dw2 = dh2.T @ h1
    db2 = dh2.sum(axis=0)
    dh1 = (dh2 @ w2) * (h1 > 0)
    dw1 = dh1.T @ x
    db1 = dh1.sum(axis=0)
    g = np.concatenate([dw1.ravel(), db1, dw2.ravel(), db2, dw3, [db3]])
    return loss, g


def features(width: int, height: int, colors: Sequence[Sequence[int]], order: Sequence[int], kind_members,
             prefix: Sequence[int], t: int) -> np.ndarray:
    """Feature row of candidate t placed at level len(prefix) after `prefix` (transitions
    kind_index << 2 | orientation per level of `order`).  kind_members[k] lists the piece
    indices of kind k (0 centre, 1 border, 2 corner) in kind-index order.

    Layout: one-hot side colours of the oriented candidate (4 x 32), neighbour state per
    side outside/placed/free (4 x 3), for free sides the number of edges of that colour
    left on unplaced pieces capped at 15 (4 x 16), x and y (16 each), depth l*16/n (16),
    kind (3), a constant 1 at 255, and the first two free sides' colours hashed
    (c1 * 32 + c2) mod 256 (or c1 alone for one free side) into [256, 512)."""
    n = width * height
    l = len(prefix)
    level_of = {pos: i for i, pos in enumerate(order)}

    def kind_at(pos):
        x, y = pos % width, pos // width
        return (x == 0) + (x == width - 1) + (y == 0) + (y == height - 1)

    def oriented(level, tt):
        pos = order[level]
        piece = kind_members[kind_at(pos)][tt >> 2]
        o = tt & 3
        return [colors[piece][(s + o) % 4] for s in range(4)]

    totals = np.zeros(32, dtype=np.int64)
    for p in range(n):
        for c in colors[p]:
            totals[c] += 1
    pos = order[l]
    x, y = pos % width, pos // width
    kind = kind_at(pos)
    col = oriented(l, t)
    placed_cols = [oriented(j, prefix[j]) for j in range(l)]
    nbr = [(x, y - 1), (x + 1, y), (x, y + 1), (x - 1, y)]
    f = np.zeros(INPUTS)
    free = []
    for s in range(4):
        c = col[s]
        f[32 * s + c] = 1
        nx, ny = nbr[s]
        if not (0 <= nx < width and 0 <= ny < height):
            state = 0
        else:
            state = 1 if level_of[ny * width + nx] < l else 2
        f[128 + 3 * s + state] = 1
        if state == 2:
            used = sum(pc.count(c) for pc in placed_cols) + col.count(c)
            f[140 + 16 * s + min(int(totals[c]) - used, 15)] = 1
            if len(free) < 2:
                free.append(c)
    f[204 + min(x, 15)] = 1
    f[220 + min(y, 15)] = 1
    f[236 + min(l * 16 // n, 15)] = 1
    f[252 + min(kind, 2)] = 1
    f[255] = 1
    if len(free) == 2:
        f[256 + ((free[0] * 32 + free[1]) & 255)] = 1
    elif len(free) == 1:
        f[256 + free[0]] = 1
    return f
