"""CPU tests of the host side: the C-ABI library loads and exports every declared
symbol, the generator matches its Python mirror, and the GPU tables built on the host
reproduce the reference's constraint table exactly (no GPU needed: host code only)."""
from __future__ import annotations

import ctypes
import os
import random
import re

import pytest

from edge_matching_puzzle_b200 import native
from edge_matching_puzzle_b200.puzzle import Puzzle, generate, row_major_order, spiral_order
from oracle.oracle import OraclePuzzle

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    with open(os.path.join(ROOT, "include", "emp_b200.h")) as f:
        text = f.read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(emp_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol(native_lib):
    names = declared_functions()
    assert len(names) >= 15
    for name in names:
        assert hasattr(native_lib, name), name
        assert name in native.SIGNATURES, name
    assert native_lib.emp_abi_version() == 1


def test_generator_matches_python_mirror():
    for args in [(5, 5, 3, 5, 0), (8, 8, 4, 8, 3), (16, 16, 5, 17, 7), (12, 12, 4, 10, 100), (4, 9, 3, 4, 5)]:
        assert native.generate(*args) == generate(*args).colors


def test_config0_shape():
    pz = generate(5, 5, 3, 5, 0)
    kinds = [sum(1 for c in p if c == 0) for p in pz.colors]
    assert (kinds.count(2), kinds.count(1), kinds.count(0)) == (4, 12, 9)
    # every internal edge appears twice, frame colours 1..3, interior 4..8
    for p, k in zip(pz.colors, kinds):
        for c in p:
            assert c == 0 or 1 <= c <= 8


def test_invalid_puzzles_rejected():
    pz = generate(4, 4, 3, 4, 1)
    bad = [list(p) for p in pz.colors]
    bad[0] = [0, 0, 0, bad[0][3] or 1]  # a piece with three frame sides
    with pytest.raises(native.EmpError) as e:
        native.NativePuzzle(4, 4, bad)
    assert e.value.status == native.EMP_ERR_INVALID
    odd = [list(p) for p in pz.colors]
    for p in odd:  # change one interior colour: that colour count becomes odd
        if all(c for c in p):
            p[0] = 30
            break
    with pytest.raises(native.EmpError):
        native.NativePuzzle(4, 4, odd)
    with pytest.raises(native.EmpError):
        native.NativePuzzle(4, 4, pz.colors, order=[0] * 16)


def _decode(blob):
    hdr = blob[:32]
    return dict(n=hdr[1], ncol=hdr[2], kw=hdr[3:6], aoff=hdr[6:9], aw=hdr[9], side=hdr[10:13], pair=hdr[13],
                desc=hdr[14], tinfo=hdr[15:18], extra=hdr[18:21], init=hdr[21], w=hdr[22], h=hdr[23])


def _u64(blob, off, count):
    return [blob[off + 2 * i] | (blob[off + 2 * i + 1] << 32) for i in range(count)]


def _candidates_from_tables(blob, h, level, neighbour_colours, order, w):
    """Decodes a level descriptor and returns (kind, candidate bits, placed sides):
    pair-table row for the first two placed neighbours & side masks of the others."""
    d = blob[h["desc"] + 16 * level: h["desc"] + 16 * level + 16]
    kind, kw, nextra = (d[0] >> 8) & 3, d[0] & 0xFF, (d[0] >> 13) & 7
    pos = order[level]

    def side_of(nb_level):  # side of this position facing the neighbour placed at nb_level
        q = order[nb_level]
        return {pos - w: 0, pos + 1: 1, pos + w: 2, pos - 1: 3}[q]

    lev_a, lev_b = d[1] & 0xFF, (d[1] >> 8) & 0xFF
    stride_a, stride_b = d[3] & 0xFFFF, d[3] >> 16
    sides = []
    row = d[2]
    if stride_a:
        sa = side_of(lev_a)
        sides.append(sa)
        assert (d[1] >> 16) & 0xFF == 5 * ((sa + 2) % 4)
        row += neighbour_colours[sa] * stride_a
    if stride_b:
        sb = side_of(lev_b)
        sides.append(sb)
        assert d[1] >> 24 == 5 * ((sb + 2) % 4)
        row += neighbour_colours[sb] * stride_b
    words = _u64(blob, row, kw)
    for j in range(nextra):
        sd = (d[7] >> (2 * j)) & 3
        sides.append(sd)
        off = d[4] + (sd * h["ncol"] + neighbour_colours[sd]) * kw * 2
        words = [a & b for a, b in zip(words, _u64(blob, off, kw))]
    return kind, sum(v << (64 * i) for i, v in enumerate(words)), sides


@pytest.mark.parametrize("seed", [0, 1, 2, 3])
@pytest.mark.parametrize("shape", [(5, 5, 3, 5), (6, 4, 3, 4), (8, 8, 4, 8)])
@pytest.mark.parametrize("order_name", ["basic", "spiral"])
def test_side_masks_equal_reference_table(shape, seed, order_name):
    """For every level and neighbour colouring, base & side masks == table[code]."""
    w, h, B, I = shape
    pz = generate(w, h, B, I, seed)
    order = row_major_order(w, h) if order_name == "basic" else spiral_order(w, h)
    npz = native.NativePuzzle(w, h, pz.colors, order=order)
    op = OraclePuzzle(w, h, pz.colors)
    blob = npz.export_tables()
    hd = _decode(blob)
    border = op.border_color_id()
    cs = op.color_id_size()
    colours = list(range(1, border))
    rng = random.Random(seed)
    for level in range(w * h):
        pos = order[level]
        x, y = pos % w, pos // w
        frame = [y == 0, x == w - 1, y == h - 1, x == 0]
        for _ in range(12):
            nb = {s: rng.choice(colours) for s in range(4)}
            kind, got, placed = _candidates_from_tables(blob, hd, level, nb, order, w)
            code = 0
            for s in range(4):
                slot = (s + 2) % 4
                if frame[s]:
                    code |= border << (cs * slot)
                elif s in placed:
                    code |= nb[s] << (cs * slot)
            bits, want_words = op.table_entry(code)
            want = sum(v << (64 * i) for i, v in enumerate(want_words))
            assert bits == 4 * op.nb_kind(kind)
            assert got == want, (level, nb)


@pytest.mark.parametrize("seed", range(6))
def test_identical_masks_match_oracle(seed):
    """Transitions flagged with extra clears and their masks equal the reference's masks."""
    rng = random.Random(seed)
    n = rng.randint(4, 7)
    pz = generate(n, n, rng.randint(3, 4), rng.randint(3, 5), seed)
    npz = native.NativePuzzle(n, n, pz.colors)
    op = OraclePuzzle(n, n, pz.colors)
    blob = npz.export_tables()
    hd = _decode(blob)
    assert bool(npz.info().has_identical) == op.has_identical
    for kind in range(3):
        kw = hd["kw"][kind]
        bits = 4 * op.nb_kind(kind)
        for t in range(bits):
            m64 = op.identical_mask(kind, t)
            m = sum(v << (64 * i) for i, v in enumerate(m64)) & ((1 << bits) - 1)
            got = sum(v << (64 * i) for i, v in enumerate(_u64(blob, hd["extra"][kind] + t * kw * 2, kw)))
            assert got & ((1 << bits) - 1) == m
