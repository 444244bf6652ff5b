"""Puzzle model on the host side: the reference's CSV format and the seeded generator.

The CSV layout is the one the reference parses in include/emp_pieces_parser.h:53-101
(``Width,Height`` header, dimensions, ``I,N,E,S,O`` header, one ``id,N,E,S,W`` line per
piece, colour 0 for the frame).  Piece ids are 1..n in file order, which is also the order
that defines kind indices (include/emp_piece_db.h:540-610).

The generator builds the seeded workloads of this project: every internal edge of a w x h
grid gets a colour, frame-to-frame edges from ``border_colors`` colours (ids 1..B) and all
other internal edges from ``interior_colors`` colours (ids B+1..B+I); outer edges are 0.
The grid is cut into pieces, shuffled (Fisher-Yates) and each piece is rotated by a
uniform quarter turn.  The random stream is splitmix64 seeded with the seed, and every
draw is ``next() % bound``, in this order: horizontal edges row by row, vertical edges row
by row, the shuffle from the last index down, then one rotation per piece.  The C++
library (``emp_generate_puzzle``) implements the same stream; the tests check both agree.
"""
from __future__ import annotations

from dataclasses import dataclass
from typing import List, Sequence

_MASK = (1 << 64) - 1


class SplitMix64:
    """splitmix64 (Steele, Lea, Flood 2014): the project's reproducible random stream."""

    def __init__(self, seed: int) -> None:
        self.state = seed & _MASK

    def next(self) -> int:
        self.state = (self.state + 0x9E3779B97F4A7C15) & _MASK
        z = self.state
        z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & _MASK
        z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & _MASK
        return z ^ (z >> 31)

    def below(self, bound: int) -> int:
        return self.next() % bound


@dataclass
class Puzzle:
    """A w x h edge-matching puzzle: ``colors[i]`` = (N, E, S, W) of piece id i+1."""

    width: int
    height: int
    colors: List[List[int]]

    @property
    def nb_pieces(self) -> int:
        return self.width * self.height

    def flat_colors(self) -> bytes:
        return bytes(c for piece in self.colors for c in piece)

    def to_csv(self) -> str:
        lines = ["Width,Height", f"{self.width},{self.height}", "I,N,E,S,O"]
        for i, (n, e, s, w) in enumerate(self.colors):
            lines.append(f"{i + 1},{n},{e},{s},{w}")
        return "\n".join(lines) + "\n"

    @staticmethod
    def from_csv(text: str) -> "Puzzle":
        """Parse the reference CSV format; raises ValueError like the reference parser
        raises quicky_logic_exception (emp_pieces_parser.h:60-78)."""
        lines = text.split("\n")
        if not lines or lines[0].strip() != "Width,Height":
            raise ValueError(f'Unsupported puzzle header "{lines[0] if lines else ""}" : should be "Width,Height"')
        if len(lines) < 2:
            raise ValueError("Truncated file after puzzle header")
        width, height = (int(v) for v in lines[1].split(",")[:2])
        if len(lines) < 3 or lines[2].strip() != "I,N,E,S,O":
            raise ValueError('Unsupported pieces header : should be "I,N,E,S,O"')
        pieces = {}
        for line in lines[3:]:
            if line.strip():
                pid, n, e, s, w = (int(v) for v in line.split(",")[:5])
                pieces[pid] = [n, e, s, w]
        if sorted(pieces) != list(range(1, width * height + 1)):
            raise ValueError("piece ids must be 1..width*height")
        return Puzzle(width, height, [pieces[i] for i in range(1, width * height + 1)])

    @staticmethod
    def load(path: str) -> "Puzzle":
        with open(path) as f:
            return Puzzle.from_csv(f.read())


def generate(width: int, height: int, border_colors: int, interior_colors: int, seed: int) -> Puzzle:
    """Seeded puzzle generator (see module docstring for the exact stream)."""
    if width < 2 or height < 2:
        raise ValueError("puzzle must be at least 2x2")
    if border_colors < 1 or interior_colors < 1:
        raise ValueError("need at least one border and one interior colour")
    rng = SplitMix64(seed)
    hor = [[0] * (width - 1) for _ in range(height)]
    ver = [[0] * width for _ in range(height - 1)]
    for y in range(height):
        for x in range(width - 1):
            frame = y == 0 or y == height - 1
            hor[y][x] = 1 + rng.below(border_colors) if frame else border_colors + 1 + rng.below(interior_colors)
    for y in range(height - 1):
        for x in range(width):
            frame = x == 0 or x == width - 1
            ver[y][x] = 1 + rng.below(border_colors) if frame else border_colors + 1 + rng.below(interior_colors)
    pieces: List[List[int]] = []
    for y in range(height):
        for x in range(width):
            n = 0 if y == 0 else ver[y - 1][x]
            e = 0 if x == width - 1 else hor[y][x]
            s = 0 if y == height - 1 else ver[y][x]
            w = 0 if x == 0 else hor[y][x - 1]
            pieces.append([n, e, s, w])
    for i in range(len(pieces) - 1, 0, -1):
        j = rng.below(i + 1)
        pieces[i], pieces[j] = pieces[j], pieces[i]
    out = []
    for c in pieces:
        r = rng.below(4)
        out.append([c[(s + r) % 4] for s in range(4)])
    return Puzzle(width, height, out)


def row_major_order(width: int, height: int) -> List[int]:
    """Strategy ``basic`` (include/emp_basic_strategy_generator.h:44-53)."""
    return list(range(width * height))


def spiral_order(width: int, height: int) -> List[int]:
    """Strategy ``spiral`` (include/emp_spiral_strategy_generator.h:52-100)."""
    used = [False] * (width * height)
    order: List[int] = []
    x = y = 0
    n = width * height
    for i in range(n):
        used[y * width + x] = True
        order.append(y * width + x)
        if n > i + 1:
            if x >= y:
                if x + 1 < width and not used[y * width + x + 1]:
                    x += 1
                elif y + 1 < height and not used[(y + 1) * width + x]:
                    y += 1
                else:
                    x -= 1
            else:
                if x and not used[y * width + x - 1]:
                    x -= 1
                elif y and not used[(y - 1) * width + x]:
                    y -= 1
                else:
                    x += 1
    return order


def board_string(width: int, height: int, cells: Sequence[int]) -> str:
    """The reference's board string (include/situation_string_formatter.h:51-70): per
    position in row-major order the piece id right-aligned on digits(n) characters plus
    its orientation letter, or dashes when empty.  ``cells`` holds (id-1)<<2|o or -1."""
    n = width * height
    wd = len(str(n)) + 1
    out = []
    for c in cells[:n]:
        if c is None or c < 0 or c == 0xFFFFFFFF:
            out.append("-" * wd)
        else:
            out.append(f"{(c >> 2) + 1:>{wd - 1}d}{'NESW'[c & 3]}")
    return "".join(out)


def parse_board_string(width: int, height: int, text: str) -> List[int]:
    """Inverse of board_string, as the reference reads a situation string
    (include/situation_string_formatter.h:80-121): per row-major position a piece id on
    digits(n) characters and an orientation letter, dashes for an empty cell.  Returns
    (id-1)<<2|o per position, -1 when empty.  Raises ValueError on a malformed string
    (the reference throws quicky_logic_exception)."""
    n = width * height
    wd = len(str(n)) + 1
    if len(text) != n * wd:
        raise ValueError(f"situation string of length {len(text)}, expected {n * wd}")
    cells = []
    for i in range(n):
        cell = text[i * wd:(i + 1) * wd]
        if cell[:-1] == "-" * (wd - 1):
            cells.append(-1)
            continue
        if cell[-1] not in "NESW":
            raise ValueError(f"bad orientation '{cell[-1]}' at position {i}")
        pid = int(cell[:-1])
        if not 1 <= pid <= n:
            raise ValueError(f"bad piece id {pid} at position {i}")
        cells.append(((pid - 1) << 2) | "NESW".index(cell[-1]))
    return cells


def situation_transitions(puzzle: "Puzzle", order: Sequence[int], cells: Sequence[int]) -> List[int]:
    """Transitions t = kind_index << 2 | o of the situation's pieces along a position
    order, up to the first empty position (include/emp_strategy.h:431-441)."""
    kinds = [sum(1 for c in p if c == 0) for p in puzzle.colors]
    kind_index, seen = [], [0, 0, 0]
    for k in kinds:
        kind_index.append(seen[k])
        seen[k] += 1
    out = []
    for pos in order:
        c = cells[pos]
        if c < 0:
            break
        out.append((kind_index[c >> 2] << 2) | (c & 3))
    return out


def mixed_batch(count: int = 4096, seed: int = 2) -> List[Puzzle]:
    """The batched workload: ``count`` square puzzles whose side is drawn uniformly from
    4..9, border colours from 3..5 and interior colours from 4..10.  Instance i takes
    four draws of one splitmix64 stream seeded with ``seed``: side, border colours,
    interior colours and the generator seed of the puzzle."""
    sm = SplitMix64(seed)
    out = []
    for _ in range(count):
        side = 4 + sm.below(6)
        border = 3 + sm.below(3)
        interior = 4 + sm.below(7)
        out.append(generate(side, side, border, interior, sm.next()))
    return out
