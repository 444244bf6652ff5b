"""ctypes binding of the CPU oracle (oracle/libemp_oracle.so) -- TEST INFRASTRUCTURE ONLY.

Only tests/, the smoke check and the CPU-baseline leg of bench.py import this module; the
product path never does.  ``ensure_built()`` runs oracle/Makefile when the shared library
is missing.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from typing import List, Optional, Sequence, Tuple

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libemp_oracle.so")
CLI_PATH = os.path.join(HERE, "emp_oracle_cli")


class BtResult(ctypes.Structure):
    _fields_ = [
        ("nodes", ctypes.c_uint64),
        ("solutions", ctypes.c_uint64),
        ("first_solution_nodes", ctypes.c_uint64),
        ("max_index", ctypes.c_uint32),
        ("status", ctypes.c_int32),
        ("first_solution", ctypes.c_uint16 * 256),
        ("first_board", ctypes.c_uint32 * 256),
    ]


class GmResult(ctypes.Structure):
    _fields_ = [
        ("placements", ctypes.c_uint64),
        ("max_level", ctypes.c_uint32),
        ("level", ctypes.c_uint32),
        ("status", ctypes.c_int32),
        ("played", ctypes.c_uint32 * 256),
        ("max_played", ctypes.c_uint32 * 256),
        ("pushes", ctypes.c_uint64),
        ("pops", ctypes.c_uint64),
        ("levels_evaluated", ctypes.c_uint64),
    ]


def ensure_built() -> None:
    src = [os.path.join(HERE, f) for f in ("emp_oracle.c", "emp_oracle.h", "emp_oracle_cli.c")]
    newest = max(os.path.getmtime(f) for f in src)
    if (not os.path.exists(LIB_PATH) or os.path.getmtime(LIB_PATH) < newest
            or not os.path.exists(CLI_PATH) or os.path.getmtime(CLI_PATH) < newest):
        subprocess.run(["make", "-s", "-C", HERE], check=True)


_lib = None


def lib():
    global _lib
    if _lib is None:
        ensure_built()
        L = ctypes.CDLL(LIB_PATH)
        vp, u32, u64 = ctypes.c_void_p, ctypes.c_uint32, ctypes.c_uint64
        L.op_puzzle_create.restype = vp
        L.op_puzzle_create.argtypes = [u32, u32, ctypes.c_char_p, ctypes.c_char_p, ctypes.c_size_t]
        L.op_puzzle_destroy.argtypes = [vp]
        L.op_has_identical.argtypes = [vp]
        for f in ("op_nb_kind", "op_kind_index", "op_border_color_id", "op_color_id_size", "op_orientation_step"):
            getattr(L, f).restype = u32
        L.op_nb_kind.argtypes = [vp, u32]
        L.op_kind_index.argtypes = [vp, u32]
        L.op_piece_of.restype = u32
        L.op_piece_of.argtypes = [vp, u32, u32]
        L.op_border_color_id.argtypes = [vp]
        L.op_color_id_size.argtypes = [vp]
        L.op_orientation_step.argtypes = [vp, u32]
        L.op_identical_mask.restype = u32
        L.op_identical_mask.argtypes = [vp, u32, u32, ctypes.POINTER(u64), u32]
        L.op_table_entry.restype = u32
        L.op_table_entry.argtypes = [vp, u32, ctypes.POINTER(u64), u32]
        L.op_bt_run.argtypes = [vp, ctypes.POINTER(u32), u64, ctypes.POINTER(BtResult), ctypes.c_char_p,
                                ctypes.c_char_p, ctypes.c_size_t]
        L.op_bt_resume.argtypes = [vp, ctypes.POINTER(u32), ctypes.POINTER(ctypes.c_uint16), u32, u64,
                                   ctypes.POINTER(BtResult), ctypes.c_char_p]
        L.op_vs_trace.argtypes = [vp, u32, ctypes.POINTER(u32), ctypes.POINTER(u32), ctypes.POINTER(u32),
                                  ctypes.POINTER(u32), ctypes.POINTER(u32), u64]
        L.op_bt_expand.restype = u64
        L.op_bt_expand.argtypes = [vp, ctypes.POINTER(u32), u32, ctypes.POINTER(ctypes.c_uint16), u64,
                                   ctypes.POINTER(u64), ctypes.POINTER(u64)]
        L.op_bt_subtree.argtypes = [vp, ctypes.POINTER(u32), ctypes.POINTER(ctypes.c_uint16), u32, u64,
                                    ctypes.POINTER(u64), ctypes.POINTER(u64)]
        L.op_bt_subtrees_parallel.argtypes = [vp, ctypes.POINTER(u32), ctypes.POINTER(ctypes.c_uint16), u32, u64, u64,
                                              ctypes.c_int, ctypes.POINTER(u64), ctypes.POINTER(u64),
                                              ctypes.POINTER(u64), ctypes.POINTER(u64), ctypes.POINTER(u64)]
        L.op_bt_estimate.restype = ctypes.c_double
        L.op_bt_estimate.argtypes = [vp, ctypes.POINTER(u32), u32, u64, ctypes.POINTER(ctypes.c_double)]
        L.op_gm_run.argtypes = [vp, u64, u64, ctypes.POINTER(GmResult)]
        L.op_gm_initial.argtypes = [vp, ctypes.POINTER(u32)]
        _lib = L
    return _lib


class OraclePuzzle:
    """Owns an op_puzzle built from (width, height, colours)."""

    def __init__(self, width: int, height: int, colors: Sequence[Sequence[int]]):
        self.width, self.height = width, height
        self.n = width * height
        flat = bytes(c for p in colors for c in p)
        err = ctypes.create_string_buffer(256)
        self._p = lib().op_puzzle_create(width, height, flat, err, 256)
        if not self._p:
            raise ValueError(err.value.decode())

    def __del__(self):
        if getattr(self, "_p", None):
            lib().op_puzzle_destroy(self._p)
            self._p = None

    def _order(self, order: Optional[Sequence[int]]):
        order = list(range(self.n)) if order is None else list(order)
        return (ctypes.c_uint32 * self.n)(*order)

    @property
    def has_identical(self) -> bool:
        return bool(lib().op_has_identical(self._p))

    def nb_kind(self, k: int) -> int:
        return lib().op_nb_kind(self._p, k)

    def kind_index(self, piece_index: int) -> int:
        return lib().op_kind_index(self._p, piece_index)

    def piece_of(self, kind: int, kind_index: int) -> int:
        return lib().op_piece_of(self._p, kind, kind_index)

    def border_color_id(self) -> int:
        return lib().op_border_color_id(self._p)

    def color_id_size(self) -> int:
        return lib().op_color_id_size(self._p)

    def orientation_step(self, piece_index: int) -> int:
        return lib().op_orientation_step(self._p, piece_index)

    def identical_mask(self, kind: int, t: int) -> List[int]:
        buf = (ctypes.c_uint64 * 32)()
        nw = lib().op_identical_mask(self._p, kind, t, buf, 32)
        return list(buf)[:nw]

    def table_entry(self, code: int) -> Tuple[int, List[int]]:
        buf = (ctypes.c_uint64 * 32)()
        bits = lib().op_table_entry(self._p, code, buf, 32)
        return bits, list(buf)[: (bits + 63) // 64]

    def run(self, order=None, node_limit: int = 0, results_bin: Optional[str] = None, with_log: bool = False):
        r = BtResult()
        cap = 1 << 22 if with_log else 0
        log = ctypes.create_string_buffer(cap) if cap else None
        lib().op_bt_run(self._p, self._order(order), node_limit, ctypes.byref(r),
                        results_bin.encode() if results_bin else None, log, cap)
        return r, (log.value.decode() if log is not None else "")

    def resume(self, situation: Sequence[int], order=None, node_limit: int = 0, results_bin: Optional[str] = None):
        """emp_strategy::set_initial_state + specific_run: ``situation`` holds the
        transition placed at each of the first levels of the order."""
        r = BtResult()
        arr = (ctypes.c_uint16 * max(1, len(situation)))(*situation)
        st = lib().op_bt_resume(self._p, self._order(order), arr, len(situation), node_limit, ctypes.byref(r),
                                results_bin.encode() if results_bin else None)
        if st:
            raise ValueError(f"situation not reachable (status {st})")
        return r

    def vs_trace(self, max_events: int = 4096, max_selections: int = 0):
        """The reference's variable-space CUDA backtracker restated: (events, board) with
        events (lane, variable id, step) and the first solution's board (None if none)."""
        la, va, st = ((ctypes.c_uint32 * max_events)() for _ in range(3))
        ne = ctypes.c_uint32()
        board = (ctypes.c_uint32 * self.n)()
        r = lib().op_vs_trace(self._p, max_events, la, va, st, ctypes.byref(ne), board, max_selections)
        if r < 0:
            raise ValueError("puzzle too large")
        ev = [(la[i], va[i], st[i]) for i in range(min(ne.value, max_events))]
        return ev, (list(board) if r == 0 else None)

    def expand(self, depth: int, order=None, max_prefixes: int = 0):
        nn, ss = ctypes.c_uint64(), ctypes.c_uint64()
        o = self._order(order)
        count = lib().op_bt_expand(self._p, o, depth, None, 0, ctypes.byref(nn), ctypes.byref(ss))
        pref = None
        if max_prefixes:
            m = min(count, max_prefixes)
            buf = (ctypes.c_uint16 * (max(1, m) * depth))()
            lib().op_bt_expand(self._p, o, depth, buf, m, ctypes.byref(nn), ctypes.byref(ss))
            pref = buf
        return count, nn.value, ss.value, pref

    def subtree(self, prefix: Sequence[int], order=None, node_limit: int = 0):
        d = len(prefix)
        arr = (ctypes.c_uint16 * max(1, d))(*prefix)
        nn, ss = ctypes.c_uint64(), ctypes.c_uint64()
        st = lib().op_bt_subtree(self._p, self._order(order), arr, d, node_limit, ctypes.byref(nn), ctypes.byref(ss))
        return nn.value, ss.value, st

    def subtrees_parallel(self, prefixes, depth: int, begin: int, end: int, threads: int, order=None,
                          per_item: bool = False, kinds: bool = False):
        nn, ss = ctypes.c_uint64(), ctypes.c_uint64()
        pn = (ctypes.c_uint64 * max(1, end - begin))() if per_item else None
        ps = (ctypes.c_uint64 * max(1, end - begin))() if per_item else None
        kn = (ctypes.c_uint64 * 3)()
        lib().op_bt_subtrees_parallel(self._p, self._order(order), prefixes, depth, begin, end, threads,
                                      ctypes.byref(nn), ctypes.byref(ss), pn, ps, kn)
        out = (nn.value, ss.value)
        if per_item:
            out = out + (list(pn), list(ps))
        if kinds:
            out = out + (list(kn),)
        return out

    def estimate(self, probes: int, seed: int = 1, order=None) -> float:
        return lib().op_bt_estimate(self._p, self._order(order), probes, seed, None)

    def glutton(self, budget: int = 0, push_budget: int = 0) -> GmResult:
        r = GmResult()
        lib().op_gm_run(self._p, budget, push_budget, ctypes.byref(r))
        return r

    def glutton_initial(self):
        """The glutton search's first situation (what CUDA glutton wide prints): per
        position its 32 info words."""
        out = (ctypes.c_uint32 * (32 * self.n))()
        lib().op_gm_initial(self._p, out)
        return [list(out[32 * j:32 * j + 32]) for j in range(self.n)]
