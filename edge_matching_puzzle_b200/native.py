"""ctypes binding of the C ABI in include/emp_b200.h (libemp_b200.so).

There is no Python or CPU implementation of the search behind these calls: if the
native library is missing or cannot load, ``load()`` raises.  The calls mirror the
reference's launchers (launch_CUDA_backtracker, launch_CUDA_glutton_max) with results
returned instead of printed.
"""
from __future__ import annotations

import ctypes
import os
from typing import List, Optional, Sequence

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libemp_b200.so")

EMP_OK = 0
EMP_INCOMPLETE = 1
EMP_FIRST_LOST = 2
EMP_ERR_INVALID = -1
EMP_ERR_UNSUPPORTED = -2
EMP_ERR_CUDA = -3
EMP_ERR_NOMEM = -4

u8p = ctypes.POINTER(ctypes.c_uint8)
u16p = ctypes.POINTER(ctypes.c_uint16)
u64p = ctypes.POINTER(ctypes.c_uint64)


class EmpError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"emp status {status}: {message}")
        self.status = status


class PuzzleDesc(ctypes.Structure):
    _fields_ = [("width", ctypes.c_uint32), ("height", ctypes.c_uint32), ("colours", u8p), ("order", u16p)]


class PuzzleInfo(ctypes.Structure):
    _fields_ = [(n, ctypes.c_uint32) for n in ("width", "height", "nb_pieces", "nb_center", "nb_border", "nb_corner",
                                               "border_color_id", "has_identical", "identical_masks_with_extra")]


class BtConfig(ctypes.Structure):
    _fields_ = [
        ("split_depth", ctypes.c_uint32),
        ("threads_per_block", ctypes.c_uint32),
        ("blocks_per_sm", ctypes.c_uint32),
        ("stop_at_first", ctypes.c_uint32),
        ("reserved_budget", ctypes.c_uint64),
        ("timeout_ms", ctypes.c_uint32),
        ("device", ctypes.c_int32),
        ("keep_subtree_counts", ctypes.c_uint32),
        ("split_budget", ctypes.c_uint32),
        ("sample_stride", ctypes.c_uint32),
        ("sample_first", ctypes.c_uint32),
        ("table_placement", ctypes.c_uint32),
        ("split_subtrees", ctypes.c_uint32),
        ("use_graph", ctypes.c_uint32),
        ("stop_at_any", ctypes.c_uint32),
        ("first_lock_wait_us", ctypes.c_uint32),
        ("hold_first_lock", ctypes.c_uint32),
        ("stack_placement", ctypes.c_uint32),
    ]


class BtResult(ctypes.Structure):
    _fields_ = [
        ("solutions", ctypes.c_uint64),
        ("nodes", ctypes.c_uint64),
        ("subtrees", ctypes.c_uint64),
        ("expansion_nodes", ctypes.c_uint64),
        ("status", ctypes.c_int32),
        ("split_depth", ctypes.c_uint32),
        ("has_first_solution", ctypes.c_uint32),
        ("first_solution", ctypes.c_uint32 * 256),
        ("kernel_ms", ctypes.c_double),
        ("total_ms", ctypes.c_double),
        ("rounds", ctypes.c_uint32),
        ("first_found_us", ctypes.c_uint32),
        ("dfs_busy_ms", ctypes.c_double),
        ("work_records", ctypes.c_uint64),
        ("handed_back", ctypes.c_uint64),
    ]


class BtSolution(ctypes.Structure):
    _fields_ = [("node_index", ctypes.c_uint64), ("board", ctypes.c_uint32 * 256)]


class VsEvent(ctypes.Structure):
    _fields_ = [("lane", ctypes.c_uint32), ("variable", ctypes.c_uint32), ("step", ctypes.c_uint32)]


class TuneResult(ctypes.Structure):
    _fields_ = [
        ("best", BtConfig),
        ("best_rate", ctypes.c_double),
        ("default_rate", ctypes.c_double),
        ("trials", ctypes.c_uint32),
        ("reserved", ctypes.c_uint32),
    ]


class MlpTrainConfig(ctypes.Structure):
    _fields_ = [("epochs", ctypes.c_uint32), ("batch", ctypes.c_uint32), ("learning_rate", ctypes.c_float),
                ("seed", ctypes.c_uint32), ("max_level", ctypes.c_uint32), ("reserved", ctypes.c_uint32 * 3)]


class MlpTrainReport(ctypes.Structure):
    _fields_ = [("samples", ctypes.c_uint64), ("positives", ctypes.c_uint64), ("puzzles", ctypes.c_uint32),
                ("epochs", ctypes.c_uint32), ("first_loss", ctypes.c_double), ("last_loss", ctypes.c_double),
                ("train_ms", ctypes.c_double)]


MLP_INPUTS = 512
MLP_HIDDEN = 256
MLP_PARAMS = 256 * 512 + 256 + 256 * 256 + 256 + 256 + 1


class GmConfig(ctypes.Structure):
    _fields_ = [("push_budget", ctypes.c_uint64), ("timeout_ms", ctypes.c_uint32), ("device", ctypes.c_int32),
                ("placement_budget", ctypes.c_uint64), ("blocks", ctypes.c_uint32), ("reserved", ctypes.c_uint32 * 5)]


class GmResult(ctypes.Structure):
    _fields_ = [
        ("status", ctypes.c_int32),
        ("max_level", ctypes.c_uint32),
        ("level", ctypes.c_uint32),
        ("reserved0", ctypes.c_uint32),
        ("best_board", ctypes.c_uint32 * 256),
        ("final_board", ctypes.c_uint32 * 256),
        ("trials", ctypes.c_uint64),
        ("pushes", ctypes.c_uint64),
        ("pops", ctypes.c_uint64),
        ("passes", ctypes.c_uint64),
        ("levels", ctypes.c_uint64),
        ("kernel_ms", ctypes.c_double),
    ]


# name -> (restype, argtypes); every symbol declared in include/emp_b200.h
SIGNATURES = {
    "emp_abi_version": (ctypes.c_uint32, []),
    "emp_glutton_wide_situation": (ctypes.c_int32, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_uint32), ctypes.c_uint64]),
    "emp_last_error": (ctypes.c_char_p, []),
    "emp_generate_puzzle": (ctypes.c_int32, [ctypes.c_uint32] * 4 + [ctypes.c_uint64, u8p]),
    "emp_puzzle_create": (ctypes.c_int32, [ctypes.POINTER(PuzzleDesc), ctypes.POINTER(ctypes.c_void_p)]),
    "emp_puzzle_destroy": (None, [ctypes.c_void_p]),
    "emp_puzzle_get_info": (ctypes.c_int32, [ctypes.c_void_p, ctypes.POINTER(PuzzleInfo)]),
    "emp_puzzle_export_tables": (ctypes.c_int32, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_uint32), ctypes.c_uint64,
                                                  u64p]),
    "emp_bt_count": (ctypes.c_int32, [ctypes.c_void_p, ctypes.POINTER(BtConfig), ctypes.POINTER(BtResult)]),
    "emp_bt_variable_space": (ctypes.c_int32, [ctypes.c_void_p, ctypes.c_int32, ctypes.c_uint64, ctypes.c_uint32,
                                               ctypes.POINTER(VsEvent), ctypes.c_uint64, u64p,
                                               ctypes.POINTER(ctypes.c_uint32), ctypes.POINTER(ctypes.c_uint32)]),
    "emp_bt_resume": (ctypes.c_int32, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_uint16), ctypes.c_uint32,
                                       ctypes.POINTER(BtConfig), ctypes.POINTER(BtResult)]),
    "emp_bt_resume_solutions": (ctypes.c_int32, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_uint16), ctypes.c_uint32,
                                                 ctypes.POINTER(BtConfig), ctypes.POINTER(BtSolution),
                                                 ctypes.c_uint64, u64p, ctypes.POINTER(BtResult)]),
    "emp_bt_count_batch": (ctypes.c_int32, [ctypes.POINTER(ctypes.c_void_p), ctypes.c_uint32, ctypes.POINTER(BtConfig),
                                            ctypes.POINTER(BtResult)]),
    "emp_bt_plan_create": (ctypes.c_int32, [ctypes.POINTER(ctypes.c_void_p), ctypes.c_uint32, ctypes.POINTER(BtConfig),
                                            ctypes.POINTER(ctypes.c_void_p)]),
    "emp_bt_plan_subtrees": (ctypes.c_int32, [ctypes.c_void_p, u64p]),
    "emp_bt_plan_select": (ctypes.c_int32, [ctypes.c_void_p, ctypes.c_uint64, ctypes.c_uint64, ctypes.c_uint64]),
    "emp_bt_plan_run": (ctypes.c_int32, [ctypes.c_void_p, ctypes.c_void_p]),
    "emp_bt_plan_results": (ctypes.c_int32, [ctypes.c_void_p, ctypes.POINTER(BtResult)]),
    "emp_bt_plan_subtree_counts": (ctypes.c_int32, [ctypes.c_void_p, u64p, u64p, ctypes.c_uint64]),
    "emp_bt_plan_subtree_prefix": (ctypes.c_int32, [ctypes.c_void_p, ctypes.c_uint64, u16p, ctypes.c_uint32]),
    "emp_bt_plan_destroy": (None, [ctypes.c_void_p]),
    "emp_bt_solutions": (ctypes.c_int32, [ctypes.c_void_p, ctypes.POINTER(BtConfig), ctypes.POINTER(BtSolution),
                                          ctypes.c_uint64, ctypes.POINTER(ctypes.c_uint64), ctypes.POINTER(BtResult)]),
    "emp_bt_autotune": (ctypes.c_int32, [ctypes.c_void_p, ctypes.c_uint32, ctypes.POINTER(BtConfig), ctypes.c_uint32,
                                         ctypes.POINTER(TuneResult)]),
    "emp_mlp_create": (ctypes.c_int32, [ctypes.c_uint64, ctypes.c_int32, ctypes.POINTER(ctypes.c_void_p)]),
    "emp_mlp_destroy": (None, [ctypes.c_void_p]),
    "emp_mlp_get_params": (ctypes.c_int32, [ctypes.c_void_p, ctypes.c_void_p]),
    "emp_mlp_set_params": (ctypes.c_int32, [ctypes.c_void_p, ctypes.c_void_p]),
    "emp_mlp_features": (ctypes.c_int32, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint32, ctypes.c_void_p,
                                          ctypes.c_void_p, ctypes.c_uint64, ctypes.c_void_p]),
    "emp_mlp_score": (ctypes.c_int32, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint64, ctypes.c_void_p]),
    "emp_mlp_score_f32": (ctypes.c_int32, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint64, ctypes.c_void_p]),
    "emp_mlp_loss_grad": (ctypes.c_int32, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                           ctypes.c_uint64, ctypes.POINTER(ctypes.c_double), ctypes.c_void_p]),
    "emp_mlp_train": (ctypes.c_int32, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint32, ctypes.c_void_p,
                                       ctypes.POINTER(MlpTrainConfig), ctypes.POINTER(MlpTrainReport)]),
    "emp_bt_plan_order": (ctypes.c_int32, [ctypes.c_void_p, ctypes.c_void_p]),
    "emp_glutton_max": (ctypes.c_int32, [ctypes.c_void_p, ctypes.POINTER(GmConfig), ctypes.POINTER(GmResult)]),
    "emp_glutton_max_noalloc": (ctypes.c_int32, [ctypes.c_void_p, ctypes.POINTER(GmConfig), ctypes.POINTER(GmResult)]),
}

_lib = None


def load():
    """Load libemp_b200.so (raises when it is missing: there is no fallback)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing; build it with python -m edge_matching_puzzle_b200.build")
        lib = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _lib = lib
    return _lib


def check(status: int) -> int:
    if status < 0:
        raise EmpError(status, load().emp_last_error().decode())
    return status


def generate(width: int, height: int, border_colors: int, interior_colors: int, seed: int) -> List[List[int]]:
    buf = (ctypes.c_uint8 * (4 * width * height))()
    check(load().emp_generate_puzzle(width, height, border_colors, interior_colors, seed, buf))
    raw = list(buf)
    return [raw[4 * i:4 * i + 4] for i in range(width * height)]


class NativePuzzle:
    """Owns an emp_puzzle handle."""

    def __init__(self, width: int, height: int, colors: Sequence[Sequence[int]], order: Optional[Sequence[int]] = None):
        L = load()
        n = width * height
        self._colours = (ctypes.c_uint8 * (4 * n))(*[c for p in colors for c in p])
        self._order = (ctypes.c_uint16 * n)(*order) if order is not None else None
        desc = PuzzleDesc(width, height, ctypes.cast(self._colours, u8p),
                          ctypes.cast(self._order, u16p) if self._order is not None else None)
        h = ctypes.c_void_p()
        check(L.emp_puzzle_create(ctypes.byref(desc), ctypes.byref(h)))
        self.handle = h
        self.width, self.height, self.n = width, height, n

    def close(self):
        if getattr(self, "handle", None):
            load().emp_puzzle_destroy(self.handle)
            self.handle = None

    def __del__(self):
        self.close()

    def export_tables(self) -> List[int]:
        words = ctypes.c_uint64()
        check(load().emp_puzzle_export_tables(self.handle, None, 0, ctypes.byref(words)))
        buf = (ctypes.c_uint32 * words.value)()
        check(load().emp_puzzle_export_tables(self.handle, buf, words.value, ctypes.byref(words)))
        return list(buf)

    def max_kind_words(self) -> int:
        """64-bit words of the widest kind bitfield (4 bits per piece)."""
        i = self.info()
        return (4 * max(i.nb_center, i.nb_border, i.nb_corner) + 63) // 64

    def table_bytes(self) -> int:
        return 4 * len(self.export_tables())

    def info(self) -> PuzzleInfo:
        i = PuzzleInfo()
        check(load().emp_puzzle_get_info(self.handle, ctypes.byref(i)))
        return i


def bt_config(**kw) -> BtConfig:
    c = BtConfig()
    c.device = -1
    for k, v in kw.items():
        setattr(c, k, v)
    return c


def bt_count(puzzle: NativePuzzle, **kw) -> BtResult:
    r = BtResult()
    cfg = bt_config(**kw)
    check(load().emp_bt_count(puzzle.handle, ctypes.byref(cfg), ctypes.byref(r)))
    return r


def bt_variable_space(puzzle: NativePuzzle, capacity: int = 4096, max_selections: int = 0, timeout_ms: int = 0,
                      device: int = -1):
    """emp_bt_variable_space (debug mode): ([(lane, variable, step)], board or None, status)."""
    ev = (VsEvent * max(capacity, 1))()
    ne = ctypes.c_uint64()
    board = (ctypes.c_uint32 * puzzle.n)()
    found = ctypes.c_uint32()
    st = check(load().emp_bt_variable_space(puzzle.handle, device, max_selections, timeout_ms, ev, capacity,
                                            ctypes.byref(ne), board, ctypes.byref(found)))
    events = [(ev[i].lane, ev[i].variable, ev[i].step) for i in range(min(ne.value, capacity))]
    return events, (list(board) if found.value else None), st


def bt_resume(puzzle: NativePuzzle, situation: Sequence[int], **kw) -> BtResult:
    """emp_bt_resume: the search resumed from a partial situation (the transitions placed
    at the first levels of the puzzle's order), as --initial_situation does."""
    r = BtResult()
    cfg = bt_config(**kw)
    arr = (ctypes.c_uint16 * max(1, len(situation)))(*situation)
    check(load().emp_bt_resume(puzzle.handle, arr, len(situation), ctypes.byref(cfg), ctypes.byref(r)))
    return r


def bt_resume_solutions(puzzle: NativePuzzle, situation: Sequence[int], capacity: int = 4096, **kw):
    """emp_bt_resume_solutions: (found, [(node_index, board)], result) of the resumed search."""
    out = (BtSolution * max(capacity, 1))()
    found = ctypes.c_uint64()
    res = BtResult()
    cfg = bt_config(**kw)
    arr = (ctypes.c_uint16 * max(1, len(situation)))(*situation)
    check(load().emp_bt_resume_solutions(puzzle.handle, arr, len(situation), ctypes.byref(cfg), out, capacity,
                                         ctypes.byref(found), ctypes.byref(res)))
    n = min(found.value, capacity)
    return found.value, [(out[i].node_index, list(out[i].board)) for i in range(n)], res


def bt_count_batch(puzzles: Sequence[NativePuzzle], **kw) -> List[BtResult]:
    arr = (ctypes.c_void_p * len(puzzles))(*[p.handle for p in puzzles])
    res = (BtResult * len(puzzles))()
    cfg = bt_config(**kw)
    check(load().emp_bt_count_batch(arr, len(puzzles), ctypes.byref(cfg), res))
    return list(res)


def bt_solutions(puzzle: NativePuzzle, capacity: int = 4096, **kw):
    """emp_bt_solutions: (found, [(node_index, board)], result) in the reference's order."""
    out = (BtSolution * max(capacity, 1))()
    found = ctypes.c_uint64()
    res = BtResult()
    cfg = bt_config(**kw)
    check(load().emp_bt_solutions(puzzle.handle, ctypes.byref(cfg), out, capacity, ctypes.byref(found),
                                  ctypes.byref(res)))
    n = min(found.value, capacity)
    return found.value, [(out[i].node_index, list(out[i].board)) for i in range(n)], res


def bt_autotune(puzzles: Sequence[NativePuzzle], trial_ms: int = 200, **kw) -> TuneResult:
    """emp_bt_autotune: the fastest launch parameters for these puzzles (timed trials)."""
    arr = (ctypes.c_void_p * len(puzzles))(*[p.handle for p in puzzles])
    cfg = bt_config(**kw)
    out = TuneResult()
    check(load().emp_bt_autotune(arr, len(puzzles), ctypes.byref(cfg), trial_ms, ctypes.byref(out)))
    return out


def _f32(a, n=None):
    import numpy as np
    arr = np.ascontiguousarray(a, dtype=np.float32)
    if n is not None and arr.size != n:
        raise ValueError(f"expected {n} values, got {arr.size}")
    return arr


class Mlp:
    """emp_mlp: the candidate-scoring network of the learned value ordering."""

    def __init__(self, seed: int = 1, device: int = -1):
        h = ctypes.c_void_p()
        check(load().emp_mlp_create(seed, device, ctypes.byref(h)))
        self.handle = h.value

    def close(self) -> None:
        if self.handle:
            load().emp_mlp_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def params(self):
        import numpy as np
        out = np.empty(MLP_PARAMS, dtype=np.float32)
        check(load().emp_mlp_get_params(self.handle, out.ctypes.data))
        return out

    def set_params(self, params) -> None:
        arr = _f32(params, MLP_PARAMS)
        check(load().emp_mlp_set_params(self.handle, arr.ctypes.data))

    def score(self, features):
        """Tensor-core scores (BF16 operands, FP32 accumulation)."""
        import numpy as np
        x = _f32(features)
        n = x.size // MLP_INPUTS
        out = np.empty(n, dtype=np.float32)
        check(load().emp_mlp_score(self.handle, x.ctypes.data, n, out.ctypes.data))
        return out

    def score_f32(self, features):
        import numpy as np
        x = _f32(features)
        n = x.size // MLP_INPUTS
        out = np.empty(n, dtype=np.float32)
        check(load().emp_mlp_score_f32(self.handle, x.ctypes.data, n, out.ctypes.data))
        return out

    def loss_grad(self, features, labels, weights):
        import numpy as np
        x = _f32(features)
        n = x.size // MLP_INPUTS
        y = _f32(labels, n)
        w = _f32(weights, n)
        loss = ctypes.c_double()
        grads = np.empty(MLP_PARAMS, dtype=np.float32)
        check(load().emp_mlp_loss_grad(self.handle, x.ctypes.data, y.ctypes.data, w.ctypes.data, n,
                                       ctypes.byref(loss), grads.ctypes.data))
        return loss.value, grads

    def train(self, puzzles: Sequence[NativePuzzle], solutions, epochs: int = 0, batch: int = 0,
              learning_rate: float = 0.0, seed: int = 1, max_level: int = 0) -> MlpTrainReport:
        """solutions: one emp_bt_result.first_solution board (256 values) per puzzle."""
        import numpy as np
        arr = (ctypes.c_void_p * len(puzzles))(*[p.handle for p in puzzles])
        boards = np.ascontiguousarray(solutions, dtype=np.uint32).reshape(len(puzzles), 256)
        cfg = MlpTrainConfig()
        cfg.epochs, cfg.batch, cfg.learning_rate, cfg.seed = epochs, batch, learning_rate, seed
        cfg.max_level = max_level
        rep = MlpTrainReport()
        check(load().emp_mlp_train(self.handle, arr, len(puzzles), boards.ctypes.data, ctypes.byref(cfg),
                                   ctypes.byref(rep)))
        return rep


def mlp_features(puzzle: NativePuzzle, prefixes: Sequence[Sequence[int]], cands: Sequence[int]):
    """emp_mlp_features: one row per (prefix, candidate placed right after it)."""
    import numpy as np
    n = len(prefixes)
    stride = max([len(p) for p in prefixes] + [1])
    pre = np.zeros((n, stride), dtype=np.uint16)
    for i, p in enumerate(prefixes):
        pre[i, :len(p)] = p
    lens = np.array([len(p) for p in prefixes], dtype=np.uint16)
    cd = np.array(cands, dtype=np.uint16)
    out = np.empty((n, MLP_INPUTS), dtype=np.float32)
    check(load().emp_mlp_features(puzzle.handle, pre.ctypes.data, stride, lens.ctypes.data, cd.ctypes.data, n,
                                  out.ctypes.data))
    return out


def config_dict(cfg: BtConfig) -> dict:
    return {name: getattr(cfg, name) for name, _ in BtConfig._fields_}


def glutton_max(puzzle: NativePuzzle, push_budget: int = 0, timeout_ms: int = 0, device: int = -1,
                placement_budget: int = 0, blocks: int = 0) -> GmResult:
    cfg = GmConfig()
    cfg.push_budget = push_budget
    cfg.blocks = blocks
    cfg.placement_budget = placement_budget
    cfg.timeout_ms = timeout_ms
    cfg.device = device
    r = GmResult()
    check(load().emp_glutton_max(puzzle.handle, ctypes.byref(cfg), ctypes.byref(r)))
    return r


def glutton_wide_situation(puzzle: NativePuzzle, n: int):
    """emp_glutton_wide_situation: the n positions' level-0 infos, 32 words each."""
    out = (ctypes.c_uint32 * (32 * n))()
    check(load().emp_glutton_wide_situation(puzzle.handle, out, 32 * n))
    return [list(out[32 * j:32 * j + 32]) for j in range(n)]


def glutton_max_noalloc(puzzle: NativePuzzle, push_budget: int = 0, timeout_ms: int = 0,
                        device: int = -1) -> GmResult:
    """emp_glutton_max_noalloc: the same search in the library's fixed device array."""
    cfg = GmConfig()
    cfg.push_budget = push_budget
    cfg.timeout_ms = timeout_ms
    cfg.device = device
    r = GmResult()
    check(load().emp_glutton_max_noalloc(puzzle.handle, ctypes.byref(cfg), ctypes.byref(r)))
    return r


class BtPlan:
    """emp_bt_plan: prefix expansion done once, kernel runs on demand."""

    def __init__(self, puzzles: Sequence[NativePuzzle], **kw):
        self.puzzles = list(puzzles)
        arr = (ctypes.c_void_p * len(puzzles))(*[p.handle for p in puzzles])
        self.cfg = bt_config(**kw)
        h = ctypes.c_void_p()
        check(load().emp_bt_plan_create(arr, len(puzzles), ctypes.byref(self.cfg), ctypes.byref(h)))
        self.handle = h
        self.selected = None

    def subtrees(self) -> int:
        n = ctypes.c_uint64()
        check(load().emp_bt_plan_subtrees(self.handle, ctypes.byref(n)))
        return n.value

    def select(self, first: int, stride: int, count: int) -> None:
        check(load().emp_bt_plan_select(self.handle, first, stride, count))
        self.selected = count

    def run(self, stream: int = 0) -> None:
        check(load().emp_bt_plan_run(self.handle, ctypes.c_void_p(stream) if stream else None))

    def results(self) -> List[BtResult]:
        res = (BtResult * len(self.puzzles))()
        check(load().emp_bt_plan_results(self.handle, res))
        return list(res)

    def order(self, model: "Mlp") -> None:
        """emp_bt_plan_order: queue the subtrees best first by the model's scores."""
        check(load().emp_bt_plan_order(self.handle, model.handle))

    def subtree_counts(self, count: int):
        nn = (ctypes.c_uint64 * count)()
        ss = (ctypes.c_uint64 * count)()
        check(load().emp_bt_plan_subtree_counts(self.handle, nn, ss, count))
        return list(nn), list(ss)

    def subtree_prefix(self, index: int, depth: int) -> List[int]:
        buf = (ctypes.c_uint16 * depth)()
        check(load().emp_bt_plan_subtree_prefix(self.handle, index, buf, depth))
        return list(buf)

    def rec_words(self) -> int:
        """32-bit words per work record (header, prefix, remaining set)."""
        n = max(p.n for p in self.puzzles)
        kw = max(p.max_kind_words() for p in self.puzzles)
        return 4 + (n + 1) // 2 + 2 * kw

    def close(self):
        if getattr(self, "handle", None):
            load().emp_bt_plan_destroy(self.handle)
            self.handle = None

    def __del__(self):
        self.close()
