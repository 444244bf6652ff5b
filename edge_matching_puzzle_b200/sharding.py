"""Sharding of the searches over ranks (one process per GPU).

The exhaustive search splits into independent subtrees and puzzles, so ranks share no
data: rank r takes slices r, r+N, r+2N, ... of the subtree slices (or every N-th puzzle
of a batch), and the only collective is the final reduction of each rank's device time
(max) and counts (sum)."""
from __future__ import annotations

from typing import List, Sequence, Tuple, TypeVar

T = TypeVar("T")


def slice_for_step(step: int, rank: int, world: int, slices: int) -> int:
    """Subtree slice that `rank` searches at `step`: consecutive steps of all ranks
    walk the slices in order, each slice once per `slices // world` steps."""
    return (step * world + rank) % slices


def items_for_rank(items: Sequence[T], rank: int, world: int) -> List[T]:
    """Every world-th item starting at rank (instances of a batch)."""
    return list(items[rank::world])


def reduce_time_and_counts(dist, device, seconds: float, counts: Sequence[float]) -> Tuple[float, List[float]]:
    """Max over ranks of the timed region and sum over ranks of the counts (one
    all-reduce each).  `dist` is torch.distributed (or None for one process); device is
    where the reduction tensors live ("cpu" for gloo, the rank's GPU for NCCL)."""
    if dist is None:
        return seconds, list(counts)
    import torch
    mx = torch.tensor([seconds], dtype=torch.float64, device=device)
    dist.all_reduce(mx, op=dist.ReduceOp.MAX)
    if not counts:
        return mx.item(), []
    sm = torch.tensor(list(counts), dtype=torch.float64, device=device)
    dist.all_reduce(sm, op=dist.ReduceOp.SUM)
    return mx.item(), sm.tolist()
