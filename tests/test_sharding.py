"""Multi-rank path of the benchmark on CPU: two gloo ranks check that the slices and
instances they take cover the work once, and that the reduction gives the max of the
ranks' times and the sum of their counts."""
from __future__ import annotations

import os
import socket

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from edge_matching_puzzle_b200.sharding import items_for_rank, reduce_time_and_counts, slice_for_step


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        steps, slices = 16, 64
        mine = [slice_for_step(i, rank, world, slices) for i in range(steps)]
        gathered = [None] * world
        dist.all_gather_object(gathered, mine)
        inst = items_for_rank(list(range(101)), rank, world)
        all_inst = [None] * world
        dist.all_gather_object(all_inst, inst)
        t, c = reduce_time_and_counts(dist, "cpu", 1.0 + rank, [10.0 * (rank + 1), 1.0])
        if rank == 0:
            out.put((gathered, all_inst, t, c))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_cover_the_work_once():
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    gathered, all_inst, t, c = q.get(timeout=120)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    slices = [s for rank_slices in gathered for s in rank_slices]
    assert sorted(slices) == list(range(32))  # 16 steps x 2 ranks = the first 32 slices, once each
    inst = sorted(i for r in all_inst for i in r)
    assert inst == list(range(101))
    assert t == 2.0 and c == [30.0, 2.0]


def test_single_process_reduction_is_identity():
    assert reduce_time_and_counts(None, "cpu", 3.5, [1, 2]) == (3.5, [1, 2])
    assert slice_for_step(5, 0, 1, 64) == 5
