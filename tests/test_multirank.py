"""The sharded batched solves as two gloo ranks on the CPU: each rank builds the rooms of its part,
and the ranks' parts together are every room once, their air cells summed by a collective the
same way bench.py sums them."""

from __future__ import annotations

import os

import torch
import torch.distributed as dist
import torch.multiprocessing as mp


def _rank(rank: int, world: int, port: int, out) -> None:
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        from acoustic_spaces_b200 import layouts

        batch = layouts.batched_rooms(7, rooms=5, sources=1, cell=0.25, steps=10, part=(rank, world))
        air = torch.tensor([float(batch.description["air_cells"])], dtype=torch.float64)
        dist.all_reduce(air, op=dist.ReduceOp.SUM)
        rooms = [None] * world
        dist.all_gather_object(rooms, batch.description["rooms_here"])
        out[rank] = (float(air.item()), rooms)
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_share_the_batched_solves():
    from acoustic_spaces_b200 import layouts

    whole = layouts.batched_rooms(7, rooms=5, sources=1, cell=0.25, steps=10).description["air_cells"]
    ctx = mp.get_context("spawn")
    with ctx.Manager() as manager:
        out = manager.dict()
        port = 29500 + os.getpid() % 1000
        procs = [ctx.Process(target=_rank, args=(r, 2, port, out)) for r in range(2)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(timeout=240)
        assert all(p.exitcode == 0 for p in procs)
        results = dict(out)
    assert results[0][0] == results[1][0] == float(whole)
    assert sum(results[0][1]) == 5
