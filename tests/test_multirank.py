"""The multi-GPU path's host logic on CPU: two gloo ranks.

The path shards by independent searches (weak scaling, no data-path
collective): each rank builds its own instances with disjoint seeds, and
the only collectives are the timing reductions -- the slowest rank's time
and the sum of all ranks' moves.
"""
import os
import socket

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    import sys
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import bench
    from datetime import timedelta
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        seeds = [j["seed"] for j in bench.make_jobs(rank)]
        gathered = [None] * world
        dist.all_gather_object(gathered, seeds)
        ms = 100.0 + 50.0 * rank            # rank 1 is the slow one
        moves = 1e9 * (rank + 1)
        (mx,), (total,) = bench.reduce_over_ranks(world, "cpu", [ms], [moves])
        out.put((rank, gathered, mx, total))
    finally:
        dist.destroy_process_group()


def test_two_ranks_shard_disjoint_searches_and_reduce_timing():
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, gathered, mx, total in res:
        assert len(set(gathered[0]) & set(gathered[1])) == 0
        assert len(gathered[0]) == len(gathered[1]) > 0
        assert mx == 150.0 and total == 3e9


def test_single_rank_needs_no_process_group():
    import bench
    assert bench.reduce_over_ranks(1, "cpu", [2.0], [3.0, 4.0]) == ([2.0], [3.0, 4.0])
