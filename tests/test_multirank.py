"""Replicas over ranks (the N > 1 bench path): two gloo ranks on the CPU.

The solver does not shard; every rank solves its own right-hand sides and the
ranks only agree on the timing (max over ranks) at the barrier."""
import os
import socket

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        bench.barrier(world)
        # each rank times a different duration; all see the slowest
        ms = bench.max_over_ranks(100.0 + 50.0 * rank, world)
        seed = bench.replica_seed(rank)
        seeds = [None] * world
        dist.all_gather_object(seeds, seed)
        out[rank] = (ms, bench.job_throughput(world, 3, 4, ms), tuple(seeds))
        bench.barrier(world)
    finally:
        dist.destroy_process_group()


def test_two_rank_replicas_agree_on_timing():
    world = 2
    port = _free_port()
    ctx = mp.get_context("spawn")
    with ctx.Manager() as manager:
        out = manager.dict()
        mp.start_processes(_rank_main, args=(world, port, out), nprocs=world, join=True,
                           start_method="spawn")
        res = dict(out)
    assert set(res) == {0, 1}
    for rank in range(world):
        ms, value, seeds = res[rank]
        assert ms == pytest.approx(150.0)              # the slowest rank
        assert value == pytest.approx(2 * 3 * 4 / 0.150)  # whole-job solves/s
        assert len(set(seeds)) == world                 # distinct right-hand sides
