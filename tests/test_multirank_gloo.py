"""The N > 1 bench plumbing on CPU: two gloo ranks, each timing its own
replica, agree on the slowest rank's step time and the whole-job throughput."""
import os
import socket

import torch.distributed as dist
import torch.multiprocessing as mp

import bench


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank: int, world: int, port: int, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        ms = bench.max_over_ranks(100.0 + 50.0 * rank, world, device="cpu")
        dist.barrier()
        out[rank] = (ms, bench.job_throughput(1_000_000, world, ms))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_take_the_slowest_step():
    world = 2
    manager = mp.get_context("spawn").Manager()
    out = manager.dict()
    mp.spawn(_rank, args=(world, _free_port(), out), nprocs=world, join=True)
    assert out[0] == out[1] == (150.0, 1_000_000 * 2 / 0.150)


def test_single_rank_is_identity():
    assert bench.max_over_ranks(12.5, 1) == 12.5
    assert bench.job_throughput(10, 1, 1000.0) == 10.0
