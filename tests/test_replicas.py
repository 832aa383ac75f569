"""The multi-GPU form is N independent replicas: the job's time is the slowest rank's.

Two gloo ranks on the CPU run the bench's barrier and max-over-ranks reduction.
"""

import os

import torch
import torch.distributed as dist
import torch.multiprocessing as mp


def _rank(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        import bench

        dist.barrier()
        out[rank] = bench.max_over_ranks(1.0 + rank, dist, "cpu")
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_with_two_gloo_ranks():
    import socket

    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    ctx = mp.get_context("spawn")
    out = ctx.Manager().dict()
    mp.start_processes(_rank, args=(2, port, out), nprocs=2, join=True, start_method="spawn")
    assert dict(out) == {0: 2.0, 1: 2.0}
