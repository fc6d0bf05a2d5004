"""bench.py's multi-rank timing on CPU: world_size-2 gloo ranks (replicas only).

Each rank reports its own elapsed time; the job's time is the slowest rank's,
and whole-job throughput divides all ranks' answers by it.
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


def _rank(rank, world, port, out):
    import sys

    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import bench

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        mine = 1.0 + rank  # rank 1 is the slow replica
        out[rank] = bench.max_over_ranks(mine, dist, "cpu")
    finally:
        dist.destroy_process_group()


def test_job_time_is_the_slowest_rank():
    ctx = mp.get_context("spawn")
    out = ctx.Manager().dict()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    assert out[0] == out[1] == 2.0


def test_single_rank_is_unchanged():
    import bench

    assert bench.max_over_ranks(3.5, None, "cpu") == 3.5
