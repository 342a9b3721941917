"""The multi-rank logic of bench.py (replicas, one per rank): max over ranks
and whole-job throughput, on two gloo ranks on the CPU."""
import os
import socket

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, out):
    import sys

    sys.path.insert(0, ROOT)
    import bench

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        seconds = 1.0 + rank  # rank 1 is the slow one
        m = bench.max_over_ranks(seconds, dist, None)
        out[rank] = m
        out[world + rank] = bench.job_throughput(100, 10, world, m)
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_and_job_throughput_two_ranks():
    world = 2
    out = mp.get_context("spawn").Array("d", 2 * world)
    mp.spawn(_worker, args=(world, _free_port(), out), nprocs=world, join=True)
    assert list(out[:world]) == [2.0, 2.0]
    assert list(out[world:]) == [pytest.approx(1000.0), pytest.approx(1000.0)]


def test_single_rank_is_identity():
    import sys

    sys.path.insert(0, ROOT)
    import bench

    assert bench.max_over_ranks(3.5) == 3.5
    assert bench.job_throughput(8, 2, 1, 4.0) == 4.0
