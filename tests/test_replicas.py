"""Multi-GPU replicas, host side: bench.py's cross-rank timing (max over ranks) and whole-job
throughput, run as two gloo ranks on the CPU (the search itself exchanges nothing between GPUs)."""
import os
import socket
import sys

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        sys.path.insert(0, REPO)
        import bench
        local_seconds = 1.0 + rank  # rank 1 is the slowest replica
        slowest = bench.max_over_ranks(local_seconds)
        out[rank] = (slowest, bench.job_throughput(4096 * 10, world, slowest))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_replicas_time_by_slowest_rank():
    world, port = 2, _free_port()
    out = mp.get_context("spawn").Manager().dict()
    mp.spawn(_rank, args=(world, port, out), nprocs=world, join=True)
    assert out[0] == out[1]
    slowest, qps = out[0]
    assert slowest == pytest.approx(2.0)
    assert qps == pytest.approx(4096 * 10 * 2 / 2.0)


def test_single_process_needs_no_group():
    sys.path.insert(0, REPO)
    import bench
    assert bench.max_over_ranks(3.5) == 3.5
    assert bench.job_throughput(100, 1, 2.0) == 50.0
