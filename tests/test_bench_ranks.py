"""The replica job arithmetic of bench.py under torch.distributed: world-size-2
gloo ranks on the CPU (the GPU run uses NCCL with the same calls). Every rank
reports the slowest rank's time, and the job rate counts all ranks' cells."""
import os
import socket

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

import bench


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import datetime

    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    ms = [120.0, 150.0][rank]
    slow = bench.max_over_ranks(ms, dist, "cpu")
    out[rank] = (slow, bench.job_rate(1000, 10, world, slow))
    dist.barrier()
    dist.destroy_process_group()


def test_replicas_report_the_slowest_rank():
    world = 2
    port = _free_port()
    with mp.Manager() as mgr:
        out = mgr.dict()
        mp.spawn(_rank, args=(world, port, out), nprocs=world, join=True)
        res = dict(out)
    for r in range(world):
        slow, rate = res[r]
        assert slow == 150.0
        assert rate == pytest.approx(1000 * 10 * 2 / 0.150)


def test_single_process_needs_no_group():
    assert bench.max_over_ranks(12.5, None, "cpu") == 12.5
    assert bench.job_rate(100, 4, 1, 1000.0) == pytest.approx(400.0)
