"""The bench's multi-GPU bookkeeping on two CPU ranks (gloo): each rank's
device time is reduced to the job's time as the maximum over ranks, and the
weak-scaling throughput counts every rank's rows against that time."""
from __future__ import annotations

import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank(rank, world, port, q):
    import datetime
    import sys

    import torch.distributed as dist
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import bench
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        times = [12.5, 20.0, 7.0, 9.5]  # ms of each rank's timed region
        job_ms = bench.max_over_ranks(times[rank], dist, "cpu")
        dist.barrier()
        value = bench.job_mtuples(world, 1000, 10, job_ms / 1e3)
        q.put((rank, job_ms, value))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 4])
def test_max_over_ranks_and_weak_scaling(world):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=120) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    slowest = max([12.5, 20.0, 7.0, 9.5][:world])
    for rank, job_ms, value in out:
        assert job_ms == slowest  # every rank reports the slowest rank's time
        assert value == pytest.approx(world * 1000 * 10 / (slowest / 1e3) / 1e6)


def test_single_process_needs_no_group():
    import bench
    assert bench.max_over_ranks(3.0, None, "cpu") == 3.0
    assert bench.job_mtuples(1, 2 ** 20, 4, 2.0) == pytest.approx(2 ** 22 / 2.0 / 1e6)
