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


def _sharded_rank(rank, world, port, q):
    import datetime
    import sys

    import numpy as np
    import torch
    import torch.distributed as dist
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, root)
    sys.path.insert(0, os.path.join(root, "oracle"))
    import bench
    import oracle as O
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        nR, nS = 5000, 40001
        rng = np.random.default_rng(5)  # every rank draws the same S; each keeps its shard
        R_rows = np.zeros(nR, dtype=O.ROW)
        R_rows["key"] = rng.permutation(nR) + 1
        S_all = np.zeros(nS, dtype=O.ROW)
        S_all["key"] = rng.integers(1, 2 * nR, nS)
        lo, hi = bench.shard_rows(nS, world, rank)
        R = torch.zeros(nR, dtype=torch.int64)
        if rank == 0:  # R exists on rank 0 only until the broadcast
            R.copy_(torch.from_numpy(R_rows.view(np.int64).copy()))

        def join_count(Rt, S):
            return O.rho(Rt.numpy().view(O.ROW), S)

        m = bench.sharded_count(dist, R, S_all[lo:hi], join_count)
        q.put((rank, lo, hi, m, O.rho(R_rows, S_all)))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_sharded_join_matches_single_join(world):
    """S split over the ranks, R broadcast from rank 0, counts all-reduced:
    the total equals the oracle's count of the unsharded join."""
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_sharded_rank, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=120) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    bounds = [(lo, hi) for _, lo, hi, _, _ in out]
    assert bounds[0][0] == 0 and bounds[-1][1] == 40001
    assert all(bounds[i][1] == bounds[i + 1][0] for i in range(world - 1))
    for _, _, _, m, want in out:
        assert m == want  # every rank holds the full join's count


def test_shard_rows_cover_evenly():
    import bench
    for n in (0, 1, 7, 1 << 20, (1 << 30) + 3):
        for world in (1, 2, 3, 8):
            parts = [bench.shard_rows(n, world, r) for r in range(world)]
            assert parts[0][0] == 0 and parts[-1][1] == n
            assert all(parts[i][1] == parts[i + 1][0] for i in range(world - 1))
            sizes = [hi - lo for lo, hi in parts]
            assert max(sizes) - min(sizes) <= 1
