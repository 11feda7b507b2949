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
    import importlib
    import sys

    import numpy as np
    import torch
    import torch.distributed as dist
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, root)
    sys.path.insert(0, os.path.join(root, "oracle"))
    import bench
    import oracle as O
    tbg = importlib.import_module("tee-bench_b200")
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        nR, nS = 5000, 40001
        rng = np.random.default_rng(5)  # every rank draws the same relations; each keeps its rows
        R_all = np.zeros(nR, dtype=O.ROW)
        R_all["key"] = rng.permutation(nR) + 1
        R_all["key"][:40] = 7  # duplicate R keys
        R_all["payload"] = np.arange(nR)
        S_all = np.zeros(nS, dtype=O.ROW)
        S_all["key"] = rng.zipf(1.3, nS) % (2 * nR) + 1  # skew and misses
        S_all["payload"] = np.arange(nS)
        rlo, rhi = bench.shard_rows(nR, world, rank)
        slo, shi = bench.shard_rows(nS, world, rank)

        def as_tensor(rows):
            return torch.from_numpy(np.ascontiguousarray(rows).view(np.int64).copy())

        def split(t, nshards):  # the library's grouping, on the host
            rows = t.numpy().view(O.ROW)
            d = tbg.shard_of(rows["key"], nshards)
            order = np.argsort(d, kind="stable")
            offs = np.concatenate([[0], np.cumsum(np.bincount(d, minlength=nshards))]).tolist()
            return as_tensor(rows[order]), offs

        seen = []

        def join(Rt, St):
            Rr, Sr = Rt.numpy().view(O.ROW), St.numpy().view(O.ROW)
            seen.append((set(tbg.shard_of(Rr["key"], world).tolist()), set(tbg.shard_of(Sr["key"], world).tolist())))
            return O.rho(Rr, Sr)

        m = tbg.distributed_join_count(dist, as_tensor(R_all[rlo:rhi]), as_tensor(S_all[slo:shi]), split, join,
                                       lambda n: torch.empty(n, dtype=torch.int64))
        q.put((rank, m, O.rho(R_all, S_all), seen))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_sharded_join_matches_single_join(world):
    """R and S spread over the ranks, split by key hash, exchanged with an
    all-to-all, joined per rank and the counts summed: every rank holds the
    unsharded join's count (oracle), and each rank joined only its shard."""
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_sharded_rank, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = sorted((q.get(timeout=120) for _ in range(world)), key=lambda x: x[0])
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, m, want, seen in out:
        assert m == want  # every rank holds the full join's count
        (r_shards, s_shards), = seen
        assert r_shards <= {rank} and s_shards <= {rank}  # a rank joins only its own shard's keys


def test_shard_rows_cover_evenly():
    import bench
    for n in (0, 1, 7, 1 << 20, (1 << 30) + 3):
        for world in (1, 2, 3, 8):
            parts = [bench.shard_rows(n, world, r) for r in range(world)]
            assert parts[0][0] == 0 and parts[-1][1] == n
            assert all(parts[i][1] == parts[i + 1][0] for i in range(world - 1))
            sizes = [hi - lo for lo, hi in parts]
            assert max(sizes) - min(sizes) <= 1
