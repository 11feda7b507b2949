"""Batched joins (tbg_batch_*): per-join counts against the oracle's RHO on
the same relations, through the C ABI, for every planning mode."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import ROOT  # noqa: F401  (puts the repo root on sys.path)

ROW = np.dtype([("key", "<u4"), ("payload", "<u4")])


def _rel(keys):
    r = np.zeros(len(keys), dtype=ROW)
    r["key"] = np.asarray(keys, dtype=np.uint32)
    r["payload"] = np.arange(len(keys), dtype=np.uint32) * np.uint32(2654435761)
    return r


def mixed_joins(seed=7):
    """Joins of every shape the planner distinguishes: empty sides, one row,
    sizes around the shared-memory table capacity (8192), duplicates in R,
    misses, full-range keys, one heavy key, Zipf-skewed S."""
    rs = np.random.RandomState(seed)
    out = []
    sizes = [0, 1, 7, 100, 1000, 5000, 8191, 8192, 8193, 20000, 70000, 300000]
    for i, n in enumerate(sizes):
        k = 1 + i % 5
        kind = ["pk", "dup", "high", "zipf", "miss"][i % 5]
        if kind == "pk":
            R = _rel(rs.permutation(n) + 1)
            S = _rel(rs.randint(1, n + 1, k * n) if n else [])
        elif kind == "dup":
            dom = max(1, n // 4)
            R = _rel(rs.randint(1, dom + 1, n))
            S = _rel(rs.randint(1, dom + 1, k * n))
        elif kind == "high":
            keys = rs.randint(0, 2 ** 32, n, dtype=np.uint64).astype(np.uint32)
            R = _rel(keys)
            pick = keys[rs.randint(0, n, k * n)] if n else np.zeros(0, np.uint32)
            S = _rel(np.where(rs.random_sample(k * n) < 0.5, pick, rs.randint(0, 2 ** 32, k * n, dtype=np.uint64)))
        elif kind == "zipf":
            R = _rel(rs.permutation(n) + 1)
            z = np.minimum(rs.zipf(1.3, k * n), max(n, 1)) if n else np.zeros(0)
            S = _rel(z)
        else:
            R = _rel(rs.permutation(n) + 1)
            S = _rel(rs.randint(n + 1, 2 * n + 2, k * n))
        out.append((R, S))
    out.append((_rel([5] * 50), _rel([5] * 100 + [6] * 10)))   # cross product
    out.append((_rel([]), _rel([1, 2, 3])))
    out.append((_rel([1, 2, 3]), _rel([])))
    out.append((_rel(rs.permutation(40000) + 1), _rel([1] * 200000 + [2] * 1000)))  # one heavy key
    return out


def upload(torch, joins, misalign=True):
    """All relations in one device buffer; every other relation starts 8
    bytes past a 16-byte boundary.  Returns (buffer, [(dR, nR, dS, nS)])."""
    rels = [r for pair in joins for r in pair]
    offs, off = [], 0
    for i, r in enumerate(rels):
        if misalign and (off % 2) != (i % 2):
            off += 1
        offs.append(off)
        off += len(r) + 1
    host = np.zeros(off + 2, dtype=np.int64)
    for r, o in zip(rels, offs):
        host[o:o + len(r)] = r.view(np.int64)
    t = torch.from_numpy(host).cuda()
    base = t.data_ptr()
    out = []
    for j in range(len(joins)):
        (R, S), oR, oS = joins[j], offs[2 * j], offs[2 * j + 1]
        out.append((base + 8 * oR, len(R), base + 8 * oS, len(S)))
    return t, out


def oracle_counts(O, joins):
    return [O.rho(R, S) if len(R) and len(S) else 0 for R, S in joins]


def run_batch(tbg, torch, b, n, stream=0):
    counts = torch.full((max(n, 1),), -1, dtype=torch.int64, device="cuda")
    st = torch.cuda.current_stream().cuda_stream
    b.run(counts.data_ptr(), st)
    torch.cuda.current_stream().synchronize()
    b.sync()
    return [int(x) for x in counts[:n].cpu().numpy()]


@pytest.mark.gpu
@pytest.mark.parametrize("mode", [dict(radix_bits=-1), dict(radix_bits=0), dict(radix_bits=3),
                                  dict(radix_bits=8), dict(radix_bits=-1, algo="RHT")])
def test_batch_mixed_counts(tbg, oracle, cuda, mode):
    torch = cuda
    joins = mixed_joins()
    want = oracle_counts(oracle, joins)
    buf, dj = upload(torch, joins)
    algo = mode.pop("algo", "RHO")
    cfg = tbg.config(algo, **mode)
    b = tbg.Batch(dj, cfg, torch.cuda.current_stream().cuda_stream)
    try:
        got1 = run_batch(tbg, torch, b, len(dj))
        got2 = run_batch(tbg, torch, b, len(dj))  # graph replay resets its counters
    finally:
        b.close()
    assert got1 == want
    assert got2 == want


@pytest.mark.gpu
def test_batch_describe_and_launches(tbg, cuda):
    torch = cuda
    joins = mixed_joins(seed=3)
    buf, dj = upload(torch, joins)
    b = tbg.Batch(dj, tbg.config("RHO", radix_bits=0))
    d = b.describe()
    assert d["grid"] >= 148 and d["tickets"] > 0
    classes = {c["log2_R"]: c for c in d["classes"]}
    assert all(c["tuned"] == 1 for c in classes.values())
    assert classes[18]["bits"] >= 1  # 300000 rows never fit one shared-memory table
    l0 = tbg.kernel_launches()
    run_batch(tbg, torch, b, len(dj))
    assert tbg.kernel_launches() - l0 == 1  # the whole batch is one kernel launch
    b.close()


@pytest.mark.gpu
def test_batch_new_contents_same_plan(tbg, oracle, cuda):
    """The plan depends on sizes and addresses only: new contents written
    into the same buffers give the new counts on the next run."""
    torch = cuda
    a = mixed_joins(seed=11)
    bb = mixed_joins(seed=12)
    buf, dj = upload(torch, a)
    b = tbg.Batch(dj, tbg.config("RHO", radix_bits=-1))
    assert run_batch(tbg, torch, b, len(dj)) == oracle_counts(oracle, a)
    buf2, _ = upload(torch, bb)
    buf.copy_(buf2)
    assert run_batch(tbg, torch, b, len(dj)) == oracle_counts(oracle, bb)
    b.close()


@pytest.mark.gpu
def test_batch_arg_errors(tbg, cuda):
    torch = cuda
    t = torch.zeros(16, dtype=torch.int64, device="cuda")
    p = t.data_ptr()
    with pytest.raises(tbg.TbgError) as e:
        tbg.Batch([(p + 4, 1, p, 1)])
    assert e.value.code == tbg.ERR_ARG
    with pytest.raises(tbg.TbgError):
        tbg.Batch([(0, 5, p, 1)])
    with pytest.raises(tbg.TbgError):
        tbg.Batch([(p, 1, p, 1)], tbg.config("RSM"))
    with pytest.raises(tbg.TbgError):
        tbg.Batch([(p, 1, p, 1)], tbg.config("RHO", radix_bits=9))
    b = tbg.Batch([])  # an empty batch is valid
    b.run()
    b.sync()
    b.close()


def _c4_check(tbg, oracle, torch, njoins, lo, hi, seed, oracle_joins):
    import bench
    st = torch.cuda.current_stream().cuda_stream
    buf, dj, zipf = bench.make_batch_device(torch, tbg, njoins, lo, hi, 0.2, seed=seed, stream=st)
    b = tbg.Batch(dj, tbg.config("RHO", radix_bits=0), st)
    try:
        got = run_batch(tbg, torch, b, njoins)
        again = run_batch(tbg, torch, b, njoins)
    finally:
        b.close()
    # R_i unique keys 1..|R_i|, every S_i key in that range: count = |S_i|
    assert got == [j[3] for j in dj]
    assert again == got
    # the oracle on a few joins, read back from the device
    idx = sorted(set([0, njoins - 1] + list(np.nonzero(zipf)[0][:2]) + list(range(1, njoins, njoins // 4))))[
        :oracle_joins]
    from gpu_util import dev_to_host_rows
    flat = buf
    base = flat.data_ptr()
    for i in idx:
        pR, nR, pS, nS = dj[i]
        R = dev_to_host_rows(flat[(pR - base) // 8:], nR)
        S = dev_to_host_rows(flat[(pS - base) // 8:], nS)
        assert oracle.rho(R, S) == got[i]
    return zipf


@pytest.mark.gpu
def test_batch_c4_recipe_scaled(tbg, oracle, cuda):
    """The 4096-join recipe (log-uniform |R_i|, k in 1..16, 20% Zipf) at
    512 joins of 2^8..2^16 rows."""
    zipf = _c4_check(tbg, oracle, cuda, 512, 8, 16, seed=5, oracle_joins=8)
    assert zipf.any() and not zipf.all()


@pytest.mark.gpu
def test_batch_c4_full(tbg, oracle, cuda):
    """4096 joins, |R_i| log-uniform in [2^10, 2^20], |S_i| = k |R_i|
    (about 5.9e9 rows, 47 GB), autotuned, one graph."""
    torch = cuda
    torch.cuda.empty_cache()
    free, _ = torch.cuda.mem_get_info()
    if free < 120 * (1 << 30):
        pytest.skip("needs ~100 GB of free device memory")
    _c4_check(tbg, oracle, torch, 4096, 10, 20, seed=4, oracle_joins=3)
