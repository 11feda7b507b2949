"""tbg_join_count_static, the join count that allocates no device memory:
checked against the existing device entry point (tbg_join_device, RHO) and
against the equi-join count computed on the host (numpy) on the same
relations, over consecutive calls that share its static scratch.
The file name makes pytest collect it last; it also passes alone in a fresh
process."""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from gpu_util import to_dev

ROW = np.dtype([("key", "<u4"), ("payload", "<u4")])
MAX_ROWS = 1 << 22  # TBG_STATIC_MAX_ROWS


def _static(tbg):
    f = tbg.lib().tbg_join_count_static
    f.argtypes = [C.c_void_p, C.c_uint64, C.c_void_p, C.c_uint64, C.c_void_p, C.c_void_p, C.c_void_p]
    f.restype = C.c_int
    return f


def _rel(keys, rs):
    r = np.zeros(len(keys), dtype=ROW)
    r["key"] = keys
    r["payload"] = rs.randint(0, 2 ** 32, len(keys), dtype=np.uint64).astype(np.uint32)
    return r


def host_count(R, S):
    """Equi-join cardinality: for every S row, the R rows with its key."""
    keys, mult = np.unique(R["key"], return_counts=True)
    if len(keys) == 0:
        return 0
    pos = np.minimum(np.searchsorted(keys, S["key"]), len(keys) - 1)
    hit = keys[pos] == S["key"]
    return int(mult[pos][hit].sum())


def _cases():
    rs = np.random.RandomState(2024)
    out = []
    # radix path (|R| > 8192): duplicate R keys, S with misses
    out.append((_rel(rs.randint(1, 150000, 200000), rs), _rel(rs.randint(1, 200000, 900000), rs)))
    # direct path (|R| <= 8192)
    out.append((_rel(rs.randint(1, 4000, 6000), rs), _rel(rs.randint(1, 5000, 300000), rs)))
    # radix path again, different sizes: the previous call's scratch must not leak in
    out.append((_rel(rs.permutation(70000) + 1, rs), _rel(rs.randint(1, 90000, 500000), rs)))
    # the largest accepted input
    nR = 1 << 20
    out.append((_rel(rs.permutation(nR) + 1, rs), _rel(rs.randint(1, nR + 5000, MAX_ROWS - nR), rs)))
    # 2^21 / 2^21: 256 radix partitions of about 8192 R rows, about half of
    # them larger than one shared-memory table, so R is built in slices and
    # S probed once per slice
    n = 1 << 21
    out.append((_rel(rs.permutation(n) + 1, rs), _rel(rs.randint(1, n + 1, n), rs)))
    # skewed R: one key repeated 12000 times (its partition alone exceeds a
    # table) and S hitting it often
    kR = rs.randint(1, 300000, 400000)
    kR[:12000] = 4242
    kS = rs.randint(1, 320000, 600000)
    kS[:64] = 4242
    out.append((_rel(kR, rs), _rel(kS, rs)))
    return out


@pytest.mark.gpu
def test_static_join_matches_device_join(tbg, cuda):
    torch = cuda
    f = _static(tbg)
    st = torch.cuda.current_stream().cuda_stream
    cnt = torch.empty(1, dtype=torch.int64, device="cuda")
    status = torch.empty(1, dtype=torch.int32, device="cuda")
    for R, S in _cases():
        tR, pR = to_dev(torch, R, 1)  # 8 bytes past a 16-byte boundary
        tS, pS = to_dev(torch, S)
        rc, want, _ = tbg.join_device(tbg.config("RHO"), pR, len(R), pS, len(S), stream=st)
        assert rc == tbg.OK
        assert want == host_count(R, S)
        for _ in range(2):  # two calls in a row on the same inputs
            cnt.fill_(-1)
            status.fill_(77)
            assert f(pR, len(R), pS, len(S), cnt.data_ptr(), status.data_ptr(), st) == tbg.OK
            torch.cuda.current_stream().synchronize()
            assert int(cnt.item()) == want
            assert int(status.item()) == 0


@pytest.mark.gpu
def test_static_join_empty_and_oversized(tbg, cuda):
    torch = cuda
    f = _static(tbg)
    st = torch.cuda.current_stream().cuda_stream
    t = torch.zeros(4, dtype=torch.int64, device="cuda")
    cnt = torch.full((1,), -1, dtype=torch.int64, device="cuda")
    assert f(t.data_ptr(), 0, t.data_ptr(), 3, cnt.data_ptr(), None, st) == tbg.OK
    torch.cuda.current_stream().synchronize()
    assert int(cnt.item()) == 0
    # sizes beyond the scratch are refused before anything is launched
    assert f(t.data_ptr(), MAX_ROWS, t.data_ptr(), 1, cnt.data_ptr(), None, st) == tbg.ERR_ARG
    assert b"static scratch limit" in tbg.lib().tbg_last_error_string()
