"""tbg_shard_split, the exchange step of a join split over several GPUs:
the grouping by shard is exact (every row once, in its key's shard), and
joining shard d of R with shard d of S for every d sums to the unsharded
join's count (the oracle's).  One GPU holds every shard here; the ranks'
all-to-all only moves the groups, which the multi-rank CPU test covers."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import gen_relation
from gpu_util import dev_relation, dev_to_host_rows, to_dev

pytestmark = pytest.mark.gpu


def _split(tbg, cuda, rows, nshards, offset=0):
    t, p = to_dev(cuda, rows, offset)
    out, po = dev_relation(cuda, len(rows))
    offs = tbg.shard_split(p, len(rows), nshards, po)
    cuda.cuda.synchronize()
    return dev_to_host_rows(out, len(rows)), offs


@pytest.mark.parametrize("nshards", [1, 2, 3, 8, 256])
def test_shard_split_groups_every_row_once(tbg, oracle, cuda, nshards):
    S = gen_relation(oracle, ("zipf", 300001, 50000, 1.1), 77, 1)
    got, offs = _split(tbg, cuda, S, nshards, offset=1)  # 8 bytes past a 16-byte boundary
    assert offs[0] == 0 and offs[-1] == len(S) and all(a <= b for a, b in zip(offs, offs[1:]))
    for d in range(nshards):
        part = got[offs[d]:offs[d + 1]]
        assert np.all(tbg.shard_of(part["key"], nshards) == d)
    assert np.array_equal(np.sort(got.view(np.uint64)), np.sort(S.view(np.uint64)))
    want = np.bincount(tbg.shard_of(S["key"], nshards), minlength=nshards)
    assert np.array_equal(np.diff(offs), want)


def test_shard_split_edge_sizes(tbg, oracle, cuda):
    assert tbg.shard_split(0, 0, 4, 0) == [0] * 5
    R = gen_relation(oracle, ("pk", 1, 0, 0.0), 3, 0)
    got, offs = _split(tbg, cuda, R, 4)
    assert offs[-1] == 1 and got[0] == R[0]
    with pytest.raises(tbg.TbgError):
        tbg.shard_split(0, 0, 257, 0)


@pytest.mark.parametrize("nshards", [2, 4, 8])
def test_per_shard_joins_sum_to_the_join(tbg, oracle, cuda, nshards):
    R = gen_relation(oracle, ("pk", 1 << 18, 0, 0.0), 5, 0)
    R["key"][:100] = R["key"][100]  # duplicate R keys
    S = gen_relation(oracle, ("zipf", 1 << 21, 1 << 18, 1.0), 6, 1)
    want = oracle.rho(R, S)
    Rg, ro = _split(tbg, cuda, R, nshards)
    Sg, so = _split(tbg, cuda, S, nshards)
    total = 0
    for d in range(nshards):
        tR, pR = to_dev(cuda, Rg[ro[d]:ro[d + 1]])
        tS, pS = to_dev(cuda, Sg[so[d]:so[d + 1]])
        _, m, _ = tbg.join_device(tbg.config("RHO"), pR, ro[d + 1] - ro[d], pS, so[d + 1] - so[d])
        total += m
    assert total == want
    # even shares of skewed keys: no shard holds more than twice its share of S
    assert max(np.diff(so)) < 2 * len(S) / nshards
