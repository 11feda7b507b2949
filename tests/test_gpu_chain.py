"""Chained joins on device-resident output (the reference's three-way chain,
Enclave/TrustedJoins/secure_joins.cpp:348-399): R x S materialised,
to_relation of its rows as (key, R payload) tuples, then T x that relation.
Checked against the oracle's RHO run twice on the host."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import gen_relation
from gpu_util import dev_to_host_rows, out_rows, rows_to_host, run_join, to_dev

pytestmark = pytest.mark.gpu


def _oracle_chain(oracle, R, S, T):
    c1, rows1 = oracle.rho(R, S, materialize=True)
    rel = np.zeros(c1, dtype=oracle.ROW)
    rel["key"] = rows1[:, 0]
    rel["payload"] = rows1[:, 1]
    c2, rows2 = oracle.rho(T, rel, materialize=True) if c1 and len(T) else (0, np.zeros((0, 3), np.uint32))
    return c1, rel, c2, rows2


def test_rows_to_relation(tbg, oracle, cuda):
    torch = cuda
    R = gen_relation(oracle, ("pk", 5000, 0, 0.0), 3, 0)
    S = gen_relation(oracle, ("fk", 20000, 5000, 0.0), 4, 1)
    c1, rel, _, _ = _oracle_chain(oracle, R, S, R[:0])
    m, rows, _ = run_join(tbg, torch, "RHO", R, S, materialize=True)
    assert m == c1
    # the GPU's rows back on the device, converted there
    flat = torch.from_numpy(np.ascontiguousarray(rows).reshape(-1).view(np.int32)).cuda()
    out = torch.zeros(max(m, 1), dtype=torch.int64, device="cuda")
    tbg.rows_to_relation(flat.data_ptr(), m, out.data_ptr())
    torch.cuda.synchronize()
    got = dev_to_host_rows(out, m)
    assert np.array_equal(got["key"], rows[:, 0]) and np.array_equal(got["payload"], rows[:, 1])


@pytest.mark.parametrize("kind", ["fk", "dup"])
def test_three_way_chain_matches_oracle(tbg, oracle, cuda, kind):
    torch = cuda
    rng = np.random.default_rng(7)
    R = gen_relation(oracle, ("pk", 1 << 16, 0, 0.0), 21, 0)
    S = gen_relation(oracle, ("fk", 1 << 18, 1 << 16, 0.0), 22, 1)
    if kind == "fk":
        T = gen_relation(oracle, ("pk", 1 << 16, 0, 0.0), 23, 0)
    else:  # T with duplicate keys: the second join multiplies rows
        T = np.zeros(50000, dtype=oracle.ROW)
        T["key"] = rng.integers(1, 30000, len(T))
        oracle.fill_payloads(T, 0)
    c1, _, c2, rows2 = _oracle_chain(oracle, R, S, T)
    tR, pR = to_dev(torch, R, 1)
    tS, pS = to_dev(torch, S)
    tT, pT = to_dev(torch, T)
    cap = c2 + 16
    tO, pO = out_rows(torch, cap)
    for algo in ("RHO", "LRN", "RSM"):
        m1, m2 = tbg.join_three_way(tbg.config(algo), pR, len(R), pS, len(S), pT, len(T), pO, cap,
                                    torch.cuda.current_stream().cuda_stream)
        torch.cuda.synchronize()
        assert (m1, m2) == (c1, c2), algo
        got = rows_to_host(tO, m2)
        assert np.array_equal(oracle.sort_rows(got), oracle.sort_rows(rows2)), algo
    # count only
    m1, m2 = tbg.join_three_way(tbg.config("RHO"), pR, len(R), pS, len(S), pT, len(T))
    assert (m1, m2) == (c1, c2)
