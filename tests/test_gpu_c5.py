"""The large skewed materialising join: |R| = 2^28 unique keys, |S| = 2^31
Zipf z = 1.0 foreign keys, every match written as a (key, R payload,
S payload) row (2^31 rows, 25.8 GB).  The reference cannot materialise this
(one malloc'd node per row, int32 offsets); the oracle's direct-addressing
join on the same arrays, copied to the host, gives the row count and the
order-free row checksum that the learned (LRN) and radix (RHO) joins must
both reproduce."""
from __future__ import annotations

import numpy as np
import pytest

ROW = np.dtype([("key", "<u4"), ("payload", "<u4")])


@pytest.mark.gpu
def test_c5_materialised_learned_and_radix(tbg, oracle, cuda):
    torch = cuda
    torch.cuda.empty_cache()
    free, _ = torch.cuda.mem_get_info()
    if free < 110 * (1 << 30):
        pytest.skip("needs ~100 GB of free device memory")
    nR, nS = 1 << 28, 1 << 31
    st = torch.cuda.current_stream().cuda_stream
    tR = torch.empty(nR, dtype=torch.int64, device="cuda")
    tS = torch.empty(nS, dtype=torch.int64, device="cuda")
    tbg.gen_pk(tR.data_ptr(), nR, 11111, st)
    tbg.gen_zipf(tS.data_ptr(), nS, nR, 1.0, 0, 22222, st)
    out = torch.empty(3 * nS, dtype=torch.int32, device="cuda")
    got = {}
    for algo in ("LRN", "RHO"):
        cfg = tbg.config(algo, materialize=1)
        rc, m, stats = tbg.join_device(cfg, tR.data_ptr(), nR, tS.data_ptr(), nS, out.data_ptr(), nS, stream=st)
        assert rc == tbg.OK
        got[algo] = (m, tbg.rows_checksum(out.data_ptr(), m, st), stats.used_fallback, stats.heavy_rows_S)
    del out
    torch.cuda.empty_cache()
    R = tR.cpu().numpy().view(ROW)
    S = tS.cpu().numpy().view(ROW)
    want_count, want_sum = oracle.join_direct(R, S)
    assert want_count == nS
    for algo, (m, chk, fallback, heavy) in got.items():
        assert m == want_count, algo
        assert chk == want_sum, algo
    # the learned join routed the hot keys around partitioning
    assert got["LRN"][2] == 0 and got["LRN"][3] > nS // 4
