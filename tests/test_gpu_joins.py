"""GPU parity of the joins (RHO, RHT, RSM, PSM) against the oracle and the
reference's golden vectors, through the C ABI.  Integer work: bit-exact.

Every algorithm must return the exact equi-join (the reference's RHO result).
The reference's own RSM / PSM miscount skewed or sparse inputs (recorded as
*_observed in the golden file); matching RHO instead is deliberate."""
from __future__ import annotations

import hashlib

import numpy as np
import pytest

from conftest import gen_relation
from gpu_util import dev_relation, dev_to_host_rows, run_join

pytestmark = pytest.mark.gpu
ALGOS = ["RHO", "RHT", "RSM", "PSM"]


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


@pytest.mark.parametrize("algo", ALGOS)
@pytest.mark.parametrize("idx", range(8))
def test_golden_cases(tbg, oracle, golden, cuda, algo, idx):
    j = golden["joins"][idx]
    R = gen_relation(oracle, j["R"], j["seedR"], 0)
    S = gen_relation(oracle, j["S"], j["seedS"], 1)
    assert sha(R["key"]) == j["R_keys_sha256"] and sha(S["key"]) == j["S_keys_sha256"]
    m, _, st = run_join(tbg, cuda, algo, R, S)
    assert m == j["RHO_n1"]
    m2, rows, _ = run_join(tbg, cuda, algo, R, S, materialize=True)
    assert m2 == j["RHO_mat_count"] == len(rows)
    assert sha(oracle.sort_rows(rows)) == j["RHO_mat_sorted_sha256"]


@pytest.mark.parametrize("algo", ALGOS)
def test_dropin_matches_reference_default_config(tbg, oracle, golden, cuda, algo):
    """RHO(&R, &S, nthreads) on the reference's default inputs (native.cpp:59-127)."""
    j = golden["joins"][0]
    R = gen_relation(oracle, j["R"], j["seedR"], 0)
    S = gen_relation(oracle, j["S"], j["seedS"], 1)
    assert tbg.find(algo).join(R, S, 2) == 2097152
    c, rows = tbg.find(algo).join(R, S, 3, materialize=True)
    assert c == 2097152 and len(rows) == c
    assert sha(oracle.sort_rows(rows)) == j["RHO_mat_sorted_sha256"]


@pytest.mark.parametrize("algo", ["RHO", "RHT"])
@pytest.mark.parametrize("slices", [1, 3, 16])
def test_dropin_sliced_copies(tbg, oracle, cuda, algo, slices):
    """The drop-in copies S in slices and joins each as it lands: same count
    and row multiset as the oracle, including the materialising retry when
    the output outgrows |S| (duplicate R keys) and a slice count that does
    not divide |S|."""
    rng = np.random.default_rng(slices)
    R = np.zeros(300007, dtype=oracle.ROW)
    S = np.zeros(1000003, dtype=oracle.ROW)
    R["key"] = rng.integers(1, 100000, len(R))  # about 3 rows per key: more matches than |S|
    S["key"] = np.minimum(rng.zipf(1.2, len(S)), 250000)
    oracle.fill_payloads(R, 0)
    oracle.fill_payloads(S, 1)
    ref, ref_rows = oracle.rho(R, S, materialize=True)
    assert ref > len(S)
    prev = tbg.set_dropin_slices(slices)
    try:
        assert tbg.find(algo).join(R, S, 2) == ref
        c, rows = tbg.find(algo).join(R, S, 3, materialize=True)
    finally:
        tbg.set_dropin_slices(prev)
    assert c == ref == len(rows)
    assert np.array_equal(oracle.sort_rows(rows), oracle.sort_rows(ref_rows))
    h2d, _ = tbg.last_transfer_bytes()
    assert h2d == 8 * (len(R) + len(S))


@pytest.mark.parametrize("bits,passes", [(1, 1), (4, 1), (8, 1), (9, 2), (12, 2), (14, 2), (15, 2)])
def test_radix_geometry(tbg, oracle, cuda, bits, passes):
    rng = np.random.default_rng(bits * 10 + passes)
    R = np.zeros(30011, dtype=oracle.ROW)
    S = np.zeros(100003, dtype=oracle.ROW)
    R["key"] = rng.integers(0, 1 << 20, len(R))
    S["key"] = rng.integers(0, 1 << 20, len(S))
    oracle.fill_payloads(R, 0)
    oracle.fill_payloads(S, 1)
    ref, ref_rows = oracle.rho(R, S, materialize=True)
    m, rows, st = run_join(tbg, cuda, "RHO", R, S, materialize=True, radix_bits=bits, passes=passes)
    assert (st.radix_bits, st.passes) == (bits, passes)
    assert m == ref
    assert np.array_equal(oracle.sort_rows(rows), oracle.sort_rows(ref_rows))


def test_partition_sizes_match_oracle(tbg, oracle, cuda):
    R = gen_relation(oracle, ("pk", 1 << 18, 0, 0.0), 1, 0)
    S = gen_relation(oracle, ("zipf", 1 << 20, 1 << 18, 1.0), 2, 1)
    m, _, st = run_join(tbg, cuda, "RHO", R, S, radix_bits=10, passes=2)
    hR = oracle.radix_hist(R, 10, 2)
    hS = oracle.radix_hist(S, 10, 2)
    assert st.max_part_R == hR.max() and st.max_part_S == hS.max()
    assert m == oracle.rho(R, S)


@pytest.mark.parametrize("case", ["emptyR", "emptyS", "one", "dupes", "allsame", "highbits",
                                  "misaligned", "nomatch"])
def test_edge_cases(tbg, oracle, cuda, case):
    rng = np.random.default_rng(5)
    nR, nS = 1000, 5000
    R = np.zeros(nR, dtype=oracle.ROW)
    S = np.zeros(nS, dtype=oracle.ROW)
    R["key"] = rng.permutation(nR) + 1
    S["key"] = rng.integers(1, nR + 1, nS)
    off = 0
    if case == "emptyR":
        R = R[:0]
    elif case == "emptyS":
        S = S[:0]
    elif case == "one":
        R, S = R[:1].copy(), R[:1].copy()
    elif case == "dupes":
        R["key"] = rng.integers(1, 50, nR)
    elif case == "allsame":
        R = R[:40].copy()
        R["key"] = 7
        S["key"] = 7
    elif case == "highbits":
        R["key"] = (rng.permutation(nR).astype(np.uint64) * 4294967 + 0xFFFF0000) & 0xFFFFFFFF
        S["key"] = R["key"][rng.integers(0, nR, nS)]
        R["key"][0] = 0xFFFFFFFF
        R["key"][1] = 0
    elif case == "misaligned":
        off = 1
    elif case == "nomatch":
        S["key"] += 1 << 20
    oracle.fill_payloads(R, 0)
    oracle.fill_payloads(S, 1)
    ref, ref_rows = oracle.rho(R, S, materialize=True) if len(R) and len(S) else (0, np.zeros((0, 3), np.uint32))
    for algo in ALGOS:
        m, rows, _ = run_join(tbg, cuda, algo, R, S, materialize=True, offset=off, cap=max(ref, 1))
        assert m == ref
        assert np.array_equal(oracle.sort_rows(rows), oracle.sort_rows(ref_rows))


def test_capacity_overflow_reports_exact_count(tbg, oracle, cuda):
    R = gen_relation(oracle, ("pk", 5000, 0, 0.0), 1, 0)
    S = gen_relation(oracle, ("fk", 20000, 5000, 0.0), 2, 1)
    with pytest.raises(tbg.TbgError) as e:
        run_join(tbg, cuda, "RHO", R, S, materialize=True, cap=1000)
    assert e.value.code == tbg.ERR_CAPACITY
    from gpu_util import to_dev, out_rows
    tR, pR = to_dev(cuda, R)
    tS, pS = to_dev(cuda, S)
    tO, pO = out_rows(cuda, 1000)
    rc, m, _ = tbg.join_device(tbg.config("RHO", materialize=1), pR, len(R), pS, len(S), pO, 1000,
                               check=False)
    assert rc == tbg.ERR_CAPACITY and m == 20000


def test_async_api_and_launch_count(tbg, oracle, cuda):
    R = gen_relation(oracle, ("pk", 1 << 16, 0, 0.0), 1, 0)
    S = gen_relation(oracle, ("fk", 1 << 18, 1 << 16, 0.0), 2, 1)
    from gpu_util import to_dev
    tR, pR = to_dev(cuda, R)
    tS, pS = to_dev(cuda, S)
    out = cuda.zeros(4, dtype=cuda.int64, device="cuda")
    n0 = tbg.kernel_launches()
    s = cuda.cuda.current_stream().cuda_stream
    for k in range(3):
        tbg.join_device_async(tbg.config("RHO"), pR, len(R), pS, len(S), out.data_ptr() + 8 * k, stream=s)
    assert tbg.lib().tbg_sync_status(s) == 0
    assert out[:3].tolist() == [1 << 18] * 3
    assert tbg.kernel_launches() - n0 >= 3 * 4


@pytest.mark.parametrize("algo,sel", [("RHO", 100), ("RHO", 50), ("RSM", 100), ("PSM", 50)])
def test_full_size_headline_config(tbg, cuda, algo, sel):
    """|R| = 2^27, |S| = 2^30 from the GPU generators: a permutation of
    1..|R| against |S|/maxid permuted copies of 1..maxid (maxid = |R| at 100%
    selectivity, 2|R| at 50%).  Known answer: |S| * |R| / maxid matches."""
    nR, nS = 1 << 27, 1 << 30
    maxid = nR * 100 // sel
    tR, pR = dev_relation(cuda, nR)
    tS, pS = dev_relation(cuda, nS)
    tbg.gen_pk(pR, nR, 11111)
    tbg.gen_fk(pS, nS, maxid, 22222)
    cuda.cuda.synchronize()
    rc, m, st = tbg.join_device(tbg.config(algo), pR, nR, pS, nS)
    assert m == nS * nR // maxid
    # the generators' contract: R is a permutation of 1..|R|
    keys = tR.view(cuda.int32)[0::2]
    assert int(keys.min()) == 1 and int(keys.max()) == nR
    assert int(cuda.bincount(keys.long(), minlength=nR + 1)[1:].max()) == 1


def test_generators_contract(tbg, cuda):
    n, maxid = 3_000_001, 1_000_000
    t, p = dev_relation(cuda, n)
    tbg.gen_fk(p, n, maxid, 9)
    keys = t[:n].view(cuda.int32)[0::2].long().cpu().numpy()
    for c in range(3):
        blk = keys[c * maxid:(c + 1) * maxid]
        assert np.array_equal(np.sort(blk), np.arange(1, maxid + 1))
    assert np.array_equal(np.sort(keys[3 * maxid:]), np.arange(1, 2))
    tz, pz = dev_relation(cuda, 1 << 22)
    tbg.gen_zipf(pz, 1 << 22, 1 << 16, 1.0, 0, 5)
    kz = tz.view(cuda.int32)[0::2].long().cpu().numpy()
    assert kz.min() >= 1 and kz.max() <= 1 << 16
    freq = np.bincount(kz, minlength=(1 << 16) + 1)[1:] / len(kz)
    H = np.sum(1.0 / np.arange(1, (1 << 16) + 1))
    expect = 1.0 / (np.arange(1, 9) * H)
    assert np.allclose(freq[:8], expect, rtol=0.02)


@pytest.mark.parametrize("algo", ["RHO", "RHT"])
@pytest.mark.parametrize("bits", [3, 4])
def test_join_table_size_gate(tbg, oracle, cuda, algo, bits):
    """Counting joins launch a 4096-row and a 5120-row table kernel, each
    gated on the largest R partition: 3 radix bits over 36000 keys give
    partitions of about 4500 rows (the 5120-row kernel runs), 4 bits about
    2250 (the 4096-row kernel runs).  Both running would double the count."""
    rng = np.random.default_rng(bits)
    R = np.zeros(36000, dtype=oracle.ROW)
    S = np.zeros(300007, dtype=oracle.ROW)
    R["key"] = rng.integers(0, 1 << 30, len(R), dtype=np.uint64).astype(np.uint32)
    S["key"] = np.where(rng.random(len(S)) < 0.8, R["key"][rng.integers(0, len(R), len(S))],
                        rng.integers(0, 1 << 30, len(S), dtype=np.uint64).astype(np.uint32))
    oracle.fill_payloads(R, 0)
    oracle.fill_payloads(S, 1)
    ref = oracle.rho(R, S)
    m, _, st = run_join(tbg, cuda, algo, R, S, radix_bits=bits)
    assert m == ref
    assert (st.max_part_R > 4096) == (bits == 3)


PSM_PLANS = [(12, 0), (20, 0), (21, 0), (27, 0), (28, 0), (32, 0), (27, 1), (20, 3_000_000_000)]


def psm_passes(bits):
    """Passes PSM reports for a key range of `bits` bits above its minimum:
    MSD (radix passes over the top B <= 15 bits, then one bucket-sort pass
    over the low 12, at most 13, bits) when the range has bits above the low
    ones; otherwise the LSD sort's passes of at most 9 bits."""
    low = min(bits, 12)
    B = bits - low
    if B > 15:
        B, low = 15, bits - 15
    if B < 1 or low > 13:
        return (bits + 8) // 9
    return (1 if B <= 8 else 2) + 1


@pytest.mark.parametrize("span,low", PSM_PLANS, ids=[f"span{s}-low{lo}" for s, lo in PSM_PLANS])
def test_psm_digit_plans(tbg, oracle, cuda, span, low):
    """PSM's sort covers the bits of key - min that vary.  Ranges of 13 to 28
    bits take the MSD sort (one or two radix passes over the top bits, one
    bucket sort over the low 12 or 13); a 12-bit range (no bits above the low
    ones) and a 32-bit one (too many low bits) take the LSD sort (9-bit digits
    when they save a pass, 7-bit at an equal count).  Keys 1..2^27 (low = 1)
    span 28 bits raw but 27 above their minimum; a range high in the key space
    takes the passes its width needs.  Every plan must give the oracle's count
    and rows."""
    rng = np.random.default_rng(span)
    width = 1 << span
    R = np.zeros(150001, dtype=oracle.ROW)
    S = np.zeros(400003, dtype=oracle.ROW)
    R["key"] = (low + rng.integers(0, width, len(R), dtype=np.uint64)).astype(np.uint32)
    R["key"][0] = low + width - 1  # the range's top key
    R["key"][1] = low              # and its bottom one
    pick = R["key"][rng.integers(0, len(R), len(S))]
    other = (low + rng.integers(0, width, len(S), dtype=np.uint64)).astype(np.uint32)
    S["key"] = np.where(rng.random(len(S)) < 0.7, pick, other)
    oracle.fill_payloads(R, 0)
    oracle.fill_payloads(S, 1)
    ref, ref_rows = oracle.rho(R, S, materialize=True)
    m, _, st = run_join(tbg, cuda, "PSM", R, S)
    assert m == ref
    bits = int(width - 1).bit_length()
    assert st.passes == psm_passes(bits), (bits, st.passes)
    m, rows, _ = run_join(tbg, cuda, "PSM", R, S, materialize=True, cap=ref)
    assert m == ref
    assert np.array_equal(oracle.sort_rows(rows), oracle.sort_rows(ref_rows))


@pytest.mark.parametrize("materialize", [False, True])
def test_psm_heavy_key_takes_lsd(tbg, oracle, cuda, materialize):
    """A Zipf S whose hottest key fills one MSD bucket past a million rows is
    sorted by the LSD passes, while R keeps the MSD sort; count and rows match
    the oracle either way."""
    import torch

    nR, nS = 1 << 18, 1 << 22
    st = torch.cuda.current_stream().cuda_stream
    tR = torch.empty(nR, dtype=torch.int64, device="cuda")
    tS = torch.empty(nS, dtype=torch.int64, device="cuda")
    tbg.gen_pk(tR.data_ptr(), nR, 3, st)
    tbg.gen_zipf(tS.data_ptr(), nS, nR, 1.5, 0, 4, st)
    R = tR.cpu().numpy().view(oracle.ROW)
    S = tS.cpu().numpy().view(oracle.ROW)
    assert np.bincount(S["key"]).max() > 1 << 20
    if materialize:
        ref, ref_rows = oracle.rho(R, S, materialize=True)
        m, rows, _ = run_join(tbg, cuda, "PSM", R, S, materialize=True, cap=ref)
        assert m == ref
        assert np.array_equal(oracle.sort_rows(rows), oracle.sort_rows(ref_rows))
    else:
        ref = oracle.rho(R, S)
        m, _, _ = run_join(tbg, cuda, "PSM", R, S)
        assert m == ref == nS


@pytest.mark.parametrize("materialize", [False, True])
def test_psm_bucket_past_group_stage(tbg, oracle, cuda, materialize):
    """MSD buckets averaging 4K rows are sorted four per CTA, each group with a
    5K-row stage; a key repeated tens of thousands of times in R (and another
    in S) makes one bucket of each relation outgrow its group's stage, so most
    of its rows go straight to their sorted place.  Count and rows match the
    oracle."""
    rng = np.random.default_rng(43)
    n = 1 << 22
    R = np.zeros(n, dtype=oracle.ROW)
    S = np.zeros(n, dtype=oracle.ROW)
    R["key"] = rng.permutation(np.arange(1, n + 1, dtype=np.uint32))
    S["key"] = rng.integers(1, n + 1, n).astype(np.uint32)
    R["key"][:30000] = 777
    S["key"][:40000] = 888
    oracle.fill_payloads(R, 0)
    oracle.fill_payloads(S, 1)
    if materialize:
        ref, ref_rows = oracle.rho(R, S, materialize=True)
        m, rows, _ = run_join(tbg, cuda, "PSM", R, S, materialize=True, cap=ref)
        assert m == ref
        assert np.array_equal(oracle.sort_rows(rows), oracle.sort_rows(ref_rows))
    else:
        ref = oracle.rho(R, S)
        m, _, _ = run_join(tbg, cuda, "PSM", R, S)
        assert m == ref


@pytest.mark.parametrize("materialize", [False, True])
def test_psm_s_keys_outside_r_range(tbg, oracle, cuda, materialize):
    """PSM first bins both relations by R's key range; S keys below and above
    it send the sort back to both relations' range.  Count and rows match
    the oracle."""
    rng = np.random.default_rng(7)
    R = np.zeros(200003, dtype=oracle.ROW)
    S = np.zeros(500009, dtype=oracle.ROW)
    R["key"] = rng.integers(1 << 20, 1 << 22, len(R)).astype(np.uint32)
    inside = R["key"][rng.integers(0, len(R), len(S))]
    anywhere = rng.integers(0, 1 << 24, len(S)).astype(np.uint32)
    S["key"] = np.where(rng.random(len(S)) < 0.8, inside, anywhere)
    assert S["key"].min() < R["key"].min() and S["key"].max() > R["key"].max()
    oracle.fill_payloads(R, 0)
    oracle.fill_payloads(S, 1)
    ref, ref_rows = oracle.rho(R, S, materialize=True)
    if materialize:
        m, rows, _ = run_join(tbg, cuda, "PSM", R, S, materialize=True, cap=ref)
        assert m == ref
        assert np.array_equal(oracle.sort_rows(rows), oracle.sort_rows(ref_rows))
    else:
        m, _, _ = run_join(tbg, cuda, "PSM", R, S)
        assert m == ref


@pytest.mark.parametrize("materialize", [False, True])
def test_rsm_wide_key_spans(tbg, oracle, cuda, materialize):
    """Full-range 32-bit keys: inside a radix partition the varying key bits
    span more than the 12 a single counting pass sorts, so every tile takes
    the stable multi-pass sort (count-only on bare keys, materialising on
    packed rows).  Both sides hold duplicate keys."""
    rng = np.random.default_rng(29)
    R = np.zeros(200003, dtype=oracle.ROW)
    S = np.zeros(700001, dtype=oracle.ROW)
    R["key"] = rng.integers(0, 1 << 32, len(R), dtype=np.uint64).astype(np.uint32)
    R["key"][:5000] = R["key"][5000:10000]  # duplicates in R
    pick = R["key"][rng.integers(0, len(R), len(S))]
    S["key"] = np.where(rng.random(len(S)) < 0.6, pick,
                        rng.integers(0, 1 << 32, len(S), dtype=np.uint64).astype(np.uint32))
    oracle.fill_payloads(R, 0)
    oracle.fill_payloads(S, 1)
    ref, ref_rows = oracle.rho(R, S, materialize=True)
    m, rows, _ = run_join(tbg, cuda, "RSM", R, S, materialize=materialize, cap=ref)
    assert m == ref
    if materialize:
        assert np.array_equal(oracle.sort_rows(rows), oracle.sort_rows(ref_rows))


@pytest.mark.parametrize("case", ["fk_half_outside", "zipf_s", "dup_r"])
def test_rsm_ranged_counting_sort(tbg, oracle, cuda, case):
    """Count-only RSM's ranged counting sort: R's keys in a partition span at
    most 4096 digits above the radix bits, so S is sorted in tiles of 16384
    rows ranked against R's key range.  Partitions hold about 32K S rows (two
    tiles and a ragged one); S keys outside R's range (below and above it)
    drop out of the sorted tiles; a Zipf S puts runs of one key in a warp;
    duplicate R keys make runs on both sides."""
    rng = np.random.default_rng(41)
    nR, nS = 1 << 20, (1 << 23) + 4099
    R = np.zeros(nR, dtype=oracle.ROW)
    S = np.zeros(nS, dtype=oracle.ROW)
    R["key"] = rng.permutation(np.arange(1, nR + 1, dtype=np.uint32)) + 1000
    if case == "dup_r":
        R["key"][: nR // 4] = R["key"][nR // 4: nR // 2]
    if case == "zipf_s":
        S["key"] = np.minimum(rng.zipf(1.3, nS), nR).astype(np.uint32) + 1000
    else:
        S["key"] = rng.integers(0, 2 * nR, nS).astype(np.uint32)
    oracle.fill_payloads(R, 0)
    oracle.fill_payloads(S, 1)
    ref = oracle.rho(R, S)
    m, _, _ = run_join(tbg, cuda, "RSM", R, S)
    assert m == ref


@pytest.mark.parametrize("materialize", [False, True])
@pytest.mark.parametrize("algo", ["RSM", "PSM"])
def test_sortmerge_duplicates_both_sides(tbg, oracle, cuda, algo, materialize):
    """Runs of equal keys on both sides, spanning merge tiles and partitions:
    count-only, the runs of equal R keys a merge thread starts inside begin
    in earlier tiles (found by walking back into global memory)."""
    rng = np.random.default_rng(17)
    R = np.zeros(20000, dtype=oracle.ROW)
    S = np.zeros(70000, dtype=oracle.ROW)
    R["key"] = rng.integers(0, 300, len(R))
    S["key"] = rng.integers(0, 330, len(S))
    oracle.fill_payloads(R, 0)
    oracle.fill_payloads(S, 1)
    ref, ref_rows = oracle.rho(R, S, materialize=True)
    m, rows, _ = run_join(tbg, cuda, algo, R, S, materialize=materialize, cap=ref)
    assert m == ref
    if materialize:
        assert np.array_equal(oracle.sort_rows(rows), oracle.sort_rows(ref_rows))
