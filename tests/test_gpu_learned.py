"""LRN, the learned skew-aware join: the GPU model kernels against the float64
oracle, exactness against the reference's RHO result, the fallback, and what
the trained network gains over the same method without it."""
from __future__ import annotations

import hashlib

import numpy as np
import pytest

from conftest import gen_relation
from gpu_util import dev_relation, run_join

pytestmark = pytest.mark.gpu


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def zipf_cdf_points(n=4096, N=1 << 20, z=1.0, seed=0):
    """Training points shaped like LRN's: log-key feature -> empirical CDF."""
    rng = np.random.default_rng(seed)
    w = 1.0 / np.arange(1, N + 1) ** z
    cdf = np.cumsum(w) / w.sum()
    keys = np.sort(np.searchsorted(cdf, rng.random(n)) + 1)
    x = (np.log2(keys + 1.0) / 16.0 - 1.0).astype(np.float32)
    y = ((np.arange(n) + 0.5) / n).astype(np.float32)
    return x, y


def test_gpu_gradient_matches_oracle(tbg, oracle, cuda):
    H = 32
    x, y = zipf_cdf_points(1000, seed=1)
    for seed in (1, 2, 3):
        p = tbg.mlp_init(seed)
        loss, g = tbg.mlp_grad(p, x, y)
        loss_ref, g_ref = oracle.mlp_loss_grad(H, p, x, y)
        assert abs(loss - loss_ref) <= 1e-4 * max(1.0, abs(loss_ref))
        # float32 forward/backward and float32 accumulation against float64
        err = np.abs(g.astype(np.float64) - g_ref)
        assert np.all(err <= 2e-3 * np.abs(g_ref) + 2e-5), (err.max(), np.abs(g_ref).max())


def test_gpu_forward_matches_oracle(tbg, oracle, cuda):
    # the gradient kernel's loss with y = 0 is the mean squared output
    x = np.linspace(-1, 1, 257).astype(np.float32)
    p = tbg.mlp_init(9)
    out = oracle.mlp_forward(32, p, x)
    loss, _ = tbg.mlp_grad(p, x, np.zeros_like(x))
    assert abs(loss - float(np.mean(out ** 2))) <= 1e-4 * max(1.0, float(np.mean(out ** 2)))


def test_training_reduces_loss(tbg, oracle, cuda):
    x, y = zipf_cdf_points(8192, seed=2)
    p0 = tbg.mlp_init(5)
    l0, _ = tbg.mlp_grad(p0, x, y)
    p1 = tbg.mlp_train(p0, x, y, steps=300, lr=0.01, seed=7)
    l1, _ = tbg.mlp_grad(p1, x, y)
    l1_ref, _ = oracle.mlp_loss_grad(32, p1, x, y)
    assert abs(l1 - l1_ref) <= 1e-4 * max(1.0, l1_ref)
    assert l1 < l0 / 20 and l1 < 2e-3, (l0, l1)


@pytest.mark.parametrize("idx", range(8))
def test_lrn_matches_reference_golden(tbg, oracle, golden, cuda, idx):
    j = golden["joins"][idx]
    R = gen_relation(oracle, j["R"], j["seedR"], 0)
    S = gen_relation(oracle, j["S"], j["seedS"], 1)
    m, _, st = run_join(tbg, cuda, "LRN", R, S)
    assert m == j["RHO_n1"]
    m2, rows, st2 = run_join(tbg, cuda, "LRN", R, S, materialize=True)
    assert m2 == j["RHO_mat_count"] == len(rows)
    assert sha(oracle.sort_rows(rows)) == j["RHO_mat_sorted_sha256"]
    if j["name"] == "zipf15":  # most of S sits on a few keys: the heavy path runs
        assert st.used_fallback == 0 and st.heavy_keys > 0 and st.heavy_rows_S > len(S) // 2


def test_lrn_falls_back_on_uniform_data(tbg, oracle, cuda):
    R = gen_relation(oracle, ("pk", 1 << 16, 0, 0.0), 3, 0)
    S = gen_relation(oracle, ("fk", 1 << 19, 1 << 16, 0.0), 4, 1)
    m, _, st = run_join(tbg, cuda, "LRN", R, S)
    assert m == 1 << 19 and st.used_fallback == 1 and st.heavy_rows_S == 0


def test_lrn_duplicate_R_keys_on_heavy_path(tbg, oracle, cuda):
    """Heavy keys with several R rows: every (R, S) pair is produced."""
    rng = np.random.default_rng(23)
    R = np.zeros(50000, dtype=oracle.ROW)
    R["key"] = rng.integers(1, 20000, len(R))
    R["key"][:30] = 1
    R["key"][30:40] = 2
    S = gen_relation(oracle, ("zipf", 1 << 19, 20000, 1.5), 8, 1)
    oracle.fill_payloads(R, 0)
    ref, ref_rows = oracle.rho(R, S, materialize=True)
    m, rows, st = run_join(tbg, cuda, "LRN", R, S, materialize=True, cap=ref)
    assert st.used_fallback == 0 and st.heavy_rows_S > 0
    assert m == ref and np.array_equal(oracle.sort_rows(rows), oracle.sort_rows(ref_rows))


def test_lrn_materialise_at_fifteen_bits(tbg, oracle, cuda):
    """15 radix bits with materialisation: the bypass histogram's shared
    memory (2^15 bins, filter, heavy keys and counts) must fit one block."""
    R = gen_relation(oracle, ("pk", 1 << 20, 0, 0.0), 31, 0)
    S = gen_relation(oracle, ("zipf", 1 << 22, 1 << 20, 1.0), 32, 1)
    ref, ref_rows = oracle.rho(R, S, materialize=True)
    m, rows, st = run_join(tbg, cuda, "LRN", R, S, materialize=True, cap=ref, radix_bits=15, passes=2)
    assert st.radix_bits == 15 and st.used_fallback == 0 and st.heavy_rows_S > 0
    assert m == ref and np.array_equal(oracle.sort_rows(rows), oracle.sort_rows(ref_rows))


def test_skew_split_with_several_R_chunks(tbg, oracle, cuda):
    """R partitions larger than one shared-memory table (duplicate R keys,
    few radix bits) with a hot S side: every R chunk probes every S slice."""
    rng = np.random.default_rng(41)
    R = np.zeros(60000, dtype=oracle.ROW)
    R["key"] = rng.integers(1, 4000, len(R))
    oracle.fill_payloads(R, 0)
    S = gen_relation(oracle, ("zipf", 1 << 20, 4000, 1.2), 42, 1)
    ref, ref_rows = oracle.rho(R, S, materialize=True)
    for algo in ("RHO", "RHT"):
        m, rows, st = run_join(tbg, cuda, algo, R, S, materialize=True, cap=ref, radix_bits=2, passes=1)
        assert st.max_part_R > 8192 and st.work_items > 4
        assert m == ref and np.array_equal(oracle.sort_rows(rows), oracle.sort_rows(ref_rows)), algo


def test_lrn_dropin(tbg, oracle, cuda):
    R = gen_relation(oracle, ("pk", 1 << 16, 0, 0.0), 11111, 0)
    S = gen_relation(oracle, ("zipf", 1 << 19, 1 << 16, 1.0), 22222, 1)
    ref = oracle.rho(R, S)
    assert tbg.find("LRN").join(R, S, 4) == ref
    c, rows = tbg.find("LRN").join(R, S, 2, materialize=True)
    assert c == ref and len(rows) == ref


def _ablation(tbg, cuda, nR, nS, z, scatter=0):
    tR, pR = dev_relation(cuda, nR)
    tS, pS = dev_relation(cuda, nS)
    tbg.gen_pk(pR, nR, 1)
    tbg.gen_zipf(pS, nS, nR, z, scatter, 2)
    cuda.cuda.synchronize()
    out = {}
    for name, algo, model in [("radix", "RHO", 0), ("trained", "LRN", tbg.MODEL_MLP),
                              ("untrained", "LRN", tbg.MODEL_UNTRAINED), ("sample", "LRN", tbg.MODEL_SAMPLE)]:
        cfg = tbg.config(algo, model=model)
        _, m, st = tbg.join_device(cfg, pR, nR, pS, nS)
        out[name] = {"count": m, "share": st.heavy_rows_S / nS, "fallback": st.used_fallback,
                     "loss": st.train_loss, "pred": st.heavy_rows_predicted, "sampled": st.heavy_rows_sampled}
    return out


@pytest.mark.parametrize("scatter", [0, 1], ids=["rank_is_key", "scattered"])
def test_trained_network_against_sample_counts_and_untrained(tbg, cuda, scatter):
    """Same pipeline, same data, Zipf over R's keys with the hot keys at small
    ranks or scattered.  The heavy keys are always the sample's most frequent
    ones; the model predicts how many S rows the top ranks hold, which sets
    how many keys bypass and whether the bypass runs at all.

    * Trained, the network's prediction of the heavy keys' rows is within 25%
      of the sample's own estimate at z = 1.0, and its decisions equal the
      raw-count method's: it matches the method without the network, it does
      not beat it (both pick the same keys).
    * Untrained (its initialisation), the prediction is at least four times
      further off than the trained one.
    * At z = 0.5 no key is heavy enough to pay: the trained network and the
      raw counts both fall back to plain radix.
    * Counts are identical in every case."""
    nR, nS = 1 << 22, 1 << 25
    o = _ablation(tbg, cuda, nR, nS, 1.0, scatter)
    assert len({v["count"] for v in o.values()}) == 1 and o["radix"]["count"] == nS
    t, smp, u = o["trained"], o["sample"], o["untrained"]
    assert t["fallback"] == 0 and smp["fallback"] == 0, o
    assert t["share"] > 0.30 and abs(t["share"] - smp["share"]) < 0.02, o
    err_t = abs(t["pred"] - t["sampled"]) / t["sampled"]
    assert err_t < 0.25, o
    err_u = abs(u["pred"] - u["sampled"]) / max(u["sampled"], 1.0) if u["sampled"] else float("inf")
    assert err_u > 4 * err_t, (err_u, err_t, o)
    o = _ablation(tbg, cuda, nR, nS, 0.5, scatter)
    assert len({v["count"] for v in o.values()}) == 1
    assert o["trained"]["fallback"] == 1 and o["sample"]["fallback"] == 1, o


def test_full_size_skewed_config(tbg, cuda):
    """|R| = 2^26, |S| = 2^29 Zipf z = 1.0: LRN and RHO agree with |S|."""
    nR, nS = 1 << 26, 1 << 29
    tR, pR = dev_relation(cuda, nR)
    tS, pS = dev_relation(cuda, nS)
    tbg.gen_pk(pR, nR, 11111)
    tbg.gen_zipf(pS, nS, nR, 1.0, 0, 22222)
    cuda.cuda.synchronize()
    _, m1, st1 = tbg.join_device(tbg.config("LRN"), pR, nR, pS, nS)
    _, m0, st0 = tbg.join_device(tbg.config("RHO"), pR, nR, pS, nS)
    assert m0 == m1 == nS
    assert st1.used_fallback == 0 and st1.heavy_rows_S > nS // 3


C3_CASES = [(0.0, 0), (0.5, 0), (1.5, 0), (0.5, 1), (1.0, 1), (1.5, 1)]


@pytest.mark.parametrize("z,scatter", C3_CASES, ids=[f"z{z}-{'scattered' if s else 'rank_is_key'}"
                                                    for z, s in C3_CASES])
def test_full_size_c3_configs(tbg, cuda, z, scatter):
    """|R| = 2^26, |S| = 2^29 Zipf over R's keys at every exponent of the
    skewed configuration, with the hot keys at small ranks (rank = key, as
    the reference's generator leaves them) or scattered over the key range
    by a seeded permutation.  LRN, RHO with the skew split and plain RHO all
    count |S|; what LRN chose is printed."""
    nR, nS = 1 << 26, 1 << 29
    tR, pR = dev_relation(cuda, nR)
    tS, pS = dev_relation(cuda, nS)
    tbg.gen_pk(pR, nR, 11111)
    tbg.gen_zipf(pS, nS, nR, z, scatter, 22222)
    cuda.cuda.synchronize()
    _, m1, st1 = tbg.join_device(tbg.config("LRN"), pR, nR, pS, nS)
    _, m0, _ = tbg.join_device(tbg.config("RHO"), pR, nR, pS, nS)
    _, m2, st2 = tbg.join_device(tbg.config("RHO", skew_split=0), pR, nR, pS, nS)
    assert m0 == m1 == m2 == nS
    print(f"\n[c3] z={z} scattered={scatter} lrn: fallback={st1.used_fallback} heavy_keys={st1.heavy_keys} "
          f"heavy_share={st1.heavy_rows_S / nS:.3f} loss={st1.train_loss:.3e} max_part_S={st1.max_part_S} "
          f"plain max_part_S={st2.max_part_S} mean={nS / st2.partitions:.0f}")
    if z <= 0.5:  # no key heavy enough to pay for the bypass
        assert st1.used_fallback == 1 and st1.heavy_rows_S == 0
    else:  # the heavy keys leave partitioning: about half of S at z = 1, nearly all at z = 1.5
        assert st1.used_fallback == 0 and st1.heavy_rows_S > (0.4 if z == 1.0 else 0.9) * nS
