"""The CPU oracle is pinned to the reference before anything is checked
against it: every vector in tests/golden/reference_vectors.json was produced
by the reference's own sources (tests/golden/make_golden.py)."""
from __future__ import annotations

import hashlib

import numpy as np
import pytest

from conftest import gen_relation


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def test_generators_match_reference(oracle, golden):
    for g in golden["generators"]:
        oracle.seed(g["seed"])
        rows = oracle.gen(g["kind"], g["n"], g["maxid"], g["zipf"])
        assert rows["key"][:16].tolist() == g["first_keys"], g
        assert sha(rows["key"]) == g["keys_sha256"], g
        if "keys" in g:
            assert rows["key"].tolist() == g["keys"]


@pytest.mark.parametrize("idx", range(8))
def test_restated_rho_matches_reference(oracle, golden, idx):
    j = golden["joins"][idx]
    R = gen_relation(oracle, j["R"], j["seedR"], 0)
    S = gen_relation(oracle, j["S"], j["seedS"], 1)
    assert sha(R["key"]) == j["R_keys_sha256"]
    assert sha(S["key"]) == j["S_keys_sha256"]
    assert oracle.rho(R, S) == j["RHO_n1"] == j["RHO_n4"]
    assert oracle.rho(R, S, algo="RHT") == j["RHT_n1"]
    c, rows = oracle.rho(R, S, materialize=True)
    assert c == j["RHO_mat_count"] == len(rows) == j["RHO_mat_rows"]
    assert sha(oracle.sort_rows(rows)) == j["RHO_mat_sorted_sha256"]
    assert oracle.rows_checksum(rows) == j["RHO_mat_checksum"]
    cnt, chk = oracle.join_direct(R, S, nthreads=4)
    assert cnt == j["RHO_n1"] and chk == j["RHO_mat_checksum"]


def test_default_config_known_answer(golden):
    # native.cpp:59-73 defaults, seeds 11111/22222: Matches = |S| = 2097152
    j = golden["joins"][0]
    assert j["name"] == "default_c1" and j["RHO_n1"] == 2097152


@pytest.mark.parametrize("bits,passes", [(14, 2), (8, 1), (10, 2), (3, 1)])
def test_restated_rho_is_partition_independent(oracle, bits, passes):
    rng = np.random.default_rng(7)
    R = np.zeros(5000, dtype=oracle.ROW)
    S = np.zeros(20000, dtype=oracle.ROW)
    R["key"] = rng.integers(0, 3000, 5000)  # duplicates on both sides
    S["key"] = rng.integers(0, 3000, 20000)
    oracle.fill_payloads(R, 0)
    oracle.fill_payloads(S, 1)
    ref = int(sum(np.bincount(R["key"], minlength=3000)[S["key"]]))
    assert oracle.rho(R, S, bits, passes) == ref
    c, rows = oracle.rho(R, S, bits, passes, materialize=True)
    assert c == ref and oracle.join_direct(R, S)[1] == oracle.rows_checksum(rows)


def test_oracle_catches_a_planted_mistake(oracle):
    """A wrong row changes the checksum: the digest is a real check."""
    R = gen_relation(oracle, ("pk", 1000, 0, 0.0), 1, 0)
    S = gen_relation(oracle, ("fk", 5000, 1000, 0.0), 2, 1)
    c, rows = oracle.rho(R, S, materialize=True)
    good = oracle.rows_checksum(rows)
    bad = rows.copy()
    bad[17, 1] ^= 1
    assert oracle.rows_checksum(bad) != good


def test_mlp_gradient_oracle_finite_difference(oracle):
    """The float64 gradient reference used to check the GPU backward kernel."""
    H = 8
    rng = np.random.default_rng(3)
    P = 3 * H + H * H + H + 1
    params = (rng.standard_normal(P) * 0.5).astype(np.float32)
    x = rng.random(64).astype(np.float32)
    y = np.sort(rng.random(64)).astype(np.float32)
    loss, g = oracle.mlp_loss_grad(H, params, x, y)
    eps = 1e-3
    for i in rng.choice(P, 12, replace=False):
        p1 = params.astype(np.float64).copy()
        p2 = p1.copy()
        p1[i] += eps
        p2[i] -= eps
        l1, _ = oracle.mlp_loss_grad(H, p1.astype(np.float32), x, y)
        l2, _ = oracle.mlp_loss_grad(H, p2.astype(np.float32), x, y)
        # perturbations are rounded to float32: use the rounded step
        step = float(np.float32(p1[i]) - np.float32(p2[i]))
        assert abs((l1 - l2) / step - g[i]) < 2e-3 * max(1.0, abs(g[i]))


def test_live_reference_when_present(oracle):
    """Where oracle/_ref was built (this container), cross-check more cases live."""
    if oracle.ref() is None:
        pytest.skip("reference library not built here")
    rng = np.random.default_rng(11)
    for _ in range(3):
        nR = int(rng.integers(1, 30000))
        nS = int(rng.integers(1, 90000))
        R = np.zeros(nR, dtype=oracle.ROW)
        S = np.zeros(nS, dtype=oracle.ROW)
        R["key"] = rng.permutation(nR) + 1
        S["key"] = rng.integers(1, nR + 1, nS)
        oracle.fill_payloads(R, 0)
        oracle.fill_payloads(S, 1)
        c_ref, rows_ref, _ = oracle.ref_join("RHO", R, S, nthreads=2, materialize=True)
        c, rows = oracle.rho(R, S, materialize=True)
        assert c == c_ref
        assert np.array_equal(oracle.sort_rows(rows), oracle.sort_rows(rows_ref))
