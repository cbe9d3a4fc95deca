"""The CPU oracle against the reference's own results (golden fixtures made by
the compiled reference CPU path) and against the live reference library."""
import numpy as np
import pytest

import oracle
from bsofi_b200 import flops
from bsofi_b200.hubbard import hubbard_matrix, lattice_adjacency, random_pcyclic
from conftest import (golden_cases, golden_matrix, inverse_tolerance, rel_fro, residual,
                      det_sign, split_state)

CASES = golden_cases()


def test_golden_present():
    assert len(CASES) >= 10


@pytest.mark.parametrize("case", CASES, ids=[c["name"] for c in CASES])
def test_port_matches_golden(case):
    n, L = case["n"], case["L"]
    M = golden_matrix(case)
    A, tau, info = oracle.port_bsoftri(M, n, L)
    assert info == case["info"] == 0
    np.testing.assert_allclose(tau, case["tau"], rtol=0, atol=1e-12)
    up, refl = split_state(A, n, L)
    gup, grefl = split_state(case["state"], n, L)
    tol = inverse_tolerance(M, case["inverse"])
    assert rel_fro(up, gup) < tol
    assert np.abs(refl - grefl).max() < 1e-10
    assert det_sign(A, tau) == det_sign(case["state"], case["tau"])
    X, _ = oracle.port_bsoi(A, tau, n, L)
    assert rel_fro(X, case["inverse"]) < tol
    assert residual(M, X) < 1e-13


@pytest.mark.skipif(not oracle.ref_available(), reason="reference library not built")
@pytest.mark.parametrize("case", CASES[:6], ids=[c["name"] for c in CASES[:6]])
def test_reference_library_reproduces_golden(case):
    n, L = case["n"], case["L"]
    M = golden_matrix(case)
    A, tau, info = oracle.ref_bsoftri(M, n, L)
    assert info == case["info"]
    np.testing.assert_array_equal(tau, case["tau"])
    np.testing.assert_array_equal(A, case["state"])


@pytest.mark.skipif(not oracle.ref_available(), reason="reference library not built")
@pytest.mark.parametrize("n,L,seed", [(16, 6, 1), (9, 11, 2), (32, 4, 3)])
def test_port_matches_reference_library(n, L, seed):
    M = random_pcyclic(n, L, seed=seed)
    Xr = oracle.ref_inverse(M, n, L)
    Xp = oracle.port_inverse(M, n, L)
    assert rel_fro(Xp, Xr) < inverse_tolerance(M, Xr)


def test_oracle_inverse_is_dense_inverse():
    M = hubbard_matrix(3, 6, 4.0, seed=5)
    X = oracle.port_inverse(M, 9, 6)
    assert rel_fro(X, np.linalg.inv(M)) < 1e-12


def test_hubbard_generator():
    K = lattice_adjacency(4)
    assert np.allclose(K, K.T) and np.all(K.sum(axis=1) == 4)
    M1 = hubbard_matrix(4, 8, 4.0, seed=3)
    M2 = hubbard_matrix(4, 8, 4.0, seed=3)
    assert np.array_equal(M1, M2)
    n = 16
    # identity diagonal, -B_k below, +B_p in the corner
    assert np.allclose(M1[:n, :n], np.eye(n))
    assert np.all(M1[n:2 * n, :n] <= 0) and np.all(M1[:n, 7 * n:] >= 0)


def test_flop_model_matches_reference_counts():
    # FLOPS_BSOFTRI + FLOPS_BSOI at the benchmark configurations.
    assert abs(flops.bsofi_flops(64, 16) / 5.2275e8 - 1) < 1e-4
    assert abs(flops.bsofi_flops(256, 32) / 1.2730e11 - 1) < 1e-4
    assert abs(flops.bsofi_flops(400, 64) / 1.8907e12 - 1) < 1e-4
