"""Parity of the single-precision library (libbsofi_b200_fp32.so) on the GPU.

Two kinds of checks:
* exact: the float results are the FP64 pipeline's results rounded once --
  state and tau equal float32(FP64 library's state, tau) bitwise, and the
  inverse equals float32(FP64 library's BSOI of the float state) bitwise;
* against the reference's single-precision build (-D__SINGLE_PREC__) and its
  fixtures: inverse and R^{-1} within 8 sqrt(N) kappa_F eps32, tau and
  reflectors within 1e-4 absolute, residual ||MX - I||_F/||X||_F within
  ||M||_F eps32 and within twice the FP32 reference's own residual,
  determinant sign exact.
"""
import ctypes

import numpy as np
import pytest

import oracle
from bsofi_b200 import api, fp32
from bsofi_b200.hubbard import assemble_pcyclic, hubbard_matrix, random_pcyclic
from conftest import det_sign, rel_fro, split_state
from test_fp32_abi import CASES32

pytestmark = pytest.mark.gpu
EPS32 = float(np.finfo(np.float32).eps)
_fp = ctypes.POINTER(ctypes.c_float)


def _tol32(M, X):
    N = M.shape[0]
    kappa = np.linalg.norm(M) * np.linalg.norm(X) / N
    return 8.0 * np.sqrt(N) * kappa * EPS32


def _residual(M, X):
    N = M.shape[0]
    X = X.astype(np.float64)
    return float(np.linalg.norm(M @ X - np.eye(N)) / np.linalg.norm(X))


def _check_vs_fp32_reference(M32, n, L, X, state, tau, ref_state, ref_tau, ref_X):
    M = M32.astype(np.float64)
    tol = _tol32(M, ref_X.astype(np.float64))
    np.testing.assert_allclose(tau, ref_tau, rtol=0, atol=1e-4)
    up, refl = split_state(state, n, L)
    rup, rrefl = split_state(ref_state, n, L)
    assert rel_fro(up.astype(np.float64), rup.astype(np.float64)) < tol
    assert np.abs(refl - rrefl).max() < 1e-4
    assert det_sign(state, tau) == det_sign(ref_state, ref_tau)
    assert rel_fro(X.astype(np.float64), ref_X.astype(np.float64)) < tol
    res = _residual(M, X)
    assert res < np.linalg.norm(M) * EPS32
    assert res < 2.0 * max(_residual(M, ref_X), 1e-8)


@pytest.mark.parametrize("case", CASES32, ids=[c["name"] for c in CASES32])
def test_handle_api_matches_fp32_golden(cuda_device, case):
    n, L = case["n"], case["L"]
    M32 = assemble_pcyclic(case["diag"], case["sub"]).astype(np.float32)
    X, state, tau, info = fp32.invert(M32, n, L)
    assert info == 0
    assert X.dtype == np.float32 and fp32.last_launches() > 0
    _check_vs_fp32_reference(M32, n, L, X, state, tau, case["state"], case["tau"],
                             case["inverse"])


@pytest.mark.parametrize("n,L", [(1, 2), (5, 4), (16, 6), (33, 3), (64, 16), (100, 5), (256, 8)])
def test_float_results_are_fp64_results_rounded(cuda_device, n, L):
    M32 = random_pcyclic(n, L, seed=700 + n * 10 + L).astype(np.float32)
    X32, S32, T32, info = fp32.invert(M32, n, L)
    assert info == 0
    _, S64, T64, info64 = api.invert(M32.astype(np.float64), n, L)
    assert info64 == 0
    np.testing.assert_array_equal(S32, S64.astype(np.float32))
    np.testing.assert_array_equal(T32, T64.astype(np.float32))
    # BSOI of the float state in FP64, rounded once.
    A = np.asfortranarray(S32.astype(np.float64))
    with api.Handle(n, L) as h:
        assert h.bsoi(A, T32.astype(np.float64)) == 0
    np.testing.assert_array_equal(X32, A.astype(np.float32))


def test_c_names_and_device_names_match_handle_api(cuda_device):
    """The split phases hand a float state from one phase to the next (as
    the reference's single-precision build does), so they agree with the
    handle API, which rounds once, within the FP32 bound; tau comes from BSOF
    alone and is bitwise the same.  The device-pointer names round at the same
    phase boundaries as the host split phases and agree with them bitwise."""
    import torch
    lib = fp32.load()
    n, L = 24, 5
    N = n * L
    M32 = random_pcyclic(n, L, seed=77).astype(np.float32)
    Xh, Sh, Th, info = fp32.invert(M32, n, L)
    assert info == 0
    tol = _tol32(M32.astype(np.float64), Xh.astype(np.float64))
    # lapackX* split phases on host float arrays.
    A = np.asfortranarray(M32.copy())
    tau = np.zeros(N, dtype=np.float32)
    w = np.zeros(1, dtype=np.float32)
    inf = ctypes.c_int(7)
    lib.lapackXbsof(n, L, A.ctypes.data_as(_fp), N, tau.ctypes.data_as(_fp),
                    w.ctypes.data_as(_fp), 1, ctypes.byref(inf))
    assert inf.value == 0
    lib.lapackXbstri(n, L, A.ctypes.data_as(_fp), N, ctypes.byref(inf))
    assert inf.value == 0
    np.testing.assert_array_equal(tau, Th)
    assert rel_fro(A.astype(np.float64), Sh.astype(np.float64)) < tol
    S_split = A.copy()
    lib.lapackXbsoi_ormqr(n, L, A.ctypes.data_as(_fp), N, tau.ctypes.data_as(_fp),
                          w.ctypes.data_as(_fp), 1, ctypes.byref(inf))
    assert inf.value == 0
    assert rel_fro(A.astype(np.float64), Xh.astype(np.float64)) < tol
    X_split = A.copy()
    Sh, Xh = S_split, X_split
    # gpuX* on a float device matrix with a padded leading dimension.
    ldd = N + 8
    dA = torch.zeros((N, ldd), dtype=torch.float32, device=cuda_device)
    dA[:, :N] = torch.from_numpy(np.ascontiguousarray(M32.T)).to(cuda_device)
    tau2 = np.zeros(N, dtype=np.float32)
    lib.gpuXbsof(n, L, dA.data_ptr(), ldd, tau2.ctypes.data_as(_fp), w.ctypes.data_as(_fp), 1,
                 None, ctypes.byref(inf))
    assert inf.value == 0
    lib.gpuXbstri_rseq(n, L, dA.data_ptr(), ldd, None, 0, ctypes.byref(inf))
    assert inf.value == 0
    np.testing.assert_array_equal(dA[:, :N].cpu().numpy().T, Sh)
    np.testing.assert_array_equal(tau2, Th)
    lib.gpuXbsoi_ormqr(n, L, dA.data_ptr(), ldd, tau2.ctypes.data_as(_fp), w.ctypes.data_as(_fp),
                       1, None, None, 0, ctypes.byref(inf))
    assert inf.value == 0
    np.testing.assert_array_equal(dA[:, :N].cpu().numpy().T, Xh)


def test_pinned_float_arrays_match_pageable(cuda_device):
    import torch
    n, L = 64, 6
    N = n * L
    M32 = random_pcyclic(n, L, seed=81).astype(np.float32)
    Xp, Sp, Tp, _ = fp32.invert(M32, n, L)
    A = torch.empty((N, N), dtype=torch.float32, pin_memory=True).numpy().T
    tau = torch.zeros(N, dtype=torch.float32, pin_memory=True).numpy()
    A[:] = M32
    with fp32.Handle(n, L) as h:
        assert h.bsoftri(A, tau) == 0
        np.testing.assert_array_equal(A, Sp)
        np.testing.assert_array_equal(tau, Tp)
        assert h.bsoi(A, tau) == 0
    np.testing.assert_array_equal(A, Xp)


def test_singular_R_reports_info(cuda_device):
    n, L = 8, 4
    M = random_pcyclic(n, L, seed=4).astype(np.float32)
    M[:n, :n] = 0.0
    M[n:2 * n, :n] = 0.0
    A = np.asfortranarray(M)
    tau = np.zeros(n * L, dtype=np.float32)
    with fp32.Handle(n, L) as h:
        assert h.bsoftri(A, tau) == 1


def test_hubbard_n256_p32_vs_fp32_reference(cuda_device):
    """The benchmark configuration (N = 8192) against the reference's
    single-precision CPU path."""
    if not oracle.ref32_available():
        pytest.skip("FP32 reference library not built")
    n, L = 256, 32
    M32 = hubbard_matrix(16, L, 4.0, seed=2).astype(np.float32)
    oracle.set_ref_threads(8, kind="ref32")
    Ar, taur, infor = oracle.ref32_bsoftri(M32, n, L)
    Xr, _ = oracle.ref32_bsoi(Ar, taur, n, L)
    assert infor == 0
    X, state, tau, info = fp32.invert(M32, n, L)
    assert info == 0
    _check_vs_fp32_reference(M32, n, L, X, state, tau, Ar, taur, Xr)


@pytest.mark.parametrize("L", [2, 3])
def test_largest_block_size_fp32(cuda_device, L):
    """n = BSOFI_MAX_BLOCK (768) through the single-precision library against
    the reference's single-precision build."""
    if not oracle.ref32_available():
        pytest.skip("FP32 reference library not built")
    n = 768
    M32 = random_pcyclic(n, L, seed=7680 + L).astype(np.float32)
    oracle.set_ref_threads(8, kind="ref32")
    Ar, taur, _ = oracle.ref32_bsoftri(M32, n, L)
    Xr, _ = oracle.ref32_bsoi(Ar, taur, n, L)
    X, state, tau, info = fp32.invert(M32, n, L)
    assert info == 0
    _check_vs_fp32_reference(M32, n, L, X, state, tau, Ar, taur, Xr)
