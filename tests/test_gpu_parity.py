"""Parity of the CUDA path (through the C ABI) with the reference's CPU path.

Tolerances (FP64): inverse forward error <= 8 sqrt(N) kappa_F eps
(conftest.inverse_tolerance), residual ||MX - I||_F/||X||_F <= 1e-13, tau
within 1e-12 absolute, reflectors within 1e-10, determinant sign exact.
"""
import ctypes

import numpy as np
import pytest

import oracle
from bsofi_b200 import api
from bsofi_b200.hubbard import hubbard_matrix, pcyclic_blocks, random_pcyclic
from conftest import (det_sign, golden_cases, golden_matrix, inverse_tolerance, rel_fro, residual,
                      split_state)
from gpu_util import block_residual_gpu, from_device_colmajor, to_device_colmajor

CASES = golden_cases()
pytestmark = pytest.mark.gpu


def _check_state(M, n, L, state, tau, ref_state, ref_tau, Xref):
    np.testing.assert_allclose(tau, ref_tau, rtol=0, atol=1e-12)
    up, refl = split_state(state, n, L)
    rup, rrefl = split_state(ref_state, n, L)
    assert rel_fro(up, rup) < inverse_tolerance(M, Xref)
    assert np.abs(refl - rrefl).max() < 1e-10
    assert det_sign(state, tau) == det_sign(ref_state, ref_tau)


@pytest.mark.parametrize("case", CASES, ids=[c["name"] for c in CASES])
def test_handle_api_matches_golden(cuda_device, case):
    n, L = case["n"], case["L"]
    M = golden_matrix(case)
    X, state, tau, info = api.invert(M, n, L)
    assert info == 0
    _check_state(M, n, L, state, tau, case["state"], case["tau"], case["inverse"])
    assert rel_fro(X, case["inverse"]) < inverse_tolerance(M, case["inverse"])
    assert residual(M, X) < 1e-13


@pytest.mark.parametrize("n,L", [(1, 2), (1, 7), (2, 2), (3, 3), (5, 4), (8, 16), (17, 5),
                                 (33, 3), (31, 9), (64, 4), (100, 3), (129, 2), (255, 4),
                                 (257, 3), (300, 3), (400, 3), (520, 2), (700, 2)])
def test_random_pcyclic_vs_oracle(cuda_device, n, L):
    M = random_pcyclic(n, L, seed=n * 100 + L)
    Ar, taur, infor = oracle.port_bsoftri(M, n, L)
    Xr, _ = oracle.port_bsoi(Ar, taur, n, L)
    X, state, tau, info = api.invert(M, n, L)
    assert info == 0
    _check_state(M, n, L, state, tau, Ar, taur, Xr)
    assert rel_fro(X, Xr) < inverse_tolerance(M, Xr)
    assert residual(M, X) < 1e-13


def _reference(M, n, L):
    if oracle.ref_available():
        oracle.set_ref_threads(8)
        A, tau, info = oracle.ref_bsoftri(M, n, L)
        X, _ = oracle.ref_bsoi(A, tau, n, L)
        return A, tau, X
    A, tau, info = oracle.port_bsoftri(M, n, L)
    X, _ = oracle.port_bsoi(A, tau, n, L)
    return A, tau, X


def test_hubbard_n64_p16_vs_reference(cuda_device):
    n, L = 64, 16
    M = hubbard_matrix(8, L, 4.0, seed=1)
    Ar, taur, Xr = _reference(M, n, L)
    X, state, tau, info = api.invert(M, n, L)
    assert info == 0
    _check_state(M, n, L, state, tau, Ar, taur, Xr)
    assert rel_fro(X, Xr) < inverse_tolerance(M, Xr)
    assert residual(M, X) < 1e-13


def test_hubbard_n256_p32_vs_reference(cuda_device):
    """The benchmark configuration (N = 8192) against the reference CPU path."""
    import torch
    n, L = 256, 32
    M = hubbard_matrix(16, L, 4.0, seed=2)
    Ar, taur, Xr = _reference(M, n, L)
    X, state, tau, info = api.invert(M, n, L)
    assert info == 0
    np.testing.assert_allclose(tau, taur, rtol=0, atol=1e-11)
    assert det_sign(state, tau) == det_sign(Ar, taur)
    kappa_tol = inverse_tolerance(M, Xr)
    assert rel_fro(X, Xr) < kappa_tol
    diag, sub = pcyclic_blocks(M, n, L)
    Xd = torch.from_numpy(np.ascontiguousarray(X)).to(cuda_device)
    assert block_residual_gpu(torch, diag, sub, Xd) < 1e-13


def test_device_api_matches_handle_api(cuda_device):
    import torch
    n, L = 48, 6
    N = n * L
    M = hubbard_matrix(4, L, 4.0, seed=3) if n == 16 else random_pcyclic(n, L, seed=9)
    Xh, _, tauh, info = api.invert(M, n, L)
    ldd = N + 6
    dA = to_device_colmajor(torch, M, ld=ldd)
    dtau = torch.zeros(N, dtype=torch.float64, device=cuda_device)
    ws = torch.zeros(api.workspace_bytes(n, L, ldd) // 8 + 1, dtype=torch.float64,
                     device=cuda_device)
    rc = api.device_invert(n, L, dA.data_ptr(), ldd, dtau.data_ptr(), ws.data_ptr(), 0)
    torch.cuda.synchronize()
    assert rc == 0
    assert api.last_launches() > 0
    Xd = from_device_colmajor(dA, N)
    np.testing.assert_array_equal(dtau.cpu().numpy(), tauh)
    assert rel_fro(Xd, Xh) < 1e-13


def test_singular_R_reports_info(cuda_device):
    n, L = 8, 4
    M = random_pcyclic(n, L, seed=4)
    M[:n, :n] = 0.0          # A_0 = 0 and B_0 = 0: the first panel is zero,
    M[n:2 * n, :n] = 0.0     # so R(1,1) = 0 exactly.
    A = np.asfortranarray(M.copy())
    tau = np.zeros(n * L)
    with api.Handle(n, L) as h:
        info = h.bsoftri(A, tau)
    assert info == 1


def test_split_c_names_match_handle_api(cuda_device):
    lib = api.load()
    n, L = 20, 5
    N = n * L
    M = random_pcyclic(n, L, seed=21)
    Xh, stateh, tauh, _ = api.invert(M, n, L)
    A = np.asfortranarray(M.copy())
    tau = np.zeros(N)
    w = np.zeros(1)
    info = ctypes.c_int(7)
    dp = ctypes.POINTER(ctypes.c_double)
    lib.lapackXbsof(n, L, A.ctypes.data_as(dp), N, tau.ctypes.data_as(dp), w.ctypes.data_as(dp), 1,
                    ctypes.byref(info))
    assert info.value == 0
    lib.lapackXbstri(n, L, A.ctypes.data_as(dp), N, ctypes.byref(info))
    assert info.value == 0
    assert rel_fro(A, stateh) < 1e-13
    lib.lapackXbsoi_ormqr(n, L, A.ctypes.data_as(dp), N, tau.ctypes.data_as(dp),
                          w.ctypes.data_as(dp), 1, ctypes.byref(info))
    assert info.value == 0
    assert rel_fro(A, Xh) < 1e-13


def test_gpu_names_on_device_memory(cuda_device):
    import torch
    lib = api.load()
    n, L = 16, 7
    N = n * L
    M = random_pcyclic(n, L, seed=31)
    Xh, stateh, tauh, _ = api.invert(M, n, L)
    dA = to_device_colmajor(torch, M)
    tau = np.zeros(N)
    w = np.zeros(1)
    info = ctypes.c_int(7)
    dp = ctypes.POINTER(ctypes.c_double)
    lib.gpuXbsof(n, L, dA.data_ptr(), N, tau.ctypes.data_as(dp), w.ctypes.data_as(dp), 1, None,
                 ctypes.byref(info))
    assert info.value == 0
    lib.gpuXbstri_rseq(n, L, dA.data_ptr(), N, None, 0, ctypes.byref(info))
    assert info.value == 0
    assert rel_fro(from_device_colmajor(dA, N), stateh) < 1e-13
    lib.gpuXbsoi_batched(n, L, dA.data_ptr(), N, tau.ctypes.data_as(dp), w.ctypes.data_as(dp), 1,
                         None, None, 0, ctypes.byref(info))
    assert info.value == 0
    assert rel_fro(from_device_colmajor(dA, N), Xh) < 1e-13


@pytest.mark.parametrize("n,L", [(37, 6), (128, 10), (256, 8)])
def test_handle_api_pinned_host_arrays(cuda_device, n, L):
    """Page-locked caller arrays take the direct-DMA path (BSOI pipelined
    with the copies, one GEMM launch per step); the state is bitwise the
    pageable path's and the inverse agrees within the parity tolerance."""
    import torch
    N = n * L
    M = random_pcyclic(n, L, seed=4242 + n)
    Xp, state_p, tau_p, info = api.invert(M, n, L)
    assert info == 0
    A = torch.empty((N, N), dtype=torch.float64, pin_memory=True).numpy().T
    tau = torch.zeros(N, dtype=torch.float64, pin_memory=True).numpy()
    A[:] = M
    with api.Handle(n, L) as h:
        assert h.bsoftri(A, tau) == 0
        np.testing.assert_array_equal(tau, tau_p)
        np.testing.assert_array_equal(A, state_p)
        assert h.bsoi(A, tau) == 0
        assert rel_fro(A, Xp) < inverse_tolerance(M, Xp)
        assert residual(M, A) < 1e-13
        # A second call on the same handle (events and streams reused).
        A[:] = M
        assert h.bsoftri(A, tau) == 0
        assert h.bsoi(A, tau) == 0
        assert residual(M, A) < 1e-13


@pytest.mark.parametrize("L", [2, 3])
def test_largest_block_size(cuda_device, L):
    """n = BSOFI_MAX_BLOCK (768): the tallest panels (2n = 1536 rows, six rows
    per thread in the BSOF kernel) against the oracle."""
    n = 768
    M = random_pcyclic(n, L, seed=768 + L)
    Ar, taur, Xr = _reference(M, n, L)
    X, state, tau, info = api.invert(M, n, L)
    assert info == 0
    _check_state(M, n, L, state, tau, Ar, taur, Xr)
    assert rel_fro(X, Xr) < inverse_tolerance(M, Xr)
    assert residual(M, X) < 1e-13


@pytest.mark.parametrize("pinned", [False, True])
def test_handle_bsoi_with_another_state_recomputes_q(cuda_device, pinned):
    """hybridxbsoih_ reuses the Q_k^T its handle formed during hybridxbsoftrih_
    only for the same state: a handle given another matrix's state (or a
    changed tau) forms Q again and inverts that matrix."""
    import torch
    n, L = 40, 6
    N = n * L
    M1 = random_pcyclic(n, L, seed=51)
    M2 = random_pcyclic(n, L, seed=52)

    def host(a):
        if not pinned:
            return np.asfortranarray(a.copy())
        t = torch.empty(a.shape[::-1], dtype=torch.float64, pin_memory=True).numpy().T
        t[:] = a
        return t

    X2, state2, tau2, info = api.invert(M2, n, L)
    assert info == 0
    with api.Handle(n, L) as h:
        A1 = host(M1)
        tau1 = np.zeros(N)
        assert h.bsoftri(A1, tau1) == 0
        # Another matrix's state through the same handle.
        A = host(state2)
        assert h.bsoi(A, tau2.copy()) == 0
        assert rel_fro(A, X2) < inverse_tolerance(M2, X2)
        assert residual(M2, A) < 1e-13
        # The first state again, but with one tau changed: Q must be re-formed.
        A1b = host(M1)
        tau1b = np.zeros(N)
        assert h.bsoftri(A1b, tau1b) == 0
        tau_mod = tau1b.copy()
        tau_mod[3] = 0.0
        Am = host(np.array(A1b))
        assert h.bsoi(Am, tau_mod) == 0
    # Reference for the modified state: a fresh handle (nothing to reuse).
    with api.Handle(n, L) as h2:
        Ar = host(np.array(A1b))
        assert h2.bsoi(Ar, tau_mod) == 0
    assert rel_fro(Am, Ar) < 1e-12
