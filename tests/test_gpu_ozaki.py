"""The int8 tensor-core product (tcgen05 kind::i8, Ozaki splitting) and the
mixed-precision inversion built on it, through the C ABI.

* bsofi_selftest_ozaki equals the numpy restatement (tests/ozaki_emul.py)
  bit for bit, for every slice count and for ragged shapes (M not a multiple
  of 128, N of 64, K of 32);
* a row or column holding Inf/NaN gives NaN in its output row/column;
* bsofi_device_invert_mixed: ||M X - I||_F / ||X||_F <= 1e-12 and the
  forward error against the reference's CPU path within 64 x the FP64
  tolerance (8 sqrt(N) kappa_F eps), at n = 64, p = 16 and at n = 256, p = 32;
  the state between the phases (tau, R^{-1}) is the FP64 path's, bitwise.
"""
import numpy as np
import pytest

import oracle
from bsofi_b200 import _lib, api
from bsofi_b200.hubbard import hubbard_matrix, pcyclic_blocks, random_pcyclic
from conftest import inverse_tolerance, rel_fro
from gpu_util import block_residual_colmajor, from_device_colmajor, to_device_colmajor
from ozaki_emul import ozaki_product

pytestmark = pytest.mark.gpu


def _product(torch, dev, A, B, S):
    lib = _lib.load()
    M, K = A.shape
    N = B.shape[1]
    dA = to_device_colmajor(torch, A, ld=M + 3, device=dev)
    dB = to_device_colmajor(torch, B, ld=K + 1, device=dev)
    dC = torch.full((N, M + 5), float("nan"), dtype=torch.float64, device=dev)
    scratch = torch.zeros(lib.bsofi_selftest_ozaki_scratch_bytes(M, N, K, S) // 8 + 32,
                          dtype=torch.float64, device=dev)
    derr = torch.zeros(1, dtype=torch.int32, device=dev)
    rc = lib.bsofi_selftest_ozaki(M, N, K, dA.data_ptr(), M + 3, dB.data_ptr(), K + 1,
                                  dC.data_ptr(), M + 5, S, scratch.data_ptr(), derr.data_ptr(),
                                  None)
    torch.cuda.synchronize()
    assert rc == 0
    assert int(derr.item()) == 0
    return from_device_colmajor(dC, M)


@pytest.mark.parametrize("M,N,K,S", [(128, 64, 32, 8), (300, 100, 77, 8), (1, 1, 1, 8),
                                     (257, 130, 512, 3), (257, 130, 512, 4), (257, 130, 512, 5),
                                     (257, 130, 512, 6), (257, 130, 512, 7),
                                     (1000, 1152, 1152, 8), (8192, 512, 512, 8)])
def test_product_bitwise_equals_restatement(cuda_device, M, N, K, S):
    import torch
    rng = np.random.default_rng(M * 7 + N * 3 + K + S)
    A = rng.standard_normal((M, K)) * np.exp(rng.uniform(-30, 30, (M, 1)))
    B = rng.standard_normal((K, N)) * np.exp(rng.uniform(-30, 30, (1, N)))
    if M > 2:
        A[1] = 0.0
    C = _product(torch, cuda_device, A, B, S)
    ref = ozaki_product(A, B, S)
    np.testing.assert_array_equal(C, ref)
    exact = A @ B
    # Slicing and the dropped products bound the error by K |A_i|max |B_j|max
    # (S + 3) 2^(2 - 7S); the FP64 product used as "exact" has its own K eps.
    scale = np.abs(A).max(axis=1)[:, None] * np.abs(B).max(axis=0)[None, :] * K
    assert (np.abs(C - exact) <= scale * (2.0 ** (-7 * S + 6) + K * 2.0 ** -52)).all()


def test_nonfinite_rows_and_columns_give_nan(cuda_device):
    import torch
    rng = np.random.default_rng(5)
    A = rng.standard_normal((200, 40))
    B = rng.standard_normal((40, 70))
    A[7, 3] = np.inf
    B[5, 11] = np.nan
    C = _product(torch, cuda_device, A, B, 8)
    assert np.isnan(C[7]).all()
    assert np.isnan(C[:, 11]).all()
    mask = np.ones_like(C, dtype=bool)
    mask[7] = False
    mask[:, 11] = False
    A2, B2 = A.copy(), B.copy()
    A2[7] = 0.0
    B2[:, 11] = 0.0
    np.testing.assert_array_equal(C[mask], ozaki_product(A2, B2, 8)[mask])


def _mixed(torch, dev, M, n, L, slices):
    N = n * L
    dA = to_device_colmajor(torch, M, ld=N, device=dev)
    dtau = torch.zeros(N, dtype=torch.float64, device=dev)
    nbytes = api.load().bsofi_device_workspace_bytes_mixed(n, L, N, slices)
    assert nbytes > 0
    ws = torch.zeros(nbytes // 8 + 1, dtype=torch.float64, device=dev)
    rc = api.load().bsofi_device_invert_mixed(n, L, dA.data_ptr(), N, dtau.data_ptr(),
                                              ws.data_ptr(), slices, None)
    torch.cuda.synchronize()
    assert rc == 0
    assert int(ws.view(torch.int32)[0].item()) >= 0x7f7f7f7f
    return dA, dtau


@pytest.mark.parametrize("side,L,U,slices", [(8, 16, 4.0, 8), (8, 16, 4.0, 0), (16, 32, 4.0, 8)])
def test_mixed_inversion_vs_reference(cuda_device, side, L, U, slices):
    import torch
    n = side * side
    N = n * L
    M = hubbard_matrix(side, L, U, seed=11)
    if oracle.ref_available():
        oracle.set_ref_threads(8)
        Ar, taur, _ = oracle.ref_bsoftri(M, n, L)
        Xr, _ = oracle.ref_bsoi(Ar, taur, n, L)
    else:
        Ar, taur, _ = oracle.port_bsoftri(M, n, L)
        Xr, _ = oracle.port_bsoi(Ar, taur, n, L)
    dA, dtau = _mixed(torch, cuda_device, M, n, L, slices)
    diag, sub = pcyclic_blocks(M, n, L)
    assert block_residual_colmajor(torch, diag, sub, dA, N) < 1e-12
    X = from_device_colmajor(dA, N)
    assert rel_fro(X, Xr) < 64 * inverse_tolerance(M, Xr)
    # The FP64 phases are the FP64 path's own: tau bitwise.
    X64, _, tau64, info = api.invert(M, n, L)
    assert info == 0
    np.testing.assert_array_equal(dtau.cpu().numpy(), tau64)


def test_mixed_inversion_seven_slices_and_ragged_size(cuda_device):
    import torch
    n, L = 50, 7
    M = random_pcyclic(n, L, seed=3)
    dA, _ = _mixed(torch, cuda_device, M, n, L, 7)
    X = from_device_colmajor(dA, n * L)
    res = np.linalg.norm(M @ X - np.eye(n * L)) / np.linalg.norm(X)
    assert res < 1e-11
    Xr = np.linalg.inv(M)
    assert rel_fro(X, Xr) < 1e3 * inverse_tolerance(M, Xr)


def test_mixed_rejects_bad_arguments(cuda_device):
    lib = api.load()
    assert lib.bsofi_device_workspace_bytes_mixed(64, 16, 1024, 9) == 0
    assert lib.bsofi_device_workspace_bytes_mixed(64, 16, 1023, 8) == 0
    fake = 0x1000
    assert lib.bsofi_device_invert_mixed(64, 16, fake, 1024, fake, fake, 2, None) == -1
    assert lib.bsofi_device_invert_mixed(769, 2, fake, 1538, fake, fake, 8, None) == -1
