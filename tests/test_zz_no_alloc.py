"""The allocation-free inversion entry point (bsofi_device_invert_noalloc).

It exists for callers that cannot allocate device memory while they invert
(a memory pool that already holds nearly all of HBM, or a sweep that must not
be synchronized by cudaMalloc/cudaFree).  This test calls it through the C ABI
twice in a row on the same device and checks each result against the
allocating entry point bsofi_device_invert, within the parity tolerance of the
other GPU tests.  It lives in its own file, collected last.
"""
import ctypes

import numpy as np
import pytest

from bsofi_b200 import _lib, api
from bsofi_b200.hubbard import hubbard_matrix, random_pcyclic
from conftest import inverse_tolerance, rel_fro

pytestmark = pytest.mark.gpu


def _run_allocating(torch, M, n, L, ldd, dev):
    from gpu_util import from_device_colmajor, to_device_colmajor
    N = n * L
    dA = to_device_colmajor(torch, M, ld=ldd, device=dev)
    dtau = torch.zeros(N, dtype=torch.float64, device=dev)
    ws = torch.zeros(api.workspace_bytes(n, L, ldd) // 8 + 1, dtype=torch.float64, device=dev)
    assert api.device_invert(n, L, dA.data_ptr(), ldd, dtau.data_ptr(), ws.data_ptr(), 0) == 0
    torch.cuda.synchronize()
    return from_device_colmajor(dA, N), dtau.cpu().numpy()


def test_noalloc_matches_allocating_entry_point(cuda_device):
    import torch
    from gpu_util import from_device_colmajor, to_device_colmajor
    lib = _lib.load()
    assert lib.bsofi_noalloc_scratch_bytes() >= api.workspace_bytes(64, 16, 1024)
    cases = [(hubbard_matrix(8, 16, 4.0, seed=41), 64, 16, 1024),
             (random_pcyclic(24, 7, seed=42), 24, 7, 24 * 7 + 2)]
    for M, n, L, ldd in cases:
        N = n * L
        Xref, tauref = _run_allocating(torch, M, n, L, ldd, cuda_device)
        tol = inverse_tolerance(M, Xref)
        for _ in range(2):  # two calls in a row share the static scratch
            dA = to_device_colmajor(torch, M, ld=ldd, device=cuda_device)
            dtau = torch.zeros(N, dtype=torch.float64, device=cuda_device)
            dinfo = torch.full((1,), -5, dtype=torch.int32, device=cuda_device)
            rc = lib.bsofi_device_invert_noalloc(n, L, dA.data_ptr(), ldd, dtau.data_ptr(),
                                                 dinfo.data_ptr(), None)
            torch.cuda.synchronize()
            assert rc == 0
            info = int(dinfo.item())
            assert info >= 0x7f7f7f7f  # no exactly-zero diagonal in R
            X = from_device_colmajor(dA, N)
            assert rel_fro(X, Xref) < tol
            np.testing.assert_allclose(dtau.cpu().numpy(), tauref, rtol=0, atol=1e-12)


def test_noalloc_rejects_oversized_problem(cuda_device):
    lib = _lib.load()
    n, L = 512, 64
    assert api.workspace_bytes(n, L, n * L) > lib.bsofi_noalloc_scratch_bytes()
    # Rejected before any device work: the pointers are never touched.
    rc = lib.bsofi_device_invert_noalloc(n, L, ctypes.c_void_p(16), n * L, ctypes.c_void_p(16),
                                         None, None)
    assert rc == -2000
