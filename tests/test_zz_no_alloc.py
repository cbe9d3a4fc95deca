"""The allocation-free inversion entry point (bsofi_device_invert_noalloc).

It exists for callers that cannot allocate device memory while they invert
(a memory pool that already holds nearly all of HBM, or a sweep that must not
be synchronized by cudaMalloc/cudaFree).  These tests call it through the C
ABI: after bsofi_noalloc_prepare, a call leaves the device's free memory and
torch's reserved memory exactly as they were; two calls in a row on the same
device each match the allocating entry point bsofi_device_invert within the
parity tolerance of the other GPU tests; with no device info word the call
returns the info word itself.  The file is collected last, and the first test
is meaningful in a fresh process too (it runs prepare before anything else
launches a kernel of the library).
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


def test_noalloc_after_prepare_allocates_nothing(cuda_device):
    import torch
    from gpu_util import from_device_colmajor, to_device_colmajor
    lib = _lib.load()
    n, L, ldd = 64, 16, 1024
    M = hubbard_matrix(8, L, 4.0, seed=43)
    # Every buffer the call touches exists before the measurement.
    dA = to_device_colmajor(torch, M, ld=ldd, device=cuda_device)
    dtau = torch.zeros(n * L, dtype=torch.float64, device=cuda_device)
    dinfo = torch.full((1,), -5, dtype=torch.int32, device=cuda_device)
    torch.cuda.synchronize()
    assert lib.bsofi_noalloc_prepare() == 0
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info(cuda_device)
    reserved0 = torch.cuda.memory_reserved(cuda_device)
    rc = lib.bsofi_device_invert_noalloc(n, L, dA.data_ptr(), ldd, dtau.data_ptr(),
                                         dinfo.data_ptr(), None)
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info(cuda_device)
    assert rc == 0
    assert free1 == free0, "device free memory moved by %d bytes" % (free1 - free0)
    assert torch.cuda.memory_reserved(cuda_device) == reserved0
    assert int(dinfo.item()) >= 0x7f7f7f7f
    X = from_device_colmajor(dA, n * L)
    Xref, _ = _run_allocating(torch, M, n, L, ldd, cuda_device)
    assert rel_fro(X, Xref) < inverse_tolerance(M, Xref)


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


def test_noalloc_without_info_word_returns_info(cuda_device):
    import torch
    from gpu_util import from_device_colmajor, to_device_colmajor
    lib = _lib.load()
    n, L = 24, 7
    M = random_pcyclic(n, L, seed=44)
    Xref, _ = _run_allocating(torch, M, n, L, n * L, cuda_device)
    dA = to_device_colmajor(torch, M, ld=n * L, device=cuda_device)
    dtau = torch.zeros(n * L, dtype=torch.float64, device=cuda_device)
    # dinfo = NULL: the call waits for its stream and returns the info word.
    assert lib.bsofi_device_invert_noalloc(n, L, dA.data_ptr(), n * L, dtau.data_ptr(),
                                           None, None) == 0
    assert rel_fro(from_device_colmajor(dA, n * L), Xref) < inverse_tolerance(M, Xref)
    # An exactly zero diagonal of R: block 0 of the input all zero makes R(1,1) = 0.
    Z = M.copy()
    Z[:, 0] = 0.0
    dA = to_device_colmajor(torch, Z, ld=n * L, device=cuda_device)
    info = lib.bsofi_device_invert_noalloc(n, L, dA.data_ptr(), n * L, dtau.data_ptr(), None,
                                           None)
    assert info == 1


def test_noalloc_rejects_oversized_problem(cuda_device):
    lib = _lib.load()
    n, L = 512, 64
    assert api.workspace_bytes(n, L, n * L) > lib.bsofi_noalloc_scratch_bytes()
    # Rejected before any device work: the pointers are never touched.
    rc = lib.bsofi_device_invert_noalloc(n, L, ctypes.c_void_p(16), n * L, ctypes.c_void_p(16),
                                         None, None)
    assert rc == -2000
