"""The FP64 DMMA tile engine (bsofi_selftest_gemm) against torch FP64 matmul."""
import numpy as np
import pytest

from bsofi_b200 import api


@pytest.mark.gpu
@pytest.mark.parametrize("M,N,K,lda,ldb,ldc,ua,ub,tile", [
    (128, 128, 128, 128, 128, 128, 0, 0, 1),
    (64, 64, 64, 64, 64, 64, 0, 0, 2),
    (100, 77, 33, 100, 33, 100, 0, 0, 0),
    (257, 129, 300, 260, 302, 258, 0, 0, 1),
    (513, 200, 96, 513, 97, 513, 0, 0, 2),      # odd leading dimensions
    (256, 256, 256, 256, 256, 256, 1, 0, 1),    # upper-triangular A
    (192, 320, 192, 192, 192, 192, 0, 1, 2),    # upper-triangular B
    (150, 150, 150, 151, 151, 151, 1, 1, 0),
    (1000, 512, 512, 1024, 512, 1024, 0, 0, 1),
])
def test_gemm_engine(cuda_device, M, N, K, lda, ldb, ldc, ua, ub, tile):
    import torch
    g = torch.Generator(device="cpu").manual_seed(M * 7 + N)
    At = torch.randn(K, lda, dtype=torch.float64, generator=g).to(cuda_device)
    Bt = torch.randn(N, ldb, dtype=torch.float64, generator=g).to(cuda_device)
    Ct = torch.randn(N, ldc, dtype=torch.float64, generator=g).to(cuda_device)
    A = At[:, :M].T.clone()
    B = Bt[:, :K].T.clone()
    if ua:
        A = torch.triu(A)
    if ub:
        B = torch.triu(B)
    ref = 1.5 * (A @ B) - 0.5 * Ct[:, :M].T
    rc = api.selftest_gemm(M, N, K, 1.5, At.data_ptr(), lda, ua, Bt.data_ptr(), ldb, ub, -0.5,
                           Ct.data_ptr(), ldc, tile, 0)
    torch.cuda.synchronize()
    assert rc == 0
    out = Ct[:, :M].T
    err = float((out - ref).abs().max() / ref.abs().max())
    assert err < 1e-14, err


@pytest.mark.gpu
@pytest.mark.parametrize("M,N,K,lda,ldb,ldc,ua,ub,tile", [
    (128, 128, 128, 128, 128, 128, 0, 0, 1),
    (128, 128, 128, 128, 128, 128, 0, 0, 3),
    (64, 64, 64, 64, 64, 64, 0, 0, 2),
    (257, 129, 300, 260, 302, 258, 0, 0, 3),
    (513, 200, 96, 513, 97, 513, 0, 0, 2),      # odd leading dimensions
    (256, 256, 256, 256, 256, 256, 1, 0, 3),    # upper-triangular A
    (192, 320, 192, 192, 192, 192, 0, 1, 2),    # upper-triangular B
    (150, 150, 150, 151, 151, 151, 1, 1, 0),
])
def test_gemm_engine_k16(cuda_device, M, N, K, lda, ldb, ldc, ua, ub, tile):
    """The tile engine with mma.sync m16n8k16 steps
    (bsofi_device_set_gemm_k16(1)) against torch FP64 matmul."""
    lib = api.load()
    lib.bsofi_device_set_gemm_k16(1)
    try:
        test_gemm_engine(cuda_device, M, N, K, lda, ldb, ldc, ua, ub, tile)
    finally:
        lib.bsofi_device_set_gemm_k16(0)


@pytest.mark.gpu
@pytest.mark.parametrize("n,L", [(256, 8), (100, 12), (400, 6), (33, 7)])
def test_inversion_with_k16_steps(cuda_device, n, L):
    """A whole inversion with m16n8k16 steps in every GEMM and BSOI launch
    against the default engine: within the FP64 tolerance, residual at the
    FP64 level."""
    import torch
    from bsofi_b200.hubbard import random_pcyclic
    from conftest import inverse_tolerance, rel_fro, residual
    from gpu_util import from_device_colmajor, to_device_colmajor
    lib = api.load()
    N = n * L
    M = random_pcyclic(n, L, seed=41 + n)
    out = []
    for k16 in (1, 0):
        lib.bsofi_device_set_gemm_k16(k16)
        try:
            dA = to_device_colmajor(torch, M, device=cuda_device)
            dtau = torch.zeros(N, dtype=torch.float64, device=cuda_device)
            ws = torch.empty(api.workspace_bytes(n, L, N), dtype=torch.uint8, device=cuda_device)
            assert api.device_invert(n, L, dA.data_ptr(), N, dtau.data_ptr(), ws.data_ptr()) == 0
            torch.cuda.synchronize()
            out.append(from_device_colmajor(dA, N))
        finally:
            lib.bsofi_device_set_gemm_k16(0)
    assert rel_fro(out[0], out[1]) < inverse_tolerance(M, out[1])
    assert residual(M, out[0]) < 1e-13


@pytest.mark.gpu
@pytest.mark.parametrize("n,L", [(256, 32), (256, 8), (128, 20), (64, 40), (320, 6), (192, 12),
                                 (80, 24), (240, 8), (400, 6)])
def test_bsoi_tma_is_bitwise_the_same(cuda_device, n, L):
    """The persistent BSOI with its clean tiles loaded by TMA (the default,
    bsofi_device_set_bsoi_tma(1)) computes the same products in the same
    order as with cp.async (0): the inverses are equal bit for bit
    (persistent plans, set explicitly; 128 x 160 TMA tiles where 2n is a
    multiple of 160 but not of 128: n = 80, 240, 400), with a residual at
    the FP64 level."""
    import torch
    from bsofi_b200.hubbard import random_pcyclic
    from gpu_util import to_device_colmajor
    lib = api.load()
    N = n * L
    M = random_pcyclic(n, L, seed=71 + n + L)
    saved = api.plan_get(n, L)[1]
    api.plan_set(n, L, [0] + list(saved[1:]))
    out = []
    try:
        for tma in (1, 0):
            lib.bsofi_device_set_bsoi_tma(tma)
            dA = to_device_colmajor(torch, M, device=cuda_device)
            dtau = torch.zeros(N, dtype=torch.float64, device=cuda_device)
            ws = torch.zeros(api.workspace_bytes(n, L, N), dtype=torch.uint8, device=cuda_device)
            assert api.device_invert(n, L, dA.data_ptr(), N, dtau.data_ptr(), ws.data_ptr()) == 0
            torch.cuda.synchronize()
            assert int(ws.view(torch.int32)[0].item()) >= 0x7f7f7f7f
            out.append(dA)
    finally:
        lib.bsofi_device_set_bsoi_tma(1)
        api.plan_set(n, L, list(saved))
    assert torch.equal(out[0], out[1])
    from conftest import residual
    from gpu_util import from_device_colmajor
    assert residual(M, from_device_colmajor(out[0], N)) < 1e-13
