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
