"""BSOI by row bands (bsofi_device_bsoi_rows), the GPU share of one inversion
split over ranks, emulated on one GPU by running every rank's band in turn on
its own copy of the factored state: the bands leave the other rows as they
were and together give the full BSOI bitwise (persistent BSOI plans: the same
tiles), or within 1e-13 (plans with one launch per step)."""
import numpy as np
import pytest

import oracle
from bsofi_b200 import api, shard
from bsofi_b200.hubbard import random_pcyclic
from conftest import inverse_tolerance, rel_fro, residual
from gpu_util import from_device_colmajor, to_device_colmajor

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("n,L,world", [(256, 32, 3), (196, 40, 4), (100, 12, 2), (64, 16, 8),
                                       (33, 9, 2)])
def test_row_bands_compose_the_inverse(cuda_device, n, L, world):
    import torch
    N = n * L
    M = random_pcyclic(n, L, seed=600 + n + L)
    dA = to_device_colmajor(torch, M)
    dtau = torch.zeros(N, dtype=torch.float64, device=cuda_device)
    ws = torch.zeros(api.workspace_bytes(n, L, N) // 8 + 1, dtype=torch.float64,
                     device=cuda_device)
    assert api.device_bsoftri(n, L, dA.data_ptr(), N, dtau.data_ptr(), ws.data_ptr(), 0) == 0
    full = dA.clone()
    assert api.device_bsoi(n, L, full.data_ptr(), N, dtau.data_ptr(), ws.data_ptr(), 0) == 0
    assembled = torch.full_like(dA, float("nan"))
    for r0, r1 in shard.row_bands(N, world):
        if r1 == r0:
            continue
        part = dA.clone()
        rc = api.device_bsoi_rows(n, L, part.data_ptr(), N, dtau.data_ptr(), ws.data_ptr(), r0,
                                  r1, 0)
        assert rc == 0
        torch.cuda.synchronize()
        assert torch.equal(part[:, :r0], dA[:, :r0])
        assert torch.equal(part[:, r1:], dA[:, r1:])
        assembled[:, r0:r1] = part[:, r0:r1]
    torch.cuda.synchronize()
    plan = api.plan_get(n, L)[1]
    if plan[0] in (0, 5):
        assert torch.equal(assembled, full)
    X = from_device_colmajor(assembled, N)
    Xf = from_device_colmajor(full, N)
    assert rel_fro(X, Xf) < 1e-13
    if N <= 3000:
        Ar, taur, _ = oracle.port_bsoftri(M, n, L)
        Xr, _ = oracle.port_bsoi(Ar, taur, n, L)
        assert rel_fro(X, Xr) < inverse_tolerance(M, Xr)
        assert residual(M, X) < 1e-13
