"""Launch plans on the GPU: every BSOI form and recurrence tile shape gives
the same inverse within the parity tolerance, and the autotuner stores a plan
that inverts correctly."""
import numpy as np
import pytest

from bsofi_b200 import api
from bsofi_b200.hubbard import hubbard_matrix, random_pcyclic
from conftest import inverse_tolerance, rel_fro, residual

pytestmark = pytest.mark.gpu


@pytest.fixture(autouse=True)
def _clear_plans():
    api.plan_clear()
    yield
    api.plan_clear()


def _device_invert(torch, M, n, L):
    from gpu_util import from_device_colmajor, to_device_colmajor
    N = n * L
    dA = to_device_colmajor(torch, M)
    dtau = torch.zeros(N, dtype=torch.float64, device="cuda:0")
    ws = torch.empty(api.workspace_bytes(n, L, N), dtype=torch.uint8, device="cuda:0")
    assert api.device_invert(n, L, dA.data_ptr(), N, dtau.data_ptr(), ws.data_ptr()) == 0
    torch.cuda.synchronize()
    return from_device_colmajor(dA, N)


@pytest.mark.parametrize("n,L", [(100, 7), (64, 20)])
def test_every_plan_inverts(cuda_device, n, L):
    import torch
    M = random_pcyclic(n, L, seed=n + 31 * L)
    Xref, _, _, info = api.invert(M, n, L)
    assert info == 0
    tol = inverse_tolerance(M, Xref)
    for bsoi in range(6):
        for rc in (0, 1, 2, 3, 4):
            assert api.plan_set(n, L, [bsoi, rc, 24, 0]) == 0
            X = _device_invert(torch, M, n, L)
            assert rel_fro(X, Xref) < tol, (bsoi, rc)
            assert residual(M, X) < 1e-13
            # The handle API follows the same plan.
            Xh, _, _, info = api.invert(M, n, L)
            assert info == 0 and rel_fro(Xh, Xref) < tol


def test_autotune_stores_a_working_plan(cuda_device):
    import torch
    n, L = 144, 12
    plan = api.autotune(n, L, reps=1)
    tuned, got = api.plan_get(n, L)
    assert tuned and got == plan
    assert 0 <= plan[0] <= 5 and 0 <= plan[1] <= 4 and plan[2] >= 1
    M = hubbard_matrix(12, L, 4.0, seed=3)
    X = _device_invert(torch, M, n, L)
    assert residual(M, X) < 1e-13
