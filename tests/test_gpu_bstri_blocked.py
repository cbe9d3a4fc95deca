"""The blocked BSTRI row recurrence (launch plan [3] = rows per group)
against the CPU oracle: ragged last groups, odd n (the unaligned tile path),
a group larger than L - 2 (clamped), and the benchmark's block size.  The
factorization is the same as with the one-row recurrence, so the reflectors
and tau must agree bitwise with it; R^{-1} and the inverse within the FP64
parity tolerance, residual within 1e-13."""
import numpy as np
import pytest

import oracle
from bsofi_b200 import api
from bsofi_b200.hubbard import random_pcyclic
from conftest import inverse_tolerance, rel_fro, residual, split_state

pytestmark = pytest.mark.gpu


@pytest.fixture(autouse=True)
def _clear_plans():
    api.plan_clear()
    yield
    api.plan_clear()


@pytest.mark.parametrize("persistent", [False, True], ids=["per_group", "persistent"])
@pytest.mark.parametrize("n,L,grp", [(5, 4, 2), (7, 9, 3), (16, 10, 4), (33, 7, 8), (31, 3, 4),
                                     (64, 16, 4), (100, 12, 6), (65, 13, 5), (256, 8, 4),
                                     (130, 20, 3)])
def test_blocked_recurrence_matches_oracle(cuda_device, n, L, grp, persistent):
    """persistent: all group steps in one launch (plan [1] = 4), tiles
    waiting on the previous group's top row tiles; else one launch per group."""
    M = random_pcyclic(n, L, seed=9000 + 13 * n + L)
    X0, S0, T0, info0 = api.invert(M, n, L)  # default plan
    assert info0 == 0
    _, plan = api.plan_get(n, L)
    assert api.plan_set(n, L, [plan[0], 4 if persistent else 2, plan[2], grp]) == 0
    X, S, T, info = api.invert(M, n, L)
    assert info == 0
    np.testing.assert_array_equal(T, T0)
    up, refl = split_state(S, n, L)
    up0, refl0 = split_state(S0, n, L)
    np.testing.assert_array_equal(refl, refl0)
    Ar, taur, _ = oracle.port_bsoftri(M, n, L)
    Xr, _ = oracle.port_bsoi(Ar, taur, n, L)
    rup, _ = split_state(Ar, n, L)
    tol = inverse_tolerance(M, Xr)
    assert rel_fro(up, rup) < tol
    assert rel_fro(X, Xr) < tol
    assert residual(M, X) < 1e-13


@pytest.mark.parametrize("n,L", [(324, 20), (400, 12), (196, 40)])
def test_default_blocked_plan_vs_reference(cuda_device, n, L):
    """Sizes whose default plan runs the persistent blocked recurrence with
    block rows that 128-row tiles straddle (n = 324, 400, 196), against the
    compiled reference CPU path."""
    _, plan = api.plan_get(n, L)
    assert plan[1] == 4 and plan[3] == 4
    M = random_pcyclic(n, L, seed=4400 + n + L)
    if oracle.ref_available():
        oracle.set_ref_threads(8)
        Ar, taur, _ = oracle.ref_bsoftri(M, n, L)
        Xr, _ = oracle.ref_bsoi(Ar, taur, n, L)
    else:
        Ar, taur, _ = oracle.port_bsoftri(M, n, L)
        Xr, _ = oracle.port_bsoi(Ar, taur, n, L)
    X, S, T, info = api.invert(M, n, L)
    assert info == 0
    np.testing.assert_allclose(T, taur, rtol=0, atol=1e-12)
    up, _ = split_state(S, n, L)
    rup, _ = split_state(Ar, n, L)
    tol = inverse_tolerance(M, Xr)
    assert rel_fro(up, rup) < tol
    assert rel_fro(X, Xr) < tol
    import torch
    from bsofi_b200.hubbard import pcyclic_blocks
    from gpu_util import block_residual_gpu
    Xd = torch.from_numpy(np.ascontiguousarray(X)).to(cuda_device)
    assert block_residual_gpu(torch, *pcyclic_blocks(M, n, L), Xd) < 1e-13


def _device_invert(torch, M, n, L):
    from gpu_util import from_device_colmajor, to_device_colmajor
    N = n * L
    dA = to_device_colmajor(torch, M)
    dtau = torch.zeros(N, dtype=torch.float64, device="cuda")
    ws = torch.zeros(api.workspace_bytes(n, L, N) // 8 + 1, dtype=torch.float64, device="cuda")
    assert api.device_invert(n, L, dA.data_ptr(), N, dtau.data_ptr(), ws.data_ptr(), 0) == 0
    torch.cuda.synchronize()
    return from_device_colmajor(dA, N), dtau.cpu().numpy()


@pytest.mark.parametrize("n,L,grp", [(256, 32, None), (64, 40, None), (100, 64, None),
                                     (33, 14, 3), (16, 20, 4), (100, 12, 2), (255, 16, 4),
                                     (128, 30, 8), (7, 23, 5)])
def test_overlapped_bstri_is_bitwise_the_ordered_one(cuda_device, n, L, grp):
    """Single inversions (device API and handle API) whose plan uses the
    persistent blocked recurrence split the factorization and overlap BSTRI's
    leading rows with its end; the results are bitwise those of the phases run
    in order (the same products), and agree with the oracle."""
    import torch
    lib = api.load()
    if grp is not None:
        _, plan = api.plan_get(n, L)
        assert api.plan_set(n, L, [plan[0], 4, plan[2], grp]) == 0
    M = random_pcyclic(n, L, seed=5100 + n + L)
    try:
        lib.bsofi_device_set_bstri_overlap(0)
        X0, tau0 = _device_invert(torch, M, n, L)
        _, S0, T0, info0 = api.invert(M, n, L)
        lib.bsofi_device_set_bstri_overlap(1)
        X1, tau1 = _device_invert(torch, M, n, L)
        _, S1, T1, info1 = api.invert(M, n, L)
    finally:
        lib.bsofi_device_set_bstri_overlap(1)
    assert info0 == info1 == 0
    np.testing.assert_array_equal(tau1, tau0)
    np.testing.assert_array_equal(X1, X0)
    np.testing.assert_array_equal(T1, T0)
    np.testing.assert_array_equal(S1, S0)
    if n * L <= 3000:
        Ar, taur, _ = oracle.port_bsoftri(M, n, L)
        Xr, _ = oracle.port_bsoi(Ar, taur, n, L)
        assert rel_fro(X1, Xr) < inverse_tolerance(M, Xr)
        assert residual(M, X1) < 1e-13
