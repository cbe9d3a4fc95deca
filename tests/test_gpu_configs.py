"""Parity and accuracy at the benchmark configurations' own sizes.

* n = 400, p = 64, U = 6 (N = 25600, the most ill-conditioned configuration,
  kappa_F about 3e6): the handle API's state and inverse, and the device API's
  inverse with the default launch plan of that size (per-step 64 x 64 BSOI
  tiles, the persistent one-row BSTRI recurrence), against the reference's own
  CPU path (oracle/_ref, src/bsofi_cpu.c:86-248) on the same matrix.
* The largest serving size, n = 576, p = 80 (N = 46080, 17 GB): the device
  inversion and its block residual on the GPU.  The residual bounds the
  forward error (||X - M^{-1}|| <= ||M^{-1}|| ||M X - I||), so it checks every
  column; the reference's state at n = 576 is checked at p = 10, where its CPU
  path takes seconds.
* 256 independent instances of the batched configuration (side in
  {8,...,16}, p in [8, 64], U in [2, 6]) in one batched call: every instance's
  block residual on the GPU, and 16 of them against the reference.

Tolerances as in test_gpu_parity: inverse forward error <= 8 sqrt(N) kappa_F
eps, residual <= 1e-13, reflectors within 1e-10, determinant sign exact; tau
within 1e-11 absolute (the oracle's plain-C restatement and the reference
differ by up to 5e-13 in tau at n = 400, p = 64, U = 6).
"""
import numpy as np
import pytest

import oracle
from bsofi_b200 import api
from bsofi_b200.hubbard import hubbard_blocks, hubbard_matrix
from conftest import det_sign, inverse_tolerance, rel_fro, split_state
from gpu_util import (block_residual_colmajor, from_device_colmajor, pcyclic_device,
                      to_device_colmajor)

pytestmark = pytest.mark.gpu


def _hubbard_blocks(side, L, U, seed):
    B = hubbard_blocks(side, L, U, seed=seed)
    n = side * side
    diag = np.broadcast_to(np.eye(n), (L, n, n)).copy()
    sub = -B
    sub[L - 1] = B[L - 1]
    return diag, sub


def _reference(M, n, L):
    if not oracle.ref_available():
        pytest.skip("oracle/_ref/libbsofi_ref.so not built")
    # A capped thread count: the host may be shared, and OpenBLAS slows
    # down badly when its threads outnumber the free cores.
    oracle.set_ref_threads(min(16, __import__("os").cpu_count() or 1))
    A, tau, info = oracle.ref_bsoftri(M, n, L)
    assert info == 0
    X, info = oracle.ref_bsoi(A, tau, n, L)
    assert info == 0
    return A, tau, X


def test_c4_n400_p64_U6_vs_reference(cuda_device):
    import torch
    n, L, U = 400, 64, 6.0
    N = n * L
    M = hubbard_matrix(20, L, U, seed=4)
    Ar, taur, Xr = _reference(M, n, L)
    tol = inverse_tolerance(M, Xr)
    # Handle API: the state between the two calls and the inverse.
    X, state, tau, info = api.invert(M, n, L)
    assert info == 0
    np.testing.assert_allclose(tau, taur, rtol=0, atol=1e-11)
    up, refl = split_state(state, n, L)
    rup, rrefl = split_state(Ar, n, L)
    assert rel_fro(up, rup) < tol
    assert np.abs(refl - rrefl).max() < 1e-10
    assert det_sign(state, tau) == det_sign(Ar, taur)
    assert rel_fro(X, Xr) < tol
    del X, state, up, refl, rup, rrefl, Ar
    # Device API with the default plan of this size.
    tuned, plan = api.plan_get(n, L)
    diag, sub = _hubbard_blocks(20, L, U, 4)
    dA = pcyclic_device(torch, diag, sub, N, cuda_device)
    dtau = torch.zeros(N, dtype=torch.float64, device=cuda_device)
    ws = torch.zeros(api.workspace_bytes(n, L, N) // 8 + 1, dtype=torch.float64,
                     device=cuda_device)
    assert api.device_invert(n, L, dA.data_ptr(), N, dtau.data_ptr(), ws.data_ptr()) == 0
    torch.cuda.synchronize()
    info = int(ws.view(torch.int32)[0].item())
    assert info >= 0x7f7f7f7f, (info, plan)
    assert block_residual_colmajor(torch, diag, sub, dA, N) < 1e-13
    Xd = from_device_colmajor(dA, N)
    assert rel_fro(Xd, Xr) < tol, (tuned, plan)


def test_c5_largest_serving_size_residual(cuda_device):
    """n = 576, p = 80, U = 6: one 17 GB inversion on the device."""
    import torch
    side, L, U = 24, 80, 6.0
    n = side * side
    N = n * L
    assert N == 46080
    diag, sub = _hubbard_blocks(side, L, U, 5)
    dA = pcyclic_device(torch, diag, sub, N, cuda_device)
    dtau = torch.zeros(N, dtype=torch.float64, device=cuda_device)
    ws = torch.zeros(api.workspace_bytes(n, L, N) // 8 + 1, dtype=torch.float64,
                     device=cuda_device)
    assert api.device_invert(n, L, dA.data_ptr(), N, dtau.data_ptr(), ws.data_ptr()) == 0
    torch.cuda.synchronize()
    assert int(ws.view(torch.int32)[0].item()) >= 0x7f7f7f7f
    assert bool(torch.isfinite(dA[:, :N]).all())
    assert block_residual_colmajor(torch, diag, sub, dA, N) < 1e-13
    del dA, ws
    torch.cuda.empty_cache()


def test_c5_block_size_576_vs_reference(cuda_device):
    """The largest serving block size (8-wide leaves, 1152-row panels) at
    p = 10 against the reference's state and inverse."""
    import torch
    side, L, U = 24, 10, 6.0
    n = side * side
    N = n * L
    M = hubbard_matrix(side, L, U, seed=6)
    Ar, taur, Xr = _reference(M, n, L)
    tol = inverse_tolerance(M, Xr)
    X, state, tau, info = api.invert(M, n, L)
    assert info == 0
    np.testing.assert_allclose(tau, taur, rtol=0, atol=1e-11)
    up, refl = split_state(state, n, L)
    rup, rrefl = split_state(Ar, n, L)
    assert rel_fro(up, rup) < tol
    assert np.abs(refl - rrefl).max() < 1e-10
    assert det_sign(state, tau) == det_sign(Ar, taur)
    assert rel_fro(X, Xr) < tol
    dA = to_device_colmajor(torch, M, ld=N, device=cuda_device)
    dtau = torch.zeros(N, dtype=torch.float64, device=cuda_device)
    ws = torch.zeros(api.workspace_bytes(n, L, N) // 8 + 1, dtype=torch.float64,
                     device=cuda_device)
    assert api.device_invert(n, L, dA.data_ptr(), N, dtau.data_ptr(), ws.data_ptr()) == 0
    torch.cuda.synchronize()
    assert rel_fro(from_device_colmajor(dA, N), Xr) < tol


def c3_specs(count=256, seed=2024):
    """The batched configuration: side in {8,10,12,14,16}, p uniform in
    [8, 64], U uniform in [2, 6], one seed per walker."""
    rng = np.random.default_rng(seed)
    return [(int(rng.choice([8, 10, 12, 14, 16])), int(rng.integers(8, 65)),
             float(rng.uniform(2.0, 6.0)), 40000 + i) for i in range(count)]


def test_c3_256_instances_one_batched_call(cuda_device):
    import torch
    specs = c3_specs()
    ns, Ls, lds, bufs, taus, blocks = [], [], [], [], [], []
    for side, L, U, seed in specs:
        n = side * side
        N = n * L
        ld = (N + 31) // 32 * 32
        d, s = _hubbard_blocks(side, L, U, seed)
        bufs.append(pcyclic_device(torch, d, s, ld, cuda_device))
        taus.append(torch.zeros(N, dtype=torch.float64, device=cuda_device))
        blocks.append((d, s))
        ns.append(n)
        Ls.append(L)
        lds.append(ld)
    ws = torch.zeros(api.batch_workspace_bytes(ns, Ls, lds) // 8 + 1, dtype=torch.float64,
                     device=cuda_device)
    rc = api.device_invert_batched(ns, Ls, [b.data_ptr() for b in bufs], lds,
                                   [t.data_ptr() for t in taus], ws.data_ptr(), 8, 0)
    torch.cuda.synchronize()
    assert rc == 0
    worst = 0.0
    for (d, s), b, n, L in zip(blocks, bufs, ns, Ls):
        r = block_residual_colmajor(torch, d, s, b, n * L)
        worst = max(worst, r)
    assert worst < 1e-13, worst
    # 16 instances (the smallest, where the reference is quickest) against
    # the reference's CPU path.
    order = sorted(range(len(specs)), key=lambda i: ns[i] * Ls[i])[:12] + \
        sorted(range(len(specs)), key=lambda i: -ns[i] * Ls[i])[:4]
    for i in order:
        side, L, U, seed = specs[i]
        n = side * side
        M = hubbard_matrix(side, L, U, seed=seed)
        _, taur, Xr = _reference(M, n, L)
        X = from_device_colmajor(bufs[i], n * L)
        assert rel_fro(X, Xr) < inverse_tolerance(M, Xr), specs[i]
        np.testing.assert_allclose(taus[i].cpu().numpy(), taur, rtol=0, atol=1e-10)
