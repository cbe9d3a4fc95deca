"""DQMC producer/consumer entry points on the device (bsofi_device_assemble,
bsofi_device_hubbard_assemble, bsofi_device_logdet) through the C ABI.

Checks: the assembled p-cyclic blocks equal the host generator's (bitwise
for packed blocks, within 1e-15 relative for the Hubbard exponentials); an
inversion of the assembled matrix, whose unread blocks hold NaN, matches the
handle API on the dense matrix within the parity tolerance; sign(det M) is
exact and log|det M| within 1e-12 relative of numpy's slogdet, and equals the
reference example's sign formula when N is even.
"""
import numpy as np
import pytest

from bsofi_b200 import api
from bsofi_b200.hubbard import (expm_sym, hubbard_matrix, lattice_adjacency, pcyclic_blocks,
                                random_pcyclic)
from conftest import det_sign, inverse_tolerance, rel_fro
from gpu_util import from_device_colmajor

pytestmark = pytest.mark.gpu


def _packed(torch, blocks, dev):
    """(L, n, n) row-major numpy blocks -> device buffer of L column-major blocks."""
    return torch.from_numpy(np.ascontiguousarray(np.transpose(blocks, (0, 2, 1)))).to(dev)


def _pcyclic_view(A, n, L):
    d, s = pcyclic_blocks(A, n, L)
    return d, s


def _invert_on_device(torch, dA, n, L, ldd, dev):
    dtau = torch.zeros(n * L, dtype=torch.float64, device=dev)
    ws = torch.empty(api.workspace_bytes(n, L, ldd), dtype=torch.uint8, device=dev)
    assert api.device_invert(n, L, dA.data_ptr(), ldd, dtau.data_ptr(), ws.data_ptr()) == 0
    torch.cuda.synchronize()
    return dtau


@pytest.mark.parametrize("n,L", [(1, 2), (7, 3), (16, 6), (33, 5)])
def test_assemble_packed_blocks(cuda_device, n, L):
    torch = pytest.importorskip("torch")
    M = random_pcyclic(n, L, seed=31 * n + L)
    diag, sub = pcyclic_blocks(M, n, L)
    N = n * L
    ldd = N + 3
    dA = torch.full((N, ldd), float("nan"), dtype=torch.float64, device=cuda_device)
    dD = _packed(torch, diag, cuda_device)
    dS = _packed(torch, sub, cuda_device)
    assert api.device_assemble(n, L, dD.data_ptr(), dS.data_ptr(), dA.data_ptr(), ldd) == 0
    torch.cuda.synchronize()
    A = from_device_colmajor(dA, N)
    d2, s2 = _pcyclic_view(A, n, L)
    np.testing.assert_array_equal(d2, diag)
    np.testing.assert_array_equal(s2, sub)
    # Every block off the p-cyclic pattern still holds NaN, except the ones
    # zeroed for the factorization; the inversion must not read any of them.
    _invert_on_device(torch, dA, n, L, ldd, cuda_device)
    X = from_device_colmajor(dA, N)
    Xh, _, _, info = api.invert(M, n, L)
    assert info == 0
    assert np.isfinite(X).all()
    assert rel_fro(X, Xh) < inverse_tolerance(M, Xh)


def test_assemble_identity_diagonal(cuda_device):
    torch = pytest.importorskip("torch")
    n, L = 9, 4
    M = hubbard_matrix(3, L, 4.0, seed=5)
    _, sub = pcyclic_blocks(M, n, L)
    N = n * L
    dA = torch.zeros((N, N), dtype=torch.float64, device=cuda_device)
    dS = _packed(torch, sub, cuda_device)
    assert api.device_assemble(n, L, 0, dS.data_ptr(), dA.data_ptr(), N) == 0
    torch.cuda.synchronize()
    np.testing.assert_array_equal(from_device_colmajor(dA, N), M)


@pytest.mark.parametrize("side,L,U,seed", [(2, 2, 4.0, 0), (4, 8, 4.0, 1), (6, 10, 6.0, 2)])
def test_hubbard_assemble_matches_generator(cuda_device, side, L, U, seed):
    torch = pytest.importorskip("torch")
    dtau = 0.125
    n, N = side * side, side * side * L
    M = hubbard_matrix(side, L, U, dtau=dtau, seed=seed)
    # The generator's own draw of the fields and of expm(dtau t K).
    h = np.random.default_rng(seed).choice(np.array([-1.0, 1.0]), size=(L, n))
    lam = np.arccosh(np.exp(U * dtau / 2.0))
    E = expm_sym(dtau * lattice_adjacency(side))
    dE = torch.from_numpy(np.ascontiguousarray(E.T)).to(cuda_device)
    dh = torch.from_numpy(np.ascontiguousarray(h)).to(cuda_device)
    dA = torch.zeros((N, N), dtype=torch.float64, device=cuda_device)
    assert api.device_hubbard_assemble(n, L, dE.data_ptr(), dh.data_ptr(), lam, dA.data_ptr(),
                                       N) == 0
    torch.cuda.synchronize()
    A = from_device_colmajor(dA, N)
    np.testing.assert_allclose(A, M, rtol=1e-15, atol=0)


def _logdet_device(torch, dA, n, L, ldd, dtau, inverted, dev):
    out = torch.full((2,), 7.0, dtype=torch.float64, device=dev)
    assert api.device_logdet(n, L, dA.data_ptr(), ldd, dtau.data_ptr(), inverted,
                             out.data_ptr()) == 0
    torch.cuda.synchronize()
    return out.cpu().numpy()


@pytest.mark.parametrize("inverted", [0, 1])
def test_logdet_synthetic_diagonal(cuda_device, inverted):
    torch = pytest.importorskip("torch")
    rng = np.random.default_rng(3)
    n, L = 50, 41  # N = 2050 > 1024 threads: every thread takes several entries
    N = n * L
    d = rng.uniform(0.5, 2.0, N) * rng.choice([-1.0, 1.0], N)
    tau = rng.uniform(1.0, 2.0, N)
    tau[rng.choice(N, 17, replace=False)] = 0.0
    A = np.zeros((N, N))
    A[np.arange(N), np.arange(N)] = d
    dA = torch.from_numpy(np.ascontiguousarray(A.T)).to(cuda_device)
    dt = torch.from_numpy(tau).to(cuda_device)
    sign, logabs = _logdet_device(torch, dA, n, L, N, dt, inverted, cuda_device)
    nflip = int((tau != 0).sum() + (d < 0).sum())
    assert sign == (-1.0 if nflip % 2 else 1.0)
    want = np.log(np.abs(d)).sum() * (-1.0 if inverted else 1.0)
    assert abs(logabs - want) <= 1e-12 * max(1.0, abs(want))
    # An exactly zero diagonal entry: sign 0, log|det| = -inf.
    A[5, 5] = 0.0
    dA = torch.from_numpy(np.ascontiguousarray(A.T)).to(cuda_device)
    sign, logabs = _logdet_device(torch, dA, n, L, N, dt, inverted, cuda_device)
    assert sign == 0.0 and np.isneginf(logabs)


@pytest.mark.parametrize("case", [("hubbard", 4, 8), ("hubbard", 8, 16), ("random", 5, 3),
                                  ("random", 16, 4)])
def test_logdet_after_bsoftri(cuda_device, case):
    torch = pytest.importorskip("torch")
    kind, a, L = case
    if kind == "hubbard":
        M, n = hubbard_matrix(a, L, 4.0, seed=11), a * a
    else:
        M, n = random_pcyclic(a, L, seed=9), a
    N = n * L
    dA = torch.from_numpy(np.ascontiguousarray(M.T)).to(cuda_device)
    dtau = torch.zeros(N, dtype=torch.float64, device=cuda_device)
    ws = torch.empty(api.workspace_bytes(n, L, N), dtype=torch.uint8, device=cuda_device)
    assert api.device_bsoftri(n, L, dA.data_ptr(), N, dtau.data_ptr(), ws.data_ptr()) == 0
    torch.cuda.synchronize()
    sign, logabs = _logdet_device(torch, dA, n, L, N, dtau, 1, cuda_device)
    s_ref, l_ref = np.linalg.slogdet(M)
    assert sign == s_ref
    assert abs(logabs - l_ref) <= 1e-12 * max(1.0, abs(l_ref))
    if N % 2 == 0:
        state = from_device_colmajor(dA, N)
        assert sign == det_sign(state, dtau.cpu().numpy())
