"""Storage-sharded inversion (bsofi_shard_*, bsofi_b200/shard.py) on one GPU.

Every rank's kernels run in turn on this GPU (shard.storage_sharded_local:
the compact factorization, each rank's block columns of R^{-1}, the
exchange of the same blocks by local copies, each rank's BSOI rows).  The
composed M^{-1} is checked against the ordinary single-GPU inversion and,
at small N, the reference's CPU path; the compact factorization's tau and
log-determinant against the ordinary layout's (bitwise: the same BSOF
kernel arithmetic on the same values, only the addresses differ)."""
import numpy as np
import pytest

import oracle
from bsofi_b200 import api, shard
from bsofi_b200.hubbard import (expm_sym, hubbard_blocks, hubbard_matrix, lattice_adjacency,
                                pcyclic_blocks, random_pcyclic)
from conftest import EPS, inverse_tolerance, rel_fro, residual
from gpu_util import (block_residual_colmajor, from_device_colmajor, pcyclic_device,
                      to_device_colmajor)

pytestmark = pytest.mark.gpu


def _packed(torch, blocks, dev):
    """(L, n, n) row-major numpy blocks -> device buffer of L column-major blocks."""
    return torch.from_numpy(np.ascontiguousarray(np.transpose(blocks, (0, 2, 1)))).to(dev)


def _single(torch, dA, n, L, dev):
    """The ordinary single-GPU path on the device matrix dA (ld N), in place:
    returns (tau, [sign, log|det|])."""
    N = n * L
    dtau = torch.zeros(N, dtype=torch.float64, device=dev)
    ws = torch.empty(api.workspace_bytes(n, L, N), dtype=torch.uint8, device=dev)
    assert api.device_bsoftri(n, L, dA.data_ptr(), N, dtau.data_ptr(), ws.data_ptr(), 0) == 0
    out = torch.empty(2, dtype=torch.float64, device=dev)
    assert api.device_logdet(n, L, dA.data_ptr(), N, dtau.data_ptr(), True, out.data_ptr()) == 0
    assert api.device_bsoi(n, L, dA.data_ptr(), N, dtau.data_ptr(), ws.data_ptr(), 0) == 0
    torch.cuda.synchronize()
    return dtau, out


def _compose(torch, bands, N, dev):
    Xc = torch.full((N, N), float("nan"), dtype=torch.float64, device=dev)
    for r0, r1, band in bands:
        Xc[:, r0:r1] = band
    return Xc


@pytest.mark.parametrize("n,L,world,kind", [(64, 16, 2, "hub"), (100, 12, 3, "rand"),
                                            (33, 9, 2, "rand"), (17, 5, 8, "rand"),
                                            (256, 32, 4, "hub"), (400, 8, 3, "rand"),
                                            (8, 2, 2, "rand")])
def test_storage_sharded_matches_single_gpu(cuda_device, n, L, world, kind):
    import torch
    N = n * L
    M = hubbard_matrix(int(round(n ** 0.5)), L, 4.0, seed=n + L) if kind == "hub" else \
        random_pcyclic(n, L, seed=500 + n + L)
    diag, sub = pcyclic_blocks(M, n, L)
    dD = _packed(torch, diag, cuda_device)
    dS = _packed(torch, sub, cuda_device)
    bands, rc, info = shard.storage_sharded_local(n, L, dD.data_ptr(), dS.data_ptr(), world)
    assert rc == 0 and info == 0
    torch.cuda.synchronize()
    covered = sorted((r0, r1) for r0, r1, _ in bands)
    assert covered == shard.bsoi_row_bands(n, L, world)
    Xc = _compose(torch, bands, N, cuda_device)
    assert not torch.isnan(Xc).any()
    dA = to_device_colmajor(torch, M, device=cuda_device)
    _single(torch, dA, n, L, cuda_device)
    X = from_device_colmajor(Xc, N)
    Xs = from_device_colmajor(dA, N)
    assert rel_fro(X, Xs) < inverse_tolerance(M, Xs)
    assert block_residual_colmajor(torch, diag, sub, Xc, N) < 1e-13
    if N <= 1500 and oracle.ref_available():
        Xr = oracle.ref_inverse(M, n, L)
        assert rel_fro(X, Xr) < inverse_tolerance(M, Xr)
        assert residual(M, X) < 1e-13


@pytest.mark.parametrize("n,L", [(64, 16), (256, 8), (400, 6), (36, 20)])
def test_compact_state_matches_ordinary_layout(cuda_device, n, L):
    """tau and sign/log|det M| from the compact factorization equal the
    ordinary path's bitwise; packed and Hubbard inputs give the same state."""
    import torch
    side = int(round(n ** 0.5))
    U, dtau_q, seed = 4.0, 0.125, 7 + n
    M = hubbard_matrix(side, L, U, dtau=dtau_q, seed=seed)
    diag, sub = pcyclic_blocks(M, n, L)
    # The generator's own draw of the fields and of expm(dtau t K).
    h = np.random.default_rng(seed).choice(np.array([-1.0, 1.0]), size=(L, n))
    lam = np.arccosh(np.exp(U * dtau_q / 2.0))
    expk = expm_sym(dtau_q * lattice_adjacency(side))
    dtau, ld_single = _single(torch, to_device_colmajor(torch, M, device=cuda_device), n, L,
                              cuda_device)
    dD = _packed(torch, diag, cuda_device)
    dS = _packed(torch, sub, cuda_device)
    state = torch.empty(api.shard_state_bytes(n, L), dtype=torch.uint8, device=cuda_device)
    assert api.shard_factor(n, L, dD.data_ptr(), dS.data_ptr(), state.data_ptr()) == 0
    assert api.shard_info(state, n, L) == 0
    tau_ptr = api.load().bsofi_shard_tau(state.data_ptr(), n, L)
    off = (tau_ptr - state.data_ptr()) // 8
    tau = state.view(torch.float64)[off:off + n * L].clone()
    out = torch.empty(2, dtype=torch.float64, device=cuda_device)
    assert api.shard_logdet(n, L, state.data_ptr(), out.data_ptr()) == 0
    torch.cuda.synchronize()
    assert torch.equal(tau, dtau)
    assert torch.equal(out, ld_single)
    # Hubbard input straight from expm(K) and the fields.
    dE = torch.from_numpy(np.ascontiguousarray(expk.T)).to(cuda_device)
    dh = torch.from_numpy(np.ascontiguousarray(h)).to(cuda_device)
    state2 = torch.empty_like(state)
    assert api.shard_hubbard_factor(n, L, dE.data_ptr(), dh.data_ptr(), lam,
                                    state2.data_ptr()) == 0
    assert api.shard_info(state2, n, L) == 0
    tau2 = state2.view(torch.float64)[off:off + n * L]
    assert torch.allclose(tau2, tau, rtol=1e-13, atol=1e-15)


def test_storage_sharded_over_a_process_group(cuda_device):
    """storage_sharded_invert over a one-rank NCCL group (the all-to-all and
    the status all-reduce through NCCL) gives the local emulation's rows."""
    import os
    import socket
    import torch
    import torch.distributed as dist
    if dist.is_initialized():
        pytest.skip("a process group is already initialised")
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    n, L = 100, 10
    M = random_pcyclic(n, L, seed=77)
    diag, sub = pcyclic_blocks(M, n, L)
    dD = _packed(torch, diag, cuda_device)
    dS = _packed(torch, sub, cuda_device)
    import datetime
    dist.init_process_group("nccl", rank=0, world_size=1, timeout=datetime.timedelta(seconds=60))
    try:
        res = shard.storage_sharded_invert(n, L, dD.data_ptr(), dS.data_ptr())
        torch.cuda.synchronize()
    finally:
        dist.destroy_process_group()
    assert res.rc == 0 and res.info == 0 and not res.failed
    assert res.rows == (0, n * L)
    bands, rc, info = shard.storage_sharded_local(n, L, dD.data_ptr(), dS.data_ptr(), 1)
    assert rc == 0 and info == 0
    assert torch.equal(res.band, bands[0][2])


def test_storage_sharded_c4_four_ranks(cuda_device):
    """C4 (n = 400, p = 64, U = 6, N = 25600) split over four emulated
    ranks: within the condition-relative tolerance of the single-GPU
    inverse, block residual at the FP64 level; no rank's slab or band
    reaches the N^2 doubles one GPU holds in the ordinary layout."""
    import torch
    n, L, world = 400, 64, 4
    N = n * L
    B = hubbard_blocks(20, L, 6.0, seed=4)
    diag = np.broadcast_to(np.eye(n), (L, n, n)).copy()
    sub = -B
    sub[L - 1] = B[L - 1]
    dD = _packed(torch, diag, cuda_device)
    dS = _packed(torch, sub, cuda_device)
    for c0, c1 in shard.column_slabs(L, world):
        assert c1 * (c1 - c0) * n * n < N * N / 2
    bands, rc, info = shard.storage_sharded_local(n, L, dD.data_ptr(), dS.data_ptr(), world)
    assert rc == 0 and info == 0
    torch.cuda.synchronize()
    Xc = _compose(torch, bands, N, cuda_device)
    del bands
    assert block_residual_colmajor(torch, diag, sub, Xc, N) < 1e-13
    dA = pcyclic_device(torch, diag, sub, N, cuda_device)
    _single(torch, dA, n, L, cuda_device)
    nx = float(torch.linalg.norm(dA))
    nm = float(np.sqrt((diag ** 2).sum() + (sub ** 2).sum()))
    tol = max(1e-13, 8.0 * np.sqrt(N) * (nm * nx / N) * EPS)
    diff = float(torch.linalg.norm(Xc - dA)) / nx
    assert diff < tol
