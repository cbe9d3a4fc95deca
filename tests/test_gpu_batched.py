"""Batched inversion (bsofi_device_invert_batched) against single inversions."""
import numpy as np
import pytest

from bsofi_b200 import api
from bsofi_b200.hubbard import hubbard_matrix, random_pcyclic
from conftest import inverse_tolerance, rel_fro, residual

pytestmark = pytest.mark.gpu


def test_batched_matches_single(cuda_device):
    import torch
    from gpu_util import from_device_colmajor, to_device_colmajor
    specs = [(64, 8, "hub", 3), (100, 5, "hub", 4), (36, 12, "rand", 5), (144, 3, "hub", 6),
             (17, 9, "rand", 7), (256, 4, "hub", 8), (49, 2, "hub", 9), (289, 3, "hub", 10),
             (450, 2, "rand", 11)]
    mats = []
    for n, L, kind, seed in specs:
        if kind == "hub":
            mats.append(hubbard_matrix(int(round(n ** 0.5)), L, 4.0, seed=seed))
        else:
            mats.append(random_pcyclic(n, L, seed=seed))
    ns = [sp[0] for sp in specs]
    Ls = [sp[1] for sp in specs]
    ldds = [n * L + (2 if i % 2 else 0) for i, (n, L) in enumerate(zip(ns, Ls))]
    dA = [to_device_colmajor(torch, M, ld=ld) for M, ld in zip(mats, ldds)]
    dtau = [torch.zeros(n * L, dtype=torch.float64, device=cuda_device) for n, L in zip(ns, Ls)]
    ws = torch.zeros(api.batch_workspace_bytes(ns, Ls, ldds) // 8 + 1, dtype=torch.float64,
                     device=cuda_device)
    rc = api.device_invert_batched(ns, Ls, [t.data_ptr() for t in dA], ldds,
                                   [t.data_ptr() for t in dtau], ws.data_ptr(), streams=3)
    torch.cuda.synchronize()
    assert rc == 0
    for M, n, L, A, tau in zip(mats, ns, Ls, dA, dtau):
        X = from_device_colmajor(A, n * L)
        Xs, _, taus, info = api.invert(M, n, L)
        assert info == 0
        assert rel_fro(X, Xs) < inverse_tolerance(M, Xs)
        np.testing.assert_allclose(tau.cpu().numpy(), taus, rtol=0, atol=1e-12)
        assert residual(M, X) < 1e-13


def test_batched_rejects_bad_sizes(cuda_device):
    rc = api.device_invert_batched([0], [4], [16], [4], [16], 16)
    assert rc == -1


def test_batch_graph_replays_match_direct(cuda_device):
    """A batch captured into a CUDA graph and replayed twice (inputs refilled
    between replays) gives the direct batched call's results."""
    import torch
    from gpu_util import from_device_colmajor, to_device_colmajor
    specs = [(64, 6, 11), (81, 4, 12), (144, 5, 13), (256, 3, 14), (16, 10, 15)]
    mats = [hubbard_matrix(int(round(n ** 0.5)), L, 4.0, seed=s) for n, L, s in specs]
    ns = [sp[0] for sp in specs]
    Ls = [sp[1] for sp in specs]
    ldds = [n * L for n, L in zip(ns, Ls)]
    pristine = [to_device_colmajor(torch, M) for M in mats]
    direct = [p.clone() for p in pristine]
    work = [torch.empty_like(p) for p in pristine]
    taus_d = [torch.zeros(n * L, dtype=torch.float64, device=cuda_device) for n, L in zip(ns, Ls)]
    taus_g = [torch.zeros(n * L, dtype=torch.float64, device=cuda_device) for n, L in zip(ns, Ls)]
    nbytes = api.batch_workspace_bytes(ns, Ls, ldds)
    ws_d = torch.zeros(nbytes // 8 + 1, dtype=torch.float64, device=cuda_device)
    ws_g = torch.zeros(nbytes // 8 + 1, dtype=torch.float64, device=cuda_device)
    rc = api.device_invert_batched(ns, Ls, [t.data_ptr() for t in direct], ldds,
                                   [t.data_ptr() for t in taus_d], ws_d.data_ptr(), streams=4)
    torch.cuda.synchronize()
    assert rc == 0
    g = api.BatchGraph(ns, Ls, [t.data_ptr() for t in work], ldds,
                       [t.data_ptr() for t in taus_g], ws_g.data_ptr(), streams=4)
    stream = torch.cuda.Stream()
    for _ in range(2):
        for w, p in zip(work, pristine):
            w.copy_(p)
        torch.cuda.synchronize()
        assert g.launch(stream.cuda_stream) == 0
        stream.synchronize()
        for M, n, L, A, D in zip(mats, ns, Ls, work, direct):
            X = from_device_colmajor(A, n * L)
            Xd = from_device_colmajor(D, n * L)
            assert rel_fro(X, Xd) < inverse_tolerance(M, Xd)
            assert residual(M, X) < 1e-13
    g.close()
