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


def test_grouped_bsoi_matches_per_instance(cuda_device):
    """With bsofi_device_set_batch_grouped(1) FP64 batches run BSOI as one
    grouped persistent launch per tile shape (64 x 64 for 2n not a multiple
    of 128, 128 x 128 otherwise; at most 256 instances per launch).  300
    instances of mixed sizes (so both tile shapes and two launches of the
    64 x 64 shape) against the same batch with each instance's BSOI launched
    on its own (the default): equal within the FP64 tolerance, with small
    residuals."""
    import torch
    from gpu_util import from_device_colmajor, to_device_colmajor
    lib = api.load()
    rng = np.random.default_rng(123)
    specs = [(int(rng.choice([8, 12, 16, 20, 32, 64, 17])), int(rng.integers(2, 9)))
             for _ in range(300)]
    mats = [random_pcyclic(n, L, seed=1000 + i) for i, (n, L) in enumerate(specs)]
    ns = [n for n, _ in specs]
    Ls = [L for _, L in specs]
    lds = [n * L + (i % 3) for i, (n, L) in enumerate(specs)]

    def run(grouped):
        lib.bsofi_device_set_batch_grouped(grouped)
        try:
            dA = [to_device_colmajor(torch, M, ld=ld, device=cuda_device)
                  for M, ld in zip(mats, lds)]
            dtau = [torch.zeros(n * L, dtype=torch.float64, device=cuda_device) for n, L in specs]
            ws = torch.zeros(api.batch_workspace_bytes(ns, Ls, lds) // 8 + 1, dtype=torch.float64,
                             device=cuda_device)
            rc = api.device_invert_batched(ns, Ls, [t.data_ptr() for t in dA], lds,
                                           [t.data_ptr() for t in dtau], ws.data_ptr(), streams=8)
            torch.cuda.synchronize()
            assert rc == 0
            return [from_device_colmajor(A, n * L) for A, (n, L) in zip(dA, specs)]
        finally:
            lib.bsofi_device_set_batch_grouped(0)

    Xg = run(1)
    Xp = run(0)
    for M, a, b in zip(mats, Xg, Xp):
        assert rel_fro(a, b) < inverse_tolerance(M, b)
        assert residual(M, a) < 1e-13


@pytest.mark.parametrize("precision", [0, 1])
def test_chain_gate_gives_the_same_results(cuda_device, precision):
    """bsofi_device_set_batch_chains(k) only orders the instances'
    factorization chains (event waits between instances): the same kernels
    run on the same data, so the results are bitwise those of the ungated
    batch."""
    import torch
    from gpu_util import to_device_colmajor
    lib = api.load()
    rng = np.random.default_rng(321)
    specs = [(int(rng.choice([16, 36, 64, 100, 144])), int(rng.integers(3, 12))) for _ in range(40)]
    mats = [random_pcyclic(n, L, seed=2000 + i) for i, (n, L) in enumerate(specs)]
    ns = [n for n, _ in specs]
    Ls = [L for _, L in specs]
    lds = [n * L for n, L in specs]

    def run(chains):
        lib.bsofi_device_set_batch_pipelined(0)  # the gate orders the one-stream pipelines
        lib.bsofi_device_set_batch_chains(chains)
        try:
            dA = [to_device_colmajor(torch, M, device=cuda_device) for M in mats]
            dtau = [torch.zeros(n * L, dtype=torch.float64, device=cuda_device) for n, L in specs]
            nb = api.batch_workspace_bytes(ns, Ls, lds, precision=precision)
            ws = torch.zeros(nb // 8 + 1, dtype=torch.float64, device=cuda_device)
            rc = api.device_invert_batched(ns, Ls, [t.data_ptr() for t in dA], lds,
                                           [t.data_ptr() for t in dtau], ws.data_ptr(),
                                           streams=8, precision=precision)
            torch.cuda.synchronize()
            assert rc == 0
            return dA, dtau
        finally:
            lib.bsofi_device_set_batch_chains(0)
            lib.bsofi_device_set_batch_pipelined(1)

    Ag, tg = run(3)
    Au, tu = run(0)
    for a, b in zip(Ag, Au):
        assert torch.equal(a, b)
    for a, b in zip(tg, tu):
        assert torch.equal(a, b)
    for M, A, (n, L) in zip(mats[:5], Ag[:5], specs[:5]):
        X = A[:, :n * L].T.cpu().numpy()
        assert residual(M, X) < (1e-13 if precision == 0 else 1e-12)


@pytest.mark.parametrize("precision", [0, 1])
def test_pipelined_batch_matches_default(cuda_device, precision):
    """Pipelined batches (the default: chains on high-priority streams,
    BSTRI/BSOI as per-step launches) against bsofi_device_set_batch_pipelined(0)
    (each instance on one stream, persistent GEMMs): each instance's inverse
    agrees within the FP64 tolerance (the per-step and persistent GEMMs may
    differ in rounding), tau bitwise (the same BSOF); and the pipelined batch
    captured into a CUDA graph replays to the same results."""
    import torch
    from gpu_util import from_device_colmajor, to_device_colmajor
    lib = api.load()
    rng = np.random.default_rng(654)
    specs = [(int(rng.choice([16, 36, 64, 100, 144, 256])), int(rng.integers(3, 14)))
             for _ in range(30)]
    mats = [random_pcyclic(n, L, seed=3000 + i) for i, (n, L) in enumerate(specs)]
    ns = [n for n, _ in specs]
    Ls = [L for _, L in specs]
    lds = [n * L for n, L in specs]

    def buffers():
        dA = [to_device_colmajor(torch, M, device=cuda_device) for M in mats]
        dtau = [torch.zeros(n * L, dtype=torch.float64, device=cuda_device) for n, L in specs]
        nb = api.batch_workspace_bytes(ns, Ls, lds, precision=precision)
        ws = torch.zeros(nb // 8 + 1, dtype=torch.float64, device=cuda_device)
        return dA, dtau, ws

    def run(pipelined):
        lib.bsofi_device_set_batch_pipelined(pipelined)
        try:
            dA, dtau, ws = buffers()
            rc = api.device_invert_batched(ns, Ls, [t.data_ptr() for t in dA], lds,
                                           [t.data_ptr() for t in dtau], ws.data_ptr(),
                                           streams=8, precision=precision)
            torch.cuda.synchronize()
            assert rc == 0
            return dA, dtau
        finally:
            lib.bsofi_device_set_batch_pipelined(1)

    Ap, tp = run(1)
    Ad, td = run(0)
    for M, a, b, (n, L) in zip(mats, Ap, Ad, specs):
        Xa = from_device_colmajor(a, n * L)
        Xb = from_device_colmajor(b, n * L)
        assert rel_fro(Xa, Xb) < max(inverse_tolerance(M, Xb), 1e-13 if precision == 0 else 1e-12)
    for a, b in zip(tp, td):
        assert torch.equal(a, b)
    if precision == 0:
        lib.bsofi_device_set_batch_pipelined(1)
        try:
            pristine = [to_device_colmajor(torch, M, device=cuda_device) for M in mats]
            dA, dtau, ws = buffers()
            g = api.BatchGraph(ns, Ls, [t.data_ptr() for t in dA], lds,
                               [t.data_ptr() for t in dtau], ws.data_ptr(), streams=8)
        finally:
            lib.bsofi_device_set_batch_pipelined(1)
        stream = torch.cuda.Stream()
        for w, p0 in zip(dA, pristine):
            w.copy_(p0)
        torch.cuda.synchronize()
        assert g.launch(stream.cuda_stream) == 0
        stream.synchronize()
        for a, b in zip(dA, Ap):
            assert torch.equal(a, b)
        g.close()
