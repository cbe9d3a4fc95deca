"""Continuous-batching server: every result is the same alone and in the mix.

Requests of different sizes are submitted together to a server whose
workspace pool is deliberately small, so admission by memory footprint and
slot reuse are exercised; each finished result is compared with the same
matrix inverted alone through bsofi_device_invert.
"""
import numpy as np
import pytest

from bsofi_b200 import api
from bsofi_b200.hubbard import hubbard_matrix, random_pcyclic
from conftest import inverse_tolerance, rel_fro, residual

pytestmark = pytest.mark.gpu


def _alone(torch, M, n, L, dev):
    from gpu_util import from_device_colmajor, to_device_colmajor
    ld = n * L
    dA = to_device_colmajor(torch, M, ld=ld, device=dev)
    dtau = torch.zeros(n * L, dtype=torch.float64, device=dev)
    ws = torch.zeros(api.workspace_bytes(n, L, ld) // 8 + 1, dtype=torch.float64, device=dev)
    assert api.device_invert(n, L, dA.data_ptr(), ld, dtau.data_ptr(), ws.data_ptr(), 0) == 0
    torch.cuda.synchronize()
    return from_device_colmajor(dA, n * L)


def test_server_results_match_alone(cuda_device):
    import time
    import torch
    from gpu_util import from_device_colmajor, to_device_colmajor
    specs = [(64, 8, "hub", 1), (100, 12, "hub", 2), (36, 20, "rand", 3), (144, 6, "hub", 4),
             (25, 33, "rand", 5), (196, 4, "hub", 6), (64, 16, "hub", 7), (81, 9, "hub", 8),
             (12, 50, "rand", 9), (256, 3, "hub", 10), (324, 4, "hub", 11), (400, 3, "rand", 12)]
    mats = [hubbard_matrix(int(round(n ** 0.5)), L, 3.0, seed=s) if k == "hub"
            else random_pcyclic(n, L, seed=s) for n, L, k, s in specs]
    sizes = [api.server_request_bytes(n, L, n * L) for n, L, _, _ in specs]
    pool = 2 * max(sizes) + 4096  # at most a few requests fit at once
    dAs, dtaus, ids = [], [], {}
    with api.Server(slots=4, pool_bytes=pool) as srv:
        for i, ((n, L, _, _), M) in enumerate(zip(specs, mats)):
            dAs.append(to_device_colmajor(torch, M, ld=n * L, device=cuda_device))
            dtaus.append(torch.zeros(n * L, dtype=torch.float64, device=cuda_device))
            ids[srv.submit(n, L, dAs[-1].data_ptr(), n * L, dtaus[-1].data_ptr())] = i
        done = {}
        t0 = time.time()
        while len(done) < len(specs) and time.time() - t0 < 120:
            for rid, st in srv.poll():
                done[rid] = st
            time.sleep(0.001)
        assert srv.pending() == 0
    assert sorted(done) == sorted(ids)
    assert all(st == 0 for st in done.values())
    for rid, i in ids.items():
        n, L, _, _ = specs[i]
        X = from_device_colmajor(dAs[i], n * L)
        Xa = _alone(torch, mats[i], n, L, cuda_device)
        assert rel_fro(X, Xa) < inverse_tolerance(mats[i], Xa)
        assert residual(mats[i], X) < 1e-13


def test_server_rejects(cuda_device):
    import torch
    with api.Server(slots=1, pool_bytes=1 << 20) as srv:
        buf = torch.zeros(16, dtype=torch.float64, device=cuda_device)
        with pytest.raises(RuntimeError):
            srv.submit(256, 32, buf.data_ptr(), 8192, buf.data_ptr())  # workspace > pool
        with pytest.raises(RuntimeError):
            srv.submit(0, 4, buf.data_ptr(), 16, buf.data_ptr())
        with pytest.raises(RuntimeError):
            srv.submit(2, 4, buf.data_ptr(), 8, buf.data_ptr(), precision=2)
        with pytest.raises(RuntimeError):  # footprint (matrix + workspace) > pool
            srv.submit_blocks(256, 32, buf.data_ptr())


def _packed_sub(torch, M, n, L, dev):
    """The L coupling blocks of a p-cyclic M, packed column-major on the device
    (block k at offset k n^2, as bsofi_device_assemble reads them)."""
    from bsofi_b200.hubbard import pcyclic_blocks
    diag, sub = pcyclic_blocks(M, n, L)
    assert np.array_equal(diag, np.broadcast_to(np.eye(n), diag.shape))
    return torch.from_numpy(np.ascontiguousarray(np.transpose(sub, (0, 2, 1)))).to(dev)


def _wait(srv, ids, timeout=300):
    import time
    done = {}
    t0 = time.time()
    while len(done) < len(ids) and time.time() - t0 < timeout:
        for rid, st in srv.poll():
            done[rid] = st
        time.sleep(0.001)
    return done


def test_server_owned_mixed_and_fp64_match_alone(cuda_device):
    """Server-owned requests at both precisions in one stream: each result
    equals the same request served alone (bitwise: the pipeline is
    deterministic), the mixed ones have ||M X - I|| / ||X|| <= 1e-12."""
    import torch
    from gpu_util import device_view, from_device_colmajor
    specs = [(64, 8, 0, 1), (100, 12, 1, 2), (144, 6, 1, 4), (196, 4, 0, 6), (64, 16, 1, 7),
             (81, 9, 0, 8), (256, 3, 1, 10), (324, 4, 1, 11), (36, 20, 0, 12), (400, 3, 1, 13)]
    mats = [hubbard_matrix(int(round(n ** 0.5)), L, 4.0, seed=s) for n, L, _, s in specs]
    packs = [_packed_sub(torch, M, n, L, cuda_device) for (n, L, _, _), M in zip(specs, mats)]
    foot = [api.server_footprint_bytes(n, L, p) for n, L, p, _ in specs]
    assert all(f > 0 for f in foot)

    def serve(idx, pool):
        """Finished results are copied out and released as they arrive: a
        result holds its pool memory until released, so a pool that fits two
        requests serves all ten only because finished ones are given back."""
        import time
        out = {}
        with api.Server(slots=4, pool_bytes=pool) as srv:
            ids = {srv.submit_blocks(specs[i][0], specs[i][1], packs[i].data_ptr(),
                                     precision=specs[i][2]): i for i in idx}
            t0 = time.time()
            while len(out) < len(ids) and time.time() - t0 < 300:
                for rid, st in srv.poll():
                    assert st == 0
                    i = ids[rid]
                    dA, ld, dtau = srv.result(rid)
                    n, L = specs[i][:2]
                    out[i] = from_device_colmajor(device_view(torch, dA, n * L, ld, cuda_device),
                                                  n * L)
                    assert srv.release(rid) == 0
                    assert srv.result(rid) is None
                time.sleep(0.001)
            assert len(out) == len(ids)
            assert srv.pending() == 0
        return out

    mix = serve(range(len(specs)), 2 * max(foot) + 4096)
    for i in range(len(specs)):
        alone = serve([i], foot[i] + 4096)[i]
        np.testing.assert_array_equal(mix[i], alone)
        n, L, prec, _ = specs[i]
        res = residual(mats[i], mix[i])
        assert res < (1e-12 if prec else 1e-13), (specs[i], res)


def test_server_owned_request_waits_for_memory(cuda_device):
    """Two requests of n = 576, L = 80 (17 GB matrix each) into a pool that
    holds one: the second is admitted only after the first's memory is
    released, then completes; the first result's residual is checked first."""
    import torch
    from bsofi_b200.hubbard import hubbard_blocks
    from gpu_util import block_residual_colmajor, device_view
    side, L = 24, 80
    n = side * side
    N = n * L
    foot = api.server_footprint_bytes(n, L, 0)
    assert foot > 17e9
    packs, blocks = [], []
    for seed in (21, 22):
        B = hubbard_blocks(side, L, 4.0, seed=seed)
        sub = -B
        sub[L - 1] = B[L - 1]
        blocks.append((np.broadcast_to(np.eye(n), (L, n, n)), sub))
        packs.append(torch.from_numpy(np.ascontiguousarray(np.transpose(sub, (0, 2, 1))))
                     .to(cuda_device))
    with api.Server(slots=2, pool_bytes=foot + foot // 2) as srv:
        a = srv.submit_blocks(n, L, packs[0].data_ptr(), precision=0)
        b = srv.submit_blocks(n, L, packs[1].data_ptr(), precision=1)
        done = _wait(srv, [a])
        assert done.get(a) == 0
        assert srv.pending() == 1  # b waits for memory, not for a slot
        for _ in range(50):
            assert b not in dict(srv.poll())
        dA, ld, _ = srv.result(a)
        assert ld >= N
        # The residual reads the result in place in the server's pool.
        assert block_residual_colmajor(torch, *blocks[0], device_view(torch, dA, N, ld,
                                                                      cuda_device), N) < 1e-13
        assert srv.release(a) == 0
        done = _wait(srv, [b])
        assert done.get(b) == 0
        dB, ld, _ = srv.result(b)
        assert block_residual_colmajor(torch, *blocks[1], device_view(torch, dB, N, ld,
                                                                      cuda_device), N) < 1e-12
        assert srv.release(b) == 0
