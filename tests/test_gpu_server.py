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
            srv.submit(2, 4, buf.data_ptr(), 8, buf.data_ptr(), precision=1)
