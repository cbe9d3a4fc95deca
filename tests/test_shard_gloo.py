"""Host logic of one inversion split over ranks by rows (bsofi_b200/shard.py)
on CPU ranks (gloo): the row bands cover every row once at tile-aligned
starts, and the all-gather of bands leaves every rank with every row."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from bsofi_b200 import shard


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


@pytest.mark.parametrize("N", [0, 1, 127, 128, 129, 1000, 8192, 25600])
@pytest.mark.parametrize("world", [1, 2, 3, 8])
def test_row_bands_cover_once_aligned(N, world):
    bands = shard.row_bands(N, world)
    assert len(bands) == world
    covered = []
    for r0, r1 in bands:
        assert 0 <= r0 <= r1 <= N
        assert r0 % 128 == 0 or r0 == N
        assert r1 % 128 == 0 or r1 == N
        covered.extend(range(r0, r1))
    assert covered == list(range(N))
    # Bands hold whole 128-row tiles (the last may be partial); their tile
    # counts differ by at most one.
    units = [(b - a + 127) // 128 for a, b in bands]
    assert max(units) - min(units) <= 1


def _worker(rank, world, port, N, ld, out):
    import torch
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    bands = shard.row_bands(N, world, align=8)
    # Column-major N x N matrix X(i, j) = 1000 j + i held as Xc[j, i]; each
    # rank starts with only its own rows set.
    Xc = torch.full((N, ld), -1.0, dtype=torch.float64)
    a, b = bands[rank]
    j = torch.arange(N, dtype=torch.float64).unsqueeze(1)
    i = torch.arange(a, b, dtype=torch.float64).unsqueeze(0)
    Xc[:, a:b] = 1000.0 * j + i
    shard.gather_rows(torch, dist, Xc, N, bands)
    out.put((rank, Xc[:, :N].numpy().copy()))
    dist.barrier()
    dist.destroy_process_group()


@pytest.mark.timeout(180)
@pytest.mark.parametrize("world,N", [(2, 40), (3, 37)])
def test_gather_rows_gives_every_rank_every_row(world, N):
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, N, N + 3, out)) for r in range(world)]
    for p in procs:
        p.start()
    got = dict(out.get(timeout=150) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    expect = 1000.0 * np.arange(N)[:, None] + np.arange(N)[None, :]
    for r in range(world):
        np.testing.assert_array_equal(got[r], expect)


def test_bsoi_rows_rejects_bad_ranges():
    """bsofi_device_bsoi_rows checks the row range before any CUDA call."""
    from bsofi_b200 import _lib
    lib = _lib.load()
    fake = 0x1000  # never dereferenced
    n, L = 4, 64   # N = 256
    for r0, r1 in [(64, 128), (0, 100), (0, 257), (128, 128), (-128, 128), (128, 0)]:
        assert lib.bsofi_device_bsoi_rows(n, L, fake, 256, fake, fake, r0, r1, None) == -1
