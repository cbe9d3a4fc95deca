"""Storage-sharded inversion (bsofi_b200/shard.py storage_sharded_invert) on
CPU: the column partition, the algebra of the split against the compiled
reference (tests/shard_emul.py restates each rank's work in numpy), and the
all-to-all of column slabs into row bands on gloo ranks."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

import oracle
import shard_emul
from bsofi_b200 import shard
from bsofi_b200.hubbard import hubbard_matrix, random_pcyclic
from conftest import inverse_tolerance, rel_fro

needs_ref = pytest.mark.skipif(not oracle.ref_available(), reason="reference library not built")


@pytest.mark.parametrize("L", [1, 2, 3, 7, 8, 64, 80, 200])
@pytest.mark.parametrize("world", [1, 2, 3, 8])
def test_column_slabs_cover_once(L, world):
    cols = shard.column_slabs(L, world)
    assert len(cols) == world
    covered = []
    for c0, c1 in cols:
        assert 0 <= c0 <= c1 <= L
        covered.extend(range(c0, c1))
    assert covered == list(range(L))
    if L >= world:
        assert all(c1 > c0 for c0, c1 in cols)
    # The largest slab, c1 (c1 - c0) blocks, stays under the N^2 / P of an
    # even split of the dense matrix (or the one block column of L blocks
    # that the last owner must hold), and well under it for larger L.
    worst = max(c1 * (c1 - c0) for c0, c1 in cols)
    assert worst <= max(L * L / world, L)
    if world >= 2 and L >= 8 * world:
        assert worst <= 0.8 * L * L / world


@pytest.mark.parametrize("n,L,world", [(256, 32, 4), (400, 64, 8), (576, 80, 8), (8, 5, 4),
                                       (100, 10, 1), (64, 16, 3)])
def test_bsoi_row_bands_cover_once_balanced(n, L, world):
    """Work-balanced BSOI bands: every row once, 128-aligned starts, and
    (with a few tiles per rank) each band's work, sum over its rows of
    2L - 2 - block row, within one tile's work of an equal share."""
    N = n * L
    bands = shard.bsoi_row_bands(n, L, world)
    covered = []
    for r0, r1 in bands:
        assert 0 <= r0 <= r1 <= N
        assert r0 % 128 == 0 or r0 == N
        assert r1 % 128 == 0 or r1 == N
        covered.extend(range(r0, r1))
    assert covered == list(range(N))
    work = [sum(2 * L - 2 - i // n for i in range(r0, r1)) for r0, r1 in bands]
    tile = 128 * (2 * L - 2)
    if N >= 4 * 128 * world:
        share = sum(work) / world
        assert max(abs(w - share) for w in work) <= tile


def _state(n, L, kind, seed):
    M = hubbard_matrix(int(round(n ** 0.5)), L, 4.0, seed=seed) if kind == "hub" else \
        random_pcyclic(n, L, seed=seed)
    A, tau, info = oracle.ref_bsof(M, n, L)
    assert info == 0
    return M, A, tau


@needs_ref
@pytest.mark.parametrize("n,L,world", [(16, 6, 2), (9, 8, 3), (8, 3, 2), (4, 2, 2), (16, 9, 8)])
def test_column_recurrence_matches_reference_bstri(n, L, world):
    """The owned block columns of every rank, put together, are the
    reference's R^{-1} (lapackXbstri after lapackXbsof)."""
    M, A, tau = _state(n, L, "hub" if n in (16, 9, 4) else "rand", 40 + n + L)
    Ar, _, info = oracle.ref_bsoftri(M, n, L)
    assert info == 0
    N = n * L
    terms = shard_emul.factor_terms(A, n, L)
    X = np.zeros((N, N))
    for c0, c1 in shard.column_slabs(L, world):
        if c1 > c0:
            X[:c1 * n, c0 * n:c1 * n] = shard_emul.bstri_columns(terms, n, L, c0, c1)
    # Compare R^{-1}'s nonzero part: the block upper triangle less the
    # strictly lower part of the diagonal blocks (reflectors in Ar).
    mask = np.zeros((N, N), dtype=bool)
    for i in range(L):
        for j in range(i, L):
            blk = np.ones((n, n), dtype=bool) if j > i else np.triu(np.ones((n, n), dtype=bool))
            mask[i * n:(i + 1) * n, j * n:(j + 1) * n] = blk
    ref = np.where(mask, Ar, 0.0)
    assert np.all(X[~mask] == 0.0)
    assert rel_fro(X, ref) < 1e-13 * max(1.0, np.linalg.cond(np.triu(A)) / 1e3)


@needs_ref
@pytest.mark.parametrize("n,L,world,align", [(16, 6, 2, 8), (9, 8, 3, 8), (8, 5, 4, 8)])
def test_split_composes_the_reference_inverse(n, L, world, align):
    """Every rank's slab, the exchange (done here by slicing) and every
    rank's BSOI rows give the reference's M^{-1}."""
    M, A, tau = _state(n, L, "hub" if n in (16, 9) else "rand", 70 + n + L)
    N = n * L
    Xr = oracle.ref_inverse(M, n, L)
    terms = shard_emul.factor_terms(A, n, L)
    cols = shard.column_slabs(L, world)
    bands = shard.row_bands(N, world, align)
    X = np.zeros((N, N))
    for c0, c1 in cols:
        if c1 > c0:
            X[:c1 * n, c0 * n:c1 * n] = shard_emul.bstri_columns(terms, n, L, c0, c1)
    Qs = shard_emul.panel_q(A, tau, n, L)
    out = np.full((N, N), np.nan)
    for r0, r1 in bands:
        if r1 > r0:
            out[r0:r1] = shard_emul.bsoi_rows(X[r0:r1].copy(), Qs, n, L)
    assert rel_fro(out, Xr) < inverse_tolerance(M, Xr)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, n, L, seed, use_ref, out):
    import torch
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        N = n * L
        cols = shard.column_slabs(L, world)
        bands = shard.row_bands(N, world, align=8)
        c0, c1 = cols[rank]
        if use_ref:
            # The whole split on this rank's share: factor terms (every rank
            # the same), its columns, the exchange, its rows.
            M, A, tau = _state(n, L, "rand", seed)
            terms = shard_emul.factor_terms(A, n, L)
            S = shard_emul.bstri_columns(terms, n, L, c0, c1) if c1 > c0 else \
                np.zeros((c1 * n, 0))
        else:
            # A known matrix: X(i, j) = 1000 j + i + 1 above the block
            # diagonal's lower edge (i < (j // n + 1) n), else 0.
            jj = np.arange(c0 * n, c1 * n)[None, :]
            ii = np.arange(c1 * n)[:, None]
            S = np.where(ii < (jj // n + 1) * n, 1000.0 * jj + ii + 1, 0.0)
        slab = torch.from_numpy(np.ascontiguousarray(S.T))   # slab[j, i] = X(i, c0 n + j)
        band = shard.columns_to_rows(torch, dist, slab, n, L, cols, bands)
        r0, r1 = bands[rank]
        B = band.numpy().T.copy()                              # (r1 - r0) x N
        if use_ref and r1 > r0:
            B = shard_emul.bsoi_rows(B, shard_emul.panel_q(A, tau, n, L), n, L)
        out.put((rank, r0, r1, B))
        dist.barrier()
    finally:
        dist.destroy_process_group()


@pytest.mark.timeout(240)
@pytest.mark.parametrize("world,n,L,use_ref", [(2, 8, 5, False), (3, 7, 6, False),
                                               (3, 8, 6, True), (4, 6, 7, True)])
def test_columns_to_rows_on_gloo_ranks(world, n, L, use_ref):
    if use_ref and not oracle.ref_available():
        pytest.skip("reference library not built")
    seed = 90 + n + L
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, n, L, seed, use_ref, out))
             for r in range(world)]
    for p in procs:
        p.start()
    got = [out.get(timeout=200) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    N = n * L
    full = np.full((N, N), np.nan)
    for _, r0, r1, B in got:
        full[r0:r1] = B
    if use_ref:
        M, _, _ = _state(n, L, "rand", seed)
        Xr = oracle.ref_inverse(M, n, L)
        assert rel_fro(full, Xr) < inverse_tolerance(M, Xr)
    else:
        jj = np.arange(N)[None, :]
        ii = np.arange(N)[:, None]
        expect = np.where(ii < (jj // n + 1) * n, 1000.0 * jj + ii + 1, 0.0)
        np.testing.assert_array_equal(full, expect)


@pytest.mark.parametrize("n,L", [(1, 2), (3, 2), (4, 3), (5, 7), (8, 9)])
def test_compact_band_windows_do_not_overlap(n, L):
    """The compact layout stores block columns 0..L-2 with leading dimension
    3n, element (i, j) at i + 3n j; the factorization and BSTRI touch only
    block rows m-1..m+1 of block column m (panel k reads and writes block
    rows k, k+1 of block columns k and k+1).  Those windows map to distinct
    offsets inside the 3 n (L-1) n + N doubles the state holds."""
    N = n * L
    seen = {}
    for j in range((L - 1) * n):
        m = j // n
        for i in range(max(0, (m - 1) * n), min(N, (m + 2) * n)):
            off = i + 3 * n * j
            assert 0 <= off < 3 * n * (L - 1) * n + N
            assert off not in seen, (i, j, seen.get(off))
            seen[off] = (i, j)
    # Every (panel, block column) access of BSOF lies in those windows.
    for k in range(L - 1):
        for m in (k, k + 1):
            if m <= L - 2:
                for i in range(k * n, (k + 2) * n):
                    assert (m - 1) * n <= i < (m + 2) * n


def test_shard_calls_reject_bad_arguments():
    """bsofi_shard_* check their arguments before any CUDA call."""
    from bsofi_b200 import _lib
    lib = _lib.load()
    fake = 0x1000  # never dereferenced
    assert lib.bsofi_shard_state_bytes(0, 8) == 0
    assert lib.bsofi_shard_state_bytes(16, 1) == 0
    assert lib.bsofi_shard_state_bytes(16, 8) > 0
    assert lib.bsofi_shard_factor(0, 8, None, fake, fake, None) == -1
    assert lib.bsofi_shard_factor(16, 8, None, None, fake, None) == -1
    assert lib.bsofi_shard_factor(16, 8, None, fake, None, None) == -1
    assert lib.bsofi_shard_hubbard_factor(16, 8, None, fake, 1.0, fake, None) == -1
    n, L = 16, 8
    for c0, c1, ldx in [(-1, 2, 64), (3, 3, 64), (2, 9, 200), (0, 4, 63), (5, 2, 128)]:
        assert lib.bsofi_shard_bstri_columns(n, L, c0, c1, fake, ldx, fake, None) == -1
    for r0, r1, ldb in [(64, 128, 64), (0, 100, 100), (0, 129, 129), (0, 128, 127),
                        (128, 128, 1)]:
        assert lib.bsofi_shard_bsoi_rows(n, L, r0, r1, fake, ldb, fake, None) == -1
    assert lib.bsofi_shard_logdet(16, 8, None, fake, None) == -1
    assert lib.bsofi_shard_tau(None, 16, 8) is None


def test_state_is_compact():
    """The per-rank state is O(L n^2) (about 12 L n^2 doubles: the band, G_k,
    W_i, Y_i, the BSOI carries and the last block column), against the N^2
    doubles of the ordinary layout: under a sixth of it at L = 80, a
    twentieth at L = 300."""
    from bsofi_b200 import api
    for n, L, frac in [(576, 80, 1 / 6), (400, 64, 1 / 4), (768, 300, 1 / 20)]:
        N = n * L
        b = api.shard_state_bytes(n, L)
        assert b < 8 * 13 * L * n * n
        assert b < frac * 8 * N * N
