"""One BSOF/I inversion split over the ranks of a torch.distributed group.

The split follows the row independence of BSOI: in X(:,k:k+1) <- X(:,k:k+1)
Q_k^T (reference src/bsofi_cpu.c:211-248) every row of X is transformed on
its own, so a rank that holds the factored state can compute any set of rows
of M^{-1} alone.  Every rank factors the whole matrix (BSOF + BSTRI, the
latency-bound chain, which does not split; the pipeline is deterministic, so
every rank holds the same state), then computes its band of rows with
bsofi_device_bsoi_rows, 79% of the flop model's work divided by the number of
ranks, and, if asked, the bands are all-gathered so that every rank holds the
dense M^{-1}.  The factorization and BSTRI are not split and each rank holds
the whole matrix, so this shortens one inversion; it does not raise the
largest N beyond one GPU's memory.
"""
from . import api


def row_bands(N, world, align=128):
    """Contiguous row bands [r0, r1) covering 0..N-1, one per rank, each
    starting at a multiple of `align` (the BSOI tile height), as even as that
    alignment allows.  Bands of ranks beyond the number of aligned units are
    empty (r0 == r1)."""
    if N < 0 or world < 1 or align < 1:
        raise ValueError("row_bands: N >= 0, world >= 1, align >= 1")
    units = (N + align - 1) // align
    per, extra = divmod(units, world)
    bands, u = [], 0
    for r in range(world):
        cnt = per + (1 if r < extra else 0)
        r0 = min(u * align, N)
        u += cnt
        bands.append((r0, min(u * align, N)))
    return bands


def gather_rows(torch, dist, Xc, N, bands, group=None):
    """All-gather the row bands of a column-major matrix held as the tensor
    Xc (ncols x ld, Xc[j, i] = X(i, j)): rank q's rows bands[q] are copied
    into every other rank's Xc.  Works for any backend of `dist`."""
    rank = dist.get_rank(group)
    world = dist.get_world_size(group)
    width = max((b - a for a, b in bands), default=0)
    if width == 0 or world == 1:
        return
    send = torch.zeros((Xc.shape[0], width), dtype=Xc.dtype, device=Xc.device)
    a, b = bands[rank]
    if b > a:
        send[:, :b - a] = Xc[:, a:b]
    recv = [torch.empty_like(send) for _ in range(world)]
    dist.all_gather(recv, send, group=group)
    for q, (a, b) in enumerate(bands):
        if q != rank and b > a:
            Xc[:, a:b] = recv[q][:, :b - a]


def sharded_invert(n, L, Xc, ldd, dtau, dwork, group=None, gather=True):
    """Invert the p-cyclic matrix held (column-major, leading dimension ldd)
    in the device tensor Xc (N x ldd view, Xc[j, i] = A(i, j)) on every rank
    of `group`: the factorization on every rank, BSOI by rows, then (gather)
    the rows of the others.  dtau: N doubles, dwork: the workspace of
    bsofi_device_workspace_bytes, both on the device.  Runs on torch's
    current stream.  Returns 0 or the first nonzero status of the two device
    calls (rows of ranks that failed are then unspecified on the others)."""
    import torch
    import torch.distributed as dist
    N = n * L
    stream = torch.cuda.current_stream().cuda_stream
    rc = api.device_bsoftri(n, L, Xc.data_ptr(), ldd, dtau.data_ptr(), dwork, stream)
    rank = dist.get_rank(group)
    bands = row_bands(N, dist.get_world_size(group))
    r0, r1 = bands[rank]
    if rc == 0 and r1 > r0:
        rc = api.device_bsoi_rows(n, L, Xc.data_ptr(), ldd, dtau.data_ptr(), dwork, r0, r1, stream)
    if gather:
        gather_rows(torch, dist, Xc[:N], N, bands, group)
    return rc
