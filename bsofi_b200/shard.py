"""One BSOF/I inversion split over the ranks of a torch.distributed group.

Two splits, both following the structure of the algorithm:

Row-band split (sharded_invert).  In BSOI, X(:,k:k+1) <- X(:,k:k+1) Q_k^T
(reference src/bsofi_cpu.c:211-248), every row of X is transformed on its
own, so a rank that holds the factored state can compute any set of rows of
M^{-1} alone.  Every rank factors the whole matrix in the ordinary layout
(BSOF + BSTRI; deterministic, so every rank holds the same state), computes
its band of rows with bsofi_device_bsoi_rows, and, if asked, the bands are
all-gathered.  Each rank holds the whole matrix: this shortens one
inversion, it does not raise the largest N beyond one GPU's memory.

Storage-sharded split (storage_sharded_invert).  No rank holds M or M^{-1}
whole, so N can exceed one GPU's memory:
  1. every rank factors the whole matrix in the compact layout of
     bsofi_shard_factor (R has three nonzero blocks per block row, the
     reflectors fill the panels: 3 L n^2 + N n doubles), which also forms the
     diagonal inverses, the row multipliers W_i and the last-column terms Z_i;
  2. rank r computes block columns cols[r] = [c0, c1) of X = R^{-1} (rows
     0 .. c1 n - 1; BSTRI's row recurrence, src/bsofi_cpu.c:146-177, read by
     columns: X_{i,c} = W_i X_{i+1,c}, plus Z_i in the last column), the
     column ranges chosen to minimise the largest stored slab;
  3. one all-to-all turns the column slabs into row bands (rows below c1 n
     of a slab are zero and are not sent);
  4. rank r finishes rows bands[r] of M^{-1} with bsofi_shard_bsoi_rows,
     the bands balanced by BSOI's work (the top rows cost twice the bottom).
Per rank the device holds the state, its slab (at most about 0.6 N^2 / P
doubles at P = 8) and its band (about N^2 / P), plus the exchange buffers of
the same sizes.
"""
import collections

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


def bsoi_row_bands(n, L, world, align=128):
    """Row bands [r0, r1) as row_bands gives them, but balanced by BSOI's
    work instead of the row count: a row of block row b takes the 2n-deep
    product in the L-1-b steps whose X(:,k) reaches it and only the n-deep
    carry product in the other b (the orgqr zero structure), so its work is
    proportional to 2L - 2 - b: the top rows cost about twice the bottom
    ones."""
    N = n * L
    if N < 0 or world < 1 or align < 1:
        raise ValueError("bsoi_row_bands: N >= 0, world >= 1, align >= 1")
    units = (N + align - 1) // align
    w = []
    for u in range(units):
        a, b = u * align, min((u + 1) * align, N)
        w.append(sum(2 * L - 2 - i // n for i in range(a, b)))
    total = float(sum(w))
    cuts, acc, u = [0], 0.0, 0
    for r in range(1, world):
        target = total * r / world
        while u < units and acc + w[u] / 2.0 <= target:
            acc += w[u]
            u += 1
        cuts.append(u)
    cuts.append(units)
    return [(min(cuts[r] * align, N), min(cuts[r + 1] * align, N)) for r in range(world)]


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


# ------------------------------------------------------------ storage-sharded


def column_slabs(L, world):
    """Contiguous block-column ranges [c0, c1) covering 0..L-1, one per rank.

    A rank stores its block columns with c1 n rows (X = R^{-1} is block
    upper triangular, so rows below c1 n of those columns are zero): its
    slab holds c1 (c1 - c0) n^2 doubles.  The ranges minimise the largest
    slab (greedy left to right under a bound found by bisection), so early
    ranks take more, shorter columns.  Every range is non-empty when
    L >= world; ranks beyond L get empty ranges (c0 == c1)."""
    if L < 1 or world < 1:
        raise ValueError("column_slabs: L >= 1, world >= 1")

    def cuts_under(T):
        cuts, c0 = [0], 0
        for r in range(world - 1):
            left = world - 1 - r          # ranks after this one
            c1 = c0
            while c1 < L - (left if L >= world else 0) and (c1 + 1) * (c1 + 1 - c0) <= T:
                c1 += 1
            if L >= world and c1 == c0:
                c1 = c0 + 1
            cuts.append(c1)
            c0 = c1
        cuts.append(L)
        return cuts

    def worst(cuts):
        return max(c1 * (c1 - c0) for c0, c1 in zip(cuts, cuts[1:]))

    lo, hi = 1, L * L
    while lo < hi:
        mid = (lo + hi) // 2
        if worst(cuts_under(mid)) <= mid:
            hi = mid
        else:
            lo = mid + 1
    cuts = cuts_under(lo)
    return [(cuts[r], cuts[r + 1]) for r in range(world)]


def _send_blocks(slab, n, c0, c1, bands):
    """Blocks of a rank's slab (tensor ((c1-c0) n, c1 n), slab[j, i] =
    X(i, c0 n + j)) for every destination band: rows [a, min(b, c1 n)) of
    the slab's columns, as contiguous (w, h) tensors (h may be 0)."""
    out = []
    for a, b in bands:
        h = max(0, min(b, c1 * n) - a)
        out.append(slab[:, a:a + h].contiguous() if h > 0 else slab[:, :0])
    return out


def _block_shapes(n, cols, band):
    """(w, h) of the block every source rank sends to the rank of `band`."""
    r0, r1 = band
    return [((c1 - c0) * n, max(0, min(r1, c1 * n) - r0) if r1 > r0 else 0) for c0, c1 in cols]


def _place(torch, band_t, n, cols, band, blocks):
    """Row band tensor (N, r1 - r0) (band_t[j, i - r0] = X(i, j)) from the
    blocks of every source rank; rows a slab does not reach stay zero."""
    for (c0, c1), (w, h), blk in zip(cols, _block_shapes(n, cols, band), blocks):
        if w and h:
            band_t[c0 * n:c1 * n, :h] = blk.reshape(w, h)


def columns_to_rows(torch, dist, slab, n, L, cols, bands, group=None):
    """All-to-all of the column slabs into row bands over `group` (any
    backend).  slab: this rank's block columns cols[rank] as a tensor
    ((c1-c0) n, c1 n); returns its row band bands[rank] as a tensor
    (N, r1 - r0) with band[j, i - r0] = X(i, j)."""
    rank = dist.get_rank(group)
    c0, c1 = cols[rank]
    N = n * L
    send = _send_blocks(slab, n, c0, c1, bands)
    in_sizes = [t.numel() for t in send]
    inp = torch.cat([t.reshape(-1) for t in send]) if sum(in_sizes) else \
        torch.empty(0, dtype=slab.dtype, device=slab.device)
    shapes = _block_shapes(n, cols, bands[rank])
    out_sizes = [w * h for w, h in shapes]
    out = torch.empty(sum(out_sizes), dtype=slab.dtype, device=slab.device)
    dist.all_to_all_single(out, inp, out_sizes, in_sizes, group=group)
    del inp, send
    r0, r1 = bands[rank]
    band_t = torch.zeros((N, r1 - r0), dtype=slab.dtype, device=slab.device)
    _place(torch, band_t, n, cols, bands[rank], list(torch.split(out, out_sizes)))
    return band_t


ShardResult = collections.namedtuple("ShardResult", "band rows rc info failed")


def _new_slab(torch, n, c0, c1, device):
    return torch.empty(((c1 - c0) * n, max(c1 * n, 1)), dtype=torch.float64, device=device)


def storage_sharded_invert(n, L, dD, dS, group=None, align=128):
    """Invert the p-cyclic matrix given by its packed blocks (device
    pointers dD, dS as bsofi_device_assemble takes them; dD may be 0 for
    identity diagonal blocks) with no rank holding M or M^{-1} whole.
    Runs on torch's current stream and device.  Returns ShardResult: band,
    this rank's rows (r0, r1) of M^{-1} as a tensor (N, r1 - r0) with
    band[j, i - r0] = M^{-1}(i, j); rc, the first nonzero status of this
    rank's library calls; info, the state's info word (0, i > 0 for an
    exactly zero R(i,i), or the wait-failure code); failed, True on every
    rank when any rank had rc != 0 or info != 0.  Every rank takes the same
    collective steps whatever its status."""
    import torch
    import torch.distributed as dist
    rank = dist.get_rank(group)
    world = dist.get_world_size(group)
    dev = torch.device("cuda", torch.cuda.current_device())
    stream = torch.cuda.current_stream().cuda_stream
    N = n * L
    state = torch.empty(api.shard_state_bytes(n, L), dtype=torch.uint8, device=dev)
    rc = api.shard_factor(n, L, dD, dS, state.data_ptr(), stream)
    cols = column_slabs(L, world)
    bands = bsoi_row_bands(n, L, world, align)
    c0, c1 = cols[rank]
    slab = _new_slab(torch, n, c0, c1, dev)
    if rc == 0 and c1 > c0:
        rc = api.shard_bstri_columns(n, L, c0, c1, slab.data_ptr(), slab.shape[1], state.data_ptr(),
                                     stream)
    band_t = columns_to_rows(torch, dist, slab, n, L, cols, bands, group)
    del slab
    r0, r1 = bands[rank]
    if rc == 0 and r1 > r0:
        rc = api.shard_bsoi_rows(n, L, r0, r1, band_t.data_ptr(), r1 - r0, state.data_ptr(),
                                 stream)
    info = api.shard_info(state, n, L)
    flag = torch.tensor([1 if (rc != 0 or info != 0) else 0], dtype=torch.int32, device=dev)
    dist.all_reduce(flag, op=dist.ReduceOp.MAX, group=group)
    return ShardResult(band_t, (r0, r1), rc, info, bool(flag.item()))


def storage_sharded_local(n, L, dD, dS, world, align=128):
    """The steps of storage_sharded_invert for `world` ranks run in turn on
    the current GPU, the all-to-all done by local copies of the same blocks.
    One factorization serves every rank (each rank would compute the same
    state).  Returns (bands, rc, info): bands a list of (r0, r1, tensor) as
    storage_sharded_invert returns them."""
    import torch
    dev = torch.device("cuda", torch.cuda.current_device())
    stream = torch.cuda.current_stream().cuda_stream
    N = n * L
    state = torch.empty(api.shard_state_bytes(n, L), dtype=torch.uint8, device=dev)
    rc = api.shard_factor(n, L, dD, dS, state.data_ptr(), stream)
    cols = column_slabs(L, world)
    bands = bsoi_row_bands(n, L, world, align)
    sends = []
    for c0, c1 in cols:
        slab = _new_slab(torch, n, c0, c1, dev)
        if rc == 0 and c1 > c0:
            rc = api.shard_bstri_columns(n, L, c0, c1, slab.data_ptr(), slab.shape[1],
                                         state.data_ptr(), stream)
        sends.append(_send_blocks(slab, n, c0, c1, bands))
        del slab
    out = []
    for q, (r0, r1) in enumerate(bands):
        band_t = torch.zeros((N, r1 - r0), dtype=torch.float64, device=dev)
        _place(torch, band_t, n, cols, (r0, r1), [sends[r][q] for r in range(len(cols))])
        if rc == 0 and r1 > r0:
            rc = api.shard_bsoi_rows(n, L, r0, r1, band_t.data_ptr(), r1 - r0, state.data_ptr(),
                                     stream)
        out.append((r0, r1, band_t))
    return out, rc, api.shard_info(state, n, L)
