"""Diagnostics of the device pipeline through the C ABI.

    python -m bsofi_b200.diag bsof-timeline N_BLOCK L [REPS]
    python -m bsofi_b200.diag invert N_BLOCK L [REPS] [U]
    python -m bsofi_b200.diag invert-mixed N_BLOCK L [REPS] [SLICES]
    python -m bsofi_b200.diag split-phases N_BLOCK L [REPS]
    python -m bsofi_b200.diag batch COUNT STREAMS [PRECISION [SIDE P]]
    python -m bsofi_b200.diag shard-storage N_BLOCK L WORLD [U]

bsof-timeline inverts a seeded Hubbard matrix (a random p-cyclic one when n is
not a square) with bsofi_device_invert and prints, for the last run, the BSOF
chain length and the per-leaf phases recorded by the persistent BSOF kernel's
critical CTA (bsofi_device_bsof_timeline: globaltimer stamps at loop start,
tile ready, next-tile update start and leaf published).  invert times REPS
device-resident inversions of the Hubbard matrix (U = 4 unless given) with the
size's launch plan and prints the fastest with its TFLOP/s, the BSOI time
(CUDA events around its launches) and the BSOF chain.
"""
import sys

import numpy as np

from . import _lib, api
from .hubbard import hubbard_blocks, hubbard_matrix, random_pcyclic


def bsof_leaves(n, L):
    nb = 16 if n <= 256 else 8
    nl = (n + nb - 1) // nb
    return (L - 2) * nl + 2 * nl


def bsof_timeline(n, L, reps=3):
    import torch
    side = int(round(n ** 0.5))
    N = n * L
    ldd = (N + 31) // 32 * 32
    M = hubbard_matrix(side, L, 4.0, seed=1) if side * side == n else random_pcyclic(n, L, seed=1)
    dev = torch.device("cuda:0")
    src = torch.zeros((N, ldd), dtype=torch.float64, device=dev)
    src[:, :N] = torch.from_numpy(np.ascontiguousarray(M.T)).to(dev)
    dA = torch.empty_like(src)
    dtau = torch.zeros(N, dtype=torch.float64, device=dev)
    ws = torch.empty(api.workspace_bytes(n, L, ldd), dtype=torch.uint8, device=dev)
    S = bsof_leaves(n, L)
    out = {}
    for _ in range(reps):
        dA.copy_(src)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        stream = torch.cuda.current_stream()
        e0.record(stream)
        rc = api.device_invert(n, L, dA.data_ptr(), ldd, dtau.data_ptr(), ws.data_ptr(),
                               stream.cuda_stream)
        e1.record(stream)
        torch.cuda.synchronize()
        if rc != 0:
            raise RuntimeError("bsofi_device_invert failed (%d)" % rc)
        buf = np.zeros(4 * S, dtype=np.uint64)
        cnt = _lib.load().bsofi_device_bsof_timeline(n, L, ldd, ws.data_ptr(), buf.ctypes.data, S)
        if cnt != S:
            raise RuntimeError("timeline holds %d leaves, expected %d" % (cnt, S))
        t = buf.reshape(S, 4).astype(np.int64)
        has = t[:-1]
        out = {
            "invert_ms": e0.elapsed_time(e1),
            "chain_ms": (t[-1, 2] - t[0, 0]) / 1e6,
            "leaves": S,
            "wait_tile_us": (t[:, 1] - t[:, 0]).mean() / 1e3,
            "factor_us": (has[:, 3] - has[:, 1]).mean() / 1e3,
            "update_publish_us": (has[:, 2] - has[:, 3]).mean() / 1e3,
            "to_next_leaf_us": (t[1:, 0] - t[:-1, 2]).mean() / 1e3,
        }
        wait = (t[:, 1] - t[:, 0]) / 1e3
        nl = (n + (16 if n <= 256 else 8) - 1) // (16 if n <= 256 else 8)
        first = np.arange(S) % nl == 0  # the first leaf of each regular panel
        first[(L - 2) * nl:] = False
        out.update({
            "wait_total_ms": wait.sum() / 1e3,
            "wait_first_leaf_ms": wait[first].sum() / 1e3,
            "wait_p50_us": float(np.percentile(wait, 50)),
            "wait_p90_us": float(np.percentile(wait, 90)),
            "wait_max_us": float(wait.max()),
            "factor_total_ms": (has[:, 3] - has[:, 1]).sum() / 1e6,
            "update_total_ms": (has[:, 2] - has[:, 3]).sum() / 1e6,
        })
    return out


def invert_timing(n, L, reps=3, U=4.0):
    import torch
    from .flops import bsofi_flops, flops_bsoi
    side = int(round(n ** 0.5))
    N = n * L
    ldd = (N + 31) // 32 * 32
    M = hubbard_matrix(side, L, U, seed=1) if side * side == n else random_pcyclic(n, L, seed=1)
    dev = torch.device("cuda:0")
    src = torch.zeros((N, ldd), dtype=torch.float64, device=dev)
    src[:, :N] = torch.from_numpy(np.ascontiguousarray(M.T)).to(dev)
    del M
    dA = torch.empty_like(src)
    dtau = torch.zeros(N, dtype=torch.float64, device=dev)
    ws = torch.empty(api.workspace_bytes(n, L, ldd), dtype=torch.uint8, device=dev)
    best, bsoi = float("inf"), float("inf")
    stream = torch.cuda.current_stream()
    for r in range(reps + 1):  # the first run is a warm-up
        dA.copy_(src)
        api.timing(True)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        rc = api.device_invert(n, L, dA.data_ptr(), ldd, dtau.data_ptr(), ws.data_ptr(),
                               stream.cuda_stream)
        e1.record(stream)
        torch.cuda.synchronize()
        ms, _ = api.timing_read()
        api.timing(False)
        if rc != 0:
            raise RuntimeError("bsofi_device_invert failed (%d)" % rc)
        if r > 0:
            best = min(best, e0.elapsed_time(e1))
            bsoi = min(bsoi, ms)
    S = bsof_leaves(n, L)
    buf = np.zeros(4 * S, dtype=np.uint64)
    _lib.load().bsofi_device_bsof_timeline(n, L, ldd, ws.data_ptr(), buf.ctypes.data, S)
    t = buf.reshape(S, 4).astype(np.int64)
    return {"invert_ms": best, "tflops": bsofi_flops(n, L) / best / 1e9, "bsoi_ms": bsoi,
            "bsoi_tflops": flops_bsoi(n, L) / bsoi / 1e9, "chain_ms": (t[-1, 2] - t[0, 0]) / 1e6,
            "plan": api.plan_get(n, L)}


def invert_mixed_timing(n, L, reps=3, U=4.0, slices=0):
    """Device-resident inversions with BSOI's products on the int8 tensor cores
    (bsofi_device_invert_mixed); fastest of reps, the BSOI products' time
    (split + product launches, CUDA events) and the residual."""
    import torch
    from .flops import bsofi_flops, flops_bsoi
    side = int(round(n ** 0.5))
    N = n * L
    ldd = (N + 31) // 32 * 32
    M = hubbard_matrix(side, L, U, seed=1) if side * side == n else random_pcyclic(n, L, seed=1)
    dev = torch.device("cuda:0")
    src = torch.zeros((N, ldd), dtype=torch.float64, device=dev)
    src[:, :N] = torch.from_numpy(np.ascontiguousarray(M.T)).to(dev)
    dA = torch.empty_like(src)
    dtau = torch.zeros(N, dtype=torch.float64, device=dev)
    ws = torch.empty(api.mixed_workspace_bytes(n, L, ldd, slices), dtype=torch.uint8, device=dev)
    best, bsoi = float("inf"), float("inf")
    stream = torch.cuda.current_stream()
    for r in range(reps + 1):
        dA.copy_(src)
        api.timing(True)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        rc = api.device_invert_mixed(n, L, dA.data_ptr(), ldd, dtau.data_ptr(), ws.data_ptr(),
                                     slices, stream.cuda_stream)
        e1.record(stream)
        torch.cuda.synchronize()
        ms, _ = api.timing_read()
        api.timing(False)
        if rc != 0:
            raise RuntimeError("bsofi_device_invert_mixed failed (%d)" % rc)
        if r > 0:
            best = min(best, e0.elapsed_time(e1))
            bsoi = min(bsoi, ms)
    X = dA[:, :N].T.cpu().numpy()
    res = np.linalg.norm(M @ X - np.eye(N)) / np.linalg.norm(X) if N <= 12000 else None
    return {"invert_ms": best, "tflops": bsofi_flops(n, L) / best / 1e9, "bsoi_ms": bsoi,
            "bsoi_tflops": flops_bsoi(n, L) / bsoi / 1e9, "residual": res}


def shard_storage_timing(n, L, world, U=4.0):
    """The storage-sharded inversion's phases for `world` ranks, each rank's
    share timed on its own on this GPU (CUDA events): the compact
    factorization (every rank runs it), each rank's block columns of R^{-1},
    each rank's BSOI rows, and the bytes each rank sends in the all-to-all.
    Returns a dict; a rank's device time is factor + columns + rows."""
    import torch
    from . import shard
    side = int(round(n ** 0.5))
    N = n * L
    # The packed blocks only (no dense N x N host matrix): the Hubbard chain
    # (identity diagonal, -B_k below, +B_p in the corner) or random blocks.
    if side * side == n:
        B = hubbard_blocks(side, L, U, seed=1)
        diag = np.broadcast_to(np.eye(n), (L, n, n))
        sub = -B
        sub[L - 1] = B[L - 1]
    else:
        rng = np.random.default_rng(1)
        diag = rng.standard_normal((L, n, n)) + np.eye(n)[None]
        sub = rng.standard_normal((L, n, n))
    dev = torch.device("cuda:0")
    st = torch.cuda.current_stream()
    dD = torch.from_numpy(np.ascontiguousarray(np.transpose(diag, (0, 2, 1)))).to(dev)
    dS = torch.from_numpy(np.ascontiguousarray(np.transpose(sub, (0, 2, 1)))).to(dev)
    state = torch.empty(api.shard_state_bytes(n, L), dtype=torch.uint8, device=dev)

    def timed(fn):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(st)
        rc = fn()
        e1.record(st)
        torch.cuda.synchronize()
        if rc != 0:
            raise RuntimeError("shard phase failed (%d)" % rc)
        return e0.elapsed_time(e1)

    def factor():
        return api.shard_factor(n, L, dD.data_ptr(), dS.data_ptr(), state.data_ptr(),
                                st.cuda_stream)

    timed(factor)  # warm-up
    t_factor = timed(factor)
    cols = shard.column_slabs(L, world)
    bands = shard.bsoi_row_bands(n, L, world)
    t_cols, sent, sends = [], [], []
    for r, (c0, c1) in enumerate(cols):
        slab = torch.empty(((c1 - c0) * n, max(c1 * n, 1)), dtype=torch.float64, device=dev)
        t_cols.append(timed(lambda: api.shard_bstri_columns(
            n, L, c0, c1, slab.data_ptr(), slab.shape[1], state.data_ptr(), st.cuda_stream))
            if c1 > c0 else 0.0)
        blocks = shard._send_blocks(slab, n, c0, c1, bands)
        sent.append(8 * sum(b.numel() for q, b in enumerate(blocks) if q != r))
        sends.append(blocks)
        del slab
    t_rows = []
    for q, (r0, r1) in enumerate(bands):
        band = torch.zeros((N, r1 - r0), dtype=torch.float64, device=dev)
        shard._place(torch, band, n, cols, (r0, r1), [sends[r][q] for r in range(world)])
        t_rows.append(timed(lambda: api.shard_bsoi_rows(
            n, L, r0, r1, band.data_ptr(), r1 - r0, state.data_ptr(), st.cuda_stream))
            if r1 > r0 else 0.0)
        del band
    return {"factor_ms": t_factor, "columns_ms": t_cols, "rows_ms": t_rows,
            "sent_bytes": sent, "state_bytes": api.shard_state_bytes(n, L),
            "cols": cols, "bands": bands}


def split_phases_timing(n, L, reps=2):
    """bsofi_device_bsoftri then bsofi_device_bsoi as separate calls: BSOI then
    forms every Q_k^T from the stored reflectors and tau (build_leaf_t_kernel,
    wy_apply_kernel), as the split entry points of the reference's API do."""
    import torch
    side = int(round(n ** 0.5))
    N = n * L
    ldd = (N + 31) // 32 * 32
    M = hubbard_matrix(side, L, 4.0, seed=1) if side * side == n else random_pcyclic(n, L, seed=1)
    dev = torch.device("cuda:0")
    src = torch.zeros((N, ldd), dtype=torch.float64, device=dev)
    src[:, :N] = torch.from_numpy(np.ascontiguousarray(M.T)).to(dev)
    dA = torch.empty_like(src)
    dtau = torch.zeros(N, dtype=torch.float64, device=dev)
    ws = torch.empty(api.workspace_bytes(n, L, ldd), dtype=torch.uint8, device=dev)
    best = float("inf")
    stream = torch.cuda.current_stream()
    for r in range(reps + 1):
        dA.copy_(src)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        rc = api.device_bsoftri(n, L, dA.data_ptr(), ldd, dtau.data_ptr(), ws.data_ptr(),
                                stream.cuda_stream)
        rc = rc or api.device_bsoi(n, L, dA.data_ptr(), ldd, dtau.data_ptr(), ws.data_ptr(),
                                   stream.cuda_stream)
        e1.record(stream)
        torch.cuda.synchronize()
        if rc != 0:
            raise RuntimeError("split phases failed (%d)" % rc)
        if r > 0:
            best = min(best, e0.elapsed_time(e1))
    return best


def batch_timing(count, streams, precision=0, reps=2, seed=77, fixed=None):
    """The batched configuration (side in {8,..,16}, p in [8, 64], U in [2, 6]),
    or `count` instances of one size when fixed = (side, p) (U = 4), per call
    with `streams` internal streams; inputs are re-assembled from packed
    blocks before each timed call.  Returns the best call's time in ms and
    the rate."""
    import torch
    from .hubbard import hubbard_blocks
    rng = np.random.default_rng(seed)
    if fixed:
        specs = [(fixed[0], fixed[1], 4.0, 9000 + i) for i in range(count)]
    else:
        specs = [(int(rng.choice([8, 10, 12, 14, 16])), int(rng.integers(8, 65)),
                  float(rng.uniform(2.0, 6.0)), 9000 + i) for i in range(count)]
    dev = torch.device("cuda:0")
    ns, Ls, lds, bufs, packs, taus = [], [], [], [], [], []
    for side, L, U, sd in specs:
        n = side * side
        N = n * L
        ld = (N + 31) // 32 * 32
        B = hubbard_blocks(side, L, U, seed=sd)
        sub = -B
        sub[L - 1] = B[L - 1]
        packs.append(torch.from_numpy(np.ascontiguousarray(np.transpose(sub, (0, 2, 1)))).to(dev))
        bufs.append(torch.empty((N, ld), dtype=torch.float64, device=dev))
        taus.append(torch.zeros(N, dtype=torch.float64, device=dev))
        ns.append(n)
        Ls.append(L)
        lds.append(ld)
    ws = torch.empty(api.batch_workspace_bytes(ns, Ls, lds, precision), dtype=torch.uint8,
                     device=dev)
    stream = torch.cuda.current_stream()
    best = float("inf")
    for r in range(reps + 1):
        for n, L, b, pk, ld in zip(ns, Ls, bufs, packs, lds):
            api.device_assemble(n, L, 0, pk.data_ptr(), b.data_ptr(), ld)
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        rc = api.device_invert_batched(ns, Ls, [b.data_ptr() for b in bufs], lds,
                                       [t.data_ptr() for t in taus], ws.data_ptr(), streams,
                                       stream.cuda_stream, precision)
        e1.record(stream)
        torch.cuda.synchronize()
        if rc != 0:
            raise RuntimeError("batched inversion failed (%d)" % rc)
        if r > 0:
            best = min(best, e0.elapsed_time(e1))
    return best, count / (best * 1e-3)


def main(argv):
    # --grouped=1: FP64 batches run BSOI as one grouped launch per tile shape
    # (the default, 0, launches each instance's BSOI on its own stream).
    for a in list(argv):
        if a.startswith("--grouped="):
            _lib.load().bsofi_device_set_batch_grouped(int(a.split("=", 1)[1]))
            argv = [x for x in argv if x != a]
    # --pipelined=1: batches with chains on high-priority streams and
    # non-persistent GEMM phases.
    for a in list(argv):
        if a.startswith("--pipelined="):
            _lib.load().bsofi_device_set_batch_pipelined(int(a.split("=", 1)[1]))
            argv = [x for x in argv if x != a]
    # --tma=1|0: the persistent BSOI's clean tiles loaded by TMA, or cp.async.
    for a in list(argv):
        if a.startswith("--tma="):
            _lib.load().bsofi_device_set_bsoi_tma(int(a.split("=", 1)[1]))
            argv = [x for x in argv if x != a]
    # --k16=1: the FP64 tile engine with mma.sync m16n8k16 steps.
    for a in list(argv):
        if a.startswith("--k16="):
            _lib.load().bsofi_device_set_gemm_k16(int(a.split("=", 1)[1]))
            argv = [x for x in argv if x != a]
    # --batch-workers=W: BSOF worker CTAs per batch instance.
    for a in list(argv):
        if a.startswith("--batch-workers="):
            _lib.load().bsofi_device_set_batch_workers(int(a.split("=", 1)[1]))
            argv = [x for x in argv if x != a]
    # --chains=K: at most K factorization chains of a batch in flight.
    for a in list(argv):
        if a.startswith("--chains="):
            _lib.load().bsofi_device_set_batch_chains(int(a.split("=", 1)[1]))
            argv = [x for x in argv if x != a]
    # --workers=W: BSOF worker CTAs of single inversions (the plan's otherwise).
    for a in list(argv):
        if a.startswith("--workers="):
            _lib.load().bsofi_device_set_bsof_workers(int(a.split("=", 1)[1]))
            argv = [x for x in argv if x != a]
    # --factor-warps=8: 16-wide BSOF leaves factored by all eight warps.
    for a in list(argv):
        if a.startswith("--factor-warps="):
            _lib.load().bsofi_device_set_bsof_factor_warps(int(a.split("=", 1)[1]))
            argv = [x for x in argv if x != a]
    if len(argv) >= 3 and argv[0] == "bsof-timeline":
        n, L = int(argv[1]), int(argv[2])
        reps = int(argv[3]) if len(argv) > 3 else 3
        r = bsof_timeline(n, L, reps)
        print("n %d L %d: invert %.3f ms, BSOF chain %.3f ms over %d leaves" %
              (n, L, r["invert_ms"], r["chain_ms"], r["leaves"]))
        print("per leaf: wait for tile %.2f us, factor (tile ready -> next-tile update) %.2f us, "
              "next-tile update + publish %.2f us, publish -> next leaf %.2f us" %
              (r["wait_tile_us"], r["factor_us"], r["update_publish_us"], r["to_next_leaf_us"]))
        print("totals: wait %.2f ms (first leaf of a panel %.2f ms; per leaf p50 %.2f us, p90 %.2f us,"
              " max %.1f us), factor %.2f ms, next-tile update + publish %.2f ms" %
              (r["wait_total_ms"], r["wait_first_leaf_ms"], r["wait_p50_us"], r["wait_p90_us"],
               r["wait_max_us"], r["factor_total_ms"], r["update_total_ms"]))
        return 0
    # --bsoi-plan=P (invert): the size's BSOI launch form (0 persistent
    # 128 x 128, 5 persistent 64 x 64, 1-4 one launch per step).
    bsoi_plan = None
    for a in list(argv):
        if a.startswith("--bsoi-plan="):
            bsoi_plan = int(a.split("=", 1)[1])
            argv = [x for x in argv if x != a]
    if bsoi_plan is not None and len(argv) >= 3:
        n, L = int(argv[1]), int(argv[2])
        api.plan_set(n, L, [bsoi_plan] + api.plan_get(n, L)[1][1:])
    if len(argv) >= 3 and argv[0] == "invert":
        n, L = int(argv[1]), int(argv[2])
        reps = int(argv[3]) if len(argv) > 3 else 3
        U = float(argv[4]) if len(argv) > 4 else 4.0
        r = invert_timing(n, L, reps, U)
        print("n %d L %d (plan %s): invert %.3f ms = %.2f TFLOP/s of the flop model; BSOI %.3f ms "
              "= %.2f TFLOP/s; BSOF chain %.3f ms" % (n, L, r["plan"], r["invert_ms"], r["tflops"],
                                                      r["bsoi_ms"], r["bsoi_tflops"], r["chain_ms"]))
        return 0
    if len(argv) >= 3 and argv[0] == "invert-mixed":
        n, L = int(argv[1]), int(argv[2])
        reps = int(argv[3]) if len(argv) > 3 else 3
        slices = int(argv[4]) if len(argv) > 4 else 0
        r = invert_mixed_timing(n, L, reps, 4.0, slices)
        print("n %d L %d mixed (slices %s): invert %.3f ms = %.2f TFLOP/s of the flop model; "
              "BSOI products %.3f ms = %.2f TFLOP/s effective FP64; residual %s"
              % (n, L, slices or 8, r["invert_ms"], r["tflops"], r["bsoi_ms"], r["bsoi_tflops"],
                 r["residual"]))
        return 0
    if len(argv) >= 3 and argv[0] == "batch":
        count, streams = int(argv[1]), int(argv[2])
        precision = int(argv[3]) if len(argv) > 3 else 0
        fixed = (int(argv[4]), int(argv[5])) if len(argv) > 5 else None
        ms, rate = batch_timing(count, streams, precision, fixed=fixed)
        print("batch of %d%s (streams %d, precision %d): %.1f ms = %.1f inversions/s"
              % (count, " x side %d p %d" % fixed if fixed else "", streams, precision, ms, rate))
        return 0
    if len(argv) >= 4 and argv[0] == "shard-storage":
        n, L, world = int(argv[1]), int(argv[2]), int(argv[3])
        U = float(argv[4]) if len(argv) > 4 else 4.0
        r = shard_storage_timing(n, L, world, U)
        per_rank = [r["factor_ms"] + c + w for c, w in zip(r["columns_ms"], r["rows_ms"])]
        print("n %d L %d over %d ranks: factor %.3f ms (every rank); columns %s ms; rows %s ms;"
              " device time per rank %s ms (max %.3f); sent %s MB; state %.1f MB"
              % (n, L, world, r["factor_ms"], ["%.3f" % x for x in r["columns_ms"]],
                 ["%.3f" % x for x in r["rows_ms"]], ["%.2f" % x for x in per_rank],
                 max(per_rank), ["%.0f" % (b / 1e6) for b in r["sent_bytes"]],
                 r["state_bytes"] / 1e6))
        return 0
    if len(argv) >= 3 and argv[0] == "split-phases":
        n, L = int(argv[1]), int(argv[2])
        reps = int(argv[3]) if len(argv) > 3 else 2
        print("n %d L %d: bsoftri + bsoi as separate calls %.3f ms"
              % (n, L, split_phases_timing(n, L, reps)))
        return 0
    print(__doc__)
    return 2


if __name__ == "__main__":
    sys.exit(main(sys.argv[1:]))
