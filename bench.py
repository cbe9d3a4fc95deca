"""BSOF/I benchmark: FP64 inversion of the DQMC block p-cyclic matrix.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Workload (default): one plain-FP64 inversion per step of the Hubbard matrix on
a 16x16 periodic lattice (n = 256), p = 32 time slices, U = 4, dtau = 0.125
(N = 8192), seeded synthetic fields.  A step is BSOF + BSTRI + BSOI on one
matrix already resident in HBM; every step inverts a different 537 MB buffer
(inputs larger than L2, no reuse between steps).

Multi-GPU: independent replicas (one process per GPU, no collective on the
data path); value = inversions by all ranks / max-over-ranks device time.

Printed JSON line (rank 0): value (device-resident inversions/s), tflops
(flop model of include/bsofi_flops.h), roofline of the dominant kernel (the
persistent BSOI kernel, FP64 DMMA, against cuBLAS DGEMM measured in the same run),
e2e (the reference handle API hybridxbsoftrih_ + hybridxbsoih_ on pinned host
buffers, copies included; e2e_pageable the same on pageable numpy arrays;
e2e_fp32 the single-precision library's handle API on pinned float arrays),
cpu_baseline (the reference's CPU path,
oracle/_ref, on the host cores), clocks sampled during the timed region.

--impl reference times the reference's own CPU implementation (the compiled
reference library in oracle/_ref, OpenBLAS with all host threads) on the same
workload and prints the same JSON line with "impl": "reference".
"""
import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

from bsofi_b200.flops import bsofi_flops, flops_bsof, flops_bsoi  # noqa: E402
from bsofi_b200.hubbard import hubbard_blocks  # noqa: E402

METRIC = "inversions/s (FP64 BSOF/I, n=256, p=32)"


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=30)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", choices=["ours", "reference"], default="ours")
    p.add_argument("--side", type=int, default=16)
    p.add_argument("--L", type=int, default=32)
    p.add_argument("--U", type=float, default=4.0)
    p.add_argument("--e2e-steps", type=int, default=5)
    p.add_argument("--cpu-sample", type=int, default=10, help="reference inversions in cpu_baseline")
    p.add_argument("--no-e2e", action="store_true")
    p.add_argument("--no-cpu", action="store_true")
    p.add_argument("--batch", type=int, default=16,
                   help="instances of the headline size per batched step (0 = skip)")
    p.add_argument("--batch-mixed", type=int, default=256,
                   help="instances of the mixed-size batched configuration (0 = skip)")
    p.add_argument("--batch-steps", type=int, default=3)
    p.add_argument("--mixed-steps", type=int, default=10,
                   help="timed mixed-precision inversions at the headline size (0 = skip)")
    p.add_argument("--c4-steps", type=int, default=4,
                   help="timed inversions at n=400, p=64, U=6 for the c4 key (0 = skip)")
    p.add_argument("--shard-ranks", type=int, default=4,
                   help="storage-sharded C4 emulated over this many ranks on one GPU (0: skip)")
    p.add_argument("--serve", type=int, default=1000,
                   help="requests in the served Poisson stream (0 = skip; 10000 = the full "
                        "serving configuration)")
    p.add_argument("--serve-rate", type=float, default=12.0, help="mean arrivals per second")
    p.add_argument("--serve-mixed", type=float, default=0.5,
                   help="fraction of served requests at mixed precision")
    p.add_argument("--serve-only", action="store_true",
                   help="run only the served Poisson stream and print its JSON line")
    return p.parse_args()


def config(args, n, N):
    return {"workload": "single FP64 inversion of the Hubbard DQMC p-cyclic matrix, "
                        "%dx%d lattice, n=%d, p=%d, N=%d, U=%g, dtau=0.125"
                        % (args.side, args.side, n, args.L, N, args.U),
            "n": n, "p": args.L, "N": N, "U": args.U,
            "l2": "inputs larger than L2: %d MB per matrix, a fresh buffer every step"
                  % (8 * N * N // 2 ** 20),
            "parallelism": "replicas" if args.gpus > 1 else "single"}


def pcyclic_device(torch, diag, sub, ldd, dev):
    """Column-major (ldd x N) device buffer of the p-cyclic matrix."""
    L, n, _ = diag.shape
    N = n * L
    t = torch.zeros((N, ldd), dtype=torch.float64, device=dev)  # t[col, row]
    D = torch.from_numpy(diag).to(dev)
    S = torch.from_numpy(sub).to(dev)
    for k in range(L):
        t[k * n:(k + 1) * n, k * n:(k + 1) * n] = D[k].T
        r = (k + 1) % L
        t[k * n:(k + 1) * n, r * n:(r + 1) * n] = S[k].T
    return t


def hubbard_pcyclic(side, L, U, seed):
    B = hubbard_blocks(side, L, U, seed=seed)
    n = side * side
    diag = np.broadcast_to(np.eye(n), (L, n, n)).copy()
    sub = -B
    sub[L - 1] = B[L - 1]
    return diag, sub


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), "--query-gpu=" + self.Q,
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.lines:
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for name, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": mx,
                "samples": len(sm), "reasons": sorted(reasons)}


def measure_dgemm_peak(torch, dev, size=8192, reps=6):
    """cuBLAS FP64 GEMM throughput (TFLOP/s), best of `reps` (the FP64
    denominator; the driver's peak file carries only HBM and BF16 figures)."""
    a = torch.randn(size, size, dtype=torch.float64, device=dev)
    b = torch.randn(size, size, dtype=torch.float64, device=dev)
    c = a @ b
    torch.cuda.synchronize()
    best = 0.0
    for _ in range(reps):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        torch.matmul(a, b, out=c)
        e1.record()
        e1.synchronize()
        best = max(best, 2.0 * size ** 3 / (e0.elapsed_time(e1) * 1e-3) / 1e12)
    del a, b, c
    return best


def hbm_peak():
    """Measured HBM copy bandwidth of this pool (GB/s), else the fallback."""
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        return float(json.load(open(path))["hbm_gbs"])
    except (OSError, ValueError, KeyError):
        return 6650.0


def bsof_chain_ms(api, n, L, ldd, ws):
    """Duration of the BSOF chain of the last inversion that used `ws`
    (globaltimer stamps written by the kernel's critical CTA)."""
    from bsofi_b200 import _lib
    nl = (n + 15) // 16 if n <= 256 else (n + 7) // 8
    S = (L - 2) * nl + 2 * nl
    buf = np.zeros(4 * S, dtype=np.uint64)
    cnt = _lib.load().bsofi_device_bsof_timeline(n, L, ldd, ws.data_ptr(), buf.ctypes.data, S)
    if cnt != S:
        return None
    t = buf.reshape(S, 4).astype(np.int64)
    return float(t[-1, 2] - t[0, 0]) / 1e6


def traffic_per_launch():
    """DRAM bytes per BSOI launch from the committed ncu summary, if any."""
    path = os.path.join(ROOT, "profiles", "bsoi_tma_traffic.json")
    if os.path.exists(path):
        try:
            return json.load(open(path)).get("dram_bytes_per_launch")
        except ValueError:
            return None
    return None


def cpu_reference(side, L, U, steps, threads=None):
    """Time the reference's CPU path (oracle/_ref) on `steps` inversions."""
    import oracle
    from bsofi_b200.hubbard import hubbard_matrix
    if not oracle.ref_available():
        return None
    cores = threads or os.cpu_count()
    oracle.set_ref_threads(cores)
    n = side * side
    M = hubbard_matrix(side, L, U, seed=12345)
    times = []
    for _ in range(steps):
        # The reference overwrites its input in place: a fresh copy of M and a
        # tau array are made before the clock starts, as a caller holds them.
        A = np.asfortranarray(M)
        tau = np.zeros(n * L)
        t0 = time.perf_counter()
        _, _, info = oracle.ref_bsoftri(A, n, L, inplace=True)
        oracle.ref_bsoi(A, tau, n, L, inplace=True)
        times.append(time.perf_counter() - t0)
    return {"times": times, "cores": cores}


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    n = args.side * args.side
    N = n * args.L
    out = cpu_reference(args.side, args.L, args.U, args.warmup + args.steps)
    if out is None:
        print(json.dumps({"impl": "reference", "unavailable":
                          "reference CPU library oracle/_ref/libbsofi_ref.so not built"}))
        return
    t = out["times"][args.warmup:]
    tot = sum(t)
    value = len(t) / tot
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": "inversions/s",
            "n_gpus": args.gpus, "steps": len(t), "warmup": args.warmup,
            "ms_per_step": 1e3 * tot / len(t), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64",
            "data": "synthetic: seeded Hubbard DQMC matrix",
            "config": config(args, n, N),
            "tflops": bsofi_flops(n, args.L) * value / 1e12,
            "cpu_baseline": {"value": value, "unit": "inversions/s", "cores": out["cores"],
                             "kind": "reference",
                             "sample": "%d full inversions (lapackXbsof+lapackXbstri+"
                                       "lapackXbsoi_ormqr, OpenBLAS)" % len(t)},
            "e2e": {"value": value, "unit": "inversions/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


def main():
    args = parse()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args)
        return

    import torch
    import torch.distributed as dist
    from bsofi_b200 import api

    api.load()  # the CUDA library is the only path; fail loudly if missing
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=dev)

    if args.serve_only:
        served = run_serving(api, torch, dev, args.serve, args.serve_rate, 31 + rank,
                             args.serve_mixed)
        if rank == 0:
            print(json.dumps({"metric": "served Poisson stream (inversions/s, p50/p99 latency)",
                              "n_gpus": world, "served": served}))
        if world > 1:
            dist.destroy_process_group()
        return

    side, L, U = args.side, args.L, args.U
    n = side * side
    N = n * L
    ldd = (N + 31) // 32 * 32
    nbuf = args.warmup + args.steps
    nseeds = 4
    blocks = [hubbard_pcyclic(side, L, U, seed=1000 * rank + s) for s in range(nseeds)]
    bufs = [pcyclic_device(torch, *blocks[i % nseeds], ldd, dev) for i in range(nbuf)]
    dtau = torch.zeros(N, dtype=torch.float64, device=dev)
    ws = torch.zeros(api.workspace_bytes(n, L, ldd) // 8 + 32, dtype=torch.float64, device=dev)
    stream = torch.cuda.Stream(device=dev)
    sp = stream.cuda_stream

    def step(i):
        rc = api.device_invert(n, L, bufs[i].data_ptr(), ldd, dtau.data_ptr(), ws.data_ptr(), sp)
        if rc != 0:
            raise RuntimeError("bsofi_device_invert failed: %d" % rc)

    with torch.cuda.stream(stream):
        for i in range(args.warmup):
            step(i)
    torch.cuda.synchronize()

    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    clocks = ClockSampler(local)
    clocks.start()
    api.timing(True)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    with torch.cuda.stream(stream):
        e0.record(stream)
        for i in range(args.warmup, nbuf):
            step(i)
        e1.record(stream)
    torch.cuda.synchronize()
    launches_per_step = api.last_launches()  # kernels of the last timed step
    gemm_ms, gemm_launches = api.timing_read()
    api.timing(False)
    clk = clocks.stop()
    if world > 1:
        dist.barrier()
    ms = e0.elapsed_time(e1)
    t = torch.tensor([ms], dtype=torch.float64, device=dev)
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    ms_max = float(t.item())
    value = world * args.steps / (ms_max * 1e-3)

    # Check the last output: ||M X - I||_F / ||X||_F on the device.
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from gpu_util import block_residual_gpu
    Xlast = bufs[nbuf - 1][:, :N].T  # row-major view of the column-major result
    resid = block_residual_gpu(torch, *blocks[(nbuf - 1) % nseeds], Xlast.contiguous())
    del bufs
    torch.cuda.empty_cache()

    peak = measure_dgemm_peak(torch, dev)
    achieved = flops_bsoi(n, L) * args.steps / (gemm_ms * 1e-3) / 1e12 if gemm_ms > 0 else None
    roofline = {"kernel": "bsoi_tma_kernel (all p-1 BSOI steps in one ordinary persistent "
                          "launch; clean 128x128 tiles loaded by TMA, FP64 DMMA m16n8k8); "
                          "dominant by algorithmic work (79% of the flop model)",
                "bound": "tensor", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                "frac": (achieved / peak) if achieved else None,
                "peak_source": "cuBLAS DGEMM 8192^3 measured in this run (FP64 tensor)",
                "launches": gemm_launches,
                "avg_launch_ms": gemm_ms / max(gemm_launches, 1),
                "algorithmic_flops_per_launch": flops_bsoi(n, L) * args.steps / max(gemm_launches, 1),
                "traffic": traffic_per_launch()}
    # The persistent BSOF kernel is the largest share of device time: a serial
    # Householder chain, latency bound.  Reported against HBM as the panels'
    # roofline, with its algorithmic flops beside it.
    bsof_ms = bsof_chain_ms(api, n, L, ldd, ws)
    bsof_bytes = 8.0 * ((L - 1) * 2 * n * 3 * n * 2 + 2 * L * n * n)
    roofline_bsof = {"kernel": "bsof_persistent_kernel (Householder panel chain + trailing "
                               "updates + Q_k^T formation)",
                     "bound": "latency (serial chain of N Householder columns)",
                     "chain_ms": bsof_ms,
                     "achieved_gbs": bsof_bytes / (bsof_ms * 1e-3) / 1e9 if bsof_ms else None,
                     "peak_gbs": hbm_peak(),
                     "algorithmic_bytes": bsof_bytes,
                     "achieved_tflops": flops_bsof(n, L) / (bsof_ms * 1e-3) / 1e12 if bsof_ms else None}

    c4 = None
    if args.c4_steps > 0:
        c4 = run_c4(api, torch, dev, stream, args.c4_steps, max(args.warmup, 3), peak, rank)

    batched = None
    if args.batch > 0:
        specs = [(side, L, U, 5000 + 100 * rank + i) for i in range(args.batch)]
        batched = run_batched(api, torch, dev, specs, args.batch_steps, stream)
        batched["workload"] = ("%d independent FP64 inversions per step, %dx%d lattice, n=%d, "
                               "p=%d (one walker each)" % (args.batch, side, side, n, L))
    mixed = None
    if args.mixed_steps > 0:
        mixed = run_mixed_single(api, torch, dev, stream, side, L, U, args.mixed_steps,
                                 max(args.warmup, 3), rank, value)
    batched_mp = None
    if args.batch > 0 and args.mixed_steps > 0:
        specs = [(side, L, U, 5000 + 100 * rank + i) for i in range(args.batch)]
        batched_mp = run_batched(api, torch, dev, specs, args.batch_steps, stream, precision=1)
        batched_mp["workload"] = ("%d independent inversions per step, %dx%d lattice, n=%d, p=%d;"
                                  " FP64 factorization, BSOI on the int8 tensor cores (Ozaki "
                                  "scheme, 8 slices)" % (args.batch, side, side, n, L))
        if batched and batched.get("value"):
            batched_mp["ratio_to_fp64_batched"] = batched_mp["value"] / batched["value"]
    batched_mixed = batched_mixed_mp = None
    if args.batch_mixed > 0:
        rng = np.random.default_rng(77 + rank)
        specs = [(int(rng.choice([8, 10, 12, 14, 16])), int(rng.integers(8, 65)),
                  float(rng.uniform(2.0, 6.0)), 9000 + 1000 * rank + i)
                 for i in range(args.batch_mixed)]
        wl = ("%d independent inversions per step, lattice side in {8,10,12,14,16}, p uniform "
              "in [8,64], U uniform in [2,6]%s" % (args.batch_mixed, " (the batched configuration)"
                                                   if args.batch_mixed >= 256 else ""))
        batched_mixed = run_batched_packed(api, torch, dev, specs, args.batch_steps, stream)
        batched_mixed["workload"] = wl
        if args.mixed_steps > 0:
            batched_mixed_mp = run_batched_packed(api, torch, dev, specs, args.batch_steps, stream,
                                                  precision=1)
            batched_mixed_mp["workload"] = wl
            batched_mixed_mp["ratio_to_fp64_batched"] = (batched_mixed_mp["value"] /
                                                         batched_mixed["value"])

    sharded = None
    if args.shard_ranks > 0 and world == 1:
        sharded = run_storage_sharded(args.shard_ranks, c4)

    served = None
    if args.serve > 0:
        served = run_serving(api, torch, dev, args.serve, args.serve_rate, 31 + rank,
                             args.serve_mixed if args.mixed_steps > 0 else 0.0)

    e2e = e2e_pageable = e2e_fp32 = None
    if not args.no_e2e and args.e2e_steps > 0:
        e2e = run_e2e(api, torch, dist, world, side, L, U, rank, args.e2e_steps)
        e2e_pageable = run_e2e(api, torch, dist, world, side, L, U, rank, args.e2e_steps,
                               pinned=False)
        e2e_fp32 = run_e2e_fp32(torch, dist, world, side, L, U, rank, args.e2e_steps)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu and args.cpu_sample > 0:
        out = cpu_reference(side, L, U, args.cpu_sample)
        if out is not None:
            cpu = {"value": len(out["times"]) / sum(out["times"]), "unit": "inversions/s",
                   "cores": out["cores"], "kind": "reference",
                   "sample": "%d inversions of the same workload through oracle/_ref "
                             "(reference CPU path, OpenBLAS, %d threads)"
                             % (len(out["times"]), out["cores"])}

    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": "inversions/s", "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_max / args.steps,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                "dtype": "f64",
                "data": "synthetic: seeded Hubbard DQMC matrices (random +-1 fields)",
                "config": config(args, n, N),
                "tflops": bsofi_flops(n, L) * value / world / 1e12,
                "residual": resid,
                "roofline": roofline, "roofline_bsof": roofline_bsof, "c4": c4,
                "cpu_baseline": cpu, "e2e": e2e, "e2e_pageable": e2e_pageable,
                "e2e_fp32": e2e_fp32,
                "batched": batched, "batched_mixed_sizes": batched_mixed, "served": served,
                "storage_sharded": sharded,
                "mixed": mixed, "batched_mixed_precision": batched_mp,
                "batched_mixed_sizes_mixed_precision": batched_mixed_mp,
                "gpu_launches": launches_per_step * args.steps,
                "clocks": clk}
        print(json.dumps(line))
    if world > 1:
        dist.destroy_process_group()


def run_c4(api, torch, dev, stream, steps, warmup, peak, rank):
    """The plain FP64 path at n = 400, p = 64, U = 6 (N = 25600, 5.2 GB per
    matrix, larger than L2): device-resident single inversions with the
    default launch plan, each timed with CUDA events on its stream from a
    fresh copy of the input made outside the timed window.  TFLOP/s uses the
    reference's flop model; frac is against the DGEMM peak measured in this
    run."""
    from bsofi_b200 import replicas
    side, L, U = 20, 64, 6.0
    n = side * side
    N = n * L
    blocks = hubbard_pcyclic(side, L, U, 7000 + rank)
    pristine = pcyclic_device(torch, *blocks, N, dev)
    work = torch.empty_like(pristine)
    dtau = torch.zeros(N, dtype=torch.float64, device=dev)
    ws = torch.zeros(api.workspace_bytes(n, L, N) // 8 + 1, dtype=torch.float64, device=dev)
    sp = stream.cuda_stream
    total = 0.0
    for it in range(warmup + steps):
        work.copy_(pristine)
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        with torch.cuda.stream(stream):
            e0.record(stream)
            rc = api.device_invert(n, L, work.data_ptr(), N, dtau.data_ptr(), ws.data_ptr(), sp)
            e1.record(stream)
        torch.cuda.synchronize()
        if rc != 0:
            raise RuntimeError("bsofi_device_invert (n=400, p=64) failed: %d" % rc)
        if it >= warmup:
            total += e0.elapsed_time(e1)
    ms = replicas.max_over_ranks(total, dev) / steps
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from gpu_util import block_residual_colmajor
    resid = block_residual_colmajor(torch, *blocks, work, N)
    _, plan = api.plan_get(n, L)
    tf = bsofi_flops(n, L) / (ms * 1e-3) / 1e12
    del pristine, work, ws
    torch.cuda.empty_cache()
    return {"workload": "single FP64 inversion, 20x20 lattice, n=400, p=64, N=25600, U=6 "
                        "(inputs larger than L2)",
            "steps": steps, "warmup": warmup, "ms_per_inversion": ms,
            "value": 1e3 / ms, "unit": "inversions/s", "tflops": tf,
            "frac": tf / peak if peak else None,
            "peak": peak, "peak_source": "cuBLAS DGEMM 8192^3 measured in this run",
            "residual": resid, "plan": plan}


def run_storage_sharded(ranks, c4):
    """The storage-sharded inversion at C4 (n = 400, p = 64, U = 6) for
    `ranks` ranks, each rank's share (the replicated compact factorization,
    its block columns of R^{-1}, its BSOI row band) timed in turn on this GPU
    with CUDA events.  The all-to-all between ranks is not timed (one GPU):
    its bytes per rank are reported."""
    from bsofi_b200.diag import shard_storage_timing
    r = shard_storage_timing(400, 64, ranks, 6.0)
    per_rank = [r["factor_ms"] + c + w for c, w in zip(r["columns_ms"], r["rows_ms"])]
    out = {"workload": "C4 (n=400, p=64, U=6, N=25600) split over %d ranks with no rank "
                       "holding M or M^-1 whole; each rank's kernels run in turn on this GPU"
                       % ranks,
           "factor_ms": r["factor_ms"], "columns_ms": r["columns_ms"], "rows_ms": r["rows_ms"],
           "device_ms_per_rank": per_rank, "max_device_ms": max(per_rank),
           "sent_bytes_per_rank": r["sent_bytes"], "state_bytes": r["state_bytes"],
           "not_timed": "the all-to-all of column slabs into row bands (one GPU here)"}
    if c4 and c4.get("ms_per_inversion"):
        out["single_gpu_ms"] = c4["ms_per_inversion"]
        out["speedup_device_time"] = c4["ms_per_inversion"] / max(per_rank)
    return out


def run_mixed_single(api, torch, dev, stream, side, L, U, steps, warmup, rank, fp64_value):
    """Single inversions of the headline size with BSOI on the int8 tensor
    cores (bsofi_device_invert_mixed, 8 slices), device-resident, CUDA-event
    timed on the launching stream, a fresh input copy per step made outside
    the timed window; residual and relative error against the FP64 path on
    the same matrix."""
    from bsofi_b200 import replicas
    n = side * side
    N = n * L
    ldd = (N + 31) // 32 * 32
    blocks = hubbard_pcyclic(side, L, U, 8000 + rank)
    pristine = pcyclic_device(torch, *blocks, ldd, dev)
    work = torch.empty_like(pristine)
    dtau = torch.zeros(N, dtype=torch.float64, device=dev)
    ws = torch.zeros(api.mixed_workspace_bytes(n, L, ldd) // 8 + 1, dtype=torch.float64,
                     device=dev)
    sp = stream.cuda_stream
    total = 0.0
    api.timing(True)
    for it in range(warmup + steps):
        work.copy_(pristine)
        torch.cuda.synchronize()
        if it == warmup:
            api.timing(True)  # BSOI product launches of the timed steps only
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        with torch.cuda.stream(stream):
            e0.record(stream)
            rc = api.device_invert_mixed(n, L, work.data_ptr(), ldd, dtau.data_ptr(),
                                         ws.data_ptr(), 0, sp)
            e1.record(stream)
        torch.cuda.synchronize()
        if rc != 0:
            raise RuntimeError("bsofi_device_invert_mixed failed: %d" % rc)
        if it >= warmup:
            total += e0.elapsed_time(e1)
    bsoi_ms, bsoi_launches = api.timing_read()
    api.timing(False)
    ms = replicas.max_over_ranks(total, dev) / steps
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from gpu_util import block_residual_colmajor
    resid = block_residual_colmajor(torch, *blocks, work, N)
    ref = pristine.clone()
    ws64 = torch.zeros(api.workspace_bytes(n, L, ldd) // 8 + 1, dtype=torch.float64, device=dev)
    if api.device_invert(n, L, ref.data_ptr(), ldd, dtau.data_ptr(), ws64.data_ptr(), 0) != 0:
        raise RuntimeError("bsofi_device_invert failed")
    torch.cuda.synchronize()
    relerr = float(torch.linalg.norm(work[:, :N] - ref[:, :N]) / torch.linalg.norm(ref[:, :N]))
    del pristine, work, ws, ws64, ref
    torch.cuda.empty_cache()
    value = 1e3 / ms
    return {"workload": "single inversion, %dx%d lattice, n=%d, p=%d, U=%g: FP64 BSOF/BSTRI, "
                        "BSOI products on the int8 tensor cores (Ozaki scheme, 8 slices)"
                        % (side, side, n, L, U),
            "value": value, "unit": "inversions/s", "ms_per_inversion": ms, "steps": steps,
            "ratio_to_fp64_single": value / fp64_value if fp64_value else None,
            "residual": resid, "relative_error_vs_fp64": relerr,
            "bsoi_ms_per_inversion": bsoi_ms / steps,
            "bsoi_effective_fp64_tflops": flops_bsoi(n, L) / (bsoi_ms / steps * 1e-3) / 1e12
            if bsoi_ms > 0 else None,
            "bsoi_timed_launches": bsoi_launches}


def run_batched_packed(api, torch, dev, specs, steps, stream, precision=0):
    """The batched configuration at its full size: every instance keeps only
    its packed coupling blocks on the device, and before each timed batch the
    inputs are re-assembled into the instances' matrices with
    bsofi_device_assemble (outside the timed window), so no second copy of
    the matrices is held.  Rate = instances / summed batch time (CUDA events,
    max over ranks)."""
    from bsofi_b200 import replicas
    ns, Ls, lds, bufs, packs = [], [], [], [], []
    flops = 0.0
    for side, L, U, seed in specs:
        n = side * side
        N = n * L
        ld = (N + 31) // 32 * 32
        _, sub = hubbard_pcyclic(side, L, U, seed)
        packs.append(torch.from_numpy(np.ascontiguousarray(np.transpose(sub, (0, 2, 1))))
                     .to(dev))
        bufs.append(torch.empty((N, ld), dtype=torch.float64, device=dev))
        ns.append(n)
        Ls.append(L)
        lds.append(ld)
        flops += bsofi_flops(n, L)
    taus = [torch.zeros(n * L, dtype=torch.float64, device=dev) for n, L in zip(ns, Ls)]
    ws = torch.zeros(api.batch_workspace_bytes(ns, Ls, lds, precision) // 8 + 1,
                     dtype=torch.float64, device=dev)
    sp = stream.cuda_stream
    total_ms = 0.0
    for it in range(steps + 1):  # the first batch is a warm-up
        for n, L, b, pk, ld in zip(ns, Ls, bufs, packs, lds):
            if api.device_assemble(n, L, 0, pk.data_ptr(), b.data_ptr(), ld) != 0:
                raise RuntimeError("bsofi_device_assemble failed")
        torch.cuda.synchronize()
        replicas.barrier()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        with torch.cuda.stream(stream):
            e0.record(stream)
            rc = api.device_invert_batched(ns, Ls, [b.data_ptr() for b in bufs], lds,
                                           [t.data_ptr() for t in taus], ws.data_ptr(), 16, sp,
                                           precision)
            e1.record(stream)
        torch.cuda.synchronize()
        if rc != 0:
            raise RuntimeError("bsofi_device_invert_batched_ex failed: %d" % rc)
        if it > 0:
            total_ms += e0.elapsed_time(e1)
    launches = api.last_launches()
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from gpu_util import block_residual_colmajor
    worst = 0.0
    for i in range(0, len(specs), max(1, len(specs) // 8)):  # 8 instances checked
        side, L, U, seed = specs[i]
        worst = max(worst, block_residual_colmajor(torch, *hubbard_pcyclic(side, L, U, seed),
                                                   bufs[i], ns[i] * Ls[i]))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    ms_max = replicas.max_over_ranks(total_ms, dev)
    out = {"value": world * len(specs) * steps / (ms_max * 1e-3), "unit": "inversions/s",
           "steps": steps, "ms_per_step": ms_max / steps,
           "tflops": flops * steps * world / (ms_max * 1e-3) / 1e12,
           "instances_per_step": len(specs), "worst_residual_of_8_checked": worst,
           "gpu_launches_per_step": launches, "precision": "FP64" if precision == 0 else
           "mixed (BSOI on the int8 tensor cores, 8 slices)"}
    del bufs, packs, ws, taus
    torch.cuda.empty_cache()
    return out


def run_batched(api, torch, dev, specs, steps, stream, precision=0):
    """Time bsofi_device_invert_batched_ex over `steps` batches (precision 0
    FP64, 1 mixed: BSOI on the int8 tensor cores).  Every batch starts from
    fresh inputs copied from pristine device buffers outside the timed
    window; the reported rate is instances / summed batch time, max over
    ranks."""
    from bsofi_b200 import replicas
    ns, Ls, lds, pristine = [], [], [], []
    flops = 0.0
    for side, L, U, seed in specs:
        n = side * side
        N = n * L
        ld = (N + 31) // 32 * 32
        pristine.append(pcyclic_device(torch, *hubbard_pcyclic(side, L, U, seed), ld, dev))
        ns.append(n)
        Ls.append(L)
        lds.append(ld)
        flops += bsofi_flops(n, L)
    work = [torch.empty_like(t) for t in pristine]
    taus = [torch.zeros(n * L, dtype=torch.float64, device=dev) for n, L in zip(ns, Ls)]
    ws = torch.zeros(api.batch_workspace_bytes(ns, Ls, lds, precision) // 8 + 1,
                     dtype=torch.float64, device=dev)
    sp = stream.cuda_stream
    total_ms = 0.0
    for it in range(steps + 1):  # the first batch is a warm-up
        for w, p0 in zip(work, pristine):
            w.copy_(p0)
        torch.cuda.synchronize()
        replicas.barrier()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        with torch.cuda.stream(stream):
            e0.record(stream)
            rc = api.device_invert_batched(ns, Ls, [w.data_ptr() for w in work], lds,
                                           [t.data_ptr() for t in taus], ws.data_ptr(), 8, sp,
                                           precision)
            e1.record(stream)
        torch.cuda.synchronize()
        if rc != 0:
            raise RuntimeError("bsofi_device_invert_batched failed: %d" % rc)
        if it > 0:
            total_ms += e0.elapsed_time(e1)
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from gpu_util import block_residual_gpu
    side, L, U, seed = specs[0]
    resid = block_residual_gpu(torch, *hubbard_pcyclic(side, L, U, seed),
                               work[0][:, :ns[0] * Ls[0]].T.contiguous())
    world = int(os.environ.get("WORLD_SIZE", "1"))
    ms_max = replicas.max_over_ranks(total_ms, dev)
    rate = world * len(specs) * steps / (ms_max * 1e-3)
    launches = api.last_launches()
    if precision == 1:
        # Against the FP64 inverse of the same first instance.
        ref = pristine[0].clone()
        dtau0 = torch.zeros(ns[0] * Ls[0], dtype=torch.float64, device=dev)
        ws0 = torch.zeros(api.workspace_bytes(ns[0], Ls[0], lds[0]) // 8 + 1,
                          dtype=torch.float64, device=dev)
        if api.device_invert(ns[0], Ls[0], ref.data_ptr(), lds[0], dtau0.data_ptr(),
                             ws0.data_ptr(), 0) != 0:
            raise RuntimeError("bsofi_device_invert failed")
        torch.cuda.synchronize()
        N0 = ns[0] * Ls[0]
        relerr = float(torch.linalg.norm(work[0][:, :N0] - ref[:, :N0]) /
                       torch.linalg.norm(ref[:, :N0]))
        del ref, ws0
        out = {"value": rate, "unit": "inversions/s", "steps": steps,
               "ms_per_step": ms_max / steps,
               "tflops": flops * steps * world / (ms_max * 1e-3) / 1e12,
               "instances_per_step": len(specs), "residual_first_instance": resid,
               "relative_error_vs_fp64_first_instance": relerr,
               "gpu_launches_per_step": launches,
               "slices": 8}
        del work, pristine, ws
        torch.cuda.empty_cache()
        return out
    # The same batch captured once into a CUDA graph and replayed.
    graph_ms = 0.0
    g = api.BatchGraph(ns, Ls, [w.data_ptr() for w in work], lds, [t.data_ptr() for t in taus],
                       ws.data_ptr(), 8)
    for it in range(steps + 1):
        for w, p0 in zip(work, pristine):
            w.copy_(p0)
        torch.cuda.synchronize()
        replicas.barrier()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        rc = g.launch(sp)
        e1.record(stream)
        torch.cuda.synchronize()
        if rc != 0:
            raise RuntimeError("bsofi_batch_graph_launch failed: %d" % rc)
        if it > 0:
            graph_ms += e0.elapsed_time(e1)
    g.close()
    graph_ms = replicas.max_over_ranks(graph_ms, dev)
    out = {"value": rate, "unit": "inversions/s", "steps": steps,
           "ms_per_step": ms_max / steps, "tflops": flops * steps * world / (ms_max * 1e-3) / 1e12,
           "instances_per_step": len(specs), "residual_first_instance": resid,
           "gpu_launches_per_step": launches,
           "graph_value": world * len(specs) * steps / (graph_ms * 1e-3)}
    del work, pristine, ws
    torch.cuda.empty_cache()
    return out


def run_serving(api, torch, dev, nreq, rate, seed, mixed_frac=0.5):
    """A Poisson stream of inversion requests through the continuous-batching
    server (bsofi_server_*), server-owned: each request is submitted as its
    packed coupling blocks (built on the device at its arrival), and the
    server's pool supplies matrix, tau and workspace at admission (admission
    by full memory footprint, up to 17 GB at n = 576, p = 80).  Sizes follow
    the serving configuration (lattice side uniform in 8..24, so n = 64..576;
    p uniform in 10..80; U in 2..6); a fraction mixed_frac of the requests
    runs mixed precision (BSOI on the int8 tensor cores).  Latency is wall
    clock from submission to the poll that sees the request finish; the
    result is then released."""
    from bsofi_b200 import replicas
    from bsofi_b200.hubbard import expm_sym, lattice_adjacency
    rng = np.random.default_rng(seed)
    specs = [(int(rng.integers(8, 25)), int(rng.integers(10, 81)), float(rng.uniform(2, 6)),
              int(rng.random() < mixed_frac)) for _ in range(nreq)]
    arrivals = np.cumsum(rng.exponential(1.0 / rate, nreq))
    expk = {}
    flops = sum(bsofi_flops(sd * sd, L) for sd, L, _, _ in specs)
    free, _ = torch.cuda.mem_get_info(dev)
    pool = int(min(free - (12 << 30), 140 << 30))
    srv = api.Server(slots=8, pool_bytes=pool)
    submit_t, lat, keep, prec_of = {}, [], {}, {}
    nxt, done = 0, 0
    replicas.barrier()
    t0 = time.perf_counter()
    while done < nreq:
        now = time.perf_counter() - t0
        while nxt < nreq and arrivals[nxt] <= now:
            sd, L, U, prec = specs[nxt]
            n = sd * sd
            if sd not in expk:
                expk[sd] = torch.from_numpy(expm_sym(0.125 * lattice_adjacency(sd))).to(dev)
            lam = float(np.arccosh(np.exp(U * 0.125 / 2.0)))
            h = torch.from_numpy(rng.choice(np.array([-1.0, 1.0]), size=(L, n))).to(dev)
            # Packed column-major blocks: block k is B_{k+1} = expK diag(exp(lam h_k)),
            # negated below the diagonal, +B_p in the corner.
            S = expk[sd][None, :, :] * torch.exp(lam * h)[:, :, None]
            S[:L - 1] *= -1.0
            torch.cuda.current_stream().synchronize()  # blocks in HBM before submission
            rid = srv.submit_blocks(n, L, S.data_ptr(), precision=prec)
            submit_t[rid] = time.perf_counter() - t0
            keep[rid] = S
            prec_of[rid] = prec
            nxt += 1
        for rid, st in srv.poll():
            if st != 0:
                raise RuntimeError("served request %d failed: %d" % (rid, st))
            lat.append((time.perf_counter() - t0 - submit_t[rid], prec_of[rid]))
            srv.release(rid)
            del keep[rid]
            done += 1
        time.sleep(0.0002)
    t_end = time.perf_counter() - t0
    srv.close()
    torch.cuda.empty_cache()
    ms = np.array([x for x, _ in lat]) * 1e3
    pr = np.array([p for _, p in lat])
    span = t_end - arrivals[0]

    def pct(a, q):
        return float(np.percentile(a, q)) if len(a) else None

    return {"requests": nreq, "arrival_rate_per_s": rate,
            "value": nreq / span, "unit": "inversions/s",
            "tflops": flops / span / 1e12,
            "p50_ms": pct(ms, 50), "p99_ms": pct(ms, 99), "max_ms": float(ms.max()),
            "p50_ms_fp64": pct(ms[pr == 0], 50), "p99_ms_fp64": pct(ms[pr == 0], 99),
            "p50_ms_mixed": pct(ms[pr == 1], 50), "p99_ms_mixed": pct(ms[pr == 1], 99),
            "requests_mixed": int(pr.sum()), "precision_mix": "%d%% mixed (BSOI on the int8 "
            "tensor cores), the rest FP64" % round(100 * mixed_frac),
            "pool_gib": pool / 2 ** 30,
            "workload": "Poisson stream, lattice side uniform in 8..24 (n = 64..576), p uniform "
                        "in 10..80, U uniform in 2..6; %d requests%s, 8 slots, server-owned "
                        "memory (matrix + tau + workspace per request from one pool)"
                        % (nreq, "" if nreq >= 10000 else
                           " (a sample of the 10,000-request serving configuration)")}


def run_e2e(api, torch, dist, world, side, L, U, rank, steps, pinned=True):
    """The reference-facing handle API on host buffers: hybridxbsoftrih_ +
    hybridxbsoih_ per step, every copy between host and device included.
    pinned: the caller's A and tau are page-locked (torch pinned memory);
    otherwise ordinary pageable numpy arrays."""
    from bsofi_b200.hubbard import hubbard_matrix
    n = side * side
    N = n * L
    M = hubbard_matrix(side, L, U, seed=777 + rank)
    if pinned:
        # Column-major N x N view of a pinned row-major buffer.
        A = torch.empty((N, N), dtype=torch.float64, pin_memory=True).numpy().T
        tau = torch.zeros(N, dtype=torch.float64, pin_memory=True).numpy()
    else:
        A = np.empty_like(M, order="F")
        tau = np.zeros(N)
    h = api.Handle(n, L)
    times = []
    for i in range(steps + 1):
        np.copyto(A, M)
        if world > 1:
            dist.barrier()
        t0 = time.perf_counter()
        info = h.bsoftri(A, tau)
        info2 = h.bsoi(A, tau)
        dt = time.perf_counter() - t0
        if info or info2:
            raise RuntimeError("handle API info %d %d" % (info, info2))
        if i > 0:
            times.append(dt)
    h.close()
    # The e2e result must be the inverse: residual of the last step on the GPU.
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from gpu_util import block_residual_gpu
    from bsofi_b200.hubbard import pcyclic_blocks
    resid = block_residual_gpu(torch, *pcyclic_blocks(M, n, L),
                               torch.from_numpy(np.ascontiguousarray(A)).to("cuda"))
    if not resid < 1e-12:
        raise RuntimeError("e2e result check failed: residual %g" % resid)
    tot = sum(times)
    t = torch.tensor([tot], dtype=torch.float64, device="cuda")
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    tot = float(t.item())
    state_bytes = sum(min(N, (k + 2) * n) * n for k in range(L)) * 8
    h2d = 2 * L * n * n * 8 + state_bytes + N * 8
    d2h = state_bytes + N * 8 + N * N * 8
    return {"value": world * len(times) / tot, "unit": "inversions/s",
            "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
            "api": "hybridxbsoftrih_ + hybridxbsoih_ (host %s buffers)"
                   % ("pinned" if pinned else "pageable"),
            "steps": len(times), "residual": resid}


def run_e2e_fp32(torch, dist, world, side, L, U, rank, steps):
    """The single-precision library's handle API (libbsofi_b200_fp32.so) on
    pinned float32 host buffers, copies included: same workload, half the
    host <-> device bytes of the FP64 API."""
    from bsofi_b200 import fp32
    from bsofi_b200.hubbard import hubbard_matrix, pcyclic_blocks
    n = side * side
    N = n * L
    M32 = hubbard_matrix(side, L, U, seed=777 + rank).astype(np.float32)
    A = torch.empty((N, N), dtype=torch.float32, pin_memory=True).numpy().T
    tau = torch.zeros(N, dtype=torch.float32, pin_memory=True).numpy()
    h = fp32.Handle(n, L)
    times = []
    for i in range(steps + 1):
        np.copyto(A, M32)
        if world > 1:
            dist.barrier()
        t0 = time.perf_counter()
        info = h.bsoftri(A, tau)
        info2 = h.bsoi(A, tau)
        dt = time.perf_counter() - t0
        if info or info2:
            raise RuntimeError("FP32 handle API info %d %d" % (info, info2))
        if i > 0:
            times.append(dt)
    h.close()
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from gpu_util import block_residual_gpu
    resid = block_residual_gpu(torch, *pcyclic_blocks(M32.astype(np.float64), n, L),
                               torch.from_numpy(np.ascontiguousarray(A, dtype=np.float64)).to("cuda"))
    if not resid < 1e-5:
        raise RuntimeError("FP32 e2e result check failed: residual %g" % resid)
    t = torch.tensor([sum(times)], dtype=torch.float64, device="cuda")
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    tot = float(t.item())
    state_bytes = sum(min(N, (k + 2) * n) * n for k in range(L)) * 4
    return {"value": world * len(times) / tot, "unit": "inversions/s",
            "h2d_bytes_per_step": 2 * L * n * n * 4 + state_bytes + N * 4,
            "d2h_bytes_per_step": state_bytes + N * 4 + N * N * 4,
            "api": "hybridxbsoftrih_ + hybridxbsoih_ of libbsofi_b200_fp32.so (host pinned "
                   "float32 buffers; FP64 arithmetic on the GPU, results rounded to float32)",
            "steps": len(times), "residual": resid}


if __name__ == "__main__":
    main()
