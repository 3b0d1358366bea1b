#!/usr/bin/env python3
"""Benchmark: rank-k iSVD (Gaussian projection / Gramian / Kolmogorov-Nagumo / Gramian) of a
200000 x 20000 FP32 matrix, k = 100, p = 28 (l = 128), N = 32 sketches, on one B200.  Prints one
JSON line.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference] [--size full|small]
                    [--parallel rowblock|replicas] [--dist-backend nccl|gloo]

On N GPUs (torchrun, one rank per GPU) the default is one solve of the same matrix split by rows
over the N ranks (the reference's dista = 'R' decomposition): each rank holds the rows
isvd_createParam gives it and the exchanges (block Grams, G = Qs'Qs, Z = A'Qbar) run as an NCCL
AllReduce on the library's stream through isvd_gpu_set_allreduce (strong scaling, value = solves/s
of the whole job).  --parallel replicas runs one independent solve per rank instead (weak scaling).

Inputs are synthetic and seeded: A = U diag(sigma) V' + 1e-4 G with Haar-random U (m x 2000),
V (n x 2000), sigma geometric from 1 to 1e-3 over 2000 values, G standard normal; generated on
the GPU before the timed region.  A (16 GB) is larger than L2 (126 MB), so no flush is needed
between timed solves.  A step is one full solve through the C ABI (isvd_sIsvd_ex, MIXED
precision: bf16 split tcgen05 products, FP64 l x l steps).  The FP64 path (isvd_dIsvd_ex, NATIVE)
is timed once on the same matrix and the same Omega for the speed-up and the sigma error.
"""
import argparse
import ctypes
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, REPO)

WORKLOADS = {
    # the headline workload: 200000 x 20000 FP32, rank-2000 factors, k = 100, p = 28, N = 32
    "full": dict(m=200000, n=20000, rank=2000, k=100, p=28, N=32, noise=1e-4, seed=2),
    # a reduced shape of the same construction, for quick checks
    "small": dict(m=20000, n=4000, rank=400, k=100, p=28, N=8, noise=1e-4, seed=2),
    # two sketch panels of the full shape (same n, N l and panel rows), for kernel profiles
    "panel": dict(m=26624, n=20000, rank=2000, k=100, p=28, N=32, noise=1e-4, seed=2),
}
METRIC = "rank-k iSVD solves/s (time & %roofline), mixed-prec vs plain FP64 on B200 at sigma rel err <= 1e-5"


def peaks():
    """(HBM GB/s, bf16 TFLOP/s burst, bf16 TFLOP/s sustained, kind)."""
    try:
        with open(os.path.join(REPO, "MEASURED_PEAKS.json")) as fh:
            d = json.load(fh)
        return (float(d["hbm_gbs"]), float(d["bf16_tflops"]),
                float(d.get("bf16_tflops_sustained", d["bf16_tflops"])), "measured")
    except (OSError, KeyError, ValueError):
        return 6650.0, 1590.0, 1400.0, "fallback"


# DRAM bytes (read + write) of the sketch kernel's one launch over the 200000 x 20000 matrix
# (N l = 4096, tiles in two column groups, Y written as bf16 planes), from a one-pass ncu capture
# of a full solve (dram__bytes_read.sum + dram__bytes_write.sum, `bench.py --single`)
SKETCH_LAUNCH_TRAFFIC = 69.929373696e9 + 4.996154112e9


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled every 50 ms during the timed region: entering
    waits (up to 5 s) for nvidia-smi's first line and drops it, so that the samples kept start with
    the region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu):
        self.gpu = gpu
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), "--query-gpu=" + self.FIELDS,
                                          "--format=csv,noheader,nounits", "-lms", "50"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.first = threading.Event()
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
            self.first.wait(5.0)
            self.lines.clear()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for ln in self.proc.stdout:
            self.lines.append(ln.strip())
            self.first.set()
        self.first.set()

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = max(mx, float(f[2]))
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


def make_matrix(torch, w, dev, seed):
    """A = U diag(sigma) V' + noise * G (FP32, row-major), Haar factors from QR of Gaussians."""
    g = torch.Generator(device=dev)
    g.manual_seed(seed)
    m, n, r = w["m"], w["n"], w["rank"]
    u = torch.linalg.qr(torch.randn(m, r, generator=g, device=dev, dtype=torch.float32))[0]
    v = torch.linalg.qr(torch.randn(n, r, generator=g, device=dev, dtype=torch.float32))[0]
    sig = torch.logspace(0.0, -3.0, r, device=dev, dtype=torch.float32)
    a = torch.randn(m, n, generator=g, device=dev, dtype=torch.float32)
    a.mul_(w["noise"])
    a.addmm_(u * sig, v.t())
    del u, v
    return a


def make_row_block(torch, w, dev, seed, prm):
    """This rank's rows [rowidxbegin, rowidxend) of A = U diag(sigma) V' + noise * G for a solve split
    by rows: U's row block is the orthonormal factor of a local Gaussian block scaled by
    sqrt(rows / m), so that the stacked U is exactly orthonormal (U'U = sum_j (m_j / m) I = I); V (the
    same on every rank) and sigma as make_matrix; the noise is drawn per rank."""
    m, n, r = w["m"], w["n"], w["rank"]
    rows = int(prm.nrow_proc)
    gv = torch.Generator(device=dev)
    gv.manual_seed(seed)
    v = torch.linalg.qr(torch.randn(n, r, generator=gv, device=dev, dtype=torch.float32))[0]
    g = torch.Generator(device=dev)
    g.manual_seed(seed + 7919 * (int(prm.mpi_rank) + 1))
    u = torch.linalg.qr(torch.randn(rows, r, generator=g, device=dev, dtype=torch.float32))[0]
    u.mul_((rows / m) ** 0.5)
    sig = torch.logspace(0.0, -3.0, r, device=dev, dtype=torch.float32)
    a = torch.randn(rows, n, generator=g, device=dev, dtype=torch.float32)
    a.mul_(w["noise"])
    a.addmm_(u * sig, v.t())
    del u, v
    return a


def solve(lib, x, prm, a, lda, s, ut, vt, l, seed, precision, retc=(0, 0, 2, 0)):
    retv, times, status = lib.isvd(x, prm, ("GP", "GR", "KN", "GR"), a, lda, s, ut, l, vt, l, seed=seed,
                                   retc=retc, argv=[None, None, [256, 1e-4], None], precision=precision)
    if status != 0:
        raise RuntimeError("isvd_%sIsvd_ex failed: %s" % (x, lib.last_error()))
    return retv, times


# ------------------------------------------------------------------------------ CPU reference
# The row-sample extrapolation over-estimates the full solve: on 8192 rows every stage costs more
# per row than on 200000 (cache reuse, fixed costs).  Measured once on this pool's host (16 cores,
# OpenBLAS; tests/test_gpu_parity_full.py case "cal"): the reference's isvd_sIsvd on the full
# 200000 x 20000 matrix took 51.6 / 3.9 / 91.2 / 4.0 s per stage (150.6 s, 77 KN iterations)
# against 58.0 / 6.7 / 113.0 / 4.5 s extrapolated from the 8192-row sample (182.2 s, 78): these
# per-stage ratios scale the extrapolation of that shape.
REF_CAL_SHAPE = (200000, 20000, 8192)
REF_CAL = (51.573 / 58.023, 3.922 / 6.748, 91.186 / 112.977, 3.967 / 4.455)


def reference_calibrated(w, stage_t, rows):
    """Stage seconds of the full solve from the sample's extrapolation (calibrated when measured)."""
    if (w["m"], w["n"], rows) == REF_CAL_SHAPE:
        return np.asarray(stage_t) * np.asarray(REF_CAL), True
    return np.asarray(stage_t), False


def reference_sample(w, steps, warmup, threads):
    """The reference's own CPU pipeline (oracle/_ref, OpenBLAS, 1 MPI rank, `threads` OpenMP
    threads) on a row sample of the workload; each stage time is scaled to the full row count
    (every stage's cost is linear in m).  Returns (stage seconds of a full solve, sample
    description, KN iterations of the sample, seconds per sample solve)."""
    os.environ["OMP_NUM_THREADS"] = str(threads)
    os.environ["OPENBLAS_NUM_THREADS"] = str(threads)
    sys.path.insert(0, os.path.join(REPO, "oracle"))
    import build_ref  # noqa: E402
    from isvd_b200.capi import IsvdLib
    ref = IsvdLib(build_ref.build())
    m, n, k, p, N = w["m"], w["n"], w["k"], w["p"], w["N"]
    l = k + p
    ms = int(os.environ.get("ISVD_BENCH_REF_ROWS", 8192 if m > 8192 else m))
    rng = np.random.default_rng(w["seed"])
    r = w["rank"]
    # rows of a Haar m x r factor are close to iid N(0, 1/m): the sample keeps A's row statistics
    us = rng.standard_normal((ms, r)).astype(np.float32) / np.sqrt(m)
    v = np.linalg.qr(rng.standard_normal((n, r)).astype(np.float32))[0]
    sig = np.logspace(0, -3, r).astype(np.float32)
    a = ((us * sig) @ v.T + w["noise"] * rng.standard_normal((ms, n)).astype(np.float32)).astype(np.float32)
    a = np.ascontiguousarray(a)
    prm = ref.create_param(ms, n, k, p, N)
    s = np.zeros(l, np.float32)
    ut = np.zeros((ms, l), np.float32)
    vt = np.zeros((n, l), np.float32)
    per = []
    its = []
    for i in range(warmup + steps):
        retv, times, _ = ref.isvd("s", prm, ("GP", "GR", "KN", "GR"), a, n, s, ut, l, vt, l, seed=w["seed"],
                                  argv=[None, None, [256, 1e-4], None], retc=(0, 0, 2, 0))
        if i >= warmup:
            per.append(times)
            its.append(int(retv[2][0]))
    scale = m / ms
    t = np.mean(np.array(per), axis=0) * scale
    desc = ("reference isvd_sIsvd (GP/GR/KN/GR, OpenBLAS, %d threads) on a %d x %d row sample, stage times "
            "scaled by m / %d" % (threads, ms, n, ms))
    t_cal, cal = reference_calibrated(w, t, ms)
    if cal:
        desc += " and by the per-stage ratios full / extrapolated measured once at full size (%.3f %.3f %.3f %.3f)" % REF_CAL
    return t_cal, desc, int(np.median(its)), float(np.mean(np.sum(np.array(per), axis=1))), t


def physical_cores():
    """Physical cores of this host (logical CPUs when the count is unavailable)."""
    try:
        import psutil
        n = psutil.cpu_count(logical=False)
        if n:
            return int(n)
    except ImportError:
        pass
    return os.cpu_count() or 1


def reference_arm(args, w):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    threads = physical_cores()
    t0 = time.time()
    stage_t, desc, its, step_s, raw_t = reference_sample(w, args.steps, args.warmup, threads)
    total = float(np.sum(stage_t))
    val = 1.0 / total
    out = {
        "impl": "reference", "metric": METRIC, "value": val, "unit": "solve/s", "n_gpus": args.gpus,
        # a step is one solve of the row sample (what was timed); value is the full solve's rate
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * step_s,
        "ms_per_solve_extrapolated": 1e3 * total, "higher_is_better": True,
        "scaling": "weak" if (args.gpus > 1 and args.parallel == "replicas") else "strong",
        "vs_baseline": None, "dtype": "fp32", "data": "synthetic (seeded row sample)",
        "config": config_dict(w, args.gpus, args.parallel),
        "cpu_baseline": {"value": val, "unit": "solve/s", "cores": threads, "kind": "reference", "sample": desc,
                         "stage_s": [float(x) for x in stage_t], "kn_iterations_sample": its,
                         "stage_s_uncalibrated": [float(x) for x in raw_t]},
        "e2e": {"value": val, "unit": "solve/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "wall_s": time.time() - t0,
    }
    print(json.dumps(out), flush=True)


def config_dict(w, world=1, parallel="rowblock"):
    if world == 1:
        par, ranks = "one GPU", "1 MPI rank"
    elif parallel == "rowblock":
        par = "row blocks over %d GPUs (NCCL AllReduce of the block Grams, G and Z)" % world
        ranks = "%d ranks" % world
    else:
        par, ranks = "replicas (one independent solve per GPU)", "1 MPI rank each"
    return {"workload": "iSVD %dx%d FP32, rank-%d Haar factors, sigma 1..1e-3 geometric, +%.0e noise; "
                        "k=%d p=%d N=%d; GP/GR/KN(1e-4,256)/GR, row block, %s"
                        % (w["m"], w["n"], w["rank"], w["noise"], w["k"], w["p"], w["N"], ranks),
            "m": w["m"], "n": w["n"], "k": w["k"], "p": w["p"], "N": w["N"], "seed": w["seed"],
            "l2_flush": "none needed: A (%.1f GB) is larger than L2" % (w["m"] * w["n"] * 4 / 1e9 / world),
            "parallelism": par}


# ------------------------------------------------------------------------------ B200 arm
BATCH = dict(count=256, m=(512, 8192), n=(256, 4096), k=(8, 16, 32, 64), N=8, noise=1e-4, seed=4)


SQUARE50K = dict(m=50000, n=50000, rank=5000, k=64, p=64, N=64, noise=1e-3, seed=3)


def square50k_main(args):
    """The 50000 x 50000 FP32 parity case: sigma_i = (1 + i)^(-1/2) for i < 5000 on Haar factors,
    + 1e-3 noise; k = 64, p = 64, N = 64; GP / TS / WY (tol 1e-4, maxit 512) / GR on column blocks
    (dista 'C').  One line: the MIXED solve (A resident, device-timed over K solves after W warm-up
    solves) beside one NATIVE FP64 solve on the FP64 copy of A with the same seed, and the largest
    relative difference of the k leading singular values."""
    import torch
    import isvd_b200
    w = SQUARE50K
    dev = torch.device("cuda", 0)
    lib = isvd_b200.load()
    stream = torch.cuda.current_stream(dev)
    lib.lib.isvd_gpu_set_stream(ctypes.c_void_p(stream.cuda_stream))
    g = torch.Generator(device=dev).manual_seed(w["seed"])
    m, n, r, k, p, N = w["m"], w["n"], w["rank"], w["k"], w["p"], w["N"]
    l = k + p
    u = torch.linalg.qr(torch.randn(m, r, generator=g, device=dev, dtype=torch.float32))[0]
    v = torch.linalg.qr(torch.randn(n, r, generator=g, device=dev, dtype=torch.float32))[0]
    sig = (1.0 + torch.arange(r, device=dev, dtype=torch.float32)) ** -0.5
    a = torch.randn(m, n, generator=g, device=dev, dtype=torch.float32).mul_(w["noise"])
    a.addmm_(u * sig, v.t())
    del u, v
    prm = lib.create_param(m, n, k, p, N)
    algs = ("GP", "TS", "WY", "GR")

    def run(x, mat, precision):
        dt = mat.dtype
        s = torch.zeros(l, dtype=dt, device=dev)
        ut = torch.zeros((m, l), dtype=dt, device=dev)
        vt = torch.zeros((n, l), dtype=dt, device=dev)
        retv, times, status = lib.isvd(x, prm, algs, mat, n, s, ut, l, vt, l, seed=w["seed"], dista=b"C", ordera=b"R",
                                       retc=(0, 0, 2, 0), argv=[None, None, [512, 1e-4], None], precision=precision)
        if status != 0:
            raise RuntimeError("50000 x 50000 solve failed: %s" % (lib.last_error(),))
        return s, retv, times

    for _ in range(args.warmup):
        run("s", a, 1)
    torch.cuda.synchronize()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    stage = np.zeros(4)
    with ClockSampler(0) as clk:
        ev0.record(stream)
        for _ in range(args.steps):
            s_mixed, retv, times = run("s", a, 1)
            stage += np.array(times)
        ev1.record(stream)
        torch.cuda.synchronize()
    mixed_ms = ev0.elapsed_time(ev1) / args.steps
    wy_mixed = int(retv[2][0])
    a64 = a.double()
    del a
    torch.cuda.synchronize()
    ev0.record(stream)
    s64, retv64, times64 = run("d", a64, 0)
    ev1.record(stream)
    torch.cuda.synchronize()
    fp64_ms = ev0.elapsed_time(ev1)
    s_ref = s64[:k].cpu().numpy()
    err = float(np.abs(s_mixed[:k].double().cpu().numpy() - s_ref).max() / s_ref.max())
    lib.lib.isvd_gpu_set_stream(None)
    print(json.dumps({"workload": "iSVD 50000x50000 FP32, sigma_i=(1+i)^-0.5 (i<5000) + 1e-3 noise; "
                                  "k=64 p=64 N=64; GP/TS/WY(1e-4,512)/GR, column blocks, 1 MPI rank",
                      "mixed_ms_per_solve": mixed_ms, "mixed_stage_ms": list(1e3 * stage / args.steps),
                      "mixed_wy_iterations": wy_mixed, "fp64_ms": fp64_ms,
                      "fp64_stage_ms": [1e3 * t for t in times64], "fp64_wy_iterations": int(retv64[2][0]),
                      "sigma_rel_err_max": err, "steps": args.steps, "warmup": args.warmup,
                      "note": "on this input Wen-Yin's stopping point (mu < tol^2) depends on rounding: the "
                              "reference's own result moves by 1.2e-4 in sigma (219 -> 157 iterations) under a "
                              "last-bit change of Y, so MIXED and FP64 differ by that order as well",
                      "clocks": clk.summary()}), flush=True)


def batch_main(args):
    """Batched uneven solves: 256 FP32 matrices, m log-uniform in [512, 8192], n log-uniform in
    [256, 4096] with n <= m, each rank 4k with a geometric spectrum (1 .. 1e-3) plus noise, k in
    {8, 16, 32, 64}, p = k/2, N = 8, GP / GR / KN / GR.  One line: the batch (isvd_sBatchIsvd, inputs
    resident, device-timed over K solves after W warm-up solves) beside the same 256 matrices solved
    one after another through isvd_sIsvd_ex (NATIVE FP32, one pass)."""
    import torch
    import isvd_b200
    out = run_batched(torch, isvd_b200.load(), args.steps, args.warmup, single=args.single)
    print(json.dumps(out), flush=True)


def kn_loop_main(args):
    """The MIXED Kolmogorov-Nagumo integration stage (isvd_sIntegrateKolmogorovNagumo) alone, at the
    loop shapes of the 200000 x 20000 workload (N = 32 blocks of l = 128, so G is 4096 x 4096) but on
    6000 rows, so that forming G and the final Qbar = Qs M take little of the time: W untimed calls,
    then K calls timed with CUDA events; the loop's cost per iteration without the sketch before it
    (which leaves the clock at the power cap in the full solve)."""
    import torch
    import isvd_b200
    lib = isvd_b200.load()
    lib.lib.isvd_gpu_set_precision(1)
    m, l, N = 6000, 128, 32
    dev = torch.device("cuda", 0)
    g = torch.Generator(device=dev).manual_seed(3)
    base = torch.linalg.qr(torch.randn(m, l, device=dev, dtype=torch.float64, generator=g))[0]
    qs = torch.cat([torch.linalg.qr(base + 0.05 * torch.randn(m, l, device=dev, dtype=torch.float64,
                                                               generator=g))[0] for _ in range(N)], dim=1)
    qs = qs.float().contiguous()
    qt = torch.zeros((m, l), device=dev)
    prm = lib.create_param(m, m, l, 0, N)
    stream = torch.cuda.current_stream(dev)
    lib.lib.isvd_gpu_set_stream(ctypes.c_void_p(stream.cuda_stream))
    its, ms = [], []
    for i in range(args.warmup + args.steps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        r = lib.integrate("s", "KN", prm, qs, l * N, qt, l, argv=[256, 1e-4])
        e1.record(stream)
        torch.cuda.synchronize()
        if i >= args.warmup:
            its.append(int(r[0]))
            ms.append(e0.elapsed_time(e1))
    lib.lib.isvd_gpu_set_stream(None)
    print(json.dumps({"workload": "KN integration, MIXED, N l = 4096, l = 128, 6000 rows", "kn_iterations": its[-1],
                      "ms_per_stage": float(np.median(ms)), "us_per_iteration": 1e3 * float(np.median(ms)) / its[-1],
                      "steps": args.steps, "warmup": args.warmup}), flush=True)


def run_batched(torch, lib, steps, warmup, single=False):
    """The batched-solves workload (batch_main); returns its JSON record.  single: one batch call
    and nothing else (for launch lists)."""
    from isvd_b200.capi import c_int_t
    dev = torch.device("cuda", 0)
    rng = np.random.default_rng(BATCH["seed"])
    gen = torch.Generator(device=dev).manual_seed(BATCH["seed"])
    mats = []
    for _ in range(BATCH["count"]):
        m = int(np.exp(rng.uniform(np.log(BATCH["m"][0]), np.log(BATCH["m"][1]))))
        n = int(np.exp(rng.uniform(np.log(BATCH["n"][0]), np.log(min(m, BATCH["n"][1])))))
        k = int(rng.choice(BATCH["k"]))
        p = k // 2
        r = min(n, 4 * k)
        u = torch.linalg.qr(torch.randn(m, r, device=dev, generator=gen))[0]
        v = torch.linalg.qr(torch.randn(n, r, device=dev, generator=gen))[0]
        sig = torch.logspace(0, -3, r, device=dev)
        a = ((u * sig) @ v.T + BATCH["noise"] * torch.randn(m, n, device=dev, generator=gen)).contiguous()
        l = k + p
        mats.append(dict(m=m, n=n, k=k, p=p, a=a, s=torch.zeros(l, device=dev), ut=torch.zeros((m, l), device=dev),
                         vt=torch.zeros((n, l), device=dev)))
    torch.cuda.synchronize()
    B, N = len(mats), BATCH["N"]
    vp = ctypes.c_void_p
    arr = lambda vals, ct=c_int_t: (ct * len(vals))(*vals)
    create = lib.lib.isvd_sBatchCreate
    create.argtypes = [c_int_t, vp, vp, vp, vp, c_int_t]
    create.restype = vp
    solve_b = lib.lib.isvd_sBatchIsvd
    solve_b.argtypes = [vp] * 10 + [c_int_t, vp, vp]
    solve_b.restype = ctypes.c_int
    batch = create(B, arr([d["m"] for d in mats]), arr([d["n"] for d in mats]), arr([d["k"] for d in mats]),
                   arr([d["p"] for d in mats]), N)
    assert batch, lib.last_error()
    seeds = [11 + i for i in range(B)]
    argv = np.asarray([256, 1e-4], dtype=np.float32)
    its = arr([0] * B)
    call = lambda: solve_b(batch, arr([d["a"].data_ptr() for d in mats], vp), arr([d["n"] for d in mats]),
                           arr([d["s"].data_ptr() for d in mats], vp), arr([d["ut"].data_ptr() for d in mats], vp),
                           arr([d["ut"].shape[1] for d in mats]), arr([d["vt"].data_ptr() for d in mats], vp),
                           arr([d["vt"].shape[1] for d in mats]), arr(seeds), argv.ctypes.data, 2, its, None)
    if single:
        # two calls: the first measures tile shapes and captures the graphs, the second is a
        # steady-state solve (a launch list skips the first call's launches)
        counts = []
        for _ in range(2):
            l0 = lib.lib.isvd_gpu_kernel_launch_count()
            assert call() == 0, lib.last_error()
            torch.cuda.synchronize()
            counts.append(int(lib.lib.isvd_gpu_kernel_launch_count() - l0))
        lib.lib.isvd_gpu_batch_destroy(ctypes.c_void_p(batch))
        return {"batch_launches": counts, "kn_iterations": list(its)}
    for _ in range(max(3, warmup)):
        assert call() == 0, lib.last_error()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    l0 = lib.lib.isvd_gpu_kernel_launch_count()
    e0.record()
    for _ in range(steps):
        assert call() == 0, lib.last_error()
    e1.record()
    torch.cuda.synchronize()
    launches = (lib.lib.isvd_gpu_kernel_launch_count() - l0) // steps
    ms_batch = e0.elapsed_time(e1) / steps
    s_batch = [d["s"].clone() for d in mats]
    it_batch = list(its)
    # the same matrices, one single solve each
    e0.record()
    it_seq = []
    for i, d in enumerate(mats):
        prm = lib.create_param(d["m"], d["n"], d["k"], d["p"], N)
        l = d["k"] + d["p"]
        retv, _, st = lib.isvd("s", prm, ("GP", "GR", "KN", "GR"), d["a"], d["n"], d["s"], d["ut"], l, d["vt"], l,
                               seed=seeds[i], argv=[None, None, [256, 1e-4], None], retc=(0, 0, 2, 0), precision=0)
        assert st == 0, lib.last_error()
        it_seq.append(int(retv[2][0]))
    e1.record()
    torch.cuda.synchronize()
    ms_seq = e0.elapsed_time(e1)
    # the k singular values each solve returns (s holds l = k + p; the last p are oversampling)
    err = max(float(((s_batch[i][:d["k"]] - d["s"][:d["k"]]).abs().max() / d["s"].abs().max()).item())
              for i, d in enumerate(mats))
    lib.lib.isvd_gpu_batch_destroy(ctypes.c_void_p(batch))
    out = {
        "metric": "batched iSVD matrices/s (256 uneven FP32 matrices)", "value": B / (ms_batch / 1e3),
        "unit": "matrix/s", "n_gpus": 1, "steps": steps, "warmup": max(3, warmup),
        "ms_per_step": ms_batch, "higher_is_better": True, "dtype": "fp32 (fp64 l x l)", "data": "synthetic",
        "config": {"workload": "256 matrices, m log-uniform [512, 8192], n log-uniform [256, 4096] (n <= m), "
                               "rank 4k geometric 1..1e-3 + 1e-4 noise, k in {8,16,32,64}, p = k/2, N = 8, GP/GR/KN/GR",
                   "total_elements": int(sum(d["m"] * d["n"] for d in mats)), "seed": BATCH["seed"]},
        "gpu_launches": int(launches),
        "sequential": {"ms": ms_seq, "value": B / (ms_seq / 1e3), "path": "isvd_sIsvd_ex per matrix, NATIVE FP32"},
        "speedup_vs_sequential": ms_seq / ms_batch,
        "sigma_rel_diff_max": err,
        "sigma_rel_diff_note": "batch against single FP32 solves, the k returned singular values of each matrix",
        "kn_iterations_equal": sum(int(a == b) for a, b in zip(it_batch, it_seq)),
    }
    return out


DIFF = dict(m=16384, n=4096, rank=512, k=64, p=32, N=16, noise=1e-4, xcols=32, seed=5)


def run_differentiated(torch, lib, steps, warmup, single=False):
    """The differentiated solve: A 16384 x 4096 FP32, rank 512 (sigma 1 .. 1e-2 geometric) + 1e-4
    noise, k = 64, l = 96, N = 16; loss sum_i w_i s_i + ||U U' X||_F^2 with w and X (16384 x 32)
    seeded Gaussian.  Timed (CUDA events, K steps after W warm-up steps): the MIXED forward
    (isvd_sIsvd_ex, GP/GR/KN/GR) and the MIXED FP32 adjoint (isvd_sSvdAdjoint: ds = w,
    dU = 2 X X' U).  Accuracy: the adjoint from the FP64 dense factors against the FP64 dense-SVD
    gradient (torch autograd through torch.linalg.svd), max abs error over max abs gradient."""
    import ctypes as ct
    from isvd_b200.capi import c_int_t, ptr
    w = DIFF
    dev = torch.device("cuda", 0)
    m, n, r, k, p, N = w["m"], w["n"], w["rank"], w["k"], w["p"], w["N"]
    l = k + p
    g = torch.Generator(device=dev).manual_seed(w["seed"])
    uu = torch.linalg.qr(torch.randn(m, r, device=dev, dtype=torch.float64, generator=g))[0]
    vv = torch.linalg.qr(torch.randn(n, r, device=dev, dtype=torch.float64, generator=g))[0]
    sig = torch.logspace(0, -2, r, device=dev, dtype=torch.float64)
    a64 = (uu * sig) @ vv.T + w["noise"] * torch.randn(m, n, device=dev, dtype=torch.float64, generator=g)
    del uu, vv
    wt = torch.randn(k, device=dev, dtype=torch.float64, generator=g)
    xx = torch.randn(m, w["xcols"], device=dev, dtype=torch.float64, generator=g)
    f32 = lambda t: t.to(torch.float32).contiguous()  # noqa: E731
    a = f32(a64)
    fn = lib.lib.isvd_sSvdAdjoint
    vp = ct.c_void_p
    fn.argtypes = [c_int_t, c_int_t, c_int_t, ct.c_char, vp, c_int_t, vp, vp, c_int_t, vp, c_int_t, vp, vp,
                   c_int_t, vp, c_int_t, vp, c_int_t, ct.c_int, ct.c_double, ct.POINTER(ct.c_int)]
    fn.restype = ct.c_int
    its = ct.c_int(0)

    def adjoint(s_, u_, v_, ds_, du_, da_):
        st = fn(m, n, k, b"R", ptr(a), n, ptr(s_), ptr(u_), k, ptr(v_), k, ptr(ds_), ptr(du_), k, None, k, ptr(da_),
                n, 300, 1e-6, ct.byref(its))
        if st != 0:
            raise RuntimeError("isvd_sSvdAdjoint failed: %s" % (lib.last_error(),))

    prm = lib.create_param(m, n, k, p, N)
    s = torch.zeros(l, device=dev)
    ut = torch.zeros((m, l), device=dev)
    vt = torch.zeros((n, l), device=dev)
    ds = f32(wt)
    da = torch.zeros_like(a)
    lib.lib.isvd_gpu_set_precision(1)
    try:
        def forward():
            retv, _, st = lib.isvd("s", prm, ("GP", "GR", "KN", "GR"), a, n, s, ut, l, vt, l, seed=w["seed"],
                                   argv=[None, None, [256, 1e-4], None], retc=(0, 0, 2, 0), precision=1)
            if st != 0:
                raise RuntimeError("isvd_sIsvd_ex failed: %s" % (lib.last_error(),))
            return int(retv[2][0])

        def backward():
            u_ = ut[:, :k].contiguous()
            v_ = vt[:, :k].contiguous()
            du_ = (2.0 * xx @ (xx.T @ u_.double())).to(torch.float32).contiguous()
            adjoint(s[:k].contiguous(), u_, v_, ds, du_, da)

        if single:  # one forward and one adjoint, nothing timed (for launch lists)
            kn = forward()
            backward()
            torch.cuda.synchronize()
            return {"kn_iterations": kn, "adjoint_cg_iterations": its.value}
        for _ in range(max(3, warmup)):
            forward()
            backward()
        torch.cuda.synchronize()
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
        t_fwd = t_bwd = 0.0
        for _ in range(steps):
            ev[0].record()
            kn = forward()
            ev[1].record()
            backward()
            ev[2].record()
            torch.cuda.synchronize()
            t_fwd += ev[0].elapsed_time(ev[1])
            t_bwd += ev[1].elapsed_time(ev[2])
        cg_its = its.value
        # accuracy of the adjoint: from the FP64 dense factors, against the FP64 dense gradient
        at = a64.clone().requires_grad_(True)
        U, S, Vh = torch.linalg.svd(at, full_matrices=False)
        L = (wt * S[:k]).sum() + ((U[:, :k] @ (U[:, :k].T @ xx)) ** 2).sum()
        L.backward()
        gref = at.grad
        u0, s0, v0 = U[:, :k].detach(), S[:k].detach(), Vh[:k].T.detach()
        adjoint(f32(s0), f32(u0), f32(v0), ds, f32(2.0 * xx @ (xx.T @ u0)), da)
        torch.cuda.synchronize()
        err = float((da.double() - gref).abs().max() / gref.abs().max())
        sig_err = float(((s[:k].double() - s0).abs() / s0).max())
    finally:
        lib.lib.isvd_gpu_set_precision(0)
    return {"workload": "A 16384x4096 FP32 rank 512 + 1e-4 noise, k=64 l=96 N=16; loss sum w_i s_i + ||U U' X||^2",
            "forward_ms": t_fwd / steps, "adjoint_ms": t_bwd / steps, "kn_iterations": kn,
            "adjoint_cg_iterations": cg_its, "adjoint_rel_err_vs_fp64_dense": err,
            "forward_sigma_rel_err_vs_fp64_dense": sig_err,
            "forward_sigma_note": "the rank-64 randomized approximation against the exact dense SVD of a slowly "
                                  "decaying spectrum (an approximation error, not a precision error)",
            "precision": "MIXED forward and adjoint",
            "steps": steps, "warmup": max(3, warmup)}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--size", default="full", choices=list(WORKLOADS))
    ap.add_argument("--skip-fp64", action="store_true")
    ap.add_argument("--skip-e2e", action="store_true")
    ap.add_argument("--skip-cpu", action="store_true")
    ap.add_argument("--skip-extra", action="store_true",
                    help="leave out the batched (256 uneven matrices) and differentiated-solve legs")
    ap.add_argument("--single", action="store_true",
                    help="one MIXED solve and its stage times, nothing else (for ncu launch lists / captures)")
    ap.add_argument("--differentiated", action="store_true",
                    help="the differentiated solve (forward + adjoint at 16384 x 4096) alone; with --single one "
                         "untimed forward and adjoint")
    ap.add_argument("--batched", action="store_true",
                    help="the batched-solves workload (256 uneven matrices) instead of the single large solve")
    ap.add_argument("--square50k", action="store_true",
                    help="the 50000 x 50000 TS / WY / column-block parity case, MIXED beside FP64")
    ap.add_argument("--kn-loop", action="store_true",
                    help="the Kolmogorov-Nagumo integration stage alone at the 200000 x 20000 workload's "
                         "loop shapes (N l = 4096, l = 128) on 6000 rows: time per iteration")
    ap.add_argument("--parallel", default="rowblock", choices=["rowblock", "replicas"],
                    help="N > 1: one solve split by rows over the ranks (default) or one solve per rank")
    ap.add_argument("--dist-backend", default="nccl", choices=["nccl", "gloo"],
                    help="process-group backend (gloo: device buffers staged through the host, e.g. "
                         "several ranks sharing one GPU for a functional check)")
    args = ap.parse_args()
    if args.batched:
        return batch_main(args)
    if args.square50k:
        return square50k_main(args)
    if args.kn_loop:
        return kn_loop_main(args)
    if args.differentiated:
        import torch
        import isvd_b200
        out = run_differentiated(torch, isvd_b200.load(), args.steps, args.warmup, single=args.single)
        print(json.dumps(out), flush=True)
        return
    w = WORKLOADS[args.size]
    if args.impl == "reference":
        return reference_arm(args, w)

    import torch
    import isvd_b200
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    gpu = local % max(1, torch.cuda.device_count())
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(gpu)
        dist.init_process_group(args.dist_backend, timeout=datetime.timedelta(seconds=600))
    dev = torch.device("cuda", gpu)
    torch.cuda.set_device(dev)
    lib = isvd_b200.load()
    stream = torch.cuda.current_stream(dev)
    lib.lib.isvd_gpu_set_stream(ctypes.c_void_p(stream.cuda_stream))
    rowblock = world > 1 and args.parallel == "rowblock"
    if rowblock:  # the ranks join as row blocks; every exchange is an AllReduce on the library stream
        from isvd_b200.capi import torch_device_allreduce
        lib.set_allreduce(torch_device_allreduce(), world, rank, on_device=True)

    m, n, k, p, N = w["m"], w["n"], w["k"], w["p"], w["N"]
    l = k + p
    prm = lib.create_param(m, n, k, p, N)
    if rowblock:
        a = make_row_block(torch, w, dev, w["seed"], prm)
    else:
        a = make_matrix(torch, w, dev, w["seed"] + 1000 * rank)
    torch.cuda.synchronize()
    if not rowblock:
        prm = lib.create_param(m, n, k, p, N)
    mloc = int(prm.nrow_proc) if rowblock else m
    nloc = int(prm.ncol_proc) if rowblock else n
    s = torch.zeros(l, dtype=torch.float32, device=dev)
    ut = torch.zeros((mloc, l), dtype=torch.float32, device=dev)
    vt = torch.zeros((nloc, l), dtype=torch.float32, device=dev)
    seed = w["seed"]
    if args.single:
        retv, times = solve(lib, "s", prm, a, n, s, ut, vt, l, seed, 1)
        print(json.dumps({"stage_ms": [1e3 * t for t in times], "kn_iterations": int(retv[2][0])}), flush=True)
        lib.lib.isvd_gpu_set_stream(None)
        return

    def barrier():
        if dist is not None:
            dist.barrier()

    # warm-up
    for _ in range(args.warmup):
        solve(lib, "s", prm, a, n, s, ut, vt, l, seed, 1)
    torch.cuda.synchronize()
    barrier()
    torch.cuda.synchronize()
    launches0 = lib.lib.isvd_gpu_kernel_launch_count()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    stage = np.zeros(4)
    kn_its = 0
    with ClockSampler(gpu) as clk:
        ev0.record(stream)
        for _ in range(args.steps):
            retv, times = solve(lib, "s", prm, a, n, s, ut, vt, l, seed, 1)
            stage += np.array(times)
            kn_its = int(retv[2][0])
        ev1.record(stream)
        torch.cuda.synchronize()
    barrier()
    torch.cuda.synchronize()
    launches = lib.lib.isvd_gpu_kernel_launch_count() - launches0
    ms_total = ev0.elapsed_time(ev1)
    if dist is not None:
        t = torch.tensor([ms_total], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms_total = float(t.item())
    ms_per = ms_total / args.steps
    solves_per_step = 1 if (rowblock or world == 1) else world
    value = solves_per_step * args.steps / (ms_total / 1e3)
    s_mixed = s.double().cpu().numpy()

    # per-kernel timing of the dominant kernel (separate, untimed run)
    lib.lib.isvd_gpu_profile_reset()
    lib.lib.isvd_gpu_profile_enable(1)
    solve(lib, "s", prm, a, n, s, ut, vt, l, seed, 1)
    lib.lib.isvd_gpu_profile_enable(0)
    prof = {t: lib.profile(t) for t in ("sketch", "block_gram", "block_apply", "gram_full", "kn_product",
                                        "coeff_apply", "project")}

    hbm, bf16, bf16_sus, peak_kind = peaks()
    sk = prof["sketch"]
    # the sketch runs as one launch per row panel of A: algorithmic flops per launch / average
    # launch time = total algorithmic flops / total kernel time
    sketch_ms_total = sk[0] if sk else None
    sketch_launches = sk[1] if sk else 0
    alg_flops = 2.0 * mloc * n * (l * N)  # this rank's rows
    achieved = alg_flops / (sketch_ms_total * 1e-3) / 1e12 if sketch_ms_total else None
    # bf16 plane products per algorithmic product, from the executed flops the library records
    nprod = int(round(sk[2] / alg_flops)) if sk else 2
    # the sketch runs as back-to-back launches inside the solve: the sustained bf16 figure is its
    # denominator; the burst figure is reported beside it
    peak3, peak3_burst = bf16_sus / nprod, bf16 / nprod
    headline_shape = (m, n, l * N) == (200000, 20000, 4096)
    roofline = {"bound": "tensor", "kernel": "umma_gemm_kernel (sketch Y = A Omega, %d bf16 plane products)" % nprod,
                "achieved": achieved, "peak": peak3, "unit": "TFLOP/s",
                "frac": (achieved / peak3) if achieved else None,
                "peak_burst": peak3_burst, "frac_burst": (achieved / peak3_burst) if achieved else None,
                "traffic": SKETCH_LAUNCH_TRAFFIC if headline_shape and sketch_launches == 1 else None,
                "traffic_unit": "bytes per launch (one launch over all m rows; ncu, dram read + write)",
                "alg_bytes_per_launch": float(mloc * n * 4 + mloc * l * N * 4 + n * l * N * 2),
                "convention": "algorithmic 2 m n Nl flops per solve / kernel time; peak = %s bf16 dense "
                              "sustained %.1f TFLOP/s / %d products (burst %.1f / %d also given)"
                              % (peak_kind, bf16_sus, nprod, bf16, nprod),
                "kernel_ms_total": sketch_ms_total, "kernel_launches": sketch_launches,
                "other_tcgen05_ms": {t: (v[0] / v[1] if v else None) for t, v in prof.items() if t != "sketch"}}

    out = {"metric": METRIC, "value": value, "unit": "solve/s", "n_gpus": world, "steps": args.steps,
           "warmup": args.warmup, "ms_per_step": ms_per, "higher_is_better": True,
           "scaling": "weak" if (world > 1 and not rowblock) else "strong",
           "vs_baseline": None, "dtype": "f32 via bf16 split planes (sketch: 2 A planes x exact bf16 Omega; fp32 accumulate; fp64 l x l)",
           "data": "synthetic (seeded, generated on GPU)", "config": config_dict(w, world, args.parallel),
           "stage_ms": [1e3 * x / args.steps for x in stage], "kn_iterations": kn_its,
           "gpu_launches": int(launches), "roofline": roofline}

    # FP64 path on the same matrix and Omega (one GPU)
    if not args.skip_fp64 and not rowblock:
        a64 = a.double()
        s64 = torch.zeros(l, dtype=torch.float64, device=dev)
        ut64 = torch.zeros((m, l), dtype=torch.float64, device=dev)
        vt64 = torch.zeros((n, l), dtype=torch.float64, device=dev)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        retv64, times64 = solve(lib, "d", prm, a64, n, s64, ut64, vt64, l, seed, 0)
        e1.record(stream)
        torch.cuda.synchronize()
        ms64 = e0.elapsed_time(e1)
        sv64 = s64.cpu().numpy()
        rel = np.abs(s_mixed[:k] - sv64[:k]) / sv64[:k]
        u32 = ut[:, :k].double()
        u64 = ut64[:, :k]
        # largest principal angle between span(U_mixed) and span(U_fp64)
        q1 = torch.linalg.qr(u32)[0]
        q2 = torch.linalg.qr(u64)[0]
        sin = torch.linalg.matrix_norm(q2 - q1 @ (q1.T @ q2), ord=2).item()
        out["fp64"] = {"ms_per_solve": ms64, "stage_ms": [1e3 * x for x in times64],
                       "kn_iterations": int(retv64[2][0]), "sigma_rel_err_max": float(rel.max()),
                       "u_max_principal_angle": float(np.arcsin(min(1.0, sin))),
                       "speedup_mixed_vs_fp64": ms64 / ms_per}
        del a64, ut64, vt64

    # end to end through the C ABI with host buffers (pinned), copies inside the timed region
    if not args.skip_e2e:
        ah = torch.empty((mloc, n), dtype=torch.float32, pin_memory=True)
        ah.copy_(a)
        sh = torch.zeros(l, dtype=torch.float32, pin_memory=True)
        uh = torch.zeros((mloc, l), dtype=torch.float32, pin_memory=True)
        vh = torch.zeros((nloc, l), dtype=torch.float32, pin_memory=True)
        a = None
        torch.cuda.synchronize()
        solve(lib, "s", prm, ah, n, sh, uh, vh, l, seed, 1)  # warm
        torch.cuda.synchronize()
        barrier()
        torch.cuda.synchronize()
        # device-timed on the library's stream: the panel copies run on the library's copy stream
        # but each is joined into this stream before the call returns, as are the output copies
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        reps = 2
        e0.record(stream)
        for _ in range(reps):
            solve(lib, "s", prm, ah, n, sh, uh, vh, l, seed, 1)
        e1.record(stream)
        torch.cuda.synchronize()
        te = e0.elapsed_time(e1) / 1e3 / reps
        if dist is not None:
            t = torch.tensor([te], device=dev, dtype=torch.float64)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            te = float(t.item())
        reps_job = 1 if rowblock else world  # whole-job bytes: every rank's copies
        out["e2e"] = {"value": solves_per_step / te, "unit": "solve/s", "ms_per_solve": 1e3 * te,
                      "h2d_bytes_per_step": reps_job * m * n * 4,
                      "d2h_bytes_per_step": reps_job * (l * (world if rowblock else 1) + m * k + n * k) * 4,
                      "path": "isvd_sIsvd_ex with pinned host A, s, U, V (H2D of A and D2H of s, U, V timed)"}
    out["clocks"] = clk.summary()
    if world == 1 and not args.skip_extra:
        a = None  # the headline matrix
        torch.cuda.empty_cache()
        out["batched_256_uneven"] = run_batched(torch, lib, args.steps, args.warmup)
        out["differentiated_16384x4096"] = run_differentiated(torch, lib, args.steps, args.warmup)
    if rank == 0 and world == 1 and not args.skip_cpu:
        cores = physical_cores()
        try:
            stage_t, desc, its, _, _ = reference_sample(w, 1, 0, cores)
            tot = float(np.sum(stage_t))
            out["cpu_baseline"] = {"value": 1.0 / tot, "unit": "solve/s", "cores": cores,
                                   "kind": "reference", "sample": desc, "stage_s": [float(x) for x in stage_t]}
        except Exception as e:  # the checker library may be absent on a fresh box
            out["cpu_baseline"] = {"value": None, "unit": "solve/s", "cores": cores, "kind": "reference",
                                   "sample": "unavailable: %s" % e}
    if rank == 0:
        print(json.dumps(out), flush=True)
    lib.lib.isvd_gpu_set_stream(None)
    if rowblock:
        lib.set_allreduce(None, 1, 0)
    if dist is not None:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
