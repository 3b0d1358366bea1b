"""Parity with the reference itself at the headline shapes, with the same Omega passed in.

    ISVD_PARITY_FULL=2,3,cal ISVD_PARITY_OUT=<file> python -m pytest tests/test_gpu_parity_full.py -m gpu -s

Skipped unless ISVD_PARITY_FULL names at least one case (each takes minutes of host-CPU time for the
reference; the ordinary `-m gpu` run skips them):

* ``2``: 200000 x 20000 FP32, rank-2000 Haar factors, sigma geometric 1 .. 1e-3, + 1e-4 noise;
  k = 100, p = 28, N = 32; GP / GR / KN(256, 1e-4) / GR, row blocks.  Omega (n x N l, FP64, seeded)
  is passed in to the FP64 GPU path (isvd_dIsvd_ex, NATIVE, A in FP64), to the MIXED GPU path
  (isvd_sIsvd_ex, MIXED, A and Omega in FP32) and to the built reference's own FP64 stage routines
  on the host: Y = A Omega through the BLAS the reference links (dgemm_, as its isvd_dGemm calls
  it, core/stage/@x@_sketch.h:136-139), then isvd_dOrthogonalizeGramian,
  isvd_dIntegrateKolmogorovNagumo and isvd_dPostprocessGramian
  (the pipeline of core/driver/@x@_isvd.c:243-264).
* ``3``: 50000 x 50000 FP32, sigma_i = (1 + i)^-1/2 for i < 5000 on Haar factors, + 1e-3 noise;
  k = 64, p = 64, N = 64; GP / TS / WY(512, 1e-4) / GR on column blocks (dista 'C'), the same three
  solves; plus the two GPU paths again with Wen-Yin run tighter (2048, 1e-6).
* ``3s``: the rounding sensitivity of the 50000 x 50000 Wen-Yin case: the reference's own TS / WY /
  GR stages on Y = A Omega and on Y changed at the rounding level, and the FP64 GPU stages on both.
* ``cal``: the reference's own single-precision driver (isvd_sIsvd, internal Omega, all host
  threads) timed once on the full 200000 x 20000 matrix beside the row-sample extrapolation that
  bench.py's reference arm reports.

Bars (from the precision contract): FP64 sigma within 1e-10 relative, MIXED within 1e-5, the
largest principal angle of the k leading U and V columns within 1e-4, and the FP64 iteration
count equal to the reference's.  Every measured number is written as one JSON line per case to
ISVD_PARITY_OUT (default: printed only) before the bars are checked.
"""
import ctypes
import json
import os
import time

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

CASES = set(x.strip() for x in os.environ.get("ISVD_PARITY_FULL", "").split(",") if x.strip())


def _emit(rec):
    line = json.dumps(rec)
    print(line, flush=True)
    out = os.environ.get("ISVD_PARITY_OUT")
    if out:
        with open(out, "a") as fh:
            fh.write(line + "\n")


def _blas_dgemm():
    """dgemm_ of the OpenBLAS the built reference links (the same shared object)."""
    import build_ref
    d, name = build_ref.openblas_dir()
    blas = ctypes.CDLL(os.path.join(d, name))
    f = blas.dgemm_
    f.restype = None
    return f


def _ref_sketch(a, om):
    """Y = A Omega, row-major m x Nl, as the reference's row-block sketch computes it:
    Y' := Omega' A' with column-major operands (core/stage/@x@_sketch.h:136-139)."""
    m, n = a.shape
    nl = om.shape[1]
    y = np.empty((m, nl))
    f = _blas_dgemm()
    ci = ctypes.c_int
    cd = ctypes.c_double
    f(ctypes.c_char_p(b"N"), ctypes.c_char_p(b"N"), ctypes.byref(ci(nl)), ctypes.byref(ci(m)), ctypes.byref(ci(n)),
      ctypes.byref(cd(1.0)), om.ctypes.data_as(ctypes.c_void_p), ctypes.byref(ci(nl)),
      a.ctypes.data_as(ctypes.c_void_p), ctypes.byref(ci(n)), ctypes.byref(cd(0.0)),
      y.ctypes.data_as(ctypes.c_void_p), ctypes.byref(ci(nl)))
    return y


def _angle(torch, u1, u2):
    """Largest principal angle between the column spans (FP64, on the device)."""
    q1 = torch.linalg.qr(u1.double())[0]
    q2 = torch.linalg.qr(u2.double())[0]
    s = torch.linalg.matrix_norm(q2 - q1 @ (q1.T @ q2), ord=2).item()
    return float(np.arcsin(min(1.0, s)))


def _sigma_err(s, s_ref, k):
    s = np.asarray(s, np.float64)[:k]
    r = np.asarray(s_ref, np.float64)[:k]
    return float(np.max(np.abs(s - r) / np.abs(r)))


def _gpu_solve(torch, lib, x, prm, algs, a, n, l, om, argv_i, precision, dista=b"R"):
    dev = a.device
    dt = torch.float64 if x == "d" else torch.float32
    m = a.shape[0]
    s = torch.zeros(l, dtype=dt, device=dev)
    ut = torch.zeros((m, l), dtype=dt, device=dev)
    vt = torch.zeros((a.shape[1], l), dtype=dt, device=dev)
    torch.cuda.synchronize()
    t0 = time.time()
    retv, times, status = lib.isvd(x, prm, algs, a, n, s, ut, l, vt, l, dista=dista, ordera=b"R",
                                   argv=[None, None, list(argv_i), None], retc=(0, 0, 2, 0),
                                   omega=om, ldomega=om.shape[1], precision=precision)
    torch.cuda.synchronize()
    wall = time.time() - t0
    assert status == 0, lib.last_error()
    return dict(s=s.double().cpu().numpy(), ut=ut, vt=vt, iters=int(retv[2][0]), err=float(retv[2][1]),
                stage_s=list(times), wall_s=wall)


def _ref_solve(reflib, a_h, om_h, k, p, N, alg_o, alg_i, argv_i, dista=b"R"):
    m, n = a_h.shape
    l = k + p
    prm = reflib.create_param(m, n, k, p, N)
    t = [0.0] * 4
    t0 = time.time()
    yst = _ref_sketch(a_h, om_h)
    t[0] = time.time() - t0
    t0 = time.time()
    reflib.orthogonalize("d", alg_o, prm, yst, l * N)
    t[1] = time.time() - t0
    qt = np.zeros((m, l))
    t0 = time.time()
    r = reflib.integrate("d", alg_i, prm, yst, l * N, qt, l, argv=list(argv_i))
    t[2] = time.time() - t0
    del yst
    return _ref_post(reflib, prm, a_h, qt, k, p, r, t, dista)


def _ref_post(reflib, prm, a_h, qt, k, p, r, t, dista):
    m, n = a_h.shape
    l = k + p
    s = np.zeros(l)
    ut = np.zeros((m, l))
    vt = np.zeros((n, l))
    t0 = time.time()
    reflib.postprocess("d", "GR", prm, a_h, n, qt, l, s, ut, l, vt, l, dista=dista)
    t[3] = time.time() - t0
    return dict(s=s, ut=ut, vt=vt, iters=int(r[0]), err=float(r[1]), stage_s=t)


def _compare(torch, name, g, ref, k):
    dev = g["ut"].device
    return {"path": name, "iterations": g["iters"], "final_err": g["err"],
            "sigma_rel_err_max": _sigma_err(g["s"], ref["s"], k),
            "u_max_angle": _angle(torch, g["ut"][:, :k], torch.from_numpy(ref["ut"][:, :k]).to(dev)),
            "v_max_angle": _angle(torch, g["vt"][:, :k], torch.from_numpy(ref["vt"][:, :k]).to(dev)),
            "stage_s": g["stage_s"], "wall_s": g["wall_s"]}


def _host_threads():
    return int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1))


@pytest.mark.skipif("2" not in CASES, reason="ISVD_PARITY_FULL does not name case 2")
def test_parity_200000x20000(lib, reflib):
    import torch
    import bench
    w = bench.WORKLOADS["full"]
    m, n, k, p, N = w["m"], w["n"], w["k"], w["p"], w["N"]
    l = k + p
    dev = torch.device("cuda", 0)
    a = bench.make_matrix(torch, w, dev, w["seed"])
    g = torch.Generator(device=dev).manual_seed(12345)
    om = torch.randn(n, l * N, generator=g, device=dev, dtype=torch.float64)
    prm = lib.create_param(m, n, k, p, N)
    algs = ("GP", "GR", "KN", "GR")
    kn = (256, 1e-4)
    mixed = _gpu_solve(torch, lib, "s", prm, algs, a, n, l, om.float(), kn, 1)
    a64 = a.double()
    del a
    fp64 = _gpu_solve(torch, lib, "d", prm, algs, a64, n, l, om, kn, 0)
    a_h = a64.cpu().numpy()
    del a64
    torch.cuda.empty_cache()
    om_h = om.cpu().numpy()
    ref = _ref_solve(reflib, a_h, om_h, k, p, N, "GR", "KN", kn)
    rec = {"case": "200000x20000 FP32 rank-2000, k=100 p=28 N=32, GP/GR/KN(256,1e-4)/GR, row blocks, Omega passed in",
           "reference": {"iterations": ref["iters"], "final_err": ref["err"], "stage_s": ref["stage_s"],
                         "host_threads": _host_threads(),
                         "sigma_head": [float(x) for x in ref["s"][:3]]},
           "fp64": _compare(torch, "isvd_dIsvd_ex NATIVE", fp64, ref, k),
           "mixed": _compare(torch, "isvd_sIsvd_ex MIXED", mixed, ref, k),
           "mixed_vs_fp64_sigma": _sigma_err(mixed["s"], fp64["s"], k)}
    _emit(rec)
    f, x = rec["fp64"], rec["mixed"]
    assert f["iterations"] == ref["iters"]
    assert f["sigma_rel_err_max"] <= 1e-10
    assert max(f["u_max_angle"], f["v_max_angle"]) <= 1e-4
    assert x["sigma_rel_err_max"] <= 1e-5
    assert max(x["u_max_angle"], x["v_max_angle"]) <= 1e-4


@pytest.mark.skipif("3" not in CASES, reason="ISVD_PARITY_FULL does not name case 3")
def test_parity_50000x50000_wen_yin(lib, reflib):
    import torch
    import bench
    w = bench.SQUARE50K
    m, n, r, k, p, N = w["m"], w["n"], w["rank"], w["k"], w["p"], w["N"]
    l = k + p
    dev = torch.device("cuda", 0)
    g = torch.Generator(device=dev).manual_seed(w["seed"])
    u = torch.linalg.qr(torch.randn(m, r, generator=g, device=dev, dtype=torch.float32))[0]
    v = torch.linalg.qr(torch.randn(n, r, generator=g, device=dev, dtype=torch.float32))[0]
    sig = (1.0 + torch.arange(r, device=dev, dtype=torch.float32)) ** -0.5
    a = torch.randn(m, n, generator=g, device=dev, dtype=torch.float32).mul_(w["noise"])
    a.addmm_(u * sig, v.t())
    del u, v
    g2 = torch.Generator(device=dev).manual_seed(54321)
    om = torch.randn(n, l * N, generator=g2, device=dev, dtype=torch.float64)
    prm = lib.create_param(m, n, k, p, N)
    algs = ("GP", "TS", "WY", "GR")
    wy, wy_tight = (512, 1e-4), (2048, 1e-6)
    mixed = _gpu_solve(torch, lib, "s", prm, algs, a, n, l, om.float(), wy, 1, dista=b"C")
    mixed_t = _gpu_solve(torch, lib, "s", prm, algs, a, n, l, om.float(), wy_tight, 1, dista=b"C")
    a64 = a.double()
    del a
    fp64 = _gpu_solve(torch, lib, "d", prm, algs, a64, n, l, om, wy, 0, dista=b"C")
    fp64_t = _gpu_solve(torch, lib, "d", prm, algs, a64, n, l, om, wy_tight, 0, dista=b"C")
    a_h = a64.cpu().numpy()
    del a64
    torch.cuda.empty_cache()
    ref = _ref_solve(reflib, a_h, om.cpu().numpy(), k, p, N, "TS", "WY", wy, dista=b"C")
    rec = {"case": "50000x50000 FP32 sigma_i=(1+i)^-0.5 (i<5000) + 1e-3 noise, k=64 p=64 N=64, "
                   "GP/TS/WY(512,1e-4)/GR, column blocks, Omega passed in",
           "reference": {"iterations": ref["iters"], "final_err": ref["err"], "stage_s": ref["stage_s"],
                         "host_threads": _host_threads(),
                         "sigma_head": [float(x) for x in ref["s"][:3]]},
           "fp64": _compare(torch, "isvd_dIsvd_ex NATIVE", fp64, ref, k),
           "mixed": _compare(torch, "isvd_sIsvd_ex MIXED", mixed, ref, k),
           "mixed_vs_fp64_sigma": _sigma_err(mixed["s"], fp64["s"], k),
           "tight_wy_2048_1e-6": {"fp64_iterations": fp64_t["iters"], "mixed_iterations": mixed_t["iters"],
                                  "mixed_vs_fp64_sigma": _sigma_err(mixed_t["s"], fp64_t["s"], k),
                                  "fp64_tight_vs_fp64_sigma": _sigma_err(fp64_t["s"], fp64["s"], k),
                                  "mixed_u_angle_vs_fp64": _angle(torch, mixed_t["ut"][:, :k], fp64_t["ut"][:, :k]),
                                  "fp64_final_mu": fp64_t["err"], "mixed_final_mu": mixed_t["err"]}}
    _emit(rec)
    f = rec["fp64"]
    assert f["sigma_rel_err_max"] <= 1e-10
    assert max(f["u_max_angle"], f["v_max_angle"]) <= 1e-4


def _square50k(torch, dev):
    import bench
    w = bench.SQUARE50K
    m, n, r = w["m"], w["n"], w["rank"]
    g = torch.Generator(device=dev).manual_seed(w["seed"])
    u = torch.linalg.qr(torch.randn(m, r, generator=g, device=dev, dtype=torch.float32))[0]
    v = torch.linalg.qr(torch.randn(n, r, generator=g, device=dev, dtype=torch.float32))[0]
    sig = (1.0 + torch.arange(r, device=dev, dtype=torch.float32)) ** -0.5
    a = torch.randn(m, n, generator=g, device=dev, dtype=torch.float32).mul_(w["noise"])
    a.addmm_(u * sig, v.t())
    return w, a


@pytest.mark.skipif("3s" not in CASES, reason="ISVD_PARITY_FULL does not name the sensitivity case")
def test_wen_yin_50000x50000_rounding_sensitivity(lib, reflib):
    """How far the reference's own TS / WY(512, 1e-4) / GR result moves when its input Y = A Omega
    changes at the rounding level (each entry times 1 + d, d in {-2^-52, 0, 2^-52}), on the
    50000 x 50000 case; the FP64 GPU stages on the same two Y beside it.  Measurement only: it
    records iteration counts, final mu and the sigma / U differences between the runs."""
    import torch
    dev = torch.device("cuda", 0)
    w, a = _square50k(torch, dev)
    m, n, k, p, N = w["m"], w["n"], w["k"], w["p"], w["N"]
    l = k + p
    a64 = a.double()
    del a
    g2 = torch.Generator(device=dev).manual_seed(54321)
    om = torch.randn(n, l * N, generator=g2, device=dev, dtype=torch.float64)
    a_h = a64.cpu().numpy()
    y1 = _ref_sketch(a_h, om.cpu().numpy())
    rng = np.random.default_rng(1)
    y2 = y1 * (1.0 + rng.integers(-1, 2, size=y1.shape) * 2.0 ** -52)
    wy = (512, 1e-4)
    prm_r = reflib.create_param(m, n, k, p, N)
    prm = lib.create_param(m, n, k, p, N)
    out = {}
    for name, y in (("y", y1), ("y_perturbed", y2)):
        ys = np.ascontiguousarray(y)
        t0 = time.time()
        reflib.orthogonalize("d", "TS", prm_r, ys, l * N)
        qt = np.zeros((m, l))
        r = reflib.integrate("d", "WY", prm_r, ys, l * N, qt, l, argv=list(wy))
        del ys
        ref = _ref_post(reflib, prm_r, a_h, qt, k, p, r, [0.0, 0.0, time.time() - t0, 0.0], b"C")
        yd = torch.from_numpy(y).to(dev)
        lib.orthogonalize("d", "TS", prm, yd, l * N)
        qd = torch.zeros((m, l), dtype=torch.float64, device=dev)
        rg = lib.integrate("d", "WY", prm, yd, l * N, qd, l, argv=list(wy))
        del yd
        sd = torch.zeros(l, dtype=torch.float64, device=dev)
        ud = torch.zeros((m, l), dtype=torch.float64, device=dev)
        vd = torch.zeros((n, l), dtype=torch.float64, device=dev)
        lib.postprocess("d", "GR", prm, a64, n, qd, l, sd, ud, l, vd, l, dista=b"C")
        out[name] = (ref, dict(s=sd.cpu().numpy(), ut=ud, iters=int(rg[0]), err=float(rg[1])))
    (r1, g1), (r2, g2_) = out["y"], out["y_perturbed"]
    ang = lambda u1, u2: _angle(torch, torch.as_tensor(u1[:, :k]).to(dev), torch.as_tensor(u2[:, :k]).to(dev))  # noqa
    rec = {"case": "50000x50000 TS/WY(512,1e-4)/GR: Y and Y with rounding-level relative changes (2^-52)",
           "reference": {"iterations": [r1["iters"], r2["iters"]], "final_mu": [r1["err"], r2["err"]],
                         "sigma_rel_diff": _sigma_err(r2["s"], r1["s"], k), "u_angle": ang(r1["ut"], r2["ut"]),
                         "wy_seconds": [r1["stage_s"][2], r2["stage_s"][2]]},
           "gpu_fp64": {"iterations": [g1["iters"], g2_["iters"]], "final_mu": [g1["err"], g2_["err"]],
                        "sigma_rel_diff": _sigma_err(g2_["s"], g1["s"], k), "u_angle": ang(g1["ut"], g2_["ut"])},
           "gpu_vs_reference_same_y": {"sigma_rel_diff": [_sigma_err(g1["s"], r1["s"], k),
                                                          _sigma_err(g2_["s"], r2["s"], k)],
                                       "u_angle": [ang(g1["ut"], r1["ut"]), ang(g2_["ut"], r2["ut"])]},
           "host_threads": _host_threads()}
    _emit(rec)


@pytest.mark.skipif("cal" not in CASES, reason="ISVD_PARITY_FULL does not name the calibration case")
def test_reference_arm_calibration(reflib):
    """One full-size single-precision reference solve, timed on the bench's own matrix, beside
    bench.py's row-sample figure."""
    import torch
    import bench
    w = bench.WORKLOADS["full"]
    m, n, k, p, N = w["m"], w["n"], w["k"], w["p"], w["N"]
    l = k + p
    a_d = bench.make_matrix(torch, w, torch.device("cuda", 0), w["seed"])
    a = a_d.cpu().numpy()
    del a_d
    torch.cuda.empty_cache()
    prm = reflib.create_param(m, n, k, p, N)
    s = np.zeros(l, np.float32)
    ut = np.zeros((m, l), np.float32)
    vt = np.zeros((n, l), np.float32)
    t0 = time.time()
    retv, times, _ = reflib.isvd("s", prm, ("GP", "GR", "KN", "GR"), a, n, s, ut, l, vt, l, seed=w["seed"],
                                 argv=[None, None, [256, 1e-4], None], retc=(0, 0, 2, 0))
    wall = time.time() - t0
    del a, ut
    _, desc, its_x, _, stage_x = bench.reference_sample(w, 1, 0, _host_threads())
    rec = {"case": "reference isvd_sIsvd at 200000x20000 (internal Omega) vs the row-sample extrapolation",
           "full": {"stage_s": list(times), "total_s": float(sum(times)), "wall_s": wall,
                    "kn_iterations": int(retv[2][0])},
           "sample": {"stage_s": [float(x) for x in stage_x], "total_s": float(np.sum(stage_x)),
                      "kn_iterations": its_x, "desc": desc},
           "extrapolation_over_full": float(np.sum(stage_x)) / float(sum(times)),
           "host_threads": _host_threads()}
    _emit(rec)
    assert int(retv[2][0]) >= 1
