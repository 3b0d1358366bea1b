"""Kolmogorov-Nagumo integration on static device scratch (isvd_dIntegrateKolmogorovNagumo_noalloc).

The entry point is called through the C ABI and checked against isvd_dIntegrateKolmogorovNagumo
on the same device operands.  The file name sorts last so that the tests also run after every
other test of the suite; the first test makes the first library call when the file runs alone
in a fresh process, which is when the per-device set-up of the scratch happens.
"""
import ctypes
import json
import subprocess
import sys

import numpy as np
import pytest

from conftest import REPO
from isvd_b200.capi import Param, c_int_t

pytestmark = pytest.mark.gpu

TOL = 1e-10            # FP64; the two entry points may split the Gram product differently
ARG, OK = 1, 0         # ISVD_GPU_ERROR_ARGUMENT, ISVD_GPU_SUCCESS


def _entry(lib):
    fn = lib.lib.isvd_dIntegrateKolmogorovNagumo_noalloc
    fn.argtypes = [Param, ctypes.c_void_p, c_int_t, ctypes.c_void_p, c_int_t, ctypes.c_void_p, c_int_t,
                   ctypes.c_void_p, c_int_t, ctypes.c_void_p]
    fn.restype = ctypes.c_int
    return fn


def _noalloc(lib, prm, ys, ldys, qt, ldqt, argv=(256, 1e-4), stream=None):
    import torch
    av = np.ascontiguousarray(argv, dtype=np.float64)
    rv = np.zeros(2)
    if stream is None:
        stream = torch.cuda.current_stream().cuda_stream
    torch.cuda.synchronize()
    st = _entry(lib)(prm, av.ctypes.data, len(av), rv.ctypes.data, 2, ys, ldys, qt, ldqt, stream)
    return st, rv


def _blocks(seed, m, l, N, noise):
    """N orthonormal m x l blocks scattered around a common l-dimensional subspace."""
    rng = np.random.default_rng(seed)
    base = np.linalg.qr(rng.standard_normal((m, l)))[0]
    qs = np.empty((m, N * l))
    for i in range(N):
        qs[:, i * l:(i + 1) * l] = np.linalg.qr(base + noise / np.sqrt(m) * rng.standard_normal((m, l)))[0]
    return qs


def test_noalloc_two_calls_match_stage(lib):
    """Two calls in a row: identical to each other, equal to the ordinary stage within TOL, and the
    second call leaves the device's free memory unchanged."""
    import torch
    m, l, N = 20000, 32, 8
    prm = lib.create_param(m, m, l, 0, N)
    ys = torch.from_numpy(_blocks(3, m, l, N, 0.5)).cuda()
    q1 = torch.full((m, l), np.nan, dtype=torch.float64, device="cuda")
    q2 = torch.full((m, l), np.nan, dtype=torch.float64, device="cuda")
    st1, r1 = _noalloc(lib, prm, ys.data_ptr(), N * l, q1.data_ptr(), l)
    assert st1 == OK, lib.last_error()
    free_before = torch.cuda.mem_get_info()[0]
    st2, r2 = _noalloc(lib, prm, ys.data_ptr(), N * l, q2.data_ptr(), l)
    free_after = torch.cuda.mem_get_info()[0]
    assert st2 == OK, lib.last_error()
    assert free_after == free_before
    assert torch.equal(q1, q2) and r1[0] == r2[0] and r1[1] == r2[1]

    q0 = torch.zeros((m, l), dtype=torch.float64, device="cuda")
    lib.clear_error()
    r0 = lib.integrate("d", "KN", prm, ys, N * l, q0, l, argv=[256, 1e-4])
    assert lib.last_error()[0] == 0
    assert int(r1[0]) == int(r0[0]) > 1
    assert abs(r1[1] - r0[1]) <= 1e-12 + 1e-8 * abs(r0[1])
    for q in (q1, q2):
        assert (q - q0).abs().max().item() < TOL


def test_noalloc_golden(lib, golden):
    """The reference's own case: 81 iterations and Qbar equal to the reference's to 1e-12."""
    import torch
    qs = golden["qs"]
    m, L, N = qs.shape[0], 11, 12
    prm = lib.create_param(m, m, L, 0, N)
    ys = torch.from_numpy(np.ascontiguousarray(qs)).cuda()
    qt = torch.zeros((m, L + 3), dtype=torch.float64, device="cuda")
    qt[:, L:] = 7.0
    st, r = _noalloc(lib, prm, ys.data_ptr(), L * N, qt.data_ptr(), L + 3)
    assert st == OK, lib.last_error()
    assert int(r[0]) == 81
    out = qt.cpu().numpy()
    assert np.abs(out[:, :L] - golden["q_kn"]).max() < 1e-12
    assert (out[:, L:] == 7.0).all()
    # maxit reached: retv[0] = maxit + 1, as the ordinary stage
    st, r = _noalloc(lib, prm, ys.data_ptr(), L * N, qt.data_ptr(), L + 3, argv=(10, 1e-4))
    q0 = np.zeros((m, L))
    r0 = lib.integrate("d", "KN", prm, np.ascontiguousarray(qs), L * N, q0, L, argv=[10, 1e-4])
    assert st == OK and int(r[0]) == int(r0[0]) == 11
    assert np.abs(qt.cpu().numpy()[:, :L] - q0).max() < TOL


def test_noalloc_rejects(lib):
    """Sizes beyond the static scratch and host operands fail with an argument error and a message;
    the next valid call still succeeds."""
    import torch
    lib.clear_error()
    m, l, N = 64, 32, 32           # N l = 1024: (N l)^2 alone is the whole 8 MiB
    prm = lib.create_param(m, m, l, 0, N)
    ys = torch.zeros((m, N * l), dtype=torch.float64, device="cuda")
    qt = torch.zeros((m, l), dtype=torch.float64, device="cuda")
    st, _ = _noalloc(lib, prm, ys.data_ptr(), N * l, qt.data_ptr(), l)
    code, msg = lib.last_error()
    assert st == ARG and code == ARG and "static scratch" in msg and "8 MiB" in msg

    lib.clear_error()
    m, l, N = 200, 8, 4
    prm = lib.create_param(m, m, l, 0, N)
    ys_h = _blocks(5, m, l, N, 0.5)
    qt_h = np.zeros((m, l))
    st, _ = _noalloc(lib, prm, ys_h.ctypes.data, N * l, qt_h.ctypes.data, l)
    code, msg = lib.last_error()
    assert st == ARG and code == ARG and "device" in msg

    lib.clear_error()
    ys = torch.from_numpy(ys_h).cuda()
    qt = torch.zeros((m, l), dtype=torch.float64, device="cuda")
    st, r = _noalloc(lib, prm, ys.data_ptr(), N * l, qt.data_ptr(), l)
    assert st == OK and int(r[0]) >= 1
    r0 = lib.integrate("d", "KN", prm, ys_h, N * l, qt_h, l, argv=[256, 1e-4])
    assert int(r[0]) == int(r0[0])
    assert np.abs(qt.cpu().numpy() - qt_h).max() < TOL


# Run in a fresh process (a fresh CUDA context, no earlier library call): the first call has a
# small shape (64 x 64 product tiles, no split-K), the second a larger one (128 x 128 tiles and a
# split-K reduction for the l x l products), so the second call is the first to need those
# kernels.  Free device memory must not move across the second and third calls.
_FRESH = r"""
import ctypes, json, sys
import numpy as np
import torch
sys.path.insert(0, sys.argv[1])
import isvd_b200
from isvd_b200.capi import Param, c_int_t
lib = isvd_b200.load()
fn = lib.lib.isvd_dIntegrateKolmogorovNagumo_noalloc
fn.argtypes = [Param, ctypes.c_void_p, c_int_t, ctypes.c_void_p, c_int_t, ctypes.c_void_p, c_int_t,
               ctypes.c_void_p, c_int_t, ctypes.c_void_p]
fn.restype = ctypes.c_int

def blocks(seed, m, l, N):
    rng = np.random.default_rng(seed)
    base = np.linalg.qr(rng.standard_normal((m, l)))[0]
    return np.concatenate([np.linalg.qr(base + 0.5 / np.sqrt(m) * rng.standard_normal((m, l)))[0]
                           for _ in range(N)], axis=1)

shapes = [(120, 32, 3), (60000, 128, 4)]
cases = []
for i, (m, l, N) in enumerate(shapes):
    ys = torch.from_numpy(blocks(7 + i, m, l, N)).cuda()
    qs = [torch.full((m, l), float("nan"), dtype=torch.float64, device="cuda") for _ in range(2)]
    cases.append((lib.create_param(m, m, l, 0, N), ys, qs, m, l, N))
argv = np.asarray([256, 1e-4])
stream = torch.cuda.current_stream().cuda_stream
torch.cuda.synchronize()
out = {"status": [], "free": [], "iters": []}

def call(c, j):
    prm, ys, qs, m, l, N = c
    rv = np.zeros(2)
    st = fn(prm, argv.ctypes.data, 2, rv.ctypes.data, 2, ys.data_ptr(), N * l, qs[j].data_ptr(), l, stream)
    out["status"].append(int(st))
    out["iters"].append(int(rv[0]))
    out["free"].append(int(torch.cuda.mem_get_info()[0]))

call(cases[0], 0)
call(cases[1], 0)
call(cases[1], 1)
# the ordinary stage on the same operands (it allocates; only after the checks above)
out["diff"] = []
out["iters_stage"] = []
for prm, ys, qs, m, l, N in cases:
    q0 = torch.zeros((m, l), dtype=torch.float64, device="cuda")
    r0 = lib.integrate("d", "KN", prm, ys, N * l, q0, l, argv=[256, 1e-4])
    out["iters_stage"].append(int(r0[0]))
    out["diff"].append(max(float((q - q0).abs().max().item()) for q in qs if not torch.isnan(q).any()))
print(json.dumps(out))
"""


def test_noalloc_fresh_process_shapes():
    """In a fresh process: a small call, then two calls of a larger shape that needs other kernel
    variants (tile size, split-K); free device memory is the same before and after the larger calls,
    every call succeeds, and the results equal the ordinary stage's within TOL with the same
    iteration counts."""
    r = subprocess.run([sys.executable, "-c", _FRESH, REPO], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-3000:]
    out = json.loads(r.stdout.strip().splitlines()[-1])
    assert out["status"] == [OK, OK, OK]
    assert out["free"][1] == out["free"][0] and out["free"][2] == out["free"][0], out["free"]
    assert out["iters"][0] == out["iters_stage"][0] > 1
    assert out["iters"][1] == out["iters"][2] == out["iters_stage"][1] > 1
    assert max(out["diff"]) < TOL, out["diff"]
