"""Out-of-core A (reference gpu/stage/@x@_sketch_gpu.h:65-135: A streamed through the device in
panels sized by isvd_gpu_memory_limit).  With the limit set below what a resident copy of A needs,
a host A is streamed in row panels by the sketch and again by the projection; the results match
the in-core solve of the same host A (FP64 to 1e-12, MIXED to 1e-6; same iteration counts) and
more kernels launch (one product per panel).  A limit below one 128-row panel is refused with
ISVD_GPU_ERROR_MEMORY before any device work."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

M, N_, K, P, NS = 3000, 1000, 16, 8, 8
L = K + P


def lowrank(m, n, seed):
    rng = np.random.default_rng(seed)
    u = np.linalg.qr(rng.standard_normal((m, 200)))[0]
    v = np.linalg.qr(rng.standard_normal((n, 200)))[0]
    return (u * 0.97 ** np.arange(200)) @ v.T + 1e-6 * rng.standard_normal((m, n))


@pytest.fixture
def limit(lib):
    var = ctypes.c_size_t.in_dll(lib.lib, "isvd_gpu_memory_limit")
    yield var
    var.value = 0


def launches(lib):
    lib.lib.isvd_gpu_kernel_launch_count.restype = ctypes.c_ulonglong
    return lib.lib.isvd_gpu_kernel_launch_count()


def run(lib, x, a_host, lda, ordera, precision, algs=("GP", "GR", "KN", "GR")):
    dt = np.float32 if x == "s" else np.float64
    prm = lib.create_param(M, N_, K, P, NS)
    s = np.zeros(L, dt)
    ut = np.zeros((M, L), dt)
    vt = np.zeros((N_, L), dt)
    om = np.random.default_rng(5).standard_normal((N_, L * NS)).astype(dt)
    c0 = launches(lib)
    retv, _, st = lib.isvd(x, prm, algs, a_host, lda, s, ut, L, vt, L, ordera=ordera,
                           argv=[None, None, [256, 1e-4] if algs[2] == "KN" else None, None], retc=(0, 0, 2, 0),
                           omega=om, ldomega=L * NS, precision=precision)
    return st, s.astype(np.float64), ut[:, :K].astype(np.float64), vt[:, :K].astype(np.float64), \
        list(retv[2]), launches(lib) - c0


@pytest.mark.parametrize("x,precision,ordera,lim_mb", [("d", 0, b"R", 100), ("d", 0, b"C", 100),
                                                      ("s", 1, b"R", 80), ("s", 1, b"C", 80)])
def test_driver_streams_host_a_in_row_panels(lib, oracle, limit, x, precision, ordera, lim_mb):
    dt = np.float32 if x == "s" else np.float64
    a = lowrank(M, N_, 1).astype(dt)
    a_host, lda = (a, N_) if ordera == b"R" else (np.ascontiguousarray(a.T), M)
    limit.value = 0
    st0, s0, u0, v0, r0, n0 = run(lib, x, a_host, lda, ordera, precision)
    assert st0 == 0, lib.last_error()
    limit.value = lim_mb << 20
    st1, s1, u1, v1, r1, n1 = run(lib, x, a_host, lda, ordera, precision)
    assert st1 == 0, lib.last_error()
    tol_s, tol_a = (1e-12, 1e-9) if x == "d" else (1e-6, 1e-4)
    assert np.abs(s1 - s0).max() <= tol_s * s0.max()
    assert r1[0] == r0[0]
    assert oracle.column_angles(u1, u0).max() < tol_a
    assert oracle.column_angles(v1, v0).max() < tol_a
    assert n1 > n0  # one product per panel, in the sketch and in the projection
    # and the in-core solve agrees with the oracle on the same Omega
    om = np.random.default_rng(5).standard_normal((N_, L * NS)).astype(dt).astype(np.float64)
    ref = oracle.isvd(a.astype(np.float64), om, K, P, NS)
    assert np.abs(s1[:K] - ref["s"][:K]).max() <= (1e-10 if x == "d" else 1e-5) * ref["s"][0]


def test_limit_below_one_panel_is_refused(lib, limit):
    a = lowrank(M, N_, 2)
    limit.value = 1 << 20
    lib.clear_error()
    st, *_ = run(lib, "d", a, N_, b"R", 0)
    assert st == 3 and lib.last_error()[0] == 3  # ISVD_GPU_ERROR_MEMORY
    assert "not enough GPU memory" in lib.last_error()[1]
    limit.value = 0
    lib.clear_error()
    st, *_ = run(lib, "d", a, N_, b"R", 0)
    assert st == 0


@pytest.mark.parametrize("x,sketch_mb,post_mb", [("d", 100, 75), ("s", 85, 75)])
def test_stages_stream_host_a(lib, oracle, limit, x, sketch_mb, post_mb):
    """isvd_?SketchGaussianProjectionOmega and isvd_?PostprocessGramian on a host A under the limit."""
    dt = np.float32 if x == "s" else np.float64
    a = lowrank(M, N_, 3).astype(dt)
    prm = lib.create_param(M, N_, K, P, NS)
    om = np.random.default_rng(6).standard_normal((N_, L * NS)).astype(dt)
    q = np.linalg.qr(np.random.default_rng(7).standard_normal((M, L)))[0].astype(dt)
    out, count = [], []
    for lims in ((0, 0), (sketch_mb << 20, post_mb << 20)):
        c0 = launches(lib)
        limit.value = lims[0]
        y = np.zeros((M, L * NS), dt)
        lib.sketch_omega(x, prm, a, N_, om, L * NS, y, L * NS)
        c1 = launches(lib)
        limit.value = lims[1]
        s = np.zeros(L, dt)
        ut = np.zeros((M, L), dt)
        vt = np.zeros((N_, L), dt)
        lib.postprocess(x, "GR", prm, a, N_, q, L, s, ut, L, vt, L)
        assert lib.last_error()[0] == 0, lib.last_error()
        out.append((y.astype(np.float64), s.astype(np.float64), vt[:, :K].astype(np.float64)))
        count.append((c1 - c0, launches(lib) - c1))
    assert count[1][0] > count[0][0] and count[1][1] > count[0][1]
    tol = 1e-12 if x == "d" else 1e-5
    assert np.abs(out[1][0] - out[0][0]).max() <= tol * np.abs(out[0][0]).max()
    assert np.abs(out[1][1] - out[0][1]).max() <= tol * out[0][1].max()
    assert oracle.column_angles(out[1][2], out[0][2]).max() < (1e-9 if x == "d" else 1e-3)
