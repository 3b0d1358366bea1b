"""The ILP64 build (libisvd_gpu_b200_64.so: isvd_int_t = int64, the reference's `_64` variant,
cmake/options.cmake:50-61) computes what the LP64 build computes: the same driver and stage calls
on the same inputs give bit-identical results and the same iteration counts."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def lowrank(m, n, rank, decay, noise, seed):
    rng = np.random.default_rng(seed)
    u = np.linalg.qr(rng.standard_normal((m, rank)))[0]
    v = np.linalg.qr(rng.standard_normal((n, rank)))[0]
    return (u * decay ** np.arange(rank)) @ v.T + noise * rng.standard_normal((m, n))


def run_driver(L, x, a, om, k, p, N, algs, precision):
    m, n = a.shape
    l = k + p
    dt = np.float32 if x == "s" else np.float64
    prm = L.create_param(m, n, k, p, N)
    s = np.zeros(l, dt)
    ut = np.zeros((m, l), dt)
    vt = np.zeros((n, l), dt)
    retv, _, st = L.isvd(x, prm, algs, np.ascontiguousarray(a.astype(dt)), n, s, ut, l, vt, l,
                         argv=[None, None, [256, 1e-4] if algs[2] == "KN" else None, None],
                         retc=(0, 0, 2, 0), omega=np.ascontiguousarray(om.astype(dt)), ldomega=l * N,
                         precision=precision)
    assert st == 0, L.last_error()
    return s, ut, vt, retv


@pytest.mark.parametrize("x,precision", [("d", 0), ("s", 1)])
@pytest.mark.parametrize("algs", [("GP", "GR", "KN", "GR"), ("GP", "TS", "WY", "TS")])
def test_ilp64_driver_matches_lp64(lib, lib64, x, precision, algs):
    m, n, k, p, N = 1200, 700, 16, 8, 8
    a = lowrank(m, n, 300, 0.97, 1e-6, 3)
    om = np.random.default_rng(4).standard_normal((n, (k + p) * N))
    r32 = run_driver(lib, x, a, om, k, p, N, algs, precision)
    r64 = run_driver(lib64, x, a, om, k, p, N, algs, precision)
    for u, v in zip(r32[:3], r64[:3]):
        assert np.array_equal(u, v)
    assert [list(v) for v in r32[3]] == [list(v) for v in r64[3]]


def test_ilp64_stage_call(lib, lib64, golden):
    """Kolmogorov-Nagumo stage on the reference golden (81 iterations) through both builds."""
    qs = np.ascontiguousarray(golden["qs"])
    m = qs.shape[0]
    L_, N_ = 11, 12
    out = []
    for L in (lib, lib64):
        prm = L.create_param(m, m, L_, 0, N_)
        qt = np.zeros((m, L_))
        r = L.integrate("d", "KN", prm, qs.copy(), L_ * N_, qt, L_, argv=[256, 1e-4])
        out.append((int(r[0]), qt))
    assert out[0][0] == out[1][0] == 81
    assert np.array_equal(out[0][1], out[1][1])
