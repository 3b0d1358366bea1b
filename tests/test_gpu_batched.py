"""Batched iSVD (isvd_?BatchIsvd) against single solves (isvd_?Isvd_ex, NATIVE precision) of the
same matrices with the same seeds: the batch runs every stage as grouped launches, so its results
must be those of the single solves to rounding, with the same Kolmogorov-Nagumo iteration counts."""
import ctypes

import numpy as np
import pytest

from isvd_b200.capi import c_int_t

pytestmark = pytest.mark.gpu

VP = ctypes.c_void_p


def _fns(lib, x):
    create = getattr(lib.lib, "isvd_%sBatchCreate" % x)
    create.argtypes = [c_int_t, VP, VP, VP, VP, c_int_t]
    create.restype = VP
    solve = getattr(lib.lib, "isvd_%sBatchIsvd" % x)
    solve.argtypes = [VP, VP, VP, VP, VP, VP, VP, VP, VP, VP, c_int_t, VP, VP]
    solve.restype = ctypes.c_int
    destroy = lib.lib.isvd_gpu_batch_destroy
    destroy.argtypes = [VP]
    destroy.restype = None
    return create, solve, destroy


def make_batch(count, seed, dt):
    """Matrices of uneven sizes: m log-uniform in [300, 1500], n log-uniform in [150, min(m, 800)],
    k in {4, 8, 16}, p = k / 2, each low-rank (3k) plus noise with a geometric spectrum."""
    torch = pytest.importorskip("torch")
    rng = np.random.default_rng(seed)
    mats = []
    for _ in range(count):
        m = int(np.exp(rng.uniform(np.log(300), np.log(1500))))
        n = int(np.exp(rng.uniform(np.log(150), np.log(min(m, 800)))))
        k = int(rng.choice([4, 8, 16]))
        r = 3 * k
        u = np.linalg.qr(rng.standard_normal((m, r)))[0]
        v = np.linalg.qr(rng.standard_normal((n, r)))[0]
        a = (u * np.geomspace(1.0, 1e-2, r)) @ v.T + 1e-5 * rng.standard_normal((m, n))
        mats.append(dict(m=m, n=n, k=k, p=k // 2, a=torch.tensor(a, dtype=dt, device="cuda")))
    return mats


def arr(vals, ct=c_int_t):
    return (ct * len(vals))(*vals)


def run_batch(lib, x, mats, N, seeds, argv=(256, 1e-4), solves=1):
    torch = pytest.importorskip("torch")
    create, solve, destroy = _fns(lib, x)
    B = len(mats)
    dt = mats[0]["a"].dtype
    batch = create(B, arr([d["m"] for d in mats]), arr([d["n"] for d in mats]), arr([d["k"] for d in mats]),
                   arr([d["p"] for d in mats]), N)
    assert batch, lib.last_error()
    outs = []
    for d in mats:
        l = d["k"] + d["p"]
        outs.append(dict(s=torch.zeros(l, dtype=dt, device="cuda"), ut=torch.zeros((d["m"], l), dtype=dt, device="cuda"),
                         vt=torch.zeros((d["n"], l), dtype=dt, device="cuda")))
    npdt = np.float32 if x == "s" else np.float64
    av = np.asarray(argv, dtype=npdt)
    results = []
    for _ in range(solves):
        its = arr([0] * B)
        errs = (ctypes.c_float if x == "s" else ctypes.c_double) * B
        errs = errs()
        torch.cuda.synchronize()
        st = solve(batch, arr([d["a"].data_ptr() for d in mats], VP), arr([d["n"] for d in mats]),
                   arr([o["s"].data_ptr() for o in outs], VP), arr([o["ut"].data_ptr() for o in outs], VP),
                   arr([o["ut"].shape[1] for o in outs]), arr([o["vt"].data_ptr() for o in outs], VP),
                   arr([o["vt"].shape[1] for o in outs]), arr(seeds), av.ctypes.data, len(av), its, errs)
        assert st == 0, lib.last_error()
        results.append(([o["s"].cpu().numpy().copy() for o in outs], [o["ut"].cpu().numpy().copy() for o in outs],
                        [o["vt"].cpu().numpy().copy() for o in outs], list(its), list(errs)))
    destroy(batch)
    return results


def single(lib, x, d, N, seed, argv=(256, 1e-4)):
    torch = pytest.importorskip("torch")
    m, n, k, p = d["m"], d["n"], d["k"], d["p"]
    l = k + p
    dt = d["a"].dtype
    prm = lib.create_param(m, n, k, p, N)
    s = torch.zeros(l, dtype=dt, device="cuda")
    ut = torch.zeros((m, l), dtype=dt, device="cuda")
    vt = torch.zeros((n, l), dtype=dt, device="cuda")
    torch.cuda.synchronize()
    retv, _, st = lib.isvd(x, prm, ("GP", "GR", "KN", "GR"), d["a"], n, s, ut, l, vt, l, seed=seed,
                           argv=[None, None, list(argv), None], retc=(0, 0, 2, 0), precision=0)
    assert st == 0, lib.last_error()
    return s.cpu().numpy(), ut.cpu().numpy(), vt.cpu().numpy(), int(retv[2][0])


@pytest.mark.parametrize("x", ["d", "s"])
def test_batch_matches_single_solves(lib, oracle, x):
    torch = pytest.importorskip("torch")
    dt = torch.float64 if x == "d" else torch.float32
    N = 8
    mats = make_batch(12, 4, dt)
    seeds = [100 + i for i in range(len(mats))]
    (s_b, u_b, v_b, it_b, _), = run_batch(lib, x, mats, N, seeds)
    tol_s = 1e-10 if x == "d" else 1e-5
    tol_a = 1e-8 if x == "d" else 1e-3
    for i, d in enumerate(mats):
        s1, u1, v1, it1 = single(lib, x, d, N, seeds[i])
        k = d["k"]
        if x == "d":
            assert it_b[i] == it1
        else:
            assert abs(it_b[i] - it1) <= 1
        assert np.abs(s_b[i] - s1).max() <= tol_s * s1.max()
        assert oracle.column_angles(u_b[i][:, :k].astype(np.float64), u1[:, :k].astype(np.float64)).max() < tol_a
        assert oracle.column_angles(v_b[i][:, :k].astype(np.float64), v1[:, :k].astype(np.float64)).max() < tol_a


def test_batch_graph_replay(lib):
    """Later solves replay the graphs captured by the second one: the same inputs give the same bits."""
    torch = pytest.importorskip("torch")
    N = 8
    mats = make_batch(6, 9, torch.float64)
    seeds = [7 * i + 1 for i in range(len(mats))]
    r = run_batch(lib, "d", mats, N, seeds, solves=3)
    for j in (1, 2):
        for i in range(len(mats)):
            assert np.array_equal(r[0][0][i], r[j][0][i])
            assert np.array_equal(r[0][1][i], r[j][1][i])
            assert r[0][3][i] == r[j][3][i]


def test_batch_rejects_bad_shapes(lib):
    create, _, _ = _fns(lib, "d")
    lib.clear_error()
    assert not create(1, arr([500]), arr([300]), arr([80]), arr([40]), 8)  # l = 120 > 96
    code, msg = lib.last_error()
    assert code == 6 and "l = 120" in msg
    lib.clear_error()
    assert not create(1, arr([50]), arr([30]), arr([30]), arr([10]), 8)  # l > n
    assert lib.last_error()[0] == 1
    lib.clear_error()
