"""Parity of the tall-skinny QR stages (TS orthogonalization, TS postprocessing) and Wen-Yin
integration with the reference built from source (same inputs) and the reference's goldens
(check/check/libisvd/core/stage/*.cxx: d 1e-8, s 1e-3, WY 21 iterations at tol 1e-3)."""
import numpy as np
import pytest

from test_gpu_driver import lowrank, reference_pipeline

pytestmark = pytest.mark.gpu

L, N = 11, 12
TOL = {"d": 1e-8, "s": 1e-3}
DT = {"d": np.float64, "s": np.float32}


@pytest.fixture(autouse=True)
def _native(lib):
    lib.lib.isvd_gpu_set_precision(0)
    lib.clear_error()
    yield
    lib.lib.isvd_gpu_set_precision(0)
    assert lib.last_error()[0] == 0, lib.last_error()


def _ts(lib, x, y, l, N):
    m = y.shape[0]
    prm = lib.create_param(m, m, l, 0, N)
    out = np.ascontiguousarray(y.astype(DT[x]))
    lib.orthogonalize(x, "TS", prm, out, l * N)
    return out


@pytest.mark.parametrize("x", ["d", "s"])
def test_orthogonalize_tsqr_matches_reference(lib, reflib, golden, x):
    """Same Q factors as the reference's Householder LQ, column signs included."""
    ys = golden["ys"]
    q = _ts(lib, x, ys, L, N)
    q_ref = _ts(reflib, x, ys, L, N)
    assert np.abs(q.astype(np.float64) - q_ref).max() < (1e-11 if x == "d" else 1e-4)
    for i in range(N):
        blk = q[:, i * L:(i + 1) * L].astype(np.float64)
        assert np.abs(blk.T @ blk - np.eye(L)).max() < (1e-13 if x == "d" else 1e-5)


def test_orthogonalize_tsqr_ill_conditioned(lib, reflib):
    """Blocks with condition numbers up to 1e7 (shifted first pass) still give the Householder factor."""
    rng = np.random.default_rng(4)
    m, l, N = 3000, 24, 5
    ys = np.empty((m, l * N))
    for i in range(N):
        u = np.linalg.qr(rng.standard_normal((m, l)))[0]
        v = np.linalg.qr(rng.standard_normal((l, l)))[0]
        ys[:, i * l:(i + 1) * l] = (u * np.logspace(0, -(i + 3), l)) @ v.T
    q = _ts(lib, "d", ys, l, N)
    q_ref = _ts(reflib, "d", ys, l, N)
    for i in range(N):
        blk = slice(i * l, (i + 1) * l)
        assert np.abs(q[:, blk].T @ q[:, blk] - np.eye(l)).max() < 1e-13
        assert np.abs(q[:, blk] - q_ref[:, blk]).max() < 1e-15 * 10.0 ** (i + 3) * 100


@pytest.mark.parametrize("x", ["d", "s"])
def test_wen_yin_golden(lib, golden, x):
    qs = golden["qs"]
    m = qs.shape[0]
    prm = lib.create_param(m, m, L, 0, N)
    qt = np.zeros((m, L), DT[x])
    r = lib.integrate(x, "WY", prm, np.ascontiguousarray(qs.astype(DT[x])), L * N, qt, L, argv=[256, 1e-3])
    assert int(r[0]) == 21
    assert np.abs(qt - golden["q_wy"]).max() < TOL[x]
    if x == "d":
        assert np.abs(qt - golden["q_wy"]).max() < 1e-9


def _blocks(seed, m, l, N, noise):
    """N orthonormal m x l blocks scattered around a common l-dimensional subspace."""
    rng = np.random.default_rng(seed)
    base = np.linalg.qr(rng.standard_normal((m, l)))[0]
    qs = np.empty((m, N * l))
    for i in range(N):
        qs[:, i * l:(i + 1) * l] = np.linalg.qr(base + noise / np.sqrt(m) * rng.standard_normal((m, l)))[0]
    return qs


@pytest.mark.parametrize("argv", [[512, 1e-4], [512, 1e-6], [5, 1e-6],
                                  [256, 1e-5, 0.25, 1e3, 1e-6, 8, 0.3, 1e-3, 0.7]])
def test_wen_yin_matches_reference(lib, reflib, argv):
    """Iteration count, mu and Qbar against the reference built from source: tight tolerances,
    non-default line-search parameters and maxit exhaustion (retv[0] = maxit + 1).

    The blocks have m = 2000 rows.  (On the golden Qs, 101 rows for N l = 132 columns, the
    iteration at tol <= 1e-4 is chaotic: a relative perturbation of 1e-15 of the input moves the
    reference's own iteration count between 60 and 63 and its Qbar by 2e-3.)"""
    m, l, N = 2000, 10, 8
    qs = _blocks(1, m, l, N, 3.0)
    prm = lib.create_param(m, m, l, 0, N)
    qt, q_ref = np.zeros((m, l)), np.zeros((m, l))
    r = lib.integrate("d", "WY", prm, qs, l * N, qt, l, argv=argv)
    r_ref = reflib.integrate("d", "WY", prm, qs, l * N, q_ref, l, argv=argv)
    assert int(r[0]) == int(r_ref[0]) > 2
    if argv[0] == 5:
        assert int(r[0]) == 6
    else:
        assert r[1] < argv[1] ** 2
    assert np.abs(qt - q_ref).max() < 1e-11
    assert abs(r[1] - r_ref[1]) < 1e-12 + 1e-6 * abs(r_ref[1])


@pytest.mark.parametrize("x", ["d", "s"])
def test_postprocess_tsqr(lib, reflib, golden, oracle, x):
    a0 = golden["a"].astype(DT[x])
    m, n = a0.shape
    prm = lib.create_param(m, n, L, 0, 1)
    q = np.ascontiguousarray(golden["q"].astype(DT[x]))
    s, ut, vt = np.zeros(L, DT[x]), np.zeros((m, L), DT[x]), np.zeros((n, L), DT[x])
    lib.postprocess(x, "TS", prm, np.ascontiguousarray(a0), n, q, L, s, ut, L, vt, L)
    s_ref = golden["s"][:, 0]
    assert np.abs(s - s_ref).max() < TOL[x] * (s_ref.max() if x == "s" else 1.0)
    s_o, u_o, v_o = oracle.postprocess_tall_skinny_qr(golden["a"], golden["q"], L)
    # U up to column signs; V mixes the rows of the small SVD's U (the reference's pairing), so only
    # its span is independent of the SVD's sign convention
    tol = 1e-10 if x == "d" else 1e-4
    assert np.abs(s - s_o).max() < tol * s_o.max()
    assert oracle.column_angles(ut.astype(np.float64), u_o).max() < tol
    assert oracle.projector_err(vt.astype(np.float64), v_o) < tol
    s_r, ut_r, vt_r = np.zeros(L, DT[x]), np.zeros((m, L), DT[x]), np.zeros((n, L), DT[x])
    reflib.postprocess(x, "TS", prm, np.ascontiguousarray(a0), n, q, L, s_r, ut_r, L, vt_r, L)
    assert np.abs(s - s_r).max() < tol * s_r.max()
    assert oracle.column_angles(ut.astype(np.float64), ut_r.astype(np.float64)).max() < tol


@pytest.mark.parametrize("algs", [("GP", "TS", "WY", "TS"), ("GP", "TS", "KN", "GR"), ("GP", "GR", "WY", "TS")])
def test_driver_qr_wy_matches_reference(lib, reflib, oracle, algs):
    m, n, k, p, N = 1500, 700, 12, 8, 8
    l = k + p
    a = lowrank(m, n, 300, 0.97, 1e-6, seed=21)
    om = np.random.default_rng(8).standard_normal((n, l * N))
    argv_i = (256, 1e-4) if algs[2] == "KN" else (256, 1e-3)
    s_r, u_r, v_r, r_r = reference_pipeline(reflib, a, om, k, p, N, algs[1], algs[2], algs[3], argv_i)
    prm = lib.create_param(m, n, k, p, N)
    s, ut, vt = np.zeros(l), np.zeros((m, l)), np.zeros((n, l))
    retv, times, status = lib.isvd("d", prm, algs, np.ascontiguousarray(a), n, s, ut, l, vt, l,
                                   argv=[None, None, list(argv_i), None], retc=(0, 0, 2, 0),
                                   omega=np.ascontiguousarray(om), ldomega=l * N, precision=0)
    assert status == 0, lib.last_error()
    assert int(retv[2][0]) == int(r_r[0])
    assert np.abs(s[:k] - s_r[:k]).max() <= 1e-9 * s_r.max()
    if algs[1] == "GR" and algs[3] == "TS":
        # The reference's TS postprocessing forms U = Qbar V_L[:, :k] and V = Qz U_L' (see
        # oracle.postprocess_tall_skinny_qr): neither is invariant under a change of Qbar's basis,
        # and after GR orthogonalization Qbar's column signs follow the small eigensolver's sign
        # convention (LAPACK's there, this library's here).  Only sigma is comparable.
        return
    assert oracle.max_principal_angle(ut[:, :k], u_r) < 1e-4
    if algs[3] != "TS":  # TS postprocessing's V columns depend on the small SVD's sign convention
        assert oracle.max_principal_angle(vt[:, :k], v_r) < 1e-4


@pytest.mark.parametrize("algs", [("GP", "TS", "WY", "GR"), ("GP", "TS", "KN", "TS")])
def test_driver_qr_wy_mixed(lib, oracle, algs):
    """MIXED precision (bf16 split tensor-core products) against the FP64 path on FP32 input."""
    m, n, k, p, N = 4000, 2000, 16, 16, 8
    l = k + p
    a = lowrank(m, n, 600, 0.99, 1e-5, seed=33).astype(np.float32)
    om = np.random.default_rng(2).standard_normal((n, l * N))
    out = {}
    for prec, x in ((0, "d"), (1, "s")):
        prm = lib.create_param(m, n, k, p, N)
        dt = DT[x]
        s, ut, vt = np.zeros(l, dt), np.zeros((m, l), dt), np.zeros((n, l), dt)
        argv_i = [256, 1e-4] if algs[2] == "KN" else [256, 1e-3]
        retv, _, status = lib.isvd(x, prm, algs, np.ascontiguousarray(a.astype(dt)), n, s, ut, l, vt, l,
                                   argv=[None, None, argv_i, None], retc=(0, 0, 2, 0),
                                   omega=np.ascontiguousarray(om.astype(dt)), ldomega=l * N, precision=prec)
        assert status == 0, lib.last_error()
        out[prec] = (s.astype(np.float64), ut.astype(np.float64), vt.astype(np.float64))
    s0, u0, v0 = out[0]
    s1, u1, v1 = out[1]
    assert np.abs(s1[:k] - s0[:k]).max() <= 1e-5 * s0.max()
    assert oracle.max_principal_angle(u1[:, :k], u0[:, :k]) < 1e-3
    assert oracle.projector_err(v1, v0) < 1e-3


def _rank5(seed=17):
    """A 101 x 1001 matrix of rank 5 (the golden shape), sigma 1 .. 0.2."""
    rng = np.random.default_rng(seed)
    u = np.linalg.qr(rng.standard_normal((101, 5)))[0]
    v = np.linalg.qr(rng.standard_normal((1001, 5)))[0]
    return (u * np.array([1.0, 0.8, 0.6, 0.4, 0.2])) @ v.T


@pytest.mark.parametrize("x", ["d", "s"])
def test_orthogonalize_tsqr_rank_deficient(lib, reflib, x):
    """Blocks of rank 5 < l = 11 (Y = A Omega with A of rank 5), a block whose third column repeats
    its first, and a zero block: the factor is orthonormal and contains span(Y_i), as Householder QR
    (gelqf / orglq) gives, and its leading independent columns are the reference's.  The completing
    columns are any orthonormal completion, in the reference as here."""
    a = _rank5()
    om = np.random.default_rng(3).standard_normal((1001, L * N))
    ys = a @ om
    ys[:, 4 * L + 2] = ys[:, 4 * L]          # block 4: column 2 = column 0
    ys[:, 7 * L:8 * L] = 0.0                  # block 7: zero
    q = _ts(lib, x, ys, L, N).astype(np.float64)
    q_ref = _ts(reflib, x, ys, L, N).astype(np.float64)
    orth, lead = (1e-13, 1e-10) if x == "d" else (1e-5, 1e-3)
    for i in range(N):
        blk = slice(i * L, (i + 1) * L)
        qi = q[:, blk]
        assert np.abs(qi.T @ qi - np.eye(L)).max() < orth, i
        yi = ys[:, blk]
        if np.abs(yi).max() > 0:
            assert np.linalg.norm(yi - qi @ (qi.T @ yi)) <= orth * 10 * np.linalg.norm(yi), i
        nlead = {4: 2, 7: 0}.get(i, 5)
        if nlead:
            assert np.abs(qi[:, :nlead] - q_ref[:, blk][:, :nlead]).max() < lead, i


def test_driver_ts_rank_deficient_matches_reference(lib, reflib, oracle):
    """GP / TS / KN / GR on a rank-5 A with l = 11 (the golden shape), Omega passed in: the five
    nonzero singular values and their U, V columns equal the reference's; the others are zero."""
    a = _rank5()
    m, n = a.shape
    k, p = 8, 3
    l = k + p
    om = np.random.default_rng(9).standard_normal((n, l * N))
    s_r, u_r, v_r, _ = reference_pipeline(reflib, a, om, k, p, N, "TS", "KN", "GR")
    for prec, x in ((0, "d"), (1, "s")):
        dt = DT[x]
        prm = lib.create_param(m, n, k, p, N)
        s, ut, vt = np.zeros(l, dt), np.zeros((m, l), dt), np.zeros((n, l), dt)
        retv, _, status = lib.isvd(x, prm, ("GP", "TS", "KN", "GR"), np.ascontiguousarray(a.astype(dt)), n, s, ut,
                                   l, vt, l, argv=[None, None, [256, 1e-4], None], retc=(0, 0, 2, 0),
                                   omega=np.ascontiguousarray(om.astype(dt)), ldomega=l * N, precision=prec)
        assert status == 0, lib.last_error()
        assert 1 <= int(retv[2][0]) <= 256
        tol = 1e-10 if x == "d" else 1e-5
        s = s.astype(np.float64)
        assert np.abs(s[:5] - s_r[:5]).max() <= tol * s_r[0]
        assert np.abs(s[5:k]).max() <= (1e-12 if x == "d" else 1e-5) * s_r[0]
        assert oracle.max_principal_angle(ut[:, :5].astype(np.float64), u_r[:, :5]) < (1e-8 if x == "d" else 1e-3)
        assert oracle.max_principal_angle(vt[:, :5].astype(np.float64), v_r[:, :5]) < (1e-8 if x == "d" else 1e-3)


@pytest.mark.parametrize("x", ["d", "s"])
def test_postprocess_tsqr_rank_deficient(lib, reflib, oracle, x):
    """TS postprocessing of Z = A' Qbar of rank 5 < l (reference gelqf of Z' is total): five
    singular values and U columns equal the reference's, the other singular values are zero."""
    a = _rank5().astype(DT[x])
    m, n = a.shape
    q = np.linalg.qr(np.random.default_rng(6).standard_normal((m, L)))[0].astype(DT[x])
    prm = lib.create_param(m, n, L, 0, 1)
    out = {}
    for name, lb in (("gpu", lib), ("ref", reflib)):
        s, ut, vt = np.zeros(L, DT[x]), np.zeros((m, L), DT[x]), np.zeros((n, L), DT[x])
        lb.postprocess(x, "TS", prm, np.ascontiguousarray(a), n, q, L, s, ut, L, vt, L)
        out[name] = (s.astype(np.float64), ut.astype(np.float64))
    (s, ut), (s_r, ut_r) = out["gpu"], out["ref"]
    tol = 1e-10 if x == "d" else 1e-5
    assert np.abs(s[:5] - s_r[:5]).max() <= tol * s_r[0]
    assert np.abs(s[5:]).max() <= (1e-12 if x == "d" else 1e-5) * s_r[0]
    assert oracle.column_angles(ut[:, :5], ut_r[:, :5]).max() < (1e-8 if x == "d" else 1e-3)
