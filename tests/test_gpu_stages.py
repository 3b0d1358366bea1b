"""Stage-by-stage parity of libisvd_gpu_b200 (NATIVE precision) with the reference's goldens
and tolerances (check/check/libisvd/core/stage/*.cxx: d 1e-8, s 1e-3, KN 81 iterations) and,
tighter, with the oracle.  All calls go through the C ABI."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

L, N = 11, 12
TOL = {"d": 1e-8, "s": 1e-3}
DT = {"d": np.float64, "s": np.float32}


def _a_layout(a, ordera):
    """A (m x n) stored per ordera with its leading dimension."""
    if ordera == b"R":
        return np.ascontiguousarray(a), a.shape[1]
    return np.asfortranarray(a), a.shape[0]


@pytest.fixture(autouse=True)
def _native(lib):
    lib.lib.isvd_gpu_set_precision(0)
    lib.clear_error()
    yield
    assert lib.last_error()[0] == 0, lib.last_error()


@pytest.mark.parametrize("x", ["d", "s"])
@pytest.mark.parametrize("dista", [b"R", b"C"])
@pytest.mark.parametrize("ordera", [b"R", b"C"])
def test_sketch_omega_golden(lib, golden, x, dista, ordera):
    a0, om = golden["a"].astype(DT[x]), golden["o_gp"].astype(DT[x])
    m, n = a0.shape
    a, lda = _a_layout(a0, ordera)
    prm = lib.create_param(m, n, L, 0, N)
    y = np.zeros((m, L * N), DT[x])
    lib.sketch_omega(x, prm, a, lda, np.ascontiguousarray(om), L * N, y, L * N, dista=dista, ordera=ordera)
    assert np.abs(y - golden["ys_gp"]).max() < (1e-8 if x == "d" else 1e-2)
    if x == "d":
        assert np.abs(y - golden["a"] @ golden["o_gp"]).max() < 1e-12 * np.abs(y).max()


@pytest.mark.parametrize("x", ["d", "s"])
def test_sketch_internal_rng_is_gaussian(lib, x):
    """Internal Omega: Y = A Omega with A = I (m = n) returns Omega itself."""
    m = n = 256
    prm = lib.create_param(m, n, 8, 8, 16)
    a = np.eye(m, dtype=DT[x])
    y = np.zeros((m, 256), DT[x])
    lib.sketch(x, prm, a, n, y, 256, seed=1234)
    assert abs(y.mean()) < 0.02 and abs(y.std() - 1.0) < 0.02
    y2 = np.zeros_like(y)
    lib.sketch(x, prm, a, n, y2, 256, seed=1234, gpu=True)
    assert np.array_equal(y, y2)
    y3 = np.zeros_like(y)
    lib.sketch(x, prm, a, n, y3, 256, seed=99)
    assert not np.allclose(y, y3)


@pytest.mark.parametrize("x", ["d", "s"])
def test_orthogonalize_gramian_golden(lib, golden, oracle, x):
    ys = golden["ys"]
    m = ys.shape[0]
    prm = lib.create_param(m, m, L, 0, N)
    y = np.ascontiguousarray(ys.astype(DT[x]))
    lib.orthogonalize(x, "GR", prm, y, L * N)
    for i in range(N):
        blk = slice(i * L, (i + 1) * L)
        assert oracle.projector_err(y[:, blk].astype(np.float64), golden["qs"][:, blk]) < TOL[x]
        if x == "d":
            assert np.abs(y[:, blk].T @ y[:, blk] - np.eye(L)).max() < 1e-10


@pytest.mark.parametrize("x", ["d", "s"])
def test_kn_golden(lib, golden, x):
    qs = golden["qs"]
    m = qs.shape[0]
    prm = lib.create_param(m, m, L, 0, N)
    qt = np.zeros((m, L), DT[x])
    r = lib.integrate(x, "KN", prm, np.ascontiguousarray(qs.astype(DT[x])), L * N, qt, L, argv=[256, 1e-4])
    assert int(r[0]) == 81
    assert np.abs(qt - golden["q_kn"]).max() < TOL[x]
    if x == "d":
        assert np.abs(qt - golden["q_kn"]).max() < 1e-12


def test_kn_maxit_semantics(lib, golden, oracle):
    """retv[0] = maxit + 1 when maxit is reached (reference :238-241)."""
    qs = golden["qs"]
    m = qs.shape[0]
    prm = lib.create_param(m, m, L, 0, N)
    qt = np.zeros((m, L))
    r = lib.integrate("d", "KN", prm, np.ascontiguousarray(qs), L * N, qt, L, argv=[10, 1e-4])
    qb, it, err = oracle.integrate_kolmogorov_nagumo(qs, L, N, 10, 1e-4)
    assert int(r[0]) == it == 11
    assert abs(r[1] - err) < 1e-12
    assert np.abs(qt - qb).max() < 1e-12


def test_kn_leading_dimensions(lib, golden, oracle):
    """ldyst > Nl and ldqt > l (padded row-major buffers) give the same result."""
    qs = golden["qs"]
    m = qs.shape[0]
    prm = lib.create_param(m, m, L, 0, N)
    ys = np.full((m, L * N + 5), np.nan)
    ys[:, :L * N] = qs
    qt = np.full((m, L + 3), 7.0)
    r = lib.integrate("d", "KN", prm, ys, L * N + 5, qt, L + 3, argv=[256, 1e-4])
    assert int(r[0]) == 81
    assert np.abs(qt[:, :L] - golden["q_kn"]).max() < 1e-12
    assert (qt[:, L:] == 7.0).all()


@pytest.mark.parametrize("x", ["d", "s"])
def test_hr_golden(lib, golden, oracle, x):
    qs = golden["qs"]
    m = qs.shape[0]
    prm = lib.create_param(m, m, L, 0, N)
    qt = np.zeros((m, L), DT[x])
    y = np.ascontiguousarray(qs.astype(DT[x]))
    lib.integrate(x, "HR", prm, y, L * N, qt, L)
    assert oracle.projector_err(qt.astype(np.float64), golden["q_hr"]) < TOL[x]
    if x == "d":
        qb, _ = oracle.integrate_hierarchical_reduction(qs, L, N)
        assert oracle.projector_err(qt, qb) < 1e-12


MODES = {"gather": (0, 0), "block": (-1, -1), "none": (-2, -2)}


@pytest.mark.parametrize("x", ["d", "s"])
@pytest.mark.parametrize("dista", [b"R", b"C"])
@pytest.mark.parametrize("ordera", [b"R", b"C"])
@pytest.mark.parametrize("mode", list(MODES))
def test_postprocess_gramian_golden(lib, golden, oracle, x, dista, ordera, mode):
    a0 = golden["a"].astype(DT[x])
    m, n = a0.shape
    a, lda = _a_layout(a0, ordera)
    prm = lib.create_param(m, n, L, 0, 1)
    s = np.zeros(L, DT[x])
    ut = np.zeros((m, L), DT[x])
    vt = np.zeros((n, L), DT[x])
    ur, vr = MODES[mode]
    lib.postprocess(x, "GR", prm, a, lda, np.ascontiguousarray(golden["q"].astype(DT[x])), L, s, ut, L, vt, L,
                    dista=dista, ordera=ordera, ut_root=ur, vt_root=vr)
    s_ref = golden["s"][:, 0]
    assert np.abs(s - s_ref).max() < TOL[x] * (s_ref.max() if x == "s" else 1.0)
    if mode == "none":
        assert not ut.any() and not vt.any()
        return
    assert oracle.projector_err(ut.astype(np.float64), golden["u"]) < TOL[x]
    assert oracle.projector_err(vt.astype(np.float64), golden["v"]) < TOL[x]
    if x == "d":
        s_o, u_o, v_o = oracle.postprocess_gramian(golden["a"], golden["q"], L)
        assert np.abs(s - s_o).max() < 1e-12 * s_o.max()
        assert oracle.column_angles(ut, u_o).max() < 1e-10
        assert oracle.column_angles(vt, v_o).max() < 1e-10
        # U and V carry the same column signs: A V = U diag(s)
        assert np.abs(ut.T @ golden["a"] @ vt - np.diag(s)).max() < 1e-9 * s.max()


@pytest.mark.parametrize("x", ["d", "s"])
def test_postprocess_symmetric_golden(lib, golden, oracle, x):
    a0 = golden["a_sym"].astype(DT[x])
    m = a0.shape[0]
    prm = lib.create_param(m, m, L, 0, 1)
    s = np.zeros(L, DT[x])
    ut = np.zeros((m, L), DT[x])
    vt = np.zeros((m, L), DT[x])
    lib.postprocess(x, "SY", prm, np.ascontiguousarray(a0), m, np.ascontiguousarray(golden["q"].astype(DT[x])), L,
                    s, ut, L, vt, L, ut_root=-1, vt_root=-1)
    lam = golden["s_sym"][:, 0]
    assert np.abs(s - lam).max() < TOL[x] * np.abs(lam).max()
    assert oracle.projector_err(ut.astype(np.float64), golden["u_sym"]) < TOL[x]
    assert np.array_equal(ut, vt)


def test_invalid_leading_dimension_reports_error(lib, golden):
    qs = golden["qs"]
    m = qs.shape[0]
    prm = lib.create_param(m, m, L, 0, N)
    qt = np.zeros((m, L))
    lib.integrate("d", "KN", prm, np.ascontiguousarray(qs), L * N - 1, qt, L, argv=[256, 1e-4])
    code, msg = lib.last_error()
    assert code == 1 and "ldyst" in msg
    lib.clear_error()


@pytest.mark.parametrize("l", [64, 65, 97, 128, 129, 160])
def test_postprocess_wide_sketch_eigensolver(lib, oracle, l):
    """Gramian and symmetric postprocessing at l = 64..160 (the l x l eigensolver on a thread-block
    cluster when the device allows one; odd l pairs one row with a dummy in every round): FP64
    results against the oracle, eigenvalues to 1e-12 and vectors to 1e-9."""
    rng = np.random.default_rng(l)
    m, n = 400, 900
    a = rng.standard_normal((m, n)) * 0.99 ** np.arange(n)
    q = np.linalg.qr(rng.standard_normal((m, l)))[0]
    prm = lib.create_param(m, n, l, 0, 1)
    s = np.zeros(l)
    ut = np.zeros((m, l))
    vt = np.zeros((n, l))
    lib.postprocess("d", "GR", prm, a, n, q, l, s, ut, l, vt, l)
    assert lib.last_error()[0] == 0, lib.last_error()
    s_o, u_o, v_o = oracle.postprocess_gramian(a, q, l)
    assert np.abs(s - s_o).max() < 1e-12 * s_o.max()
    assert oracle.column_angles(ut, u_o).max() < 1e-9
    assert oracle.column_angles(vt, v_o).max() < 1e-9
    sym = a[:, :m] @ a[:, :m].T / m - 0.3 * np.eye(m)  # indefinite: ascending order with signs
    prm = lib.create_param(m, m, l, 0, 1)
    s = np.zeros(l)
    u = np.zeros((m, l))
    lib.postprocess("d", "SY", prm, sym, m, q, l, s, u, l, None, l, ut_root=-1, vt_root=-2)
    assert lib.last_error()[0] == 0, lib.last_error()
    lam, u_s = oracle.postprocess_symmetric(sym, q, l)
    assert np.abs(s - lam).max() < 1e-12 * np.abs(lam).max()
    assert oracle.column_angles(u, u_s).max() < 1e-9
