"""Pins the NumPy restatement (oracle/isvd_oracle.py) and the built reference library
(oracle/_ref) against the reference's own golden fixtures (data/*.mtx) and tolerances
(check/check/libisvd/core/stage/*.cxx: s 1e-3, d 1e-8; KN 81 and WY 21 iterations)."""
import numpy as np
import pytest

L, N = 11, 12


def test_sketch_golden(golden, oracle):
    y = oracle.sketch_gaussian_projection(golden["a"], golden["o_gp"])
    assert np.abs(y - golden["ys_gp"]).max() < 1e-8


def test_orthogonalize_golden(golden, oracle):
    for fn in (oracle.orthogonalize_gramian, oracle.orthogonalize_tall_skinny_qr):
        q = fn(golden["ys"], L, N)
        for i in range(N):
            blk = slice(i * L, (i + 1) * L)
            assert oracle.projector_err(q[:, blk], golden["qs"][:, blk]) < 1e-8


def test_kn_golden(golden, oracle):
    qb, it, err = oracle.integrate_kolmogorov_nagumo(golden["qs"], L, N, 256, 1e-4)
    assert it == int(golden["kn_iter"]) == 81
    assert np.abs(qb - golden["q_kn"]).max() < 1e-8
    assert err <= 1e-4


def test_wy_golden(golden, oracle):
    qb, it, mu = oracle.integrate_wen_yin(golden["qs"], L, N, tol=1e-3)
    assert it == int(golden["wy_iter"]) == 21
    assert np.abs(qb - golden["q_wy"]).max() < 1e-8


def test_hr_golden(golden, oracle):
    qb, _ = oracle.integrate_hierarchical_reduction(golden["qs"], L, N)
    assert oracle.projector_err(qb, golden["q_hr"]) < 1e-8


@pytest.mark.parametrize("alg", ["GR", "TS"])
def test_postprocess_golden(golden, oracle, alg):
    fn = oracle.postprocess_gramian if alg == "GR" else oracle.postprocess_tall_skinny_qr
    s, u, v = fn(golden["a"], golden["q"], L)
    assert np.abs(s - golden["s"][:, 0]).max() < 1e-8 * s.max()
    assert oracle.projector_err(u, golden["u"]) < 1e-8
    assert oracle.projector_err(v, golden["v"]) < 1e-8


def test_postprocess_symmetric_golden(golden, oracle):
    lam, u = oracle.postprocess_symmetric(golden["a_sym"], golden["q"], L)
    assert np.abs(lam - golden["s_sym"][:, 0]).max() < 1e-8 * np.abs(lam).max()
    assert oracle.projector_err(u, golden["u_sym"]) < 1e-8


# ------------------------------------------------------------------ the built reference itself
def test_reflib_kn_wy_golden(golden, reflib):
    m = golden["qs"].shape[0]
    p = reflib.create_param(m, m, L, 0, N)
    qst = np.ascontiguousarray(golden["qs"])
    for alg, tol, key, iters in (("KN", 1e-4, "q_kn", 81), ("WY", 1e-3, "q_wy", 21)):
        qt = np.zeros((m, L))
        r = reflib.integrate("d", alg, p, qst, L * N, qt, L, argv=[256, tol])
        assert int(r[0]) == iters
        assert np.abs(qt - golden[key]).max() < 1e-8


def test_reflib_query_defaults(reflib):
    assert list(reflib.query("d", "KN", 2)) == [256, 1e-4]
    assert list(reflib.query("d", "WY", 9)) == [256, 1e-3, 1.0, 1e14, 1e-14, 20, 0.5, 1e-4, 0.85]


def test_oracle_matches_reflib_pipeline(oracle, reflib):
    """Stage by stage on a seeded tall problem (m > n, the configuration the upstream param check
    rejects): the restatement and the reference agree to FP64 rounding."""
    rng = np.random.default_rng(7)
    m, n, k, p_, Nn = 300, 120, 6, 4, 5
    l = k + p_
    a = rng.standard_normal((m, 40)) @ rng.standard_normal((40, n)) + 1e-3 * rng.standard_normal((m, n))
    om = rng.standard_normal((n, l * Nn))
    y = a @ om
    prm = reflib.create_param(m, n, k, p_, Nn)
    yst = np.ascontiguousarray(y)
    reflib.orthogonalize("d", "GR", prm, yst, l * Nn)
    q_o = oracle.orthogonalize_gramian(y, l, Nn)
    for i in range(Nn):
        blk = slice(i * l, (i + 1) * l)
        assert oracle.projector_err(yst[:, blk], q_o[:, blk]) < 1e-10
    qt = np.zeros((m, l))
    r = reflib.integrate("d", "KN", prm, yst, l * Nn, qt, l, argv=[256, 1e-4])
    qb, it, _ = oracle.integrate_kolmogorov_nagumo(yst, l, Nn, 256, 1e-4)
    assert int(r[0]) == it
    assert np.abs(qt - qb).max() < 1e-10
    s = np.zeros(l)
    ut = np.zeros((m, l))
    vt = np.zeros((n, l))
    reflib.postprocess("d", "GR", prm, np.ascontiguousarray(a), n, qt, l, s, ut, l, vt, l)
    s_o, u_o, v_o = oracle.postprocess_gramian(a, qb, k)
    assert np.abs(s - s_o).max() < 1e-12 * s.max()
    assert oracle.column_angles(ut[:, :k], u_o).max() < 1e-8
    assert oracle.column_angles(vt[:, :k], v_o).max() < 1e-8
