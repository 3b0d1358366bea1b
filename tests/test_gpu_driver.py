"""End-to-end parity of the isvd_?Isvd driver with the reference pipeline, same inputs and the
same Omega (passed in): singular values within 1e-10 relative (FP64) and the largest
principal angle of U and V within 1e-4."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def lowrank(m, n, rank, decay, noise, seed):
    rng = np.random.default_rng(seed)
    u = np.linalg.qr(rng.standard_normal((m, rank)))[0]
    v = np.linalg.qr(rng.standard_normal((n, rank)))[0]
    sig = decay ** np.arange(rank)
    return (u * sig) @ v.T + noise * rng.standard_normal((m, n))


def reference_pipeline(reflib, a, om, k, p, N, alg_o="GR", alg_i="KN", alg_p="GR", argv_i=(256, 1e-4)):
    """The built reference's own stage routines on Y = A Omega (FP64)."""
    m, n = a.shape
    l = k + p
    prm = reflib.create_param(m, n, k, p, N)
    yst = np.ascontiguousarray(a @ om)
    reflib.orthogonalize("d", alg_o, prm, yst, l * N)
    qt = np.zeros((m, l))
    r = reflib.integrate("d", alg_i, prm, yst, l * N, qt, l, argv=list(argv_i))
    s = np.zeros(l)
    ut = np.zeros((m, l))
    vt = np.zeros((n, l))
    reflib.postprocess("d", alg_p, prm, np.ascontiguousarray(a), n, qt, l, s, ut, l, vt, l)
    return s, ut[:, :k], vt[:, :k], r


@pytest.mark.parametrize("shape", [(600, 300, 10, 6, 8), (2000, 1000, 20, 12, 16), (257, 513, 7, 5, 6)])
@pytest.mark.parametrize("ordera", [b"R", b"C"])
def test_driver_fp64_matches_reference(lib, reflib, oracle, shape, ordera):
    m, n, k, p, N = shape
    l = k + p
    a = lowrank(m, n, min(m, n) // 2, 0.97, 1e-6, seed=m + n)
    om = np.random.default_rng(5).standard_normal((n, l * N))
    s_r, u_r, v_r, r_r = reference_pipeline(reflib, a, om, k, p, N)
    prm = lib.create_param(m, n, k, p, N)
    s = np.zeros(l)
    ut = np.zeros((m, l))
    vt = np.zeros((n, l))
    aa = np.ascontiguousarray(a) if ordera == b"R" else np.asfortranarray(a)
    lda = n if ordera == b"R" else m
    retv, times, status = lib.isvd("d", prm, ("GP", "GR", "KN", "GR"), aa, lda, s, ut, l, vt, l,
                                   ordera=ordera, argv=[None, None, [256, 1e-4], None], retc=(0, 0, 2, 0),
                                   omega=np.ascontiguousarray(om), ldomega=l * N, precision=0)
    assert status == 0, lib.last_error()
    assert int(retv[2][0]) == int(r_r[0])
    assert np.abs(s - s_r).max() <= 1e-10 * s_r.max()
    assert oracle.max_principal_angle(ut[:, :k], u_r) < 1e-4
    assert oracle.max_principal_angle(vt[:, :k], v_r) < 1e-4
    assert oracle.column_angles(ut[:, :k], u_r).max() < 1e-8
    assert all(t >= 0 for t in times)


def test_driver_stream_output(lib, capfd):
    m, n, k, p, N = 300, 200, 5, 3, 4
    a = lowrank(m, n, 50, 0.3, 1e-9, 3)
    prm = lib.create_param(m, n, k, p, N)
    l = k + p
    s = np.zeros(l)
    ut = np.zeros((m, l))
    vt = np.zeros((n, l))
    lib.isvd("d", prm, ("gp_gpu", "gr", "kn", "gr_gpu"), np.ascontiguousarray(a), n, s, ut, l, vt, l, seed=7)
    assert lib.last_error()[0] == 0
    # internal Omega: the leading singular values are those of A to randomized-SVD accuracy
    sv = np.linalg.svd(a, compute_uv=False)[:k]
    assert np.abs(s[:k] - sv).max() < 1e-3 * sv[0]


def test_device_pointers(lib, oracle):
    torch = pytest.importorskip("torch")
    m, n, k, p, N = 500, 300, 8, 4, 6
    l = k + p
    a = lowrank(m, n, 100, 0.95, 1e-6, 11)
    om = np.random.default_rng(1).standard_normal((n, l * N))
    prm = lib.create_param(m, n, k, p, N)
    s_h, ut_h, vt_h = np.zeros(l), np.zeros((m, l)), np.zeros((n, l))
    r_h, _, st = lib.isvd("d", prm, ("GP", "GR", "KN", "GR"), np.ascontiguousarray(a), n, s_h, ut_h, l, vt_h, l,
                          omega=np.ascontiguousarray(om), ldomega=l * N, precision=0)
    assert st == 0
    dev = torch.device("cuda:0")
    a_d = torch.from_numpy(np.ascontiguousarray(a)).to(dev)
    om_d = torch.from_numpy(np.ascontiguousarray(om)).to(dev)
    s_d = torch.zeros(l, dtype=torch.float64, device=dev)
    ut_d = torch.zeros((m, l), dtype=torch.float64, device=dev)
    vt_d = torch.zeros((n, l), dtype=torch.float64, device=dev)
    torch.cuda.synchronize()
    r_d, _, st = lib.isvd("d", prm, ("GP", "GR", "KN", "GR"), a_d, n, s_d, ut_d, l, vt_d, l, omega=om_d,
                          ldomega=l * N, precision=0)
    assert st == 0
    assert np.array_equal(s_d.cpu().numpy(), s_h)
    assert np.array_equal(ut_d.cpu().numpy(), ut_h)
    assert int(r_d[2][0]) == int(r_h[2][0])
