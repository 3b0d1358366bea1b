"""MIXED precision (bf16 split planes on tcgen05 tensor cores, FP32 accumulation, FP64 l x l steps)
against FP64: every stage on the reference goldens, and end to end against the FP64 path with
the same Omega.  Tolerance: singular values within 1e-5 relative, largest principal angle of U
and V within 1e-4 (the mixed-precision bar); products within FP32 rounding (1e-6 relative)."""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
L, N = 11, 12


@pytest.fixture(autouse=True)
def _mixed(lib):
    lib.lib.isvd_gpu_set_precision(1)
    lib.clear_error()
    yield
    lib.lib.isvd_gpu_set_precision(0)
    assert lib.last_error()[0] == 0, lib.last_error()


def lowrank(m, n, rank, decay, noise, seed):
    rng = np.random.default_rng(seed)
    u = np.linalg.qr(rng.standard_normal((m, rank)))[0]
    v = np.linalg.qr(rng.standard_normal((n, rank)))[0]
    return (u * decay ** np.arange(rank)) @ v.T + noise * rng.standard_normal((m, n))


@pytest.mark.parametrize("x", ["s", "d"])
@pytest.mark.parametrize("ordera", [b"R", b"C"])
@pytest.mark.parametrize("shape", [(101, 1001, 132), (1000, 777, 300), (300, 2000, 512)])
def test_mixed_sketch_omega(lib, x, ordera, shape):
    """Y = A Omega with A split into 2 planes and Omega into 3 (5 products): FP32-level accuracy
    (the FP32 tensor-core accumulation bounds it, as it bounds an FP32 GEMM: ~1e-6 relative at
    K = 1e3..2e4), across M/N/K tails and both storage orders of A."""
    m, n, nl = shape
    dt = np.float32 if x == "s" else np.float64
    rng = np.random.default_rng(m + n)
    a = rng.standard_normal((m, n)).astype(dt)
    om = rng.standard_normal((n, nl)).astype(dt)
    aa = np.ascontiguousarray(a) if ordera == b"R" else np.asfortranarray(a)
    lda = n if ordera == b"R" else m
    prm = lib.create_param(m, n, nl, 0, 1)
    y = np.zeros((m, nl), dt)
    lib.sketch_omega(x, prm, aa, lda, np.ascontiguousarray(om), nl, y, nl, ordera=ordera)
    ref = a.astype(np.float64) @ om.astype(np.float64)
    err = np.abs(y - ref).max() / np.abs(ref).max()
    assert err < 1e-5, err


@pytest.mark.parametrize("bk", ["64", "32"])
def test_mixed_sketch_cta_pair(lib, monkeypatch, bk):
    """A sketch large enough for the CTA-pair kernel (ISVD_UMMA_PAIR=1; 80 tiles of 256 x 256; M, N
    and K tails): the one-CTA kernel's products (ISVD_UMMA_PAIR=0) to the tensor cores' FP32
    accumulation error over 512-deep chunks (M = 256 and M = 128 instructions may add in different
    orders; 5e-6 of max |Y|), and the FP64 product to the sketch's bar."""
    m, n, nl = 4000, 1500, 1200
    rng = np.random.default_rng(8)
    a = rng.standard_normal((m, n)).astype(np.float32)
    om = rng.standard_normal((n, nl)).astype(np.float32)
    prm = lib.create_param(m, n, nl, 0, 1)
    monkeypatch.setenv("ISVD_UMMA_PAIR", "1")
    monkeypatch.setenv("ISVD_UMMA_PAIR_BK", bk)
    y2 = np.zeros((m, nl), np.float32)
    lib.sketch_omega("s", prm, a, n, om, nl, y2, nl)
    monkeypatch.setenv("ISVD_UMMA_PAIR", "0")
    y1 = np.zeros((m, nl), np.float32)
    lib.sketch_omega("s", prm, a, n, om, nl, y1, nl)
    ref = a.astype(np.float64) @ om.astype(np.float64)
    scale = np.abs(ref).max()
    assert np.abs(y2 - y1).max() < 5e-6 * scale
    assert np.abs(y2 - ref).max() < 1e-5 * scale


@pytest.mark.parametrize("order", [("3", "0"), ("3", "1"), ("16", "1"), ("0", "1")])
def test_mixed_sketch_tile_order_bitwise(lib, monkeypatch, order):
    """The sketch's column-grouped tile order (ISVD_GPU_SKETCH_NGROUP: 3 N tiles per group over 16,
    so the last group is one tile wide; 16: one group) and its L2 cache policies
    (ISVD_GPU_SKETCH_L2HINT) change which CTA runs a tile and when, not the tile's arithmetic:
    bitwise the row-major order's Y."""
    m, n, nl = 1100, 900, 4096
    rng = np.random.default_rng(21)
    a = rng.standard_normal((m, n)).astype(np.float32)
    om = rng.standard_normal((n, nl)).astype(np.float32)
    prm = lib.create_param(m, n, nl, 0, 1)
    monkeypatch.setenv("ISVD_GPU_SKETCH_NGROUP", "0")
    monkeypatch.setenv("ISVD_GPU_SKETCH_L2HINT", "0")
    y0 = np.zeros((m, nl), np.float32)
    lib.sketch_omega("s", prm, a, n, om, nl, y0, nl)
    monkeypatch.setenv("ISVD_GPU_SKETCH_NGROUP", order[0])
    monkeypatch.setenv("ISVD_GPU_SKETCH_L2HINT", order[1])
    y1 = np.zeros((m, nl), np.float32)
    lib.sketch_omega("s", prm, a, n, om, nl, y1, nl)
    assert np.array_equal(y0, y1)
    ref = a.astype(np.float64) @ om.astype(np.float64)
    assert np.abs(y1 - ref).max() < 1e-5 * np.abs(ref).max()


def test_mixed_kn_gram_cta_pair(lib, monkeypatch):
    """KN at N l = 4096 (the Gram matrix Qs'Qs has 136 upper 256 x 256 tiles): with the Gram on
    the MN-major CTA-pair kernel (the default), the same iteration count and Qbar as with the
    one-CTA kernel (ISVD_UMMA_PAIR_MN=0)."""
    torch = pytest.importorskip("torch")
    m, l, Nn = 6000, 128, 32
    g = torch.Generator(device="cuda").manual_seed(3)
    base = torch.linalg.qr(torch.randn(m, l, device="cuda", dtype=torch.float64, generator=g))[0]
    blocks = []
    for _ in range(Nn):  # perturbed copies of one subspace, re-orthonormalised
        blocks.append(torch.linalg.qr(base + 0.05 * torch.randn(m, l, device="cuda", dtype=torch.float64,
                                                                 generator=g))[0])
    qs = torch.cat(blocks, dim=1).float().contiguous()
    prm = lib.create_param(m, m, l, 0, Nn)

    def run():
        qt = torch.zeros((m, l), device="cuda")
        torch.cuda.synchronize()
        r = lib.integrate("s", "KN", prm, qs, l * Nn, qt, l, argv=[256, 1e-4])
        return int(r[0]), qt.double()

    monkeypatch.setenv("ISVD_UMMA_PAIR_MN", "1")
    it2, q2 = run()
    monkeypatch.setenv("ISVD_UMMA_PAIR_MN", "0")
    it1, q1 = run()
    assert it2 == it1
    assert (q2 - q1).abs().max().item() < 1e-5


def test_kn_update_planes_bitwise(lib, monkeypatch):
    """The next Bc's bf16 planes written by the [M | B] update's epilogue (the default when N l is a
    multiple of 64) give bitwise the iteration count and Qbar of the separate transposed split
    (ISVD_GPU_KN_UPDATE_PLANES=0)."""
    torch = pytest.importorskip("torch")
    m, l, Nn = 3000, 128, 16
    g = torch.Generator(device="cuda").manual_seed(5)
    base = torch.linalg.qr(torch.randn(m, l, device="cuda", dtype=torch.float64, generator=g))[0]
    qs = torch.cat([torch.linalg.qr(base + 0.05 * torch.randn(m, l, device="cuda", dtype=torch.float64,
                                                               generator=g))[0] for _ in range(Nn)], dim=1)
    qs = qs.float().contiguous()
    prm = lib.create_param(m, m, l, 0, Nn)

    def run():
        qt = torch.zeros((m, l), device="cuda", dtype=qs.dtype)
        torch.cuda.synchronize()
        r = lib.integrate("s", "KN", prm, qs, l * Nn, qt, l, argv=[256, 1e-4])
        return int(r[0]), qt.cpu().numpy()

    monkeypatch.setenv("ISVD_GPU_KN_UPDATE_PLANES", "1")
    it1, q1 = run()
    monkeypatch.setenv("ISVD_GPU_KN_UPDATE_PLANES", "0")
    it0, q0 = run()
    assert it1 == it0 and it1 > 3
    assert np.array_equal(q1, q0)


def test_mixed_sketch_internal_omega_matches_native(lib):
    """The internal Omega is drawn exactly in bf16, identical in both precision modes."""
    m, n, k, p, Nn = 700, 500, 20, 12, 4
    a = np.random.default_rng(3).standard_normal((m, n))
    prm = lib.create_param(m, n, k, p, Nn)
    y_mixed = np.zeros((m, (k + p) * Nn))
    lib.sketch("d", prm, a, n, y_mixed, (k + p) * Nn, seed=42)
    lib.lib.isvd_gpu_set_precision(0)
    y_native = np.zeros_like(y_mixed)
    lib.sketch("d", prm, a, n, y_native, (k + p) * Nn, seed=42)
    lib.lib.isvd_gpu_set_precision(1)
    assert np.abs(y_mixed - y_native).max() < 1e-5 * np.abs(y_native).max()


@pytest.mark.parametrize("x", ["s", "d"])
def test_mixed_orthogonalize_golden(lib, golden, oracle, x):
    dt = np.float32 if x == "s" else np.float64
    ys = golden["ys"]
    m = ys.shape[0]
    prm = lib.create_param(m, m, L, 0, N)
    y = np.ascontiguousarray(ys.astype(dt))
    lib.orthogonalize(x, "GR", prm, y, L * N)
    for i in range(N):
        blk = slice(i * L, (i + 1) * L)
        q = y[:, blk].astype(np.float64)
        assert oracle.projector_err(q, golden["qs"][:, blk]) < 1e-5
        assert np.abs(q.T @ q - np.eye(L)).max() < 1e-5


@pytest.mark.parametrize("l", [64, 128])
def test_mixed_orthogonalize_wide_blocks(lib, oracle, l):
    """Gramian orthogonalization with l a multiple of 64, where the N block applies Y_i Wp_i run as
    one tensor-core launch that loops over the blocks inside each CTA: the blocks agree with the
    FP64 orthogonalization of the same Y (projector distance) and are orthonormal."""
    m, Nn = 3000, 6
    rng = np.random.default_rng(l)
    y = rng.standard_normal((m, l * Nn)) @ np.diag(np.geomspace(1.0, 1e-2, l * Nn))
    y32 = np.ascontiguousarray(y.astype(np.float32))
    prm = lib.create_param(m, m, l, 0, Nn)
    lib.orthogonalize("s", "GR", prm, y32, l * Nn)
    lib.lib.isvd_gpu_set_precision(0)
    y64 = np.ascontiguousarray(y.astype(np.float32).astype(np.float64))
    lib.orthogonalize("d", "GR", prm, y64, l * Nn)
    lib.lib.isvd_gpu_set_precision(1)
    for i in range(Nn):
        blk = slice(i * l, (i + 1) * l)
        q = y32[:, blk].astype(np.float64)
        assert oracle.projector_err(q, y64[:, blk]) < 1e-4
        assert np.abs(q.T @ q - np.eye(l)).max() < 1e-5


@pytest.mark.parametrize("x", ["s", "d"])
def test_mixed_kn_golden(lib, golden, x):
    dt = np.float32 if x == "s" else np.float64
    qs = golden["qs"]
    m = qs.shape[0]
    prm = lib.create_param(m, m, L, 0, N)
    qt = np.zeros((m, L), dt)
    r = lib.integrate(x, "KN", prm, np.ascontiguousarray(qs.astype(dt)), L * N, qt, L, argv=[256, 1e-4])
    assert abs(int(r[0]) - 81) <= 2
    assert np.abs(qt - golden["q_kn"]).max() < 1e-3


@pytest.mark.parametrize("x", ["s", "d"])
@pytest.mark.parametrize("ordera", [b"R", b"C"])
def test_mixed_postprocess_golden(lib, golden, oracle, x, ordera):
    dt = np.float32 if x == "s" else np.float64
    a0 = golden["a"].astype(dt)
    m, n = a0.shape
    aa = np.ascontiguousarray(a0) if ordera == b"R" else np.asfortranarray(a0)
    lda = n if ordera == b"R" else m
    prm = lib.create_param(m, n, L, 0, 1)
    s = np.zeros(L, dt)
    ut = np.zeros((m, L), dt)
    vt = np.zeros((n, L), dt)
    lib.postprocess(x, "GR", prm, aa, lda, np.ascontiguousarray(golden["q"].astype(dt)), L, s, ut, L, vt, L,
                    ordera=ordera)
    s_ref = golden["s"][:, 0]
    assert np.abs(s - s_ref).max() < 1e-5 * s_ref.max()
    assert oracle.max_principal_angle(ut.astype(np.float64), golden["u"]) < 1e-4
    assert oracle.max_principal_angle(vt.astype(np.float64), golden["v"]) < 1e-4


@pytest.mark.parametrize("x", ["s", "d"])
def test_mixed_driver_vs_fp64(lib, oracle, x):
    """End to end: same A, same Omega; mixed vs the FP64 path."""
    m, n, k, p, Nn = 3000, 1500, 20, 12, 8
    l = k + p
    a = lowrank(m, n, 400, 10 ** (-3 / 400), 1e-6, 17)
    om = np.random.default_rng(9).standard_normal((n, l * Nn))
    dt = np.float32 if x == "s" else np.float64
    prm = lib.create_param(m, n, k, p, Nn)
    res = {}
    for prec in (0, 1):
        s = np.zeros(l, np.float64)
        ut = np.zeros((m, l))
        vt = np.zeros((n, l))
        if prec == 0:
            retv, _, st = lib.isvd("d", prm, ("GP", "GR", "KN", "GR"), np.ascontiguousarray(a), n, s, ut, l, vt, l,
                                   omega=np.ascontiguousarray(om), ldomega=l * Nn, precision=0)
        else:
            s = s.astype(dt); ut = ut.astype(dt); vt = vt.astype(dt)
            retv, _, st = lib.isvd(x, prm, ("GP", "GR", "KN", "GR"), np.ascontiguousarray(a.astype(dt)), n, s, ut,
                                   l, vt, l, omega=np.ascontiguousarray(om.astype(dt)), ldomega=l * Nn,
                                   precision=1)
        assert st == 0, lib.last_error()
        res[prec] = (s.astype(np.float64), ut.astype(np.float64), vt.astype(np.float64), int(retv[2][0]))
    s0, u0, v0, it0 = res[0]
    s1, u1, v1, it1 = res[1]
    assert np.abs(s1 - s0).max() / s0.max() < 1e-5
    assert oracle.max_principal_angle(u1[:, :k], u0[:, :k]) < 1e-4
    assert oracle.max_principal_angle(v1[:, :k], v0[:, :k]) < 1e-4


@pytest.mark.parametrize("integ", ["KN", "WY"])
@pytest.mark.parametrize("where", ["host", "device"])
def test_mixed_plane_handoff_bitwise(lib, monkeypatch, where, integ):
    """The MIXED driver hands Y (sketch -> Gramian orthogonalization) and Qs (-> integration) over
    as the bf16 planes the next stage would split them into: with the hand-off and without it
    (ISVD_GPU_PLANE_HANDOFF=0) the results are bitwise the same, with A on the device (one sketch
    launch) and in host memory (one launch per streamed panel)."""
    torch = pytest.importorskip("torch")
    m, n, k, p, Nn = 2000, 1200, 40, 24, 4  # l = 64, N l = 256
    l = k + p
    a = np.ascontiguousarray(lowrank(m, n, 300, 10 ** (-3 / 300), 1e-6, 31).astype(np.float32))
    aa = torch.from_numpy(a).cuda() if where == "device" else a
    if where == "host":
        monkeypatch.setenv("ISVD_GPU_PANEL_ROWS", "512")
    prm = lib.create_param(m, n, k, p, Nn)
    argv = [None, None, [256, 1e-4] if integ == "KN" else [256, 1e-3], None]
    out = []
    for off in ("1", "0"):
        monkeypatch.setenv("ISVD_GPU_PLANE_HANDOFF", off)
        s = np.zeros(l, np.float32); u = np.zeros((m, l), np.float32); v = np.zeros((n, l), np.float32)
        retv, _, st = lib.isvd("s", prm, ("GP", "GR", integ, "GR"), aa, n, s, u, l, v, l, seed=7, argv=argv,
                               retc=(0, 0, 2, 0), precision=1)
        assert st == 0, lib.last_error()
        out.append((s, u, v, int(retv[2][0])))
    (s1, u1, v1, i1), (s0, u0, v0, i0) = out
    assert i1 == i0
    assert np.array_equal(s1, s0) and np.array_equal(u1, u0) and np.array_equal(v1, v0)


@pytest.mark.parametrize("where", ["host", "device"])
def test_mixed_driver_wide_blocks(lib, oracle, where):
    """l = 64 (device A: one sketch launch; host A: one per streamed 512-row panel): the Gramian
    orthogonalization's block applies read only Y's planes and write Qs in place.  Against the
    FP64 path with the same Omega."""
    torch = pytest.importorskip("torch")
    m, n, k, p, Nn = 3000, 1500, 40, 24, 8
    l = k + p
    a = lowrank(m, n, 400, 10 ** (-3 / 400), 1e-6, 29)
    om = np.random.default_rng(5).standard_normal((n, l * Nn))
    prm = lib.create_param(m, n, k, p, Nn)
    s0 = np.zeros(l); u0 = np.zeros((m, l)); v0 = np.zeros((n, l))
    retv0, _, st = lib.isvd("d", prm, ("GP", "GR", "KN", "GR"), np.ascontiguousarray(a), n, s0, u0, l, v0, l,
                            omega=np.ascontiguousarray(om), ldomega=l * Nn, precision=0)
    assert st == 0, lib.last_error()
    a32 = np.ascontiguousarray(a.astype(np.float32))
    if where == "device":
        a32 = torch.from_numpy(a32).cuda()
    else:
        os.environ["ISVD_GPU_PANEL_ROWS"] = "512"
    try:
        s1 = np.zeros(l, np.float32); u1 = np.zeros((m, l), np.float32); v1 = np.zeros((n, l), np.float32)
        retv1, _, st = lib.isvd("s", prm, ("GP", "GR", "KN", "GR"), a32, n, s1, u1, l, v1, l,
                                omega=np.ascontiguousarray(om.astype(np.float32)), ldomega=l * Nn, precision=1)
    finally:
        os.environ.pop("ISVD_GPU_PANEL_ROWS", None)
    assert st == 0, lib.last_error()
    assert abs(int(retv1[2][0]) - int(retv0[2][0])) <= 1
    assert np.abs(s1 - s0).max() / s0.max() < 1e-5
    assert oracle.max_principal_angle(u1[:, :k].astype(np.float64), u0[:, :k]) < 1e-4
    assert oracle.max_principal_angle(v1[:, :k].astype(np.float64), v0[:, :k]) < 1e-4


@pytest.mark.parametrize("ordera", [b"R", b"C"])
@pytest.mark.parametrize("where", ["host", "device"])
def test_mixed_streamed_panels(lib, oracle, ordera, where, monkeypatch):
    """A in many row panels (panel size forced to 256 rows): host A streams through the copy stream;
    the result equals the single-panel device result."""
    torch = pytest.importorskip("torch")
    m, n, k, p, Nn = 3000, 1500, 12, 8, 6
    l = k + p
    a = lowrank(m, n, 300, 0.98, 1e-6, 23)
    om = np.random.default_rng(4).standard_normal((n, l * Nn))
    aa = np.ascontiguousarray(a) if ordera == b"R" else np.asfortranarray(a)
    lda = n if ordera == b"R" else m
    prm = lib.create_param(m, n, k, p, Nn)

    def run(arr):
        s = np.zeros(l)
        ut = np.zeros((m, l))
        vt = np.zeros((n, l))
        retv, _, st = lib.isvd("d", prm, ("GP", "GR", "KN", "GR"), arr, lda, s, ut, l, vt, l, ordera=ordera,
                               omega=np.ascontiguousarray(om), ldomega=l * Nn, precision=1)
        assert st == 0, lib.last_error()
        return s, ut, vt, int(retv[2][0])

    ref = run(aa)
    monkeypatch.setenv("ISVD_GPU_PANEL_ROWS", "256")
    if where == "host":
        got = run(aa)
    else:
        ad = torch.from_numpy(np.ascontiguousarray(aa.T) if ordera == b"C" else aa).cuda()
        got = run(ad)
    assert got[3] == ref[3]
    assert np.abs(got[0] - ref[0]).max() < 1e-6 * ref[0].max()
    assert oracle.max_principal_angle(got[1][:, :k], ref[1][:, :k]) < 1e-5
