"""Truncated-SVD adjoint (isvd_?SvdAdjoint): against the FP64 dense-SVD gradient (torch autograd
through torch.linalg.svd), central finite differences (h = 1e-3, FP64) on a 512 x 256 slice, and,
wrapped in a torch.autograd.Function over the iSVD forward, end to end.

The loss is the one of the differentiated-solve workload: L = sum_i w_i s_i + ||U U' X||_F^2, whose
cotangents are ds = w, dU = 2 X X' U, dV = 0."""
import ctypes

import numpy as np
import pytest

from isvd_b200.capi import c_int_t, ptr

pytestmark = pytest.mark.gpu


def _adjoint_fn(lib, x):
    fn = getattr(lib.lib, "isvd_%sSvdAdjoint" % x)
    vp = ctypes.c_void_p
    fn.argtypes = [c_int_t, c_int_t, c_int_t, ctypes.c_char, vp, c_int_t, vp, vp, c_int_t, vp, c_int_t, vp, vp,
                   c_int_t, vp, c_int_t, vp, c_int_t, ctypes.c_int, ctypes.c_double, ctypes.POINTER(ctypes.c_int)]
    fn.restype = ctypes.c_int
    return fn


def adjoint(lib, a, s, u, v, ds=None, du=None, dv=None, cg_iters=500, tol=1e-13, x="d", ordera=b"R"):
    """dA through the C ABI; arrays may be numpy (host) or CUDA tensors."""
    m, k = u.shape[0], u.shape[1]
    n = v.shape[0]
    if hasattr(a, "data_ptr"):
        import torch
        da = torch.zeros_like(a)
    else:
        da = np.zeros_like(a)
    lda = n if ordera == b"R" else m
    its = ctypes.c_int(0)
    if hasattr(a, "data_ptr"):  # the operands were produced on torch's stream; the library uses its own
        import torch
        torch.cuda.synchronize()
    st = _adjoint_fn(lib, x)(m, n, k, ordera, ptr(a), lda, ptr(s), ptr(u), k, ptr(v), k, ptr(ds), ptr(du), k, ptr(dv),
                             k, ptr(da), lda, cg_iters, tol, ctypes.byref(its))
    assert st == 0, lib.last_error()
    return da, its.value


def spectrum_matrix(m, n, sig, seed):
    rng = np.random.default_rng(seed)
    uu = np.linalg.qr(rng.standard_normal((m, len(sig))))[0]
    vv = np.linalg.qr(rng.standard_normal((n, len(sig))))[0]
    return (uu * sig) @ vv.T


def loss_parts(a, k, w, xx):
    u, s, vt = np.linalg.svd(a, full_matrices=False)
    u, s, v = u[:, :k], s[:k], vt[:k].T
    L = float(w @ s + np.sum((u @ (u.T @ xx)) ** 2))
    return L, u, s, v


def dense_grad(a, k, w, xx):
    torch = pytest.importorskip("torch")
    at = torch.tensor(a, dtype=torch.float64, requires_grad=True)
    uu, ss, _ = torch.linalg.svd(at, full_matrices=False)
    L = (torch.tensor(w) * ss[:k]).sum() + ((uu[:, :k] @ (uu[:, :k].T @ torch.tensor(xx))) ** 2).sum()
    L.backward()
    return at.grad.numpy()


def slice_case(seed=5):
    """A 512 x 256 slice of a rank-512-plus-noise matrix (the differentiated-solve construction)."""
    m, n, k = 512, 256, 16
    rng = np.random.default_rng(seed)
    sig = np.geomspace(1.0, 1e-2, 256) * (1.0 + 0.05 * rng.standard_normal(256) ** 2)
    a = spectrum_matrix(m, n, np.sort(sig)[::-1], seed) + 1e-4 * rng.standard_normal((m, n))
    w = rng.standard_normal(k)
    xx = rng.standard_normal((m, 32))
    return a, k, w, xx


@pytest.mark.parametrize("ordera", [b"R", b"C"])
def test_adjoint_matches_dense_svd_gradient(lib, ordera):
    a, k, w, xx = slice_case()
    L, u, s, v = loss_parts(a, k, w, xx)
    g = dense_grad(a, k, w, xx)
    du = 2.0 * xx @ (xx.T @ u)
    aa = np.ascontiguousarray(a) if ordera == b"R" else np.asfortranarray(a)
    da, its = adjoint(lib, aa, np.ascontiguousarray(s), np.ascontiguousarray(u), np.ascontiguousarray(v),
                      ds=np.ascontiguousarray(w), du=np.ascontiguousarray(du), ordera=ordera)
    assert its > 0
    assert np.abs(da - g).max() < 1e-8 * np.abs(g).max()


@pytest.mark.parametrize("ordera", [b"R", b"C"])
@pytest.mark.parametrize("precision,operator", [(0, "a"), (1, "gram"), (1, "a")],
                         ids=["native", "mixed-gram", "mixed-in-a"])
def test_adjoint_fp32_u_and_v_terms(lib, monkeypatch, ordera, precision, operator):
    """FP32 adjoint with both complement systems (dU and dV), A row- and column-major, NATIVE and
    MIXED (products on the tensor cores), against the FP64 dense gradient of
    L = w's + ||U U' X||_F^2 + ||V V' Y||_F^2.  MIXED runs the complement systems in the
    coordinates of B'B (the default for n <= m) and, with ISVD_GPU_ADJOINT_CG_A=1, with the
    operator in A (both systems in one pass over A per product)."""
    torch = pytest.importorskip("torch")
    if operator == "a":
        monkeypatch.setenv("ISVD_GPU_ADJOINT_CG_A", "1")
    a, k, w, xx = slice_case(11)
    yy = np.random.default_rng(12).standard_normal((a.shape[1], 8))
    at = torch.tensor(a, dtype=torch.float64, requires_grad=True)
    uu, ss, vh = torch.linalg.svd(at, full_matrices=False)
    uk, vk = uu[:, :k], vh[:k].T
    L = (torch.tensor(w) * ss[:k]).sum() + ((uk @ (uk.T @ torch.tensor(xx))) ** 2).sum() + \
        ((vk @ (vk.T @ torch.tensor(yy))) ** 2).sum()
    L.backward()
    g = at.grad.numpy()
    _, u, s, v = loss_parts(a, k, w, xx)
    du = 2.0 * xx @ (xx.T @ u)
    dv = 2.0 * yy @ (yy.T @ v)
    f32 = lambda x_: np.ascontiguousarray(x_, dtype=np.float32)  # noqa: E731
    aa = f32(a) if ordera == b"R" else np.asfortranarray(a, dtype=np.float32)
    lib.lib.isvd_gpu_set_precision(precision)
    try:
        da, its = adjoint(lib, aa, f32(s), f32(u), f32(v), ds=f32(w), du=f32(du), dv=f32(dv), cg_iters=300,
                          tol=1e-6, x="s", ordera=ordera)
    finally:
        lib.lib.isvd_gpu_set_precision(0)
    assert its > 0
    assert np.abs(da.astype(np.float64) - g).max() < 1e-3 * np.abs(g).max()


def test_adjoint_finite_differences(lib):
    """Central differences, h = 1e-3 in FP64, along random directions of the 512 x 256 slice."""
    a, k, w, xx = slice_case(7)
    L, u, s, v = loss_parts(a, k, w, xx)
    du = 2.0 * xx @ (xx.T @ u)
    da, _ = adjoint(lib, np.ascontiguousarray(a), s, np.ascontiguousarray(u), np.ascontiguousarray(v), ds=w,
                    du=np.ascontiguousarray(du))
    rng = np.random.default_rng(1)
    h = 1e-3
    for _ in range(3):
        e = rng.standard_normal(a.shape)
        e /= np.linalg.norm(e)
        fd = (loss_parts(a + h * e, k, w, xx)[0] - loss_parts(a - h * e, k, w, xx)[0]) / (2 * h)
        an = float(np.sum(da * e))
        assert abs(fd - an) < 1e-5 * max(1.0, abs(an))


def test_adjoint_rank_k_formula(lib):
    """cg_iters = 0 is exact when rank(A) = k: it agrees with the full solve and with the formula."""
    rng = np.random.default_rng(3)
    m, n, k = 300, 200, 10
    a = spectrum_matrix(m, n, np.geomspace(2.0, 0.3, k), 3)
    L, u, s, v = loss_parts(a, k, np.ones(k), rng.standard_normal((m, 4)))
    du, dv, ds = rng.standard_normal((m, k)), rng.standard_normal((n, k)), rng.standard_normal(k)
    args = (np.ascontiguousarray(a), s, np.ascontiguousarray(u), np.ascontiguousarray(v))
    d0, its0 = adjoint(lib, *args, ds=ds, du=du, dv=dv, cg_iters=0)
    d1, _ = adjoint(lib, *args, ds=ds, du=du, dv=dv, cg_iters=200)
    assert its0 == 0
    assert np.abs(d0 - d1).max() < 1e-9 * np.abs(d1).max()
    f = np.zeros((k, k))
    for i in range(k):
        for j in range(k):
            if i != j:
                f[i, j] = 1.0 / (s[j] ** 2 - s[i] ** 2)
    k1, k2 = u.T @ du, v.T @ dv
    jm = np.diag(ds) + (f * (k1 - k1.T)) * s[None, :] + s[:, None] * (f * (k2 - k2.T))
    ref = u @ jm @ v.T + (du - u @ k1) / s @ v.T + u @ ((dv - v @ k2) / s).T
    assert np.abs(d0 - ref).max() < 1e-10 * np.abs(ref).max()


def test_autograd_function_end_to_end(lib):
    """torch.autograd.Function over the iSVD forward (FP64) and the adjoint backward, against the
    dense-SVD gradient.  The k leading singular values lie in [0.3, 1] and the rest below 1e-5, so
    the sketch captures the k leading triplets to about sigma_(l+1) / sigma_k ~ 3e-5: the gradients
    agree to that accuracy.  (A tail far below the FP64 resolution of the sketch Gram matrices,
    e.g. rank k plus 1e-10 noise, makes the Gramian orthogonalization divide by singular values
    that are pure rounding, in the reference as here.)"""
    torch = pytest.importorskip("torch")
    m, n, k, p, N = 512, 256, 12, 4, 8
    l = k + p
    rng = np.random.default_rng(11)
    a = spectrum_matrix(m, n, np.concatenate([np.geomspace(1.0, 0.3, k), np.geomspace(1e-5, 1e-7, 100)]), 11)
    a += 1e-9 * rng.standard_normal((m, n))  # distinct small singular values for the dense gradient
    w = rng.standard_normal(k)
    xx = rng.standard_normal((m, 8))
    dev = torch.device("cuda:0")
    om = torch.tensor(rng.standard_normal((n, l * N)), device=dev)

    class TruncatedSvd(torch.autograd.Function):
        @staticmethod
        def forward(ctx, at):
            prm = lib.create_param(m, n, k, p, N)
            s = torch.zeros(l, dtype=torch.float64, device=dev)
            ut = torch.zeros((m, l), dtype=torch.float64, device=dev)
            vt = torch.zeros((n, l), dtype=torch.float64, device=dev)
            torch.cuda.synchronize()
            _, _, st = lib.isvd("d", prm, ("GP", "GR", "KN", "GR"), at.contiguous(), n, s, ut, l, vt, l,
                                argv=[None, None, [256, 1e-4], None], omega=om, ldomega=l * N, precision=0)
            assert st == 0, lib.last_error()
            u, ss, v = ut[:, :k].contiguous(), s[:k].contiguous(), vt[:, :k].contiguous()
            ctx.save_for_backward(at, u, ss, v)
            return u, ss, v

        @staticmethod
        def backward(ctx, gu, gs, gv):
            at, u, ss, v = ctx.saved_tensors
            torch.cuda.synchronize()
            da, _ = adjoint(lib, at.contiguous(), ss, u, v, ds=gs.contiguous(), du=gu.contiguous(),
                            dv=gv.contiguous())
            return da

    at = torch.tensor(a, device=dev, requires_grad=True)
    u, s, v = TruncatedSvd.apply(at)
    L = (torch.tensor(w, device=dev) * s).sum() + ((u @ (u.T @ torch.tensor(xx, device=dev))) ** 2).sum()
    L.backward()
    g = dense_grad(a, k, w, xx)
    got = at.grad.cpu().numpy()
    assert np.abs(got - g).max() < 5e-4 * np.abs(g).max()


@pytest.mark.parametrize("precision", [0, 1], ids=["native", "mixed"])
def test_adjoint_differentiated_solve_fp32(lib, precision):
    """The differentiated-solve shape: A 16384 x 4096 FP32, rank 512 plus noise, k = 64, X 16384 x 32.
    The FP32 adjoint (device buffers) from the FP64 dense factors, against the FP64 dense gradient;
    NATIVE (CUDA-core FP32 products) and MIXED (products by A on the tensor cores)."""
    torch = pytest.importorskip("torch")
    dev = torch.device("cuda:0")
    m, n, k, r = 16384, 4096, 64, 512
    g = torch.Generator(device=dev).manual_seed(5)
    uu = torch.linalg.qr(torch.randn(m, r, device=dev, dtype=torch.float64, generator=g))[0]
    vv = torch.linalg.qr(torch.randn(n, r, device=dev, dtype=torch.float64, generator=g))[0]
    sig = torch.logspace(0, -2, r, device=dev, dtype=torch.float64)
    a = (uu * sig) @ vv.T + 1e-4 * torch.randn(m, n, device=dev, dtype=torch.float64, generator=g)
    w = torch.randn(k, device=dev, dtype=torch.float64, generator=g)
    xx = torch.randn(m, 32, device=dev, dtype=torch.float64, generator=g)
    at = a.clone().requires_grad_(True)
    U, S, Vh = torch.linalg.svd(at, full_matrices=False)
    L = (w * S[:k]).sum() + ((U[:, :k] @ (U[:, :k].T @ xx)) ** 2).sum()
    L.backward()
    gref = at.grad
    u, s, v = U[:, :k].detach(), S[:k].detach(), Vh[:k].T.detach()
    du = 2.0 * xx @ (xx.T @ u)
    f32 = lambda t: t.to(torch.float32).contiguous()
    lib.lib.isvd_gpu_set_precision(precision)
    try:
        da, its = adjoint(lib, f32(a), f32(s), f32(u), f32(v), ds=f32(w), du=f32(du), cg_iters=300, tol=1e-6, x="s")
    finally:
        lib.lib.isvd_gpu_set_precision(0)
    assert its > 0
    err = (da.double() - gref).abs().max().item() / gref.abs().max().item()
    assert err < 1e-3
