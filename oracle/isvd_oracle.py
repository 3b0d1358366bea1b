"""NumPy restatement of the iSVD stage algorithms (emfomy/isvd v1.3.2), one MPI rank.

TEST INFRASTRUCTURE ONLY -- this module is the checker.  Only ``tests/``,
``__graft_entry__.smoke()`` and ``bench.py`` (its CPU-baseline / reference arm)
import it.  The product library never calls it.

Every function restates the reference stage at one MPI rank (P = 1), in float64,
on natural-orientation matrices: A is m x n, Y/Qs are m x (N*l), Qbar is m x l,
Z is n x l.  The reference stores those same matrices row-major ("yst", "qt").
Each function cites the reference lines it follows.  LAPACK kernels are replaced
by their NumPy equivalents; where LAPACK's sign/ordering conventions are not
reproducible (gesvd/gelqf column signs) the result is equal up to a right
factor diag(+-1), which the stages downstream are invariant to, and the tests
compare sign-invariant quantities (projectors, singular values) there.

Parity of this restatement is pinned by tests/test_oracle.py against
  * the reference's golden fixtures (tests/golden/isvd_golden.npz, from data/*.mtx),
  * the reference library itself built from source (oracle/_ref, build_ref.py).
"""
import numpy as np

KN_DEFAULTS = dict(maxit=256, tol=1e-4)            # core/stage/@x@_integrate_kolmogorov_nagumo.c:16-17
WY_DEFAULTS = dict(maxit=256, tol=1e-3, tau0=1.0, taumax=1e14, taumin=1e-14, taumaxit=20,
                   beta=0.5, sigma=1e-4, eta=0.85)  # core/stage/@x@_integrate_wen_yin.c:16-24


def sketch_gaussian_projection(a, omega):
    """Y = A * Omega for all N sketches in one product.

    core/stage/@x@_sketch.h:136-139 (row block: Y' := Omega' * A').  ``omega`` is
    n x Nl; the reference draws it as r[j*Nl + c] = Omega(j, c)
    (la/vsl/@x@_rng_gaussian_driver.c:16-41)."""
    return np.asarray(a, np.float64) @ np.asarray(omega, np.float64)


def orthogonalize_gramian(y, l, N):
    """Gramian orthogonalization, core/stage/@x@_orthogonalize_gramian.c:80-98.

    W_i = Y_i' Y_i (:82-84); gesvd('O') gives W_i's singular vectors and values
    (:88-90); S = sqrt(s) (:91); Q_i = Y_i W_i S^-1 (:94-98)."""
    y = np.asarray(y, np.float64)
    q = np.empty_like(y)
    for i in range(N):
        yi = y[:, i * l:(i + 1) * l]
        w = yi.T @ yi
        u, s, _ = np.linalg.svd(w)
        q[:, i * l:(i + 1) * l] = yi @ (u / np.sqrt(s))
    return q


def orthogonalize_tall_skinny_qr(y, l, N):
    """TSQR orthogonalization at P = 1, core/stage/@x@_orthogonalize_tall_skinny_qr.c:123-143:
    LQ of Y_i' (gelqf) then orglq, i.e. the orthonormal factor of a thin QR of Y_i."""
    y = np.asarray(y, np.float64)
    q = np.empty_like(y)
    for i in range(N):
        q[:, i * l:(i + 1) * l] = np.linalg.qr(y[:, i * l:(i + 1) * l])[0]
    return q


def _sym_upper(x):
    return np.triu(x) + np.triu(x, 1).T


def _local(x):
    return x


def integrate_kolmogorov_nagumo(qs, l, N, maxit=256, tol=1e-4, trace=None, allreduce=None):
    """Kolmogorov-Nagumo integration, core/stage/@x@_integrate_kolmogorov_nagumo.c:153-266.

    Returns (Qbar, iterations, error) with the reference's retv conventions:
    iterations = maxit + 1 when maxit is hit (:238-241).  With ``allreduce`` (an in-place sum over
    the ranks of a float64 array) ``qs`` holds this rank's rows and Bc, Bgc are summed where the
    reference calls MPI_Allreduce (:160, :178)."""
    ar = allreduce or _local
    qs = np.asarray(qs, np.float64)
    qc = qs[:, :l].copy()                                     # :154
    bc = ar(qs.T @ qc)                                        # :157-160
    it = 1
    err = -np.inf
    while True:
        gc = qs @ bc / N                                      # :174
        bgc = ar(qs.T @ gc)                                   # :177-178
        dc = bc.T @ bc / N                                    # :181
        z = bc.T @ bgc / N                                    # :184 (upper used)
        z = _sym_upper(z - dc @ dc)                           # :190 syrk 'U'
        lam, vec = np.linalg.eigh(z, UPLO="U")                # :193
        s = np.sqrt(0.5 + np.sqrt(0.25 - lam))                # :196-198
        ss = np.sqrt(s)                                       # :199
        c = (vec * ss) @ (vec * ss).T                         # :202-209
        cinv = (vec / ss) @ (vec / ss).T                      # :205-212
        fc = c - dc @ cinv                                    # :218
        qp = qc @ fc + gc @ cinv                              # :221-222
        bp = bc @ fc + bgc @ cinv                             # :225-226
        err = float(np.linalg.norm(s - 1.0))                  # :230-234
        if trace is not None:
            trace.append(dict(iter=it, err=err, lam_max=float(lam.max()), lam_min=float(lam.min())))
        if err <= tol:
            break
        if it == maxit:
            it += 1
            break
        qc, bc = qp, bp                                       # :244-245
        it += 1
    return qp, it, err


def integrate_wen_yin(qs, l, N, maxit=256, tol=1e-3, tau0=1.0, taumax=1e14, taumin=1e-14, taumaxit=20,
                      beta=0.5, sigma=1e-4, eta=0.85, allreduce=None):
    """Wen-Yin integration, core/stage/@x@_integrate_wen_yin.c:197-360.

    Returns (Qbar, iterations, mu).  The 2l x 2l inverse of the line-search
    matrix C (:262) is taken with numpy.linalg.inv (LU with partial pivoting,
    the same factorization as the reference's getrf+getri).  With ``allreduce`` ``qs`` holds this
    rank's rows and Bc, Bgc and the two step-size sums are summed over the ranks where the
    reference calls MPI_Allreduce (:206, :216, :303, :345)."""
    ar = allreduce or _local
    qs = np.asarray(qs, np.float64)
    I = np.eye(l)
    qc = qs[:, :l].copy()                                     # :200
    bc = ar(qs.T @ qc)                                        # :203-206
    dc = bc.T @ bc / N                                        # :209
    gc = qs @ bc / N                                          # :212
    bgc = ar(qs.T @ gc)                                       # :215-216
    dgc = bc.T @ bgc / N                                      # :219
    xc = gc - qc @ dc                                         # :222-223
    mu = np.trace(dgc) - np.sum(dc * dc)                      # :226
    taug, zeta, phi = tau0, 1.0, 0.5 / N * np.sum(bc * bc)    # :229-231
    it = 1
    while True:
        tau, phit = taug, phi
        fc = fgc = bp = None
        for _ in range(int(taumaxit)):                        # :243
            cm = np.zeros((2 * l, 2 * l))
            cm[:l, :l] = 0.5 * dc - I / tau
            cm[l:, :l] = -0.5 * dgc
            cm[:l, l:] = 0.5 * I
            cm[l:, l:] = -0.5 * dc - I / tau
            ci = np.linalg.inv(cm)                            # :262
            cs1, cs2 = ci[:, :l], ci[:, l:]
            f = cs2 @ dc - cs1                                # :266
            fgc, fc = f[:l, :].copy(), f[l:, :] + I           # :267-269
            bp = bc @ fc + bgc @ fgc                          # :272-273
            phit = 0.5 / N * np.sum(bp * bp)                  # :276
            if phit >= phi + tau * sigma * mu:                # :279
                break
            tau *= beta
        phi = (eta * zeta * phi + phit) / (eta * zeta + 1)    # :288
        zeta = eta * zeta + 1                                 # :289
        qp = qc @ fc + gc @ fgc                               # :292-293
        dc = bp.T @ bp / N                                    # :296
        gc = qs @ bp / N                                      # :299
        bgc = ar(qs.T @ gc)                                   # :302-303
        dgc = bp.T @ bgc / N                                  # :306
        mu = np.trace(dgc) - np.sum(dc * dc)                  # :309
        if mu < tol * tol:                                    # :314
            break
        if it == maxit:
            it += 1
            break
        xp = gc - qp @ dc                                     # :327-328
        d1, d2 = qc - qp, xc - xp                             # :331-332
        if it % 2:
            t = np.array([np.sum(d1 * d1), np.sum(d1 * d2)])  # :336-338
        else:
            t = np.array([np.sum(d2 * d1), np.sum(d2 * d2)])  # :339-341
        t0, t1 = ar(t)                                        # :345
        taug = min(max(abs(t0 / t1), taumin), taumax)         # :347-349
        qc, xc, bc = qp, xp, bp                               # :352-354
        it += 1
    return qp, it, float(mu)


def integrate_hierarchical_reduction(qs, l, N, allreduce=None):
    """Hierarchical reduction, core/stage/@x@_integrate_hierarchical_reduction.c:90-130.

    Q(i) := (Q(i) W + Q(i+h) T) / sqrt(2 (1 + s)) with B(i) = Q(i)' Q(i+h) = W S T'; with row
    blocks the h products B(i) of a level are summed over the ranks in one reduction (:100).
    Works on a copy; the reference overwrites yst (the returned ``qs_out``)."""
    red = allreduce or _local
    q = np.array(qs, np.float64)
    h2 = N
    while h2 > 1:
        h = h2 // 2
        bs = red(np.stack([q[:, i * l:(i + 1) * l].T @ q[:, (i + h) * l:(i + h + 1) * l] for i in range(h)]))
        for i in range(h):
            qi, qih = q[:, i * l:(i + 1) * l], q[:, (i + h) * l:(i + h + 1) * l]
            w, s, tt = np.linalg.svd(bs[i])
            q[:, i * l:(i + 1) * l] = (qi @ w + qih @ tt.T) / np.sqrt(2.0 * (1.0 + s))
        h2 = (h2 + 1) // 2
    return q[:, :l].copy(), q


def postprocess_gramian(a, qbar, k):
    """Gramian postprocessing, core/stage/@x@_postprocess_gramian.c:139-176 with
    projectBlockRow/Col (core/stage/@x@_postprocess.h): Z = A' Qbar; W = Z' Z;
    gesvd('O'); sigma = sqrt(s) (length l); U = Qbar W[:, :k]; V = Z W[:, :k] / sigma."""
    a = np.asarray(a, np.float64)
    z = a.T @ qbar
    w, s, _ = np.linalg.svd(z.T @ z)
    sig = np.sqrt(s)
    return sig, qbar @ w[:, :k], (z @ w[:, :k]) / sig[:k]


def postprocess_tall_skinny_qr(a, qbar, k):
    """TSQR postprocessing at P = 1, core/stage/@x@_postprocess_tall_skinny_qr.c:195-294.

    Z' = L Qlq (gelqf, :199); svd(L) = U_L S V_L' with U_L in ``tt`` and V_L' over
    ``wt`` (:259-266).  The reference then forms U = Qbar * wt[0:k, :]' = Qbar V_L[:, :k]
    (:270) and V = (tt * Qlq)' = Qlq' U_L' for all l columns (:286), i.e. it pairs the
    singular vectors of L' rather than L.  With k = l (the upstream test) both
    pairings span the same subspaces; this restatement reproduces the reference's
    output, including that pairing.  Here L = r' from numpy's LAPACK QR of Z (the
    same Householder sign convention as gelqf of Z').  V mixes the rows of U_L, so
    its columns depend on the sign convention of the small SVD; only span(V) (all
    l columns) and U up to column signs are convention-free.  Returns (s, U, V)
    with U m x k and V n x l."""
    a = np.asarray(a, np.float64)
    z = a.T @ qbar
    qz, r = np.linalg.qr(z)            # Z = qz r  =>  Z' = r' qz' : L = r', Qlq = qz'
    uu, s, vvt = np.linalg.svd(r.T)    # L = U_L diag(s) V_L'
    return s, qbar @ vvt.T[:, :k], qz @ uu.T


def postprocess_symmetric(a, qbar, k):
    """Symmetric postprocessing, core/stage/@x@_postprocess_symmetric.c:139-157:
    W = Z' Qbar = Qbar' A Qbar; syev (ascending eigenvalues, length l); U = Qbar W[:, :k]."""
    a = np.asarray(a, np.float64)
    z = a.T @ qbar
    lam, w = np.linalg.eigh(_sym_upper(z.T @ qbar))
    return lam, qbar @ w[:, :k]


def isvd(a, omega, k, p, N, alg_o="GR", alg_i="KN", alg_p="GR", argv_i=None):
    """The four-stage driver (core/driver/@x@_isvd.c:243-265) with Omega passed in."""
    l = k + p
    y = sketch_gaussian_projection(a, omega)
    q = orthogonalize_gramian(y, l, N) if alg_o == "GR" else orthogonalize_tall_skinny_qr(y, l, N)
    argv_i = argv_i or {}
    if alg_i == "KN":
        qbar, it, err = integrate_kolmogorov_nagumo(q, l, N, **argv_i)
    elif alg_i == "WY":
        qbar, it, err = integrate_wen_yin(q, l, N, **argv_i)
    else:
        qbar, it, err = integrate_hierarchical_reduction(q, l, N)[0], 0, 0.0
    if alg_p == "GR":
        s, u, v = postprocess_gramian(a, qbar, k)
    elif alg_p == "TS":
        s, u, v = postprocess_tall_skinny_qr(a, qbar, k)
    else:
        s, u = postprocess_symmetric(a, qbar, k)
        v = u
    return dict(s=s, u=u, v=v, qbar=qbar, iters=it, err=err)


def row_block(m, P, rank):
    """Rows [begin, end) of rank `rank` of P, core/param.c:47-55 (ceil(m / P) rows each)."""
    each = (m - 1) // P + 1
    return min(rank * each, m), min(rank * each + each, m)


def _distributed(y, project, k, p, N, allreduce, alg_i, argv_i, alg_p, row_begin):
    """Orthogonalization, integration and postprocessing on this rank's rows y of Y, every sum over
    the ranks through ``allreduce``; ``project(qbar_rows)`` returns the whole Z = A' Qbar."""
    l = k + p
    q = np.empty_like(y)
    for i in range(N):
        yi = y[:, i * l:(i + 1) * l]
        w = allreduce(yi.T @ yi)
        u, s, _ = np.linalg.svd(w)
        q[:, i * l:(i + 1) * l] = yi @ (u / np.sqrt(s))
    argv_i = dict(argv_i or {})
    if alg_i == "KN":
        qp, it, err = integrate_kolmogorov_nagumo(q, l, N, allreduce=allreduce, **argv_i)
    elif alg_i == "WY":
        qp, it, err = integrate_wen_yin(q, l, N, allreduce=allreduce, **argv_i)
    else:
        qp, it, err = integrate_hierarchical_reduction(q, l, N, allreduce=allreduce)[0], 0, 0.0
    z = project(qp)
    if alg_p == "TS":
        qz, r = np.linalg.qr(z)
        uu, s, vvt = np.linalg.svd(r.T)
        return s, qp @ vvt.T[:, :k], qz @ uu.T, it, err
    if alg_p == "SY":
        w = allreduce(z[row_begin:row_begin + qp.shape[0]].T @ qp)
        lam, ev = np.linalg.eigh(_sym_upper(w))
        return lam, qp @ ev[:, :k], None, it, err
    w, s, _ = np.linalg.svd(z.T @ z)
    sig = np.sqrt(s)
    return sig, qp @ w[:, :k], (z @ w[:, :k]) / sig[:k], it, err


def isvd_row_block(a_rows, omega, k, p, N, allreduce, alg_i="KN", argv_i=None, alg_p="GR", row_begin=0):
    """The Gramian / KN, WY or HR / GR, TS or SY driver on one rank's rows [row_begin, ...) of a
    row-distributed A (dista 'R'), with every reduction over the ranks done by ``allreduce(x)`` (an
    in-place sum of a float64 array, the reference's MPI_Allreduce with MPI_SUM):
      * orthogonalization W_i = sum_ranks Y_i' Y_i, core/stage/@x@_orthogonalize_gramian.c:82-85;
      * integration as the reference's integrate stages with ``allreduce`` (Bc, Bgc and, for WY,
        the step-size sums; for HR the products B(i) of each level);
      * postprocessing Z = A' Qbar (projectBlockRow, core/stage/@x@_postprocess.h:96-162, whose
        MPI_Reduce_scatter_block leaves each rank its column block of the sum; here every rank keeps
        the whole sum), then GR: W = Z' Z (core/stage/@x@_postprocess_gramian.c:145-146); TS: the
        QR factorization of the whole Z on every rank (the reference's TSQR tree over the ranks,
        @x@_postprocess_tall_skinny_qr.c:199-241, factors the same Z); SY: W = sum_ranks of
        Z(own rows)' Qbar_j (@x@_postprocess_symmetric.c:146-147).
    Returns (s, U rows of this rank, V (all n rows; SY: None), iterations, error or mu)."""
    a_rows = np.asarray(a_rows, np.float64)
    y = a_rows @ np.asarray(omega, np.float64)
    return _distributed(y, lambda qp: allreduce(a_rows.T @ qp), k, p, N, allreduce, alg_i, argv_i, alg_p,
                        row_begin)


def isvd_col_block(a_cols, omega, k, p, N, allreduce, rows, cols, alg_i="KN", argv_i=None, alg_p="GR"):
    """The same driver on one rank's columns ``cols`` (a slice) of a column-distributed A (dista
    'C'; a_cols holds all m rows of them), with Omega's rows of those columns:
      * sketch Y = sum_ranks A_j Omega_j, each rank keeping its row block ``rows``
        (sketchBlockCol, core/stage/@x@_sketch.h:21-90: MPI_Reduce_scatter_block at :82);
      * orthogonalization and integration on the row blocks, as isvd_row_block;
      * projection: Qbar gathered (MPI_Allgather, core/stage/@x@_postprocess.h:78), Z_j = A_j' Qbar
        for the rank's columns, Z gathered (here both gathers are sums of zero-padded copies)."""
    a_cols = np.asarray(a_cols, np.float64)
    omega = np.asarray(omega, np.float64)
    m, n, l = a_cols.shape[0], omega.shape[0], k + p
    y = allreduce(a_cols @ omega[cols])[rows]

    def project(qp):
        qf = np.zeros((m, l))
        qf[rows] = qp
        qf = allreduce(qf)
        z = np.zeros((n, l))
        z[cols] = a_cols.T @ qf
        return allreduce(z)
    return _distributed(y, project, k, p, N, allreduce, alg_i, argv_i, alg_p, rows.start)


# ---------------------------------------------------------------------------------------------
# Comparison helpers (sign- and rotation-invariant)

def projector_err(x, y):
    """max |X X' - Y Y'| for matrices with orthonormal columns."""
    return float(np.max(np.abs(x @ x.T - y @ y.T)))


def max_principal_angle(x, y):
    """Largest principal angle (radians) between span(X) and span(Y), via the sine formula
    ||(I - Qx Qx') Qy||_2 (accurate for small angles)."""
    qx = np.linalg.qr(x)[0]
    qy = np.linalg.qr(y)[0]
    r = qy - qx @ (qx.T @ qy)
    return float(np.arcsin(min(1.0, np.linalg.norm(r, 2))))


def column_angles(x, y):
    """Per-column angle between x[:, j] and +-y[:, j] (singular vectors up to sign),
    computed as atan2(|x - (x.y) y|, |x.y|) for accuracy at small angles."""
    nx = x / np.linalg.norm(x, axis=0)
    ny = y / np.linalg.norm(y, axis=0)
    c = np.sum(nx * ny, axis=0)
    r = np.linalg.norm(nx - ny * c, axis=0)
    return np.arctan2(r, np.abs(c))
