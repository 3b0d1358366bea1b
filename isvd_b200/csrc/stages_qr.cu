// QR-based stages (tall-skinny QR orthogonalization and postprocessing) and Wen-Yin integration.
//
// Tall-skinny QR: the reference factors each block with Householder reflectors (gelqf + orglq of
// Y_i').  Here the orthonormal factor comes from shifted CholeskyQR3 (Fukaya, Kannan, Nakatsukasa,
// Yamamoto, Yanagisawa, SIAM J. Sci. Comput. 42 (2020) A477-A503): three passes of Gram matrix,
// Cholesky factor and triangular solve, which read and write each block as whole tall panels
// (HBM streaming) instead of sweeping it column by column.  Each pass right-multiplies by an
// upper-triangular matrix, so the result is the Q factor of the block; the Householder sign of
// every column is then restored from the top l x l block (Ballard et al. 2015, k_chol.cu), which
// makes the output the one LAPACK's Householder QR gives, to rounding.
#include <cmath>
#include <type_traits>
#include <utility>

#include "kernels.h"
#include "mixed.h"
#include "runtime.h"
#include "stages.h"

namespace isvdb {
namespace {

void read_status(const StageCtx &c, const char *what) {
  int h = 0;
  CK(cudaMemcpyAsync(&h, c.status, sizeof(int), cudaMemcpyDeviceToHost, c.st));
  CK(cudaStreamSynchronize(c.st));
  if (h == kErrTimeout) fail(kErrTimeout, "%s: a device-side wait timed out", what);
  if (h == kStatusNotPD)
    fail(kErrNumerical, "%s: a Cholesky factor broke down (the block is numerically rank deficient)", what);
  if (h) fail(kErrNumerical, "%s: small dense solver reported status %d", what, h);
}

// C = alpha op(A) op(B) + beta C, row-major FP64; op(X) = X' when the flag is set.
void mul(cudaStream_t st, int M, int N, int K, const double *A, long long lda, bool ta, const double *B,
         long long ldb, bool tb, double *C, long long ldc, double alpha, double beta) {
  Gemm<double, double> g;
  g.M = M; g.N = N; g.K = K;
  g.alpha = alpha; g.beta = beta;
  g.A = A;
  if (ta) { g.a_rs = 1; g.a_cs = lda; } else { g.a_rs = lda; g.a_cs = 1; }
  g.B = B;
  if (tb) { g.b_rs = 1; g.b_cs = ldb; } else { g.b_rs = ldb; g.b_cs = 1; }
  g.C = C; g.c_rs = ldc; g.c_cs = 1;
  gemm(g, st);
}

template <class T>
constexpr double unit_roundoff() {
  return std::is_same<T, float>::value ? 0x1p-24 : 0x1p-53;
}

// Orthonormal completion of the null columns of a TS factor (src: rows x N l, null columns zero,
// the others orthonormal): the null columns are filled with pseudo-random values and then
// orthogonalized against the kept columns of their block and each other by two CholeskyQR passes
// in the column order "kept columns first, then the null ones" (a permuted Cholesky), which leaves
// the span of every leading set of kept columns unchanged.  Householder QR (the reference's
// gelqf / orglq) also returns some orthonormal completion for a rank-deficient block; which one
// depends on the rounding of the dependent columns, so only the kept columns are comparable.
// Products in the stage's own type on CUDA cores.  Result in src (dst is scratch).
template <class T>
void complete_null_columns(const StageCtx &c, long long rows, int l, int N, T *&src, long long &lds, T *&dst,
                           long long &ldd, const int *mask) {
  const int Nl = N * l;
  const size_t ll = (size_t)l * l;
  // each rank fills its own rows (a replicated matrix: the same values on every rank)
  const uint64_t seed = 0x5EEDC0DEull + (c.replicated ? 0 : (uint64_t)collective().rank);
  fill_null_columns<T>(src, lds, rows, Nl, mask, seed, 0, c.st);
  DBuf<int> perm((size_t)N * l);
  kept_first_perm(mask, l, N, perm.p, c.st);
  DBuf<double> W(N * ll), X(N * ll);
  DBuf<T> Xt(N * ll);
  for (int pass = 0; pass < 2; ++pass) {
    Gemm<T, double> g;
    g.M = l; g.N = l; g.K = (int)rows; g.batch = N;
    g.A = src; g.a_rs = 1; g.a_cs = lds; g.a_bs = l;
    g.B = src; g.b_rs = lds; g.b_cs = 1; g.b_bs = l;
    g.C = W.p; g.c_rs = l; g.c_cs = 1; g.c_bs = (long long)ll;
    gemm(g, c.st);
    if (!c.replicated) allreduce_sum(W.p, N * ll, c.st);
    chol_inv_batched(l, N, W.p, 1.0, 0.0, 0.0, l * unit_roundoff<T>(), X.p, 1.0, kCholFactor, c.status, c.st,
                     nullptr, nullptr, perm.p);
    copy2d<double, T>(X.p, l, 1, Xt.p, l, 1, (long long)N * l, l, c.st);
    Gemm<T, T> a;
    a.M = (int)rows; a.N = l; a.K = l; a.batch = N;
    a.A = src; a.a_rs = lds; a.a_cs = 1; a.a_bs = l;
    a.B = Xt.p; a.b_rs = l; a.b_cs = 1; a.b_bs = (long long)ll;
    a.C = dst; a.c_rs = ldd; a.c_cs = 1; a.c_bs = l;
    gemm(a, c.st);
    std::swap(src, dst);
    std::swap(lds, ldd);
  }
}

// Householder-signed Q factor of each of the N column blocks (rows x l) of y, in place.
//   pass 0: W = Y'Y,  R'R = W + s I with s = (sqrt(rows) + l + 1) u trace(W),  Y := Y R^-1
//   pass 1, 2: the same without shift (CholeskyQR2 on the now well-conditioned panels); the last
//   R^-1 carries the Householder column signs.
// A block of numerical rank r < l (a Cholesky pivot at rounding level: the column depends on the
// ones before it) does not fail: its dependent columns are marked null, left out of the factor
// (exact zeros, the later columns orthogonalized against the others only) and finally replaced by
// an orthonormal completion (complete_null_columns), so that the result is orthonormal and its
// leading independent columns are the Householder factor's, as Householder QR is total.
// MIXED precision takes the Gram matrices and products from the bf16 split-product tensor-core engine.
template <class T>
void cholqr3_blocks(const StageCtx &c, long long rows, int l, int N, T *y, long long ldy) {
  const int Nl = N * l;
  const size_t ll = (size_t)l * l;
  const bool mixed = (c.precision == kMixed);
  const double u = mixed ? 0x1p-24 : unit_roundoff<T>();
  DBuf<double> W(N * ll), X(N * ll);
  DBuf<T> Xt(N * ll), tmp((size_t)rows * Nl);
  DBuf<int> nmask((size_t)Nl + 1);  // null-column flags, then their count
  CK(cudaMemsetAsync(nmask.p, 0, ((size_t)Nl + 1) * sizeof(int), c.st));
  T *src = y, *dst = tmp.p;
  long long lds = ldy, ldd = Nl;
  for (int pass = 0; pass < 3; ++pass) {
    PlaneBuf yp;
    if (mixed) {
      make_planes<T>(yp, src, lds, rows, Nl, 3, false, c.st);
      mixed_block_gram<T>(c, yp.P, (int)rows, l, N, src, lds, W.p);
    } else {
      Gemm<T, double> g;
      g.M = l; g.N = l; g.K = (int)rows; g.batch = N;
      g.A = src; g.a_rs = 1; g.a_cs = lds; g.a_bs = l;
      g.B = src; g.b_rs = lds; g.b_cs = 1; g.b_bs = l;
      g.C = W.p; g.c_rs = l; g.c_cs = 1; g.c_bs = (long long)ll;
      gemm(g, c.st);
    }
    if (!c.replicated) allreduce_sum(W.p, N * ll, c.st);  // row blocks on several ranks: the Grams are sums
    const double mrows = c.m_total > 0 ? (double)c.m_total : (double)rows;
    const double shift_rel = (pass == 0) ? (std::sqrt(mrows) + l + 1) * u : 0.0;
    const double piv_rel = (pass == 0) ? 0.0 : l * u;
    chol_inv_batched(l, N, W.p, 1.0, 0.0, shift_rel, piv_rel, X.p, 1.0, kCholFactor, c.status, c.st, nmask.p,
                     nmask.p + Nl);
    if (pass == 2) {
      if (collective().nranks > 1 && !c.replicated) {
        // the sign rule reads the first l rows of each block, held by rank 0: every rank takes
        // them from a sum in which the other ranks contribute zeros
        DBuf<T> top((size_t)l * Nl);
        if (collective().rank == 0) {
          if (rows < l) fail(kErrUnsupported, "tall-skinny QR: rank 0 holds fewer than l rows");
          CK(cudaMemcpy2DAsync(top.p, (size_t)Nl * sizeof(T), src, lds * sizeof(T), (size_t)Nl * sizeof(T), l,
                               cudaMemcpyDeviceToDevice, c.st));
        } else {
          CK(cudaMemsetAsync(top.p, 0, (size_t)l * Nl * sizeof(T), c.st));
        }
        allreduce_sum(top.p, (size_t)l * Nl, c.st);
        hh_sign_batched<T>(l, N, top.p, Nl, l, X.p, c.st);
      } else {
        hh_sign_batched<T>(l, N, src, lds, l, X.p, c.st);
      }
    }
    copy2d<double, T>(X.p, l, 1, Xt.p, l, 1, (long long)N * l, l, c.st);
    if (mixed) {
      mixed_block_apply<T>(c, yp.P, (int)rows, l, N, src, lds, Xt.p, dst, ldd);
    } else {
      Gemm<T, T> g;
      g.M = (int)rows; g.N = l; g.K = l; g.batch = N;
      g.A = src; g.a_rs = lds; g.a_cs = 1; g.a_bs = l;
      g.B = Xt.p; g.b_rs = l; g.b_cs = 1; g.b_bs = (long long)ll;
      g.C = dst; g.c_rs = ldd; g.c_cs = 1; g.c_bs = l;
      gemm(g, c.st);
    }
    std::swap(src, dst);
    std::swap(lds, ldd);
  }
  int nulls = 0;
  CK(cudaMemcpyAsync(&nulls, nmask.p + Nl, sizeof(int), cudaMemcpyDeviceToHost, c.st));
  CK(cudaStreamSynchronize(c.st));
  if (nulls > 0) complete_null_columns<T>(c, rows, l, N, src, lds, dst, ldd, nmask.p);
  // three passes: y -> tmp -> y -> tmp (two more for a completion: -> y -> tmp)
  CK(cudaMemcpy2DAsync(y, ldy * sizeof(T), src, lds * sizeof(T), (size_t)Nl * sizeof(T), rows,
                       cudaMemcpyDeviceToDevice, c.st));
}

}  // namespace

// Tall-skinny QR orthogonalization (reference @x@_orthogonalize_tall_skinny_qr.c:123-143 at P = 1:
// Q_i = the orthonormal factor of the LQ of Y_i', in place).
template <class T>
void orth_tsqr_dev(const StageCtx &c, int m, int l, int N, T *y, long long ldy) {
  cholqr3_blocks<T>(c, m, l, N, y, ldy);
  read_status(c, "tall-skinny QR orthogonalization");
}

// Wen-Yin integration (reference @x@_integrate_wen_yin.c:197-360), carried in the coordinates of
// Qs like Kolmogorov-Nagumo: every m x l iterate is Qs M for an Nl x l coefficient matrix, G = Qs'Qs,
//   B = Qs' Q = G M,   Gc = Qs Bc / N -> coefficients Bc / N,   Bgc = Qs' Gc = G Bc / N,
//   X = Gc - Q Dc -> coefficients Bc / N - M Dc,  G X = Bgc - B Dc,
// and the inner products of the Barzilai-Borwein step are <Qs a, Qs b> = sum(a .* G b).
// The 2l x 2l system of the Cayley step (:243-269) is solved in closed form: with
// A11 = Dc/2 - I/tau, A12 = I/2, A21 = -Dgc/2, A22 = -Dc/2 - I/tau its solution F = C^-1 [-I; Dc] has
//   F1 = (2/tau) K^-1,   K = Z/2 + (2/tau^2) I,   Z = Dgc - Dc Dc (symmetric positive semidefinite),
//   F2 = -2 (I + A11 F1),   so  Fgc = F1,  Fc = F2 + I = (2/tau) F1 - I - Dc F1.
// K^-1 comes from a Cholesky factorization; when K is too ill-conditioned for it (large tau), from
// the eigendecomposition of Z with its eigenvalues clipped at zero.
template <class T>
IterResult integrate_wy_dev(const StageCtx &c, int m, int l, int N, const T *qs, long long ldq, T *qt,
                            long long ldqt, const WyArgs &w) {
  const int Nl = N * l;
  const size_t nl = (size_t)Nl * l, ll = (size_t)l * l;
  const double invN = 1.0 / N;
  const bool mixed = (c.precision == kMixed);
  cudaStream_t st = c.st;
  DBuf<double> G((size_t)Nl * Nl);
  PlaneBuf qp;  // MIXED: bf16 planes of Qs, shared by G and the final Qbar = Qs M
  if (mixed) {
    if (c.handoff && c.handoff->holds(qs, ldq)) qp.P = c.handoff->pb.P;  // the Gramian apply's planes
    else make_planes<T>(qp, qs, ldq, m, Nl, 3, false, st);
    mixed_gram_full<T>(c, qp.P, m, Nl, qs, ldq, G.p);
  } else {
    Gemm<T, double> g;
    g.M = Nl; g.N = Nl; g.K = m;
    g.A = qs; g.a_rs = 1; g.a_cs = ldq;
    g.B = qs; g.b_rs = ldq; g.b_cs = 1;
    g.C = G.p; g.c_rs = Nl; g.c_cs = 1;
    g.upper = true;  // G is symmetric: the upper triangle's tiles, then mirrored
    gemm(g, st);
    mirror_upper(G.p, Nl, Nl, st);
  }
  // row blocks on several ranks: G is the integration's one exchange (the reference exchanges Bc,
  // Bgc and two scalars per iteration, @x@_integrate_wen_yin.c:206-345)
  allreduce_sum(G.p, (size_t)Nl * Nl, st);
  DBuf<double> Xo;  // deferred second orthogonalization pass, applied in the coordinates of G
  const bool defer = (mixed && c.deferred_orth);
  if (defer) {
    Xo.alloc((size_t)N * ll);
    coeff_orthonormalize(c, Nl, l, N, G.p, Xo.p);
  }
  // out = G B / N in FP64 in both precision modes.  The iteration carries B by the recursion
  // B+ = Bc Fc + Bgc Fgc and never re-orthonormalizes, so the products must agree with one fixed G
  // to FP64 rounding: BF16x3 products (independent errors of ~1e-7 in every call) make Q drift off
  // orthonormality within tens of iterations, while a G that is itself off by ~1e-7 (the MIXED
  // Gram) only moves the result by that much.
  auto g_times = [&](const double *B, double *out) {
    mul(st, Nl, l, Nl, G.p, Nl, false, B, l, false, out, l, invN, 0.0);
  };
  DBuf<double> Mb(2 * nl), Bb(2 * nl), Bgb(2 * nl), Xb(2 * nl), GXb(2 * nl), Db(2 * ll), Dgb(2 * ll);
  DBuf<double> Z(ll), Fc(ll), Fg(ll), Vz(ll), Vd(ll), lam(l), dd(l), sc(kMaxDotJobs);
  DBuf<int> cst(1);
  double *Mc = Mb.p, *Mp = Mb.p + nl, *Bc = Bb.p, *Bp = Bb.p + nl, *Bgc = Bgb.p, *Bgp = Bgb.p + nl;
  double *Xc = Xb.p, *Xp = Xb.p + nl, *GXc = GXb.p, *GXp = GXb.p + nl;
  double *Dc = Db.p, *Dp = Db.p + ll, *Dgc = Dgb.p, *Dgp = Dgb.p + ll;
  double h[kMaxDotJobs];
  int chol_bad = 0;
  auto fetch = [&](int count) {
    CK(cudaMemcpyAsync(h, sc.p, count * sizeof(double), cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(&chol_bad, cst.p, sizeof(int), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
  };

  copy2d<double, double>(G.p, Nl, 1, Bc, l, 1, Nl, l, st);   // Bc = Qs' Q0 = G[:, 0:l]   (:203)
  set_identity<double>(Mc, Nl, l, l, st);                     // Qc = Q0                   (:200)
  mul(st, l, l, Nl, Bc, l, true, Bc, l, false, Dc, l, invN, 0.0);     // Dc = Bc'Bc / N      (:209)
  g_times(Bc, Bgc);                                                   // Bgc = Qs' Gc        (:212-215)
  mul(st, l, l, Nl, Bc, l, true, Bgc, l, false, Dgc, l, invN, 0.0);   // Dgc = Bc'Bgc / N    (:219)
  lincomb(Xc, Bc, invN, nullptr, 0.0, 0.0, Nl, l, st);                // Xc = Gc - Qc Dc     (:222-223)
  mul(st, Nl, l, l, Mc, l, false, Dc, l, false, Xc, l, -1.0, 1.0);
  lincomb(GXc, Bgc, 1.0, nullptr, 0.0, 0.0, Nl, l, st);
  mul(st, Nl, l, l, Bc, l, false, Dc, l, false, GXc, l, -1.0, 1.0);
  {
    DotJobs j;
    j.trace(Dgc, l);
    j.dot(Dc, nullptr, Dc, nullptr, ll);
    j.dot(Bc, nullptr, Bc, nullptr, nl);
    CK(cudaMemsetAsync(cst.p, 0, sizeof(int), st));
    dots(j, sc.p, st);
    fetch(j.count);
  }
  double mu = h[0] - h[1];                                    // (:226)
  double phi = 0.5 * invN * h[2], taug = w.tau0, zeta = 1.0;  // (:229-231)
  const double tol2 = w.tol * w.tol;
  const int cap = w.maxit > 0 ? w.maxit : 1000000;
  const int lsmax = w.taumaxit > 0 ? w.taumaxit : 1;
  int it = 1;
  for (;; ++it) {
    // Z = Dgc - Dc Dc
    lincomb(Z.p, Dgc, 1.0, nullptr, 0.0, 0.0, l, l, st);
    mul(st, l, l, l, Dc, l, false, Dc, l, false, Z.p, l, -1.0, 1.0);
    bool use_eig = false;
    double tau = taug, phit = phi;
    for (int ls = 0; ls < lsmax; ++ls) {  // curvilinear search (:243-284)
      for (;;) {
        const double a = 2.0 / tau, add = 2.0 / (tau * tau);
        CK(cudaMemsetAsync(cst.p, 0, sizeof(int), st));
        if (!use_eig) {
          chol_inv_batched(l, 1, Z.p, 0.5, add, 0.0, l * 0x1p-52, Fg.p, a, kCholInverse, cst.p, st);
        } else {
          recip_affine(lam.p, l, a, 0.5, add, dd.p, st);
          scale_cols_batched<double, double>(Vz.p, l, Vd.p, l, l, l, l, dd.p, kScaleMul, st);
          mul(st, l, l, l, Vd.p, l, false, Vz.p, l, true, Fg.p, l, 1.0, 0.0);
        }
        lincomb(Fc.p, Fg.p, a, nullptr, 0.0, -1.0, l, l, st);
        mul(st, l, l, l, Dc, l, false, Fg.p, l, false, Fc.p, l, -1.0, 1.0);
        mul(st, Nl, l, l, Bc, l, false, Fc.p, l, false, Bp, l, 1.0, 0.0);   // Bp = Bc Fc + Bgc Fgc (:272-273)
        mul(st, Nl, l, l, Bgc, l, false, Fg.p, l, false, Bp, l, 1.0, 1.0);
        DotJobs j;
        j.dot(Bp, nullptr, Bp, nullptr, nl);
        dots(j, sc.p, st);
        fetch(j.count);
        if (!chol_bad) break;
        // K too ill-conditioned for Cholesky: eigendecomposition of Z for the rest of this iteration
        use_eig = true;
        sym_eig_batched(l, 1, Z.p, Vz.p, lam.p, -1, false, c.status, st);
      }
      phit = 0.5 * invN * h[0];                                        // (:276)
      if (phit >= phi + tau * w.sigma * mu) break;                      // (:279)
      tau *= w.beta;
    }
    phi = (w.eta * zeta * phi + phit) / (w.eta * zeta + 1.0);          // (:288)
    zeta = w.eta * zeta + 1.0;                                         // (:289)
    mul(st, Nl, l, l, Mc, l, false, Fc.p, l, false, Mp, l, 1.0, 0.0);  // Qp = Qc Fc + Gc Fgc (:292-293)
    mul(st, Nl, l, l, Bc, l, false, Fg.p, l, false, Mp, l, invN, 1.0);
    mul(st, l, l, Nl, Bp, l, true, Bp, l, false, Dp, l, invN, 0.0);    // Dp (:296)
    g_times(Bp, Bgp);                                                  // Gp, Bgp (:299-302)
    mul(st, l, l, Nl, Bp, l, true, Bgp, l, false, Dgp, l, invN, 0.0);  // Dgp (:306)
    lincomb(Xp, Bp, invN, nullptr, 0.0, 0.0, Nl, l, st);               // Xp = Gp - Qp Dp (:327-328)
    mul(st, Nl, l, l, Mp, l, false, Dp, l, false, Xp, l, -1.0, 1.0);
    lincomb(GXp, Bgp, 1.0, nullptr, 0.0, 0.0, Nl, l, st);
    mul(st, Nl, l, l, Bp, l, false, Dp, l, false, GXp, l, -1.0, 1.0);
    {
      DotJobs j;
      j.trace(Dgp, l);                          // mu (:309)
      j.dot(Dp, nullptr, Dp, nullptr, ll);
      j.dot(Mc, Mp, Bc, Bp, nl);                // <d1, d1>, d1 = Qc - Qp (:331)
      j.dot(Mc, Mp, GXc, GXp, nl);              // <d1, d2>, d2 = Xc - Xp (:332)
      j.dot(Xc, Xp, Bc, Bp, nl);                // <d2, d1>
      j.dot(Xc, Xp, GXc, GXp, nl);              // <d2, d2>
      dots(j, sc.p, st);
      fetch(j.count);
    }
    read_status(c, "Wen-Yin integration");
    mu = h[0] - h[1];
    if (mu < tol2) break;                                              // (:314)
    if (it == cap) { ++it; break; }                                    // (:317-320)
    const double t0 = (it % 2) ? h[2] : h[4], t1 = (it % 2) ? h[3] : h[5];  // (:336-341)
    taug = std::fmin(std::fmax(std::fabs(t0 / t1), w.taumin), w.taumax);    // (:344-347)
    std::swap(Mc, Mp); std::swap(Bc, Bp); std::swap(Bgc, Bgp); std::swap(Xc, Xp);
    std::swap(GXc, GXp); std::swap(Dc, Dp); std::swap(Dgc, Dgp);
  }
  IterResult res;
  res.iterations = it;
  res.error = mu;
  // Qbar = Qs Mp
  if (mixed) {
    if (defer) {
      DBuf<double> Mt(nl);
      coeff_unorthonormalize(c, Nl, l, N, Xo.p, Mp, l, Mt.p);
      mixed_apply_coeff<T>(c, qp.P, m, Nl, l, qs, ldq, Mt.p, qt, ldqt);
    } else {
      mixed_apply_coeff<T>(c, qp.P, m, Nl, l, qs, ldq, Mp, qt, ldqt);
    }
  } else {
    DBuf<T> Mt(nl);
    copy2d<double, T>(Mp, l, 1, Mt.p, l, 1, Nl, l, st);
    Gemm<T, T> g;
    g.M = m; g.N = l; g.K = Nl;
    g.A = qs; g.a_rs = ldq; g.a_cs = 1;
    g.B = Mt.p; g.b_rs = l; g.b_cs = 1;
    g.C = qt; g.c_rs = ldqt; g.c_cs = 1;
    gemm(g, st);
  }
  return res;
}

// Tall-skinny QR postprocessing (reference @x@_postprocess_tall_skinny_qr.c:195-294):
//   Z = A' Qbar;  Z' = L Qlq (gelqf, :199), i.e. Z = Qz R with L = R';  svd(L) = U_L S V_L';
//   U = Qbar V_L[:, 0:k]  (:270);  V = Qz U_L'  (all l columns, :286);  s = S (l values).
template <class T>
void post_tsqr_dev(const StageCtx &c, int m, int n, int k, int l, char ordera, const T *a, long long lda,
                   const T *qt, long long ldqt, T *s, T *ut, long long ldut, T *vt, long long ldvt, bool wu,
                   bool wv) {
  const size_t ll = (size_t)l * l;
  DBuf<T> Z((size_t)n * l), Qz((size_t)n * l);
  // several ranks: the whole Z on every rank, which then factors it as one rank would (the
  // reference factors its distributed Z by a TSQR tree, :199-241; both give the QR factorization of
  // the same Z, up to rounding and column signs)
  project_sum<T>(c, m, n, l, ordera, a, lda, qt, ldqt, Z.p);
  CK(cudaMemcpyAsync(Qz.p, Z.p, (size_t)n * l * sizeof(T), cudaMemcpyDeviceToDevice, c.st));
  StageCtx cn = c;
  cn.precision = kNative;  // the n x l factorization: the stage's own type on CUDA cores
  cn.replicated = true;
  cn.m_total = 0;
  cholqr3_blocks<T>(cn, n, l, 1, Qz.p, l);
  DBuf<double> R(ll), L(ll), Ul(ll), Vl(ll), sv(l);
  {  // R = Qz' Z (upper triangular to rounding)
    Gemm<T, double> g;
    g.M = l; g.N = l; g.K = n;
    g.A = Qz.p; g.a_rs = 1; g.a_cs = l;
    g.B = Z.p; g.b_rs = l; g.b_cs = 1;
    g.C = R.p; g.c_rs = l; g.c_cs = 1;
    gemm(g, c.st);
  }
  copy2d<double, double>(R.p, 1, l, L.p, l, 1, l, l, c.st);  // L = R'
  svd_jacobi_batched(l, 1, L.p, Ul.p, sv.p, Vl.p, c.status, c.st);
  copy2d<double, T>(sv.p, 1, 1, s, 1, 1, l, 1, c.st);
  if (wu) {  // U = Qbar V_L[:, 0:k]
    DBuf<T> Vt(ll);
    copy2d<double, T>(Vl.p, l, 1, Vt.p, l, 1, l, l, c.st);
    Gemm<T, T> g;
    g.M = m; g.N = k; g.K = l;
    g.A = qt; g.a_rs = ldqt; g.a_cs = 1;
    g.B = Vt.p; g.b_rs = l; g.b_cs = 1;
    g.C = ut; g.c_rs = ldut; g.c_cs = 1;
    gemm(g, c.st);
  }
  if (wv) {  // V = Qz U_L'
    DBuf<T> Ut(ll);
    copy2d<double, T>(Ul.p, 1, l, Ut.p, l, 1, l, l, c.st);
    Gemm<T, T> g;
    g.M = n; g.N = l; g.K = l;
    g.A = Qz.p; g.a_rs = l; g.a_cs = 1;
    g.B = Ut.p; g.b_rs = l; g.b_cs = 1;
    g.C = vt; g.c_rs = ldvt; g.c_cs = 1;
    gemm(g, c.st);
  }
  read_status(c, "tall-skinny QR postprocessing");
}

#define ISVD_INST(T)                                                                                         \
  template void orth_tsqr_dev<T>(const StageCtx &, int, int, int, T *, long long);                           \
  template IterResult integrate_wy_dev<T>(const StageCtx &, int, int, int, const T *, long long, T *, long long, \
                                          const WyArgs &);                                                   \
  template void post_tsqr_dev<T>(const StageCtx &, int, int, int, int, char, const T *, long long, const T *,  \
                                 long long, T *, T *, long long, T *, long long, bool, bool);
ISVD_INST(float)
ISVD_INST(double)

}  // namespace isvdb
