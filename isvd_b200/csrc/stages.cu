// Device-level iSVD stages (one MPI rank).  NATIVE precision: products in the stage's type on
// CUDA cores; l x l steps in FP64.  MIXED precision routes the large products to the tcgen05
// bf16 split-product engine (mixed.cu).
#include <cmath>
#include <cstdlib>
#include <vector>

#include "kernels.h"
#include "mixed.h"
#include "panels.h"
#include "runtime.h"
#include "stages.h"

namespace isvdb {
namespace {

template <class T>
inline Gemm<T, T> gm(int M, int N, int K) {
  Gemm<T, T> g;
  g.M = M; g.N = N; g.K = K;
  return g;
}

// A(i, j) of an m x n matrix stored per ordera ('R' row-major, 'C' column-major).
template <class G>
inline void set_a(G &g, char ordera, long long lda, bool transpose) {
  const bool row = (ordera == 'R');
  long long rs = row ? lda : 1, cs = row ? 1 : lda;
  if (transpose) { long long t = rs; rs = cs; cs = t; }
  g.a_rs = rs; g.a_cs = cs;
}

void read_status(const StageCtx &c, const char *what) {
  int h = 0;
  CK(cudaMemcpyAsync(&h, c.status, sizeof(int), cudaMemcpyDeviceToHost, c.st));
  CK(cudaStreamSynchronize(c.st));
  if (h == kErrTimeout) fail(kErrTimeout, "%s: a device-side wait timed out", what);
  if (h) fail(kErrNumerical, "%s: small dense solver reported status %d", what, h);
}

}  // namespace

// ------------------------------------------------------------------------------------ sketch
template <class T>
void sketch_dev(const StageCtx &c, int m, int n, int Nl, char ordera, const T *a, long long lda, const T *omega,
                long long ldom, uint64_t seed, T *y, long long ldy) {
  if (c.precision == kMixed) {
    mixed_sketch<T>(c, m, n, Nl, ordera, a, lda, omega, ldom, seed, y, ldy, c.handoff);
    read_status(c, "Gaussian projection sketching");
    return;
  }
  DBuf<T> om;
  if (!omega) {
    om.alloc((size_t)n * Nl);
    rng_gaussian<T>(om.p, n, Nl, Nl, seed, (uint64_t)c.col_begin * Nl, c.st);  // column blocks: own rows
    omega = om.p;
    ldom = Nl;
  }
  auto rows_times_omega = [&](long long r0, long long rows, const T *ap, long long ld) {
    Gemm<T, T> g = gm<T>((int)rows, Nl, n);
    g.A = ap; set_a(g, ordera, ld, false);
    g.B = omega; g.b_rs = ldom; g.b_cs = 1;
    g.C = y + r0 * ldy; g.c_rs = ldy; g.c_cs = 1;
    gemm(g, c.st);
  };
  if (c.a_panel_rows > 0 && !is_device_pointer(a))  // out-of-core A: Y's rows panel by panel
    for_each_host_panel<T>(c, a, lda, ordera, m, n, c.a_panel_rows, rows_times_omega);
  else
    rows_times_omega(0, m, a, lda);
}

// -------------------------------------------------------------------------- orthogonalize
namespace {

// One Gramian pass on the N column blocks of y (in place):  Q_i = Y_i F(W_i),  W_i = Y_i' Y_i,
//   polar = false:  F = V S^-1           (reference :80-98: gesvd('O') vectors over sqrt(values))
//   polar = true:   F = V S^-1 V'        (re-orthogonalization that keeps Q's columns in place)
// emit (MIXED, l % 64 == 0, with c.handoff): Q goes to the hand-off as bf16 planes, y is not
// written.  Y's planes come from the hand-off when it holds them (the sketch's), else from y.
template <class T>
void gramian_pass(const StageCtx &c, int m, int l, int N, T *y, long long ldy, bool polar, bool emit) {
  const int Nl = N * l;
  const size_t ll = (size_t)l * l;
  DBuf<double> W(N * ll), V(N * ll), w((size_t)N * l);
  PlaneBuf yp;  // MIXED: bf16 planes of Y, shared by the Gram and the apply
  const bool from_hand = c.precision == kMixed && c.handoff && c.handoff->holds(y, ldy);
  if (from_hand) yp.P = c.handoff->pb.P;
  else if (c.precision == kMixed) make_planes<T>(yp, y, ldy, m, Nl, 3, false, c.st);
  // W_i = Y_i' Y_i   (reference :82-84)
  if (c.precision == kMixed) {
    mixed_block_gram<T>(c, yp.P, m, l, N, y, ldy, W.p);
  } else {
    Gemm<T, double> g;
    g.M = l; g.N = l; g.K = m; g.batch = N;
    g.A = y; g.a_rs = 1; g.a_cs = ldy; g.a_bs = l;
    g.B = y; g.b_rs = ldy; g.b_cs = 1; g.b_bs = l;
    g.C = W.p; g.c_rs = l; g.c_cs = 1; g.c_bs = (long long)ll;
    gemm(g, c.st);
  }
  allreduce_sum(W.p, N * ll, c.st);  // row blocks on several ranks: the blocks' Grams are sums
  DBuf<T> Wp(N * ll);
  bool done = false;
  if (c.chol_basis) {
    // F = R^-1 with R'R = W_i (Cholesky): another orthonormal basis of span(Y_i), for callers
    // whose result does not depend on the basis; falls back to the eigenbasis when W_i is too
    // ill-conditioned for a Cholesky factor
    DBuf<int> bad(1);
    CK(cudaMemsetAsync(bad.p, 0, sizeof(int), c.st));
    chol_inv_batched(l, N, W.p, 1.0, 0.0, 0.0, l * 0x1p-52, V.p, 1.0, kCholFactor, bad.p, c.st);
    int h = 0;
    CK(cudaMemcpyAsync(&h, bad.p, sizeof(int), cudaMemcpyDeviceToHost, c.st));
    CK(cudaStreamSynchronize(c.st));
    if (!h) {
      copy2d<double, T>(V.p, l, 1, Wp.p, l, 1, (long long)N * l, l, c.st);
      done = true;
    }
  }
  // eig(W_i) = W_i S_i^2 W_i'  (gesvd 'O' of the PSD Gram: |lambda| descending, :88-91)
  if (!done) sym_eig_batched(l, N, W.p, V.p, w.p, +1, true, c.status, c.st);
  if (done) {
  } else if (!polar) {
    // W_i / S_i with S = sqrt(s)  (:94)
    scale_cols_batched<double, T>(V.p, l, Wp.p, l, (long long)N * l, l, l, w.p, kScaleInvSqrt, c.st);
  } else {
    DBuf<double> Vs(N * ll), P(N * ll);
    scale_cols_batched<double, double>(V.p, l, Vs.p, l, (long long)N * l, l, l, w.p, kScaleInvSqrt, c.st);
    Gemm<double, double> g;
    g.M = l; g.N = l; g.K = l; g.batch = N;
    g.A = Vs.p; g.a_rs = l; g.a_cs = 1; g.a_bs = (long long)ll;
    g.B = V.p; g.b_rs = 1; g.b_cs = l; g.b_bs = (long long)ll;  // V'
    g.C = P.p; g.c_rs = l; g.c_cs = 1; g.c_bs = (long long)ll;
    gemm(g, c.st);
    copy2d<double, T>(P.p, l, 1, Wp.p, l, 1, (long long)N * l, l, c.st);
  }
  // Q_i = Y_i F_i  (:95-98).  MIXED with planes: the product reads only the planes, so it writes
  // y in place; otherwise it goes to a temporary that is copied back.
  if (c.precision == kMixed && l % 64 == 0) {
    const bool out_planes = emit && c.handoff;
    mixed_block_apply<T>(c, yp.P, m, l, N, y, ldy, Wp.p, y, ldy, out_planes ? c.handoff : nullptr);
    if (!out_planes && c.handoff && c.handoff->holds(y, ldy)) c.handoff->of = nullptr;  // y's values changed
    return;
  }
  if (from_hand) fail(kErrUnsupported, "plane hand-off into the Gramian orthogonalization needs l %% 64 == 0");
  DBuf<T> tmp((size_t)m * Nl);
  if (c.precision == kMixed) {
    mixed_block_apply<T>(c, yp.P, m, l, N, y, ldy, Wp.p, tmp.p, Nl);
  } else {
    Gemm<T, T> g = gm<T>(m, l, l);
    g.batch = N;
    g.A = y; g.a_rs = ldy; g.a_cs = 1; g.a_bs = l;
    g.B = Wp.p; g.b_rs = l; g.b_cs = 1; g.b_bs = (long long)ll;
    g.C = tmp.p; g.c_rs = Nl; g.c_cs = 1; g.c_bs = l;
    gemm(g, c.st);
  }
  CK(cudaMemcpy2DAsync(y, ldy * sizeof(T), tmp.p, (size_t)Nl * sizeof(T), (size_t)Nl * sizeof(T), m,
                       cudaMemcpyDeviceToDevice, c.st));
}

}  // namespace

// Gramian orthogonalization (reference @x@_orthogonalize_gramian.c).  In MIXED precision the
// Gram matrices carry FP32-level errors, which cost orthogonality in proportion to cond(Y_i)^2;
// a second, polar pass (the second step of CholeskyQR2, with the symmetric inverse square root in
// place of the Cholesky factor) restores orthonormality to FP32 level without moving the span.
template <class T>
void orth_gramian_dev(const StageCtx &c, int m, int l, int N, T *y, long long ldy) {
  const bool two = c.precision == kMixed && !c.deferred_orth;
  gramian_pass<T>(c, m, l, N, y, ldy, false, !two);
  if (two) gramian_pass<T>(c, m, l, N, y, ldy, true, true);
  read_status(c, "Gramian orthogonalization");
}

// ------------------------------------------------------------------------------- integrate

void coeff_orthonormalize(const StageCtx &c, int Nl, int l, int N, double *G, double *X) {
  const size_t ll = (size_t)l * l;
  DBuf<double> D(N * ll), G1((size_t)Nl * Nl);
  copy_diag_blocks(G, Nl, l, N, D.p, c.st);
  chol_inv_batched(l, N, D.p, 1.0, 0.0, 0.0, l * 0x1p-24, X, 1.0, kCholFactor, c.status, c.st);
  {  // G1 = G diag(X_j)
    Gemm<double, double> g = gm<double>(Nl, l, l);
    g.batch = N;
    g.A = G; g.a_rs = Nl; g.a_cs = 1; g.a_bs = l;
    g.B = X; g.b_rs = l; g.b_cs = 1; g.b_bs = (long long)ll;
    g.C = G1.p; g.c_rs = Nl; g.c_cs = 1; g.c_bs = l;
    gemm(g, c.st);
  }
  {  // G = diag(X_i)' G1
    Gemm<double, double> g = gm<double>(l, Nl, l);
    g.batch = N;
    g.A = X; g.a_rs = 1; g.a_cs = l; g.a_bs = (long long)ll;
    g.B = G1.p; g.b_rs = Nl; g.b_cs = 1; g.b_bs = (long long)l * Nl;
    g.C = G; g.c_rs = Nl; g.c_cs = 1; g.c_bs = (long long)l * Nl;
    gemm(g, c.st);
  }
}

void coeff_unorthonormalize(const StageCtx &c, int Nl, int l, int N, const double *X, const double *M, long long ldm,
                            double *out) {
  const size_t ll = (size_t)l * l;
  Gemm<double, double> g = gm<double>(l, l, l);
  g.batch = N;
  g.A = X; g.a_rs = l; g.a_cs = 1; g.a_bs = (long long)ll;
  g.B = M; g.b_rs = ldm; g.b_cs = 1; g.b_bs = (long long)l * ldm;
  g.C = out; g.c_rs = l; g.c_cs = 1; g.c_bs = (long long)ll;
  gemm(g, c.st);
  (void)Nl;
}

// K depth per CTA of the split-K [Dc, Dgc] product of long Kolmogorov-Nagumo loops (0: the
// generic split-K model).
static int kn_dd_kchunk() {
  const char *e = getenv("ISVD_GPU_KN_DD_KCHUNK");
  const int v = e ? atoi(e) : 128;
  return v == 0 ? 0 : (v >= 16 ? v : 128);
}
// N l from which the loop uses kn_dd_kchunk (ISVD_GPU_KN_DD_FROM overrides 2048)
static int kn_dd_from() {
  const char *e = getenv("ISVD_GPU_KN_DD_FROM");
  return e ? atoi(e) : 2048;
}

//
// Kolmogorov-Nagumo (reference @x@_integrate_kolmogorov_nagumo.c:153-266), carried in the
// coordinates of Qs: with G = Qs' Qs (Nl x Nl), every m x l iterate is Qs * M for an Nl x l
// coefficient matrix M, and
//   Bc = Qs' Qc = G Mc,  Gc = Qs Bc / N  ->  coefficients Bc / N,  Bgc = Qs' Gc = G Bc / N,
//   Q+ = Qc Fc + Gc C^-1  ->  M+ = Mc Fc + (Bc / N) C^-1,   B+ = Bc Fc + Bgc C^-1  (as the reference).
// Each iteration then costs 2 Nl^2 l flops instead of 4 m Nl l, and Qbar = Qs M at the end.
template <class T>
IterResult integrate_kn_dev(const StageCtx &c, int m, int l, int N, const T *qs, long long ldq, T *qt,
                            long long ldqt, int maxit, double tol) {
  const int Nl = N * l;
  const size_t nl = (size_t)Nl * l, ll = (size_t)l * l;
  const long long lw = 3LL * l;  // row stride of the iterate [M | B | Bgc]
  DBuf<double> G((size_t)Nl * Nl);
  PlaneBuf qp;  // MIXED: bf16 planes of Qs, shared by G and the final Qbar = Qs M
  if (c.precision == kMixed && c.handoff && c.handoff->holds(qs, ldq)) qp.P = c.handoff->pb.P;  // the apply's
  else if (c.precision == kMixed) make_planes<T>(qp, qs, ldq, m, Nl, 3, false, c.st);
  if (c.precision == kMixed) {
    mixed_gram_full<T>(c, qp.P, m, Nl, qs, ldq, G.p);
  } else {
    Gemm<T, double> g;
    g.M = Nl; g.N = Nl; g.K = m;
    g.A = qs; g.a_rs = 1; g.a_cs = ldq;
    g.B = qs; g.b_rs = ldq; g.b_cs = 1;
    g.C = G.p; g.c_rs = Nl; g.c_cs = 1;
    g.upper = true;  // G is symmetric: the upper triangle's tiles, then mirrored
    gemm(g, c.st);
    mirror_upper(G.p, Nl, Nl, c.st);
  }
  // Row blocks on several ranks: G is the one exchange of the integration (the reference
  // exchanges Bc and Bgc in every iteration, @x@_integrate_kolmogorov_nagumo.c:160,178); every
  // rank then runs the same iterations on the same G.
  allreduce_sum(G.p, (size_t)Nl * Nl, c.st);
  DBuf<double> Xo;  // deferred second orthogonalization pass, applied in the coordinates of G
  const bool defer = (c.precision == kMixed && c.deferred_orth);
  if (defer) {
    Xo.alloc((size_t)N * ll);
    coeff_orthonormalize(c, Nl, l, N, G.p, Xo.p);
  }
  // iterates W = [M | B | Bgc] (Nl x 3l, current and next), [Dc; Dgc], step outputs
  DBuf<double> Wb(6 * nl), DD(2 * ll), C(ll), Ci(ll), F(ll), Fs(4 * ll), work(kKnWorkMatrices * ll + 64);
  double *Wc = Wb.p, *Wp = Wb.p + 3 * nl;
  copy2d<double, double>(G.p, Nl, 1, Wc + l, lw, 1, Nl, l, c.st);  // Bc = Qs' Q0 = G[:, 0:l]   (:157)
  set_identity<double>(Wc, Nl, l, lw, c.st);                       // Qc = Q0 = Qs [I; 0]       (:154)
  Runtime &rt = Runtime::get();
  const double invN = 1.0 / N;
  MixedGProduct gprod;  // MIXED: G's bf16 planes, reused by every iteration
  if (c.precision == kMixed) gprod.prepare(c, Nl, G.p);
  // MIXED, Nl % 64 == 0: the update writes the bf16 planes of B+ (the next Bc) from its epilogue,
  // so that the G product reads them without a split launch (ISVD_GPU_KN_UPDATE_PLANES=0: split)
  const bool update_planes = c.precision == kMixed && dmma_enabled() && Nl % 64 == 0 && [] {
    const char *e = getenv("ISVD_GPU_KN_UPDATE_PLANES");
    return !(e && atoi(e) == 0);
  }();
  bool split_bc = true;  // the first iteration's Bc = G[:, 0:l] is split by the G product
  // One iteration: W(next) from W(cur).  After two eager iterations (which size every buffer and
  // set every kernel attribute) the iteration is captured as one CUDA graph per parity of the
  // ping-pong buffers, so that an iteration costs one graph launch plus the host read of err.
  auto iteration = [&](double *Wcur, double *Wnext, double *errp) {
    double *Bc = Wcur + l, *Bgc = Wcur + 2 * l;
    if (c.precision == kMixed) {  // Bgc = G Bc / N   (:174-177)
      gprod.apply(c, l, Bc, lw, invN, Bgc, lw, split_bc || !update_planes);
      split_bc = false;
    } else {
      Gemm<double, double> g = gm<double>(Nl, l, Nl);
      g.alpha = invN;
      g.A = G.p; g.a_rs = Nl; g.a_cs = 1;
      g.B = Bc; g.b_rs = lw; g.b_cs = 1;
      g.C = Bgc; g.c_rs = lw; g.c_cs = 1;
      gemm(g, c.st);
    }
    {  // [Dc, Dgc] = Bc' [Bc, Bgc] / N   (:181-184), one batched product
      Gemm<double, double> g = gm<double>(l, l, Nl);
      g.batch = 2;
      // long K (N l >= 2048): 128-deep K chunks per CTA, more splits than the generic split-K
      // model picks (measured at N l = 4096: 32 splits 157.7 us per iteration against 161.2 with
      // the model's 18; 24: 161.8, 12: 167.6, 6: 187.5); ISVD_GPU_KN_DD_KCHUNK overrides the depth
      if (Nl >= kn_dd_from() && kn_dd_kchunk() > 0) g.splits = std::max(1, Nl / kn_dd_kchunk());
      g.alpha = invN;
      g.A = Bc; g.a_rs = 1; g.a_cs = lw; g.a_bs = 0;
      g.B = Bc; g.b_rs = lw; g.b_cs = 1; g.b_bs = l;
      g.C = DD.p; g.c_rs = l; g.c_cs = 1; g.c_bs = (long long)ll;
      gemm(g, c.st);
    }
    // l x l step (:187-218)
    KnStep s;
    s.l = l; s.Dc = DD.p; s.Dgc = DD.p + ll; s.C = C.p; s.Cinv = Ci.p; s.F = F.p; s.err = errp;
    s.work = work.p; s.status = c.status; s.bar = rt.ctl;
    s.ns_target = (c.precision == kMixed) ? 1e-12 : 1e-18;  // MIXED carries FP32-level errors anyway
    s.fstack = Fs.p; s.fstack_scale = invN;
    kn_step(s, c.st);
    {  // [M+ | B+] = [Mc Bc] [F; C^-1 / N] , [Bc Bgc] [F; C^-1]   (:221-226), one batched product
      Gemm<double, double> g = gm<double>(Nl, l, 2 * l);
      g.batch = 2;
      g.A = Wcur; g.a_rs = lw; g.a_cs = 1; g.a_bs = l;
      g.B = Fs.p; g.b_rs = l; g.b_cs = 1; g.b_bs = 2 * (long long)ll;
      g.C = Wnext; g.c_rs = lw; g.c_cs = 1; g.c_bs = l;
      g.splits = 1;  // 2 N l / 64^2 tiles already fill the GPU: no split-K partials to add up
      if (update_planes) {  // batch 1 is B+: its transpose's planes feed the next G product
        g.pl_t = gprod.b.buf.p; g.pl_ld = gprod.b.P.ld; g.pl_ps = gprod.b.P.plane_stride; g.pl_batch = 1;
      }
      gemm(g, c.st);
    }
  };
  GraphPair graphs(c.st);
  IterResult res;
  double herr = 0.0;
  const int cap = maxit > 0 ? maxit : 1000000;
  // Iteration i + 1 is queued before the host reads the error of iteration i, so the GPU never
  // waits for the host's convergence test.  The step kernel writes the error straight into pinned
  // host memory (one slot per parity; no copy behind the iteration).  Iteration i + 1 reads W(i)
  // and writes the other buffer and error slot: when iteration i has converged, its result W(i)
  // is intact and the extra iteration is discarded.
  double *hpin = rt.host_pin;
  cudaEvent_t ev[2];
  for (int e = 0; e < 2; ++e) CK(cudaEventCreateWithFlags(&ev[e], cudaEventDisableTiming));
  auto launch = [&](int it, double *cur, double *next) {
    const int par = it & 1;
    if (graphs.usable && it > 2) graphs.run(par, [&] { iteration(cur, next, hpin + par); });
    else iteration(cur, next, hpin + par);
    CK(cudaEventRecord(ev[par], c.st));
  };
  int iter = 1;
  try {
    launch(1, Wc, Wp);
    for (;; ++iter) {
      if (iter < cap) launch(iter + 1, Wp, Wc);  // speculative next iteration
      CK(cudaEventSynchronize(ev[iter & 1]));
      herr = hpin[iter & 1];
      if (!(herr == herr) || iter % 16 == 0) read_status(c, "Kolmogorov-Nagumo integration");
      if (herr <= tol) break;                                  // (:235-237)
      if (iter == cap) { ++iter; break; }                      // (:238-241)
      std::swap(Wc, Wp);
    }
    read_status(c, "Kolmogorov-Nagumo integration");
  } catch (...) {
    for (int e = 0; e < 2; ++e) cudaEventDestroy(ev[e]);
    throw;
  }
  for (int e = 0; e < 2; ++e) cudaEventDestroy(ev[e]);
  res.iterations = iter;
  res.error = herr;
  // Qbar = Qs M+  (:251)
  if (c.precision == kMixed) {
    DBuf<double> Mt(nl);
    if (defer) coeff_unorthonormalize(c, Nl, l, N, Xo.p, Wp, lw, Mt.p);
    else copy2d<double, double>(Wp, lw, 1, Mt.p, l, 1, Nl, l, c.st);
    mixed_apply_coeff<T>(c, qp.P, m, Nl, l, qs, ldq, Mt.p, qt, ldqt);
  } else {
    DBuf<T> Mt(nl);
    copy2d<double, T>(Wp, lw, 1, Mt.p, l, 1, Nl, l, c.st);
    Gemm<T, T> g = gm<T>(m, l, Nl);
    g.A = qs; g.a_rs = ldq; g.a_cs = 1;
    g.B = Mt.p; g.b_rs = l; g.b_cs = 1;
    g.C = qt; g.c_rs = ldqt; g.c_cs = 1;
    gemm(g, c.st);
  }
  return res;
}

// Hierarchical reduction (reference @x@_integrate_hierarchical_reduction.c:90-130).
template <class T>
void integrate_hr_dev(const StageCtx &c, int m, int l, int N, T *qs, long long ldq, T *qt, long long ldqt) {
  const size_t ll = (size_t)l * l;
  const int hmax = N / 2 > 0 ? N / 2 : 1;
  DBuf<double> Bs(hmax * ll), W(hmax * ll), Vv(hmax * ll), s((size_t)hmax * l);
  DBuf<T> Wt(hmax * ll), Tt(hmax * ll), tmp((size_t)m * l * hmax);
  for (int h2 = N; h2 > 1; h2 = (h2 + 1) / 2) {
    const int h = h2 / 2;
    {  // B(i) = Q(i)' Q(i+h)
      Gemm<T, double> g;
      g.M = l; g.N = l; g.K = m; g.batch = h;
      g.A = qs; g.a_rs = 1; g.a_cs = ldq; g.a_bs = l;
      g.B = qs + (size_t)h * l; g.b_rs = ldq; g.b_cs = 1; g.b_bs = l;
      g.C = Bs.p; g.c_rs = l; g.c_cs = 1; g.c_bs = ll;
      gemm(g, c.st);
    }
    allreduce_sum(Bs.p, (size_t)h * ll, c.st);  // row blocks on several ranks: a sum (:100)
    // svd(B(i)) = W S T' (the same B on every rank: the same factors)
    svd_jacobi_batched(l, h, Bs.p, W.p, s.p, Vv.p, c.status, c.st);
    // Q(i) := (Q(i) W + Q(i+h) T) / sqrt(2 (1 + s))
    scale_cols_batched<double, T>(W.p, l, Wt.p, l, (long long)h * l, l, l, s.p, kScaleHr, c.st);
    scale_cols_batched<double, T>(Vv.p, l, Tt.p, l, (long long)h * l, l, l, s.p, kScaleHr, c.st);
    Gemm<T, T> g = gm<T>(m, l, l);
    g.batch = h;
    g.A = qs; g.a_rs = ldq; g.a_cs = 1; g.a_bs = l;
    g.B = Wt.p; g.b_rs = l; g.b_cs = 1; g.b_bs = ll;
    g.C = tmp.p; g.c_rs = (long long)l * h; g.c_cs = 1; g.c_bs = l;
    gemm(g, c.st);
    g.A = qs + (size_t)h * l; g.B = Tt.p; g.beta = 1.0;
    gemm(g, c.st);
    CK(cudaMemcpy2DAsync(qs, ldq * sizeof(T), tmp.p, (size_t)l * h * sizeof(T), (size_t)l * h * sizeof(T), m,
                         cudaMemcpyDeviceToDevice, c.st));
  }
  CK(cudaMemcpy2DAsync(qt, ldqt * sizeof(T), qs, ldq * sizeof(T), (size_t)l * sizeof(T), m,
                       cudaMemcpyDeviceToDevice, c.st));
  read_status(c, "hierarchical reduction");
}

// ----------------------------------------------------------------------------- postprocess
// Z = A' Qbar (reference @x@_postprocess.h:96-171, row block at P = 1).
template <class T>
void project(const StageCtx &c, int m, int n, int l, char ordera, const T *a, long long lda, const T *qt,
                    long long ldqt, T *z) {
  if (c.precision == kMixed) {
    mixed_project<T>(c, m, n, l, ordera, a, lda, qt, ldqt, z);
    return;
  }
  auto add_rows = [&](long long r0, long long rows, const T *ap, long long ld) {  // Z += A_p' Qbar_p
    Gemm<T, T> g = gm<T>(n, l, (int)rows);
    g.A = ap; set_a(g, ordera, ld, true);
    g.B = qt + r0 * ldqt; g.b_rs = ldqt; g.b_cs = 1;
    g.C = z; g.c_rs = l; g.c_cs = 1;
    g.beta = r0 > 0 ? 1.0 : 0.0;
    gemm(g, c.st);
  };
  if (c.a_panel_rows > 0 && !is_device_pointer(a))  // out-of-core A
    for_each_host_panel<T>(c, a, lda, ordera, m, n, c.a_panel_rows, add_rows);
  else
    add_rows(0, m, a, lda);
}

template <class T>
void project_sum(const StageCtx &c, int m, int n, int l, char ordera, const T *a, long long lda, const T *qt,
                 long long ldqt, T *z) {
  if (c.a_cols <= 0) {  // one rank, or row blocks: Z = sum of A_j' Qbar_j
    project<T>(c, m, n, l, ordera, a, lda, qt, ldqt, z);
    allreduce_sum(z, (size_t)n * l, c.st);
    return;
  }
  // column blocks (reference projectBlockCol, @x@_postprocess.h:19-94): Qbar gathered (its
  // MPI_Allgather, :78, here a sum of zero-padded copies), Z_j = A_j' Qbar for this rank's
  // columns, Z gathered likewise
  const long long M = c.m_total, nj = c.a_cols;
  DBuf<T> qf((size_t)M * l), zj((size_t)nj * l);
  CK(cudaMemsetAsync(qf.p, 0, (size_t)M * l * sizeof(T), c.st));
  CK(cudaMemcpy2DAsync(qf.p + (size_t)c.row_begin * l, (size_t)l * sizeof(T), qt, (size_t)ldqt * sizeof(T),
                       (size_t)l * sizeof(T), m, cudaMemcpyDeviceToDevice, c.st));
  allreduce_sum(qf.p, (size_t)M * l, c.st);
  project<T>(c, (int)M, (int)nj, l, ordera, a, lda, qf.p, l, zj.p);
  CK(cudaMemsetAsync(z, 0, (size_t)n * l * sizeof(T), c.st));
  CK(cudaMemcpyAsync(z + (size_t)c.col_begin * l, zj.p, (size_t)nj * l * sizeof(T), cudaMemcpyDeviceToDevice, c.st));
  allreduce_sum(z, (size_t)n * l, c.st);
}

template <class T>
void post_gramian_dev(const StageCtx &c, int m, int n, int k, int l, char ordera, const T *a, long long lda,
                      const T *qt, long long ldqt, T *s, T *ut, long long ldut, T *vt, long long ldvt, bool wu,
                      bool wv) {
  const size_t ll = (size_t)l * l;
  DBuf<T> Z((size_t)n * l);
  project_sum<T>(c, m, n, l, ordera, a, lda, qt, ldqt, Z.p);  // several ranks: the whole Z on each
  DBuf<double> W(ll), V(ll), w(l);
  {  // W = Z' Z  (reference @x@_postprocess_gramian.c:145)
    Gemm<T, double> g;
    g.M = l; g.N = l; g.K = n;
    g.A = Z.p; g.a_rs = 1; g.a_cs = l;
    g.B = Z.p; g.b_rs = l; g.b_cs = 1;
    g.C = W.p; g.c_rs = l; g.c_cs = 1;
    gemm(g, c.st);
  }
  sym_eig_batched(l, 1, W.p, V.p, w.p, +1, true, c.status, c.st);   // gesvd of W (:150)
  scale_cols_batched<double, T>(w.p, 1, s, 1, l, 1, l, w.p, kSqrtOnly, c.st);  // sigma = sqrt(s) (:151)
  if (wu) {  // U = Qbar W[:, :k]  (:158)
    DBuf<T> Wk(ll);
    copy2d<double, T>(V.p, l, 1, Wk.p, l, 1, l, l, c.st);
    Gemm<T, T> g = gm<T>(m, k, l);
    g.A = qt; g.a_rs = ldqt; g.a_cs = 1;
    g.B = Wk.p; g.b_rs = l; g.b_cs = 1;
    g.C = ut; g.c_rs = ldut; g.c_cs = 1;
    gemm(g, c.st);
  }
  if (wv) {  // V = Z W[:, :k] / sigma  (:173-174)
    DBuf<T> Ws(ll);
    scale_cols_batched<double, T>(V.p, l, Ws.p, l, l, l, l, w.p, kScaleInvSqrt, c.st);
    Gemm<T, T> g = gm<T>(n, k, l);
    g.A = Z.p; g.a_rs = l; g.a_cs = 1;
    g.B = Ws.p; g.b_rs = l; g.b_cs = 1;
    g.C = vt; g.c_rs = ldvt; g.c_cs = 1;
    gemm(g, c.st);
  }
  read_status(c, "Gramian postprocessing");
}

// Symmetric postprocessing (reference @x@_postprocess_symmetric.c:139-157): W = Qbar' A Qbar,
// syev (ascending), U = Qbar W[:, :k].  Row blocks on several ranks (this rank: rows
// [row_begin, row_begin + m) of A and Qbar, n = all rows): Z = A' Qbar summed over the ranks, then
// W = sum of Z(own rows)' Qbar_j (the reference's MPI_Allreduce of W, :147).
template <class T>
void post_symmetric_dev(const StageCtx &c, int m, int n, int k, int l, char ordera, const T *a, long long lda,
                        const T *qt, long long ldqt, T *s, T *ut, long long ldut, bool wu) {
  const size_t ll = (size_t)l * l;
  DBuf<T> Z((size_t)n * l);
  project_sum<T>(c, m, n, l, ordera, a, lda, qt, ldqt, Z.p);
  DBuf<double> W(ll), V(ll), w(l);
  {
    Gemm<T, double> g;
    g.M = l; g.N = l; g.K = m;
    g.A = Z.p + (size_t)c.row_begin * l; g.a_rs = 1; g.a_cs = l;
    g.B = qt; g.b_rs = ldqt; g.b_cs = 1;
    g.C = W.p; g.c_rs = l; g.c_cs = 1;
    gemm(g, c.st);
  }
  allreduce_sum(W.p, ll, c.st);
  sym_eig_batched(l, 1, W.p, V.p, w.p, -1, false, c.status, c.st);
  copy2d<double, T>(w.p, 1, 1, s, 1, 1, l, 1, c.st);
  if (wu) {
    DBuf<T> Wk(ll);
    copy2d<double, T>(V.p, l, 1, Wk.p, l, 1, l, l, c.st);
    Gemm<T, T> g = gm<T>(m, k, l);
    g.A = qt; g.a_rs = ldqt; g.a_cs = 1;
    g.B = Wk.p; g.b_rs = l; g.b_cs = 1;
    g.C = ut; g.c_rs = ldut; g.c_cs = 1;
    gemm(g, c.st);
  }
  read_status(c, "symmetric postprocessing");
}

#define ISVD_INST(T)                                                                                          \
  template void sketch_dev<T>(const StageCtx &, int, int, int, char, const T *, long long, const T *, long long, \
                              uint64_t, T *, long long);                                                        \
  template void orth_gramian_dev<T>(const StageCtx &, int, int, int, T *, long long);                           \
  template void project<T>(const StageCtx &, int, int, int, char, const T *, long long, const T *, long long, T *); \
  template void project_sum<T>(const StageCtx &, int, int, int, char, const T *, long long, const T *, long long,  \
                               T *);                                                                               \
  template IterResult integrate_kn_dev<T>(const StageCtx &, int, int, int, const T *, long long, T *, long long, \
                                          int, double);                                                         \
  template void integrate_hr_dev<T>(const StageCtx &, int, int, int, T *, long long, T *, long long);           \
  template void post_gramian_dev<T>(const StageCtx &, int, int, int, int, char, const T *, long long, const T *, \
                                    long long, T *, T *, long long, T *, long long, bool, bool);               \
  template void post_symmetric_dev<T>(const StageCtx &, int, int, int, int, char, const T *, long long,         \
                                      const T *, long long, T *, T *, long long, bool);
ISVD_INST(float)
ISVD_INST(double)
#undef ISVD_INST

}  // namespace isvdb
