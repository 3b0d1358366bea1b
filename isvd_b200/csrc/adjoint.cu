// Adjoint (reverse-mode derivative) of the truncated SVD.
//
// For the k leading singular triplets A ~ U diag(s) V' of A (m x n; sigma_1 > ... > sigma_k >
// sigma_(k+1)), and cotangents dU (m x k), ds (k), dV (n x k) of a scalar loss, the gradient is
//   dA = U J V'  +  Lam S V' + U Lam' Aperp  +  U S Gam' + Aperp Gam V'
// with S = diag(s), Aperp = (I - UU') A (I - VV'),
//   J = diag(ds) + (F o (U'dU - dU'U)) S + S (F o (V'dV - dV'V)),  F_ij = 1 / (s_j^2 - s_i^2) (i != j),
// and the orthogonal-complement terms from the Sylvester equations
//   Lam S^2 - Aperp Aperp' Lam = (I - UU') dU,      Gam S^2 - Aperp' Aperp Gam = (I - VV') dV.
// Column i of each is a symmetric positive definite system (s_i^2 I - Aperp Aperp') lam_i = r_i
// (the spectrum of Aperp lies below s_k), solved by conjugate gradients, all columns in one batch,
// with products by A and A'.  cg_iters = 0 keeps the leading term Lam = (I - UU') dU S^-2, exact
// when A has rank k.  The gradient is assembled as one rank-2k update
//   dA = U Q1' + P2 V',   P2 = Lam S + Aperp Gam,   Q1 = V J' + Gam S + Aperp' Lam.
// The two systems run in one loop (one host read of both residual vectors per iteration).  In
// MIXED precision with FP32 operands, A is split once into two bf16 planes and every product by A
// or A' runs on the tcgen05 engine with the other operand in three planes (products with
// p + q < 3: the operand's rounding at FP32 level; A's two planes are one fixed approximation of
// A used by both A X and A' Y, so the CG operator stays symmetric); the projections and the CG
// vector updates stay on CUDA cores in the operands' type.
#include <algorithm>
#include <cmath>
#include <utility>
#include <vector>

#include "kernels.h"
#include "mixed.h"
#include "runtime.h"
#include "stages.h"

namespace isvdb {
namespace {

// C (M x N, row-major ldc) = alpha op(A) op(B) + beta C; op(X) = X' when the flag is set.
template <class T>
void mul_t(cudaStream_t st, int M, int N, int K, const T *A, long long lda, bool ta, const T *B, long long ldb,
           bool tb, T *C, long long ldc, double alpha, double beta) {
  Gemm<T, T> g;
  g.M = M; g.N = N; g.K = K;
  g.alpha = alpha; g.beta = beta;
  g.A = A;
  if (ta) { g.a_rs = 1; g.a_cs = lda; } else { g.a_rs = lda; g.a_cs = 1; }
  g.B = B;
  if (tb) { g.b_rs = 1; g.b_cs = ldb; } else { g.b_rs = ldb; g.b_cs = 1; }
  g.C = C; g.c_rs = ldc; g.c_cs = 1;
  gemm(g, st);
}

// Y = A X (m x k) or A' X (n x k) for A m x n stored per ordera; X, Y contiguous with k columns.
template <class T>
void mul_a(cudaStream_t st, char ordera, int m, int n, const T *a, long long lda, bool transpose, int k, const T *X,
           T *Y) {
  Gemm<T, T> g;
  g.M = transpose ? n : m; g.N = k; g.K = transpose ? m : n;
  long long rs = (ordera == 'R') ? lda : 1, cs = (ordera == 'R') ? 1 : lda;
  if (transpose) std::swap(rs, cs);
  g.A = a; g.a_rs = rs; g.a_cs = cs;
  g.B = X; g.b_rs = k; g.b_cs = 1;
  g.C = Y; g.c_rs = k; g.c_cs = 1;
  gemm(g, st);
}

// J = diag(ds) + (F o (K1 - K1')) S + S (F o (K2 - K2')), F_ij = 1 / (s_j^2 - s_i^2)  (k x k).
template <class T>
__global__ void adj_core_kernel(int k, const T *__restrict__ s, const T *__restrict__ ds, const double *__restrict__ K1,
                                const double *__restrict__ K2, T *__restrict__ J) {
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < k * k; e += gridDim.x * blockDim.x) {
    const int i = e / k, j = e - i * k;
    double v;
    if (i == j) {
      v = ds ? (double)ds[i] : 0.0;
    } else {
      const double si = s[i], sj = s[j];
      const double f = 1.0 / ((sj - si) * (sj + si));
      v = f * (K1[e] - K1[j * k + i]) * sj + si * f * (K2[e] - K2[j * k + i]);
    }
    J[e] = (T)v;
  }
}

// Y = X diag(s)^power + zc Z  (rows x k, contiguous; power in {0, 1, 2, -2}; Z may be null).
// Y may alias X or Z: every entry is read and written by the same thread.
template <class T>
__global__ void colscale_add_kernel(T *Y, const T *X, const T *__restrict__ s, int power, double zc, const T *Z,
                                    long long rows, int k) {
  const long long total = rows * k;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
       e += (long long)gridDim.x * blockDim.x) {
    const double sc = s[e % k];
    const double f = power == 0 ? 1.0 : power == 1 ? sc : power == 2 ? sc * sc : 1.0 / (sc * sc);
    double v = (double)X[e] * f;
    if (Z) v += zc * (double)Z[e];
    Y[e] = (T)v;
  }
}

// Conjugate gradient updates, column c with its own scalars:
//   step 1: a_c = rr_c / pq_c;  x_c += a_c p_c;  r_c -= a_c q_c
//   step 2: b_c = rn_c / rr_c;  p_c = r_c + b_c p_c
template <class T>
__global__ void cg_step1_kernel(T *x, T *r, const T *__restrict__ p, const T *__restrict__ q, long long rows, int k,
                                const double *__restrict__ rr, const double *__restrict__ pq) {
  const long long total = rows * k;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
       e += (long long)gridDim.x * blockDim.x) {
    const int c = (int)(e % k);
    const double a = (rr[c] > 0.0 && pq[c] != 0.0) ? rr[c] / pq[c] : 0.0;
    x[e] = (T)((double)x[e] + a * (double)p[e]);
    r[e] = (T)((double)r[e] - a * (double)q[e]);
  }
}

template <class T>
__global__ void cg_step2_kernel(T *p, const T *__restrict__ r, long long rows, int k, double *__restrict__ rr,
                                const double *__restrict__ rn) {
  const long long total = rows * k;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
       e += (long long)gridDim.x * blockDim.x) {
    const int c = (int)(e % k);
    const double b = rr[c] > 0.0 ? rn[c] / rr[c] : 0.0;
    p[e] = (T)((double)r[e] + b * (double)p[e]);
  }
}

// Column dot products out_c = sum_r x(r, c) y(r, c) of two rows x k matrices (contiguous), in FP64
// and in a fixed order: CTA b sums its slice of rows per column into partial[b * k + c]
// (at most kColdotBlocks slices), then one CTA adds the slices in order.
constexpr int kColdotBlocks = 128;
constexpr int kColdotThreads = 256;

template <class T>
__global__ void __launch_bounds__(kColdotThreads)
    coldot_kernel(const T *__restrict__ x, const T *__restrict__ y, long long rows, int k, double *__restrict__ partial) {
  extern __shared__ double acc[];  // kColdotThreads values per column group
  const long long per = (rows + gridDim.x - 1) / gridDim.x;
  const long long r0 = blockIdx.x * per, r1 = min(rows, r0 + per);
  for (int c0 = 0; c0 < k; c0 += kColdotThreads) {
    // thread t handles column c0 + (t % cw) over rows r0 + t / cw, stepping kColdotThreads / cw
    const int cw = min(kColdotThreads, k - c0);
    const int lanes = kColdotThreads / cw;
    const int t = threadIdx.x;
    double v = 0.0;
    if (t < lanes * cw) {
      const int c = c0 + t % cw;
      for (long long r = r0 + t / cw; r < r1; r += lanes) v += (double)x[r * k + c] * (double)y[r * k + c];
    }
    acc[t] = v;
    __syncthreads();
    if (t < cw) {
      double s = 0.0;
      for (int j = 0; j < lanes; ++j) s += acc[j * cw + t];
      partial[(size_t)blockIdx.x * k + c0 + t] = s;
    }
    __syncthreads();
  }
}

// One warp per column: lane j adds the slices j, j + 32, ... in order, then a fixed shuffle tree.
__global__ void coldot_final_kernel(const double *__restrict__ partial, int nb, int k, double *__restrict__ out) {
  const int c = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5), lane = threadIdx.x & 31;
  if (c >= k) return;  // whole warps leave together
  double s = 0.0;
  for (int b = lane; b < nb; b += 32) s += partial[(size_t)b * k + c];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
  if (lane == 0) out[c] = s;
}

inline int egrid(long long n) {
  return (int)std::max<long long>(1, std::min<long long>((n + 255) / 256, 8LL * Runtime::get().num_sms));
}

template <class T>
void colscale_add(cudaStream_t st, T *Y, const T *X, const T *s, int power, double zc, const T *Z, long long rows,
                  int k) {
  colscale_add_kernel<T><<<egrid(rows * k), 256, 0, st>>>(Y, X, s, power, zc, Z, rows, k);
  KLAUNCHED();
}

// out_c = x_c' y_c (rows x k, contiguous); partial: kColdotBlocks * k doubles.
template <class T>
void coldot(cudaStream_t st, const T *x, const T *y, long long rows, int k, double *partial, double *out) {
  const int nb = (int)std::max<long long>(1, std::min<long long>(kColdotBlocks, (rows + 63) / 64));
  coldot_kernel<T><<<nb, kColdotThreads, kColdotThreads * sizeof(double), st>>>(x, y, rows, k, partial);
  KLAUNCHED();
  coldot_final_kernel<<<(k + 7) / 8, 256, 0, st>>>(partial, nb, k, out);
  KLAUNCHED();
}

// Products by A (m x n, stored per ordera) and A' with k-column operands (contiguous).  MIXED with
// FP32 operands: A's two bf16 planes (made once) on the tcgen05 engine; otherwise the strided GEMM.
template <class T>
struct AProducts {
  const StageCtx &c;
  int m, n;
  char ordera;
  const T *a;
  long long lda;
  bool mixed;
  PlaneBuf ap;
  PlaneBuf xpn, xpm;  // the other operand's planes (n or m rows), kept across products
  AProducts(const StageCtx &c_, int m_, int n_, char ordera_, const T *a_, long long lda_)
      : c(c_), m(m_), n(n_), ordera(ordera_), a(a_), lda(lda_),
        mixed(c_.precision == kMixed && sizeof(T) == sizeof(float)) {
    if (!mixed) return;
    if (ordera == 'R') make_planes<T>(ap, a, lda, m, n, 2, false, c.st);  // m x n, n contiguous
    else make_planes<T>(ap, a, lda, n, m, 2, true, c.st);
  }
  // Y = A X (m x k) or, transpose, A' X (n x k)
  void mul(bool transpose, int k, const T *X, T *Y) {
    if (!mixed) {
      mul_a<T>(c.st, ordera, m, n, a, lda, transpose, k, X, Y);
      return;
    }
    UmmaGemm g;
    PlaneBuf &xp = transpose ? xpm : xpn;
    if (!transpose) {  // Y (m x k) = A X: A planes M x K (K-major), X' planes N x K
      make_planes<T>(xp, X, k, n, k, 3, true, c.st);
      g.M = m; g.N = k; g.K = n;
      g.A = ap.P; g.B = xp.P;
      g.C = Y; g.c_rs = k; g.c_cs = 1;
    } else {  // Y' (k x n) = X' A: X' planes M x K, A planes as the K x N operand (MN-major)
      make_planes<T>(xp, X, k, m, k, 3, true, c.st);
      Planes b = ap.P;
      b.mn_major = true;
      g.M = k; g.N = n; g.K = m;
      g.A = xp.P; g.B = b;
      g.C = Y; g.c_rs = 1; g.c_cs = k;
    }
    g.nprod = 0;
    for (int s = 0; s < 3; ++s)  // plane pairs (p of A, q of X) with p + q < 3
      for (int p = 0; p <= s && p < 2; ++p) {
        const int q = s - p;
        if (transpose) { g.pa[g.nprod] = q; g.pb[g.nprod] = p; } else { g.pa[g.nprod] = p; g.pb[g.nprod] = q; }
        ++g.nprod;
      }
    g.c_double = false;
    g.status = c.status;
    g.tag = "adjoint_a";
    umma_gemm(g, c.st);
  }
};

// X -= B (B' X) for B (rows x k, orthonormal columns, row stride ldb); tk: k x k scratch.
template <class T>
void project_out(cudaStream_t st, long long rows, int k, const T *B, long long ldb, T *X, T *tk) {
  mul_t<T>(st, k, k, (int)rows, B, ldb, true, X, k, false, tk, k, 1.0, 0.0);
  mul_t<T>(st, (int)rows, k, k, B, ldb, false, tk, k, false, X, k, -1.0, 1.0);
}

// One of the two complement systems, (s_c^2 I - Aperp Aperp') x_c = b_c (left: m rows) or
// (s_c^2 I - Aperp' Aperp) x_c = b_c (right: n rows), all columns at once.
template <class T>
struct CgSystem {
  bool left = true, active = false;
  long long rows = 0, other = 0;
  const T *P = nullptr, *Qb = nullptr;  // projector bases: U then V (left), V then U (right)
  long long ldp = 0, ldq = 0;
  const T *b = nullptr;
  T *x = nullptr;
  DBuf<T> r, p, q, w, z, tk;
  DBuf<double> rn, pq, part;
  double *rr = nullptr, *bb = nullptr;  // rr_c = r_c' r_c, bb_c = b_c' b_c (device)
  int its = 0;
};

// Batched conjugate gradients for both complement systems in one loop, from x = b S^-2; each
// system stops when every column's residual is below tol relative to its right-hand side.
// Returns the iterations of both systems together.
template <class T>
int complement_cg(const StageCtx &c, AProducts<T> &A, int k, const T *u, long long ldu, const T *v, long long ldv,
                  const T *s, const T *bu, T *xu, const T *bv, T *xv, int maxit, double tol) {
  cudaStream_t st = c.st;
  const int m = A.m, n = A.n;
  CgSystem<T> sys[2];
  DBuf<double> scal((size_t)4 * k);  // rr and bb of both systems, one read-back
  for (int i = 0; i < 2; ++i) {
    CgSystem<T> &y = sys[i];
    y.left = (i == 0);
    y.b = y.left ? bu : bv;
    y.x = y.left ? xu : xv;
    y.rows = y.left ? m : n;
    y.other = y.left ? n : m;
    y.P = y.left ? u : v;  y.ldp = y.left ? ldu : ldv;
    y.Qb = y.left ? v : u; y.ldq = y.left ? ldv : ldu;
    y.rr = scal.p + (size_t)i * 2 * k;
    y.bb = y.rr + k;
    if (!y.b) continue;
    colscale_add<T>(st, y.x, y.b, s, -2, 0.0, nullptr, y.rows, k);
    y.active = maxit > 0;
  }
  if (maxit <= 0 || (!sys[0].active && !sys[1].active)) return 0;
  // op(X) = X S^2 - P_perp A_ Q_perp A_' X,  A_ = A (left) or A' (right).  Every X this is
  // applied to (b S^-2, the CG directions) lies in the complement of P already (b does, and op
  // ends with P_perp), so the projection before A_' is left out: P_perp A_' X = A_' X - ... would
  // only remove rounding-level components, which the final P_perp removes from the result.
  auto apply = [&](CgSystem<T> &y, const T *X, T *Y) {
    A.mul(y.left, k, X, y.w.p);
    project_out<T>(st, y.other, k, y.Qb, y.ldq, y.w.p, y.tk.p);
    A.mul(!y.left, k, y.w.p, y.z.p);
    project_out<T>(st, y.rows, k, y.P, y.ldp, y.z.p, y.tk.p);
    colscale_add<T>(st, Y, X, s, 2, -1.0, y.z.p, y.rows, k);
  };
  for (CgSystem<T> &y : sys) {
    if (!y.active) continue;
    const size_t rk = (size_t)y.rows * k;
    y.r.alloc(rk); y.p.alloc(rk); y.q.alloc(rk); y.z.alloc(rk);
    y.w.alloc((size_t)y.other * k); y.tk.alloc((size_t)k * k);
    y.rn.alloc(k); y.pq.alloc(k); y.part.alloc((size_t)kColdotBlocks * k);
    apply(y, y.x, y.q.p);
    colscale_add<T>(st, y.r.p, y.b, s, 0, -1.0, y.q.p, y.rows, k);  // r = b - op(x)
    CK(cudaMemcpyAsync(y.p.p, y.r.p, rk * sizeof(T), cudaMemcpyDeviceToDevice, st));
    coldot<T>(st, y.b, y.b, y.rows, k, y.part.p, y.bb);
    coldot<T>(st, y.r.p, y.r.p, y.rows, k, y.part.p, y.rr);
  }
  // One CG iteration of one system; after two eager iterations (which size every buffer) each
  // system's iteration is captured as a CUDA graph and replayed.
  auto body = [&](CgSystem<T> &y) {
    apply(y, y.p.p, y.q.p);
    coldot<T>(st, y.p.p, y.q.p, y.rows, k, y.part.p, y.pq.p);
    cg_step1_kernel<T><<<egrid(y.rows * k), 256, 0, st>>>(y.x, y.r.p, y.p.p, y.q.p, y.rows, k, y.rr, y.pq.p);
    KLAUNCHED();
    coldot<T>(st, y.r.p, y.r.p, y.rows, k, y.part.p, y.rn.p);
    cg_step2_kernel<T><<<egrid(y.rows * k), 256, 0, st>>>(y.p.p, y.r.p, y.rows, k, y.rr, y.rn.p);
    KLAUNCHED();
    CK(cudaMemcpyAsync(y.rr, y.rn.p, k * sizeof(double), cudaMemcpyDeviceToDevice, st));
  };
  GraphPair graphs(st);
  std::vector<double> h((size_t)4 * k);
  for (int it = 0; it < maxit; ++it) {
    CK(cudaMemcpyAsync(h.data(), scal.p, h.size() * sizeof(double), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    bool any = false;
    for (int i = 0; i < 2; ++i) {
      CgSystem<T> &y = sys[i];
      if (!y.active) continue;
      bool done = true;
      const double *rr = h.data() + (size_t)i * 2 * k, *bb = rr + k;
      for (int j = 0; j < k; ++j)
        if (rr[j] > tol * tol * bb[j]) done = false;
      if (done) y.active = false;
      any = any || y.active;
    }
    if (!any) break;
    for (int i = 0; i < 2; ++i) {
      CgSystem<T> &y = sys[i];
      if (!y.active) continue;
      ++y.its;
      if (graphs.usable && it >= 2) graphs.run(i, [&] { body(y); });
      else body(y);
    }
  }
  return sys[0].its + sys[1].its;
}

}  // namespace

template <class T>
int svd_adjoint_dev(const StageCtx &c, int m, int n, int k, char ordera, const T *a, long long lda, const T *u,
                    long long ldu, const T *s, const T *v, long long ldv, const T *du, long long lddu, const T *ds,
                    const T *dv, long long lddv, T *da, long long ldda, int cg_iters, double tol) {
  cudaStream_t st = c.st;
  const size_t mk = (size_t)m * k, nk = (size_t)n * k, kk = (size_t)k * k;
  DBuf<T> ru(mk), rv(nk), lam(mk), gam(nk), w1(nk), w2(mk), tk(kk), J(kk);
  DBuf<double> K1(kk), K2(kk);
  CK(cudaMemsetAsync(ru.p, 0, mk * sizeof(T), st));
  CK(cudaMemsetAsync(rv.p, 0, nk * sizeof(T), st));
  CK(cudaMemsetAsync(K1.p, 0, kk * sizeof(double), st));
  CK(cudaMemsetAsync(K2.p, 0, kk * sizeof(double), st));
  if (du) {  // K1 = U' dU ;  ru = (I - UU') dU
    Gemm<T, double> g;
    g.M = k; g.N = k; g.K = m;
    g.A = u; g.a_rs = 1; g.a_cs = ldu;
    g.B = du; g.b_rs = lddu; g.b_cs = 1;
    g.C = K1.p; g.c_rs = k; g.c_cs = 1;
    gemm(g, st);
    CK(cudaMemcpy2DAsync(ru.p, k * sizeof(T), du, lddu * sizeof(T), k * sizeof(T), m, cudaMemcpyDeviceToDevice, st));
    project_out<T>(st, m, k, u, ldu, ru.p, tk.p);
  }
  if (dv) {  // K2 = V' dV ;  rv = (I - VV') dV
    Gemm<T, double> g;
    g.M = k; g.N = k; g.K = n;
    g.A = v; g.a_rs = 1; g.a_cs = ldv;
    g.B = dv; g.b_rs = lddv; g.b_cs = 1;
    g.C = K2.p; g.c_rs = k; g.c_cs = 1;
    gemm(g, st);
    CK(cudaMemcpy2DAsync(rv.p, k * sizeof(T), dv, lddv * sizeof(T), k * sizeof(T), n, cudaMemcpyDeviceToDevice, st));
    project_out<T>(st, n, k, v, ldv, rv.p, tk.p);
  }
  adj_core_kernel<T><<<egrid((long long)kk), 256, 0, st>>>(k, s, ds, K1.p, K2.p, J.p);
  KLAUNCHED();
  AProducts<T> A(c, m, n, ordera, a, lda);
  if (!du) CK(cudaMemsetAsync(lam.p, 0, mk * sizeof(T), st));
  if (!dv) CK(cudaMemsetAsync(gam.p, 0, nk * sizeof(T), st));
  const int iters = complement_cg<T>(c, A, k, u, ldu, v, ldv, s, du ? ru.p : nullptr, lam.p, dv ? rv.p : nullptr,
                                     gam.p, cg_iters, tol);
  // w1 = (I - VV') A' Lam  ->  Q1 = V J' + Gam S + w1 ;  w2 = (I - UU') A Gam  ->  P2 = Lam S + w2
  A.mul(true, k, lam.p, w1.p);
  project_out<T>(st, n, k, v, ldv, w1.p, tk.p);
  colscale_add<T>(st, w1.p, gam.p, s, 1, 1.0, w1.p, n, k);
  mul_t<T>(st, n, k, k, v, ldv, false, J.p, k, true, w1.p, k, 1.0, 1.0);
  A.mul(false, k, gam.p, w2.p);
  project_out<T>(st, m, k, u, ldu, w2.p, tk.p);
  colscale_add<T>(st, w2.p, lam.p, s, 1, 1.0, w2.p, m, k);
  // dA = U Q1' + P2 V'  (stored per ordera)
  const long long crs = (ordera == 'R') ? ldda : 1, ccs = (ordera == 'R') ? 1 : ldda;
  {
    Gemm<T, T> g;
    g.M = m; g.N = n; g.K = k;
    g.A = u; g.a_rs = ldu; g.a_cs = 1;
    g.B = w1.p; g.b_rs = 1; g.b_cs = k;
    g.C = da; g.c_rs = crs; g.c_cs = ccs;
    gemm(g, st);
    g.A = w2.p; g.a_rs = k; g.a_cs = 1;
    g.B = v; g.b_rs = 1; g.b_cs = ldv;
    g.beta = 1.0;
    gemm(g, st);
  }
  return iters;
}

template int svd_adjoint_dev<float>(const StageCtx &, int, int, int, char, const float *, long long, const float *,
                                    long long, const float *, const float *, long long, const float *, long long,
                                    const float *, const float *, long long, float *, long long, int, double);
template int svd_adjoint_dev<double>(const StageCtx &, int, int, int, char, const double *, long long, const double *,
                                     long long, const double *, const double *, long long, const double *, long long,
                                     const double *, const double *, long long, double *, long long, int, double);

}  // namespace isvdb
