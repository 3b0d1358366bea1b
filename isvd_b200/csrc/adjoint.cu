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
#include <algorithm>
#include <cmath>
#include <utility>
#include <vector>

#include "kernels.h"
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

// Conjugate gradient updates, column c with its own scalars (diagonals of k x k Gram matrices):
//   step 1: a_c = rr_c / (P'Q)_cc;  x_c += a_c p_c;  r_c -= a_c q_c
//   step 2: b_c = (R'R)_cc / rr_c;  p_c = r_c + b_c p_c
template <class T>
__global__ void cg_step1_kernel(T *x, T *r, const T *__restrict__ p, const T *__restrict__ q, long long rows, int k,
                                const double *__restrict__ rr, const T *__restrict__ PQ) {
  const long long total = rows * k;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
       e += (long long)gridDim.x * blockDim.x) {
    const int c = (int)(e % k);
    const double pq = (double)PQ[c * k + c];
    const double a = (rr[c] > 0.0 && pq != 0.0) ? rr[c] / pq : 0.0;
    x[e] = (T)((double)x[e] + a * (double)p[e]);
    r[e] = (T)((double)r[e] - a * (double)q[e]);
  }
}

template <class T>
__global__ void cg_step2_kernel(T *p, const T *__restrict__ r, long long rows, int k, const double *__restrict__ rr,
                                const T *__restrict__ RR) {
  const long long total = rows * k;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
       e += (long long)gridDim.x * blockDim.x) {
    const int c = (int)(e % k);
    const double b = rr[c] > 0.0 ? (double)RR[c * k + c] / rr[c] : 0.0;
    p[e] = (T)((double)r[e] + b * (double)p[e]);
  }
}

template <class T>
__global__ void diag_to_double_kernel(const T *__restrict__ G, int k, double *__restrict__ d) {
  for (int c = threadIdx.x; c < k; c += blockDim.x) d[c] = (double)G[c * k + c];
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

// X -= B (B' X) for B (rows x k, orthonormal columns, row stride ldb); tk: k x k scratch.
template <class T>
void project_out(cudaStream_t st, long long rows, int k, const T *B, long long ldb, T *X, T *tk) {
  mul_t<T>(st, k, k, (int)rows, B, ldb, true, X, k, false, tk, k, 1.0, 0.0);
  mul_t<T>(st, (int)rows, k, k, B, ldb, false, tk, k, false, X, k, -1.0, 1.0);
}

// Batched conjugate gradients for (s_c^2 I - Aperp Aperp') x_c = b_c (left: m rows) or
// (s_c^2 I - Aperp' Aperp) x_c = b_c (right: n rows), from x = b S^-2.  Returns the iterations.
template <class T>
int complement_cg(const StageCtx &c, int m, int n, int k, char ordera, const T *a, long long lda, const T *u,
                  long long ldu, const T *v, long long ldv, const T *s, bool left, const T *b, T *x, int maxit,
                  double tol) {
  cudaStream_t st = c.st;
  const long long rows = left ? m : n, other = left ? n : m;
  const size_t rk = (size_t)rows * k;
  const T *P = left ? u : v, *Qb = left ? v : u;
  const long long ldp = left ? ldu : ldv, ldq = left ? ldv : ldu;
  colscale_add<T>(st, x, b, s, -2, 0.0, nullptr, rows, k);
  if (maxit <= 0) return 0;
  DBuf<T> r(rk), p(rk), q(rk), w((size_t)other * k), z(rk), tk((size_t)k * k), G((size_t)k * k);
  DBuf<double> rr(k), bb(k);
  // op(X) = X S^2 - P_perp A_ Q_perp A_' P_perp X,  A_ = A (left) or A' (right)
  auto apply = [&](const T *X, T *Y) {
    CK(cudaMemcpyAsync(z.p, X, rk * sizeof(T), cudaMemcpyDeviceToDevice, st));
    project_out<T>(st, rows, k, P, ldp, z.p, tk.p);
    mul_a<T>(st, ordera, m, n, a, lda, left, k, z.p, w.p);
    project_out<T>(st, other, k, Qb, ldq, w.p, tk.p);
    mul_a<T>(st, ordera, m, n, a, lda, !left, k, w.p, z.p);
    project_out<T>(st, rows, k, P, ldp, z.p, tk.p);
    colscale_add<T>(st, Y, X, s, 2, -1.0, z.p, rows, k);
  };
  auto col_norms2 = [&](const T *X, double *out) {  // out_c = x_c' x_c
    mul_t<T>(st, k, k, (int)rows, X, k, true, X, k, false, G.p, k, 1.0, 0.0);
    diag_to_double_kernel<T><<<1, 128, 0, st>>>(G.p, k, out);
    KLAUNCHED();
  };
  apply(x, q.p);
  colscale_add<T>(st, r.p, b, s, 0, -1.0, q.p, rows, k);  // r = b - op(x)
  CK(cudaMemcpyAsync(p.p, r.p, rk * sizeof(T), cudaMemcpyDeviceToDevice, st));
  col_norms2(b, bb.p);
  col_norms2(r.p, rr.p);
  std::vector<double> h_rr(k), h_b(k);
  CK(cudaMemcpyAsync(h_b.data(), bb.p, k * sizeof(double), cudaMemcpyDeviceToHost, st));
  int it = 0;
  for (; it < maxit; ++it) {
    CK(cudaMemcpyAsync(h_rr.data(), rr.p, k * sizeof(double), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    bool done = true;
    for (int i = 0; i < k; ++i)
      if (h_rr[i] > tol * tol * h_b[i]) done = false;
    if (done) break;
    apply(p.p, q.p);
    mul_t<T>(st, k, k, (int)rows, p.p, k, true, q.p, k, false, G.p, k, 1.0, 0.0);  // diagonal: p_c' q_c
    cg_step1_kernel<T><<<egrid((long long)rk), 256, 0, st>>>(x, r.p, p.p, q.p, rows, k, rr.p, G.p);
    KLAUNCHED();
    mul_t<T>(st, k, k, (int)rows, r.p, k, true, r.p, k, false, G.p, k, 1.0, 0.0);  // diagonal: r_c' r_c
    cg_step2_kernel<T><<<egrid((long long)rk), 256, 0, st>>>(p.p, r.p, rows, k, rr.p, G.p);
    KLAUNCHED();
    diag_to_double_kernel<T><<<1, 128, 0, st>>>(G.p, k, rr.p);
    KLAUNCHED();
  }
  return it;
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
  int iters = 0;
  iters += complement_cg<T>(c, m, n, k, ordera, a, lda, u, ldu, v, ldv, s, true, ru.p, lam.p, du ? cg_iters : 0, tol);
  iters += complement_cg<T>(c, m, n, k, ordera, a, lda, u, ldu, v, ldv, s, false, rv.p, gam.p, dv ? cg_iters : 0,
                            tol);
  // w1 = (I - VV') A' Lam  ->  Q1 = V J' + Gam S + w1 ;  w2 = (I - UU') A Gam  ->  P2 = Lam S + w2
  mul_a<T>(st, ordera, m, n, a, lda, true, k, lam.p, w1.p);
  project_out<T>(st, n, k, v, ldv, w1.p, tk.p);
  colscale_add<T>(st, w1.p, gam.p, s, 1, 1.0, w1.p, n, k);
  mul_t<T>(st, n, k, k, v, ldv, false, J.p, k, true, w1.p, k, 1.0, 1.0);
  mul_a<T>(st, ordera, m, n, a, lda, false, k, gam.p, w2.p);
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
