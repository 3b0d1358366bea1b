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
// vector updates stay on CUDA cores in the operands' type.  With n <= m, MIXED solves both
// systems in the n-dimensional coordinates of B'B (B = Aperp), formed once from the Gram A'A of
// the same planes (complement_gram_cg): one n x n product per iteration instead of two products by
// A and four projections.
#include <algorithm>
#include <cmath>
#include <cstdlib>
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

// Y = X diag(s)^power + zc Z  (rows x k; X and Y contiguous, Z of row stride ldz; power in
// {0, 1, 2, -2}; Z may be null).  Y may alias X or Z: every entry is read and written by the same
// thread.
template <class T>
__global__ void colscale_add_kernel(T *Y, const T *X, const T *__restrict__ s, int power, double zc, const T *Z,
                                    long long rows, int k, long long ldz) {
  const long long total = rows * k;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
       e += (long long)gridDim.x * blockDim.x) {
    const long long r = e / k, c = e - r * k;
    const double sc = s[c];
    const double f = power == 0 ? 1.0 : power == 1 ? sc : power == 2 ? sc * sc : 1.0 / (sc * sc);
    double v = (double)X[e] * f;
    if (Z) v += zc * (double)Z[r * ldz + c];
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
                  int k, long long ldz = 0) {
  colscale_add_kernel<T><<<egrid(rows * k), 256, 0, st>>>(Y, X, s, power, zc, Z, rows, k, ldz > 0 ? ldz : k);
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
  // MIXED only: one pass over A for two k-column operands side by side,
  //   Y = A [X1 | X2] (m x 2k; X1, X2: n x k)   or, transpose,   Y = A' [X1 | X2] (n x 2k; X1, X2: m x k),
  // with X1, X2 of row strides ld1, ld2 and Y of row stride ldy.  Each output column depends on its
  // own operand column only, so the two halves are the products mul() would give (to the rounding
  // of the split-K grouping).
  PlaneBuf x2n, x2m;
  void mul2(bool transpose, int k, const T *X1, long long ld1, const T *X2, long long ld2, T *Y, long long ldy) {
    const long long rows = transpose ? m : n;  // operand rows (the product's K)
    PlaneBuf &xp = transpose ? x2m : x2n;
    const long long ld = plane_ld(rows), ps = plane_rows(2LL * k) * ld;
    xp.buf.ensure((size_t)3 * ps);
    // [X1 | X2]' planes (2k x rows): the first call also zeroes every padding row and column
    split_planes<T>(X1, ld1, 1, rows, k, 3, true, xp.buf.p, ld, ps, c.st);
    split_rows<T>(X2, ld2, 1, rows, k, 3, true, xp.buf.p + (size_t)k * ld, ld, ps, c.st);
    xp.P.ptr = xp.buf.p; xp.P.np = 3; xp.P.rows = 2LL * k; xp.P.cols = rows; xp.P.ld = ld;
    xp.P.plane_stride = ps; xp.P.mn_major = false;
    UmmaGemm g;
    if (!transpose) {  // Y (m x 2k) = A [X1 | X2]
      g.M = m; g.N = 2 * k; g.K = n;
      g.A = ap.P; g.B = xp.P;
      g.C = Y; g.c_rs = ldy; g.c_cs = 1;
    } else {  // Y' (2k x n) = [X1 | X2]' A
      Planes b = ap.P;
      b.mn_major = true;
      g.M = 2 * k; g.N = n; g.K = m;
      g.A = xp.P; g.B = b;
      g.C = Y; g.c_rs = 1; g.c_cs = ldy;
    }
    g.nprod = 0;
    for (int sum = 0; sum < 3; ++sum)  // plane pairs (p of A, q of X) with p + q < 3
      for (int p = 0; p <= sum && p < 2; ++p) {
        const int q = sum - p;
        if (transpose) { g.pa[g.nprod] = q; g.pb[g.nprod] = p; } else { g.pa[g.nprod] = p; g.pb[g.nprod] = q; }
        ++g.nprod;
      }
    g.c_double = false;
    g.status = c.status;
    g.tag = "adjoint_a2";
    umma_gemm(g, c.st);
  }
};

// X -= B (B' X) for B (rows x k, orthonormal columns, row stride ldb) and X (rows x k, row stride
// ldx, default k); tk: k x k scratch.
template <class T>
void project_out(cudaStream_t st, long long rows, int k, const T *B, long long ldb, T *X, T *tk, long long ldx = 0) {
  if (ldx <= 0) ldx = k;
  mul_t<T>(st, k, k, (int)rows, B, ldb, true, X, ldx, false, tk, k, 1.0, 0.0);
  mul_t<T>(st, (int)rows, k, k, B, ldb, false, tk, k, false, X, ldx, -1.0, 1.0);
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
  // the CG update of one system after q = op(p): x, r, p and rr
  auto update = [&](CgSystem<T> &y) {
    coldot<T>(st, y.p.p, y.q.p, y.rows, k, y.part.p, y.pq.p);
    cg_step1_kernel<T><<<egrid(y.rows * k), 256, 0, st>>>(y.x, y.r.p, y.p.p, y.q.p, y.rows, k, y.rr, y.pq.p);
    KLAUNCHED();
    coldot<T>(st, y.r.p, y.r.p, y.rows, k, y.part.p, y.rn.p);
    cg_step2_kernel<T><<<egrid(y.rows * k), 256, 0, st>>>(y.p.p, y.r.p, y.rows, k, y.rr, y.rn.p);
    KLAUNCHED();
    CK(cudaMemcpyAsync(y.rr, y.rn.p, k * sizeof(double), cudaMemcpyDeviceToDevice, st));
  };
  // One CG iteration of one system; after two eager iterations (which size every buffer) each
  // system's iteration is captured as a CUDA graph and replayed.
  auto body = [&](CgSystem<T> &y) {
    apply(y, y.p.p, y.q.p);
    update(y);
  };
  std::vector<double> h((size_t)4 * k);
  // reads both systems' rr and bb; a system whose every column is below tol leaves; false when
  // neither is left
  auto check = [&]() {
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
    return any;
  };
  int it = 0;
  const char *sep = getenv("ISVD_GPU_ADJOINT_SEPARATE");  // diagnostic: one pass over A per product
  if (A.mixed && sys[0].active && sys[1].active && !(sep && atoi(sep) != 0)) {
    // Both systems in one pass over A per product: the left operator applies A' then A, the right
    // one A then A', so with the right system half an iteration behind, every product by A' takes
    // [p_L | w_R] and every product by A takes [w_L | p_R] (2k columns, one read of A's planes):
    //   A' [p_L | w_R] -> [w_L | z_R];  project;  q_R = p_R S^2 - z_R;  update R;
    //   A [w_L | p_R]  -> [z_L | w_R];  project;  q_L = p_L S^2 - z_L;  update L.
    // Each system goes through exactly its own iteration; w_R of the first iteration comes first.
    CgSystem<T> &L = sys[0], &R = sys[1];
    const long long k2 = 2LL * k;
    DBuf<T> Y1((size_t)n * k2), Y2((size_t)m * k2);  // [w_L | z_R] (n x 2k), [z_L | w_R] (m x 2k)
    auto second_half_R = [&]() { project_out<T>(st, m, k, R.Qb, R.ldq, Y2.p + k, R.tk.p, k2); };
    A.mul2(false, k, R.p.p, k, R.p.p, k, Y2.p, k2);  // w_R = A p_R (both halves)
    second_half_R();
    auto joint = [&]() {
      A.mul2(true, k, L.p.p, k, Y2.p + k, k2, Y1.p, k2);
      project_out<T>(st, n, k, L.Qb, L.ldq, Y1.p, L.tk.p, k2);
      project_out<T>(st, n, k, R.P, R.ldp, Y1.p + k, R.tk.p, k2);
      colscale_add<T>(st, R.q.p, R.p.p, s, 2, -1.0, Y1.p + k, n, k, k2);
      update(R);
      A.mul2(false, k, Y1.p, k2, R.p.p, k, Y2.p, k2);
      project_out<T>(st, m, k, L.P, L.ldp, Y2.p, L.tk.p, k2);
      colscale_add<T>(st, L.q.p, L.p.p, s, 2, -1.0, Y2.p, m, k, k2);
      update(L);
      second_half_R();
    };
    GraphPair jgraph(st);
    for (; it < maxit; ++it) {
      if (!check()) return L.its + R.its;
      if (!L.active || !R.active) break;  // the other one continues on its own below
      ++L.its;
      ++R.its;
      if (jgraph.usable && it >= 2) jgraph.run(0, joint);
      else joint();
    }
  }
  GraphPair graphs(st);
  for (; it < maxit; ++it) {
    if (!check()) break;
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

// MIXED with FP32 operands and n <= m: both complement systems in the n-dimensional
// coordinates of B'B, B = (I - UU') A (I - VV'):
//   right:  (s_c^2 I - B'B) gam_c = bv_c                                   (as it stands)
//   left:   (s_c^2 I - BB') lam_c = bu_c  <=>  lam_c = (bu_c + B mu_c) / s_c^2  with
//           (s_c^2 I - B'B) mu_c = B' bu_c                                 (push-through identity)
// B'B = (I - VV') (G - (U'A)' (U'A)) (I - VV') with G = A'A, formed once (G from all four products
// of A's two bf16 planes with FP64 results, so that it is the Gram of the same approximation of A
// the products by A use; the rank-k corrections in FP64), and kept as three bf16 planes: a CG
// iteration then costs one n x n x (k or 2k) tensor-core product, where the operator in A costs two
// m x n x k products and four projections.  Both systems run as one CG over their columns side by
// side ([mu | gam], s repeated); the count returned is the iterations times the systems.
template <class T>
int complement_gram_cg(const StageCtx &c, AProducts<T> &A, int k, const T *u, long long ldu, const T *v,
                       long long ldv, const T *s, const T *bu, T *xu, const T *bv, T *xv, int maxit, double tol) {
  cudaStream_t st = c.st;
  const int m = A.m, n = A.n;
  const int ns = (bu ? 1 : 0) + (bv ? 1 : 0), kc = ns * k;
  const size_t nk = (size_t)n * k, nc = (size_t)n * kc;
  // G = A'A, then Gp = (I - VV') (G - B1' B1) (I - VV'), B1 = U'A  (all n x n FP64)
  DBuf<double> G((size_t)n * n);
  mixed_gram_full<T>(c, A.ap.P, m, n, A.a, A.lda, G.p, 2, true);
  DBuf<T> uc, b1t(nk);
  const T *uk = u;
  if (ldu != k) {
    uc.alloc((size_t)m * k);
    copy2d<T, T>(u, ldu, 1, uc.p, k, 1, m, k, st);
    uk = uc.p;
  }
  A.mul(true, k, uk, b1t.p);  // B1' = A' U
  DBuf<double> b1d(nk), vd(nk), hv(nk), cm((size_t)k * k);
  copy2d<T, double>(b1t.p, k, 1, b1d.p, k, 1, n, k, st);
  copy2d<T, double>(v, ldv, 1, vd.p, k, 1, n, k, st);
  auto dprod = [&](int M, int N, int K, const double *A_, long long a_rs, long long a_cs, const double *B_,
                   long long b_rs, long long b_cs, double *C_, long long c_rs, double alpha, double beta) {
    Gemm<double, double> g;
    g.M = M; g.N = N; g.K = K;
    g.A = A_; g.a_rs = a_rs; g.a_cs = a_cs;
    g.B = B_; g.b_rs = b_rs; g.b_cs = b_cs;
    g.C = C_; g.c_rs = c_rs; g.c_cs = 1;
    g.alpha = alpha; g.beta = beta;
    gemm(g, st);
  };
  dprod(n, n, k, b1d.p, k, 1, b1d.p, 1, k, G.p, n, -1.0, 1.0);  // H = G - B1' B1
  dprod(n, k, n, G.p, n, 1, vd.p, k, 1, hv.p, k, 1.0, 0.0);     // H V
  dprod(k, k, n, vd.p, 1, k, hv.p, k, 1, cm.p, k, 1.0, 0.0);    // C = V' H V
  dprod(n, k, k, vd.p, k, 1, cm.p, k, 1, hv.p, k, -0.5, 1.0);   // Z = H V - V C / 2
  dprod(n, n, k, vd.p, k, 1, hv.p, 1, k, G.p, n, -1.0, 1.0);    // H - V Z'
  dprod(n, n, k, hv.p, k, 1, vd.p, 1, k, G.p, n, -1.0, 1.0);    //   - Z V'  = Gp
  PlaneBuf gp;
  make_planes<double>(gp, G.p, n, n, n, 3, false, st);
  // right-hand sides [B' bu | bv] (n x kc) and s repeated per system
  DBuf<T> b(nc), x(nc), r(nc), pv(nc), q(nc), z(nc), tn(nk), tk((size_t)k * k), s2(kc);
  int off = 0, off_l = -1, off_r = -1;
  if (bu) {
    A.mul(true, k, bu, tn.p);
    project_out<T>(st, n, k, v, ldv, tn.p, tk.p);  // B' bu = (I - VV') A' bu  (bu orthogonal to U)
    copy2d<T, T>(tn.p, k, 1, b.p + off, kc, 1, n, k, st);
    off_l = off;
    off += k;
  }
  if (bv) {
    copy2d<T, T>(bv, k, 1, b.p + off, kc, 1, n, k, st);
    off_r = off;
    off += k;
  }
  for (int i = 0; i < ns; ++i) CK(cudaMemcpyAsync(s2.p + (size_t)i * k, s, k * sizeof(T), cudaMemcpyDeviceToDevice, st));
  PlaneBuf xp;
  auto op = [&](const T *X, T *Y) {  // Y = X S^2 - Gp X
    make_planes<T>(xp, X, kc, n, kc, 3, true, st);  // X' planes (kc x n)
    UmmaGemm g;
    g.M = n; g.N = kc; g.K = n;
    g.A = gp.P; g.B = xp.P;
    g.nprod = 0;
    for (int sum = 0; sum < 3; ++sum)  // plane pairs with p + q < 3
      for (int pp = 0; pp <= sum; ++pp) { g.pa[g.nprod] = pp; g.pb[g.nprod] = sum - pp; ++g.nprod; }
    g.C = z.p; g.c_double = false; g.c_rs = kc; g.c_cs = 1;
    g.status = c.status;
    g.tag = "adjoint_gram_op";
    umma_gemm(g, st);
    colscale_add<T>(st, Y, X, s2.p, 2, -1.0, z.p, n, kc);
  };
  DBuf<double> scal((size_t)2 * kc), rn(kc), pq(kc), part((size_t)kColdotBlocks * kc);
  double *rr = scal.p, *bb = scal.p + kc;
  colscale_add<T>(st, x.p, b.p, s2.p, -2, 0.0, nullptr, n, kc);  // x = b S^-2
  op(x.p, q.p);
  colscale_add<T>(st, r.p, b.p, s2.p, 0, -1.0, q.p, n, kc);      // r = b - op(x)
  CK(cudaMemcpyAsync(pv.p, r.p, nc * sizeof(T), cudaMemcpyDeviceToDevice, st));
  coldot<T>(st, b.p, b.p, n, kc, part.p, bb);
  coldot<T>(st, r.p, r.p, n, kc, part.p, rr);
  auto body = [&]() {
    op(pv.p, q.p);
    coldot<T>(st, pv.p, q.p, n, kc, part.p, pq.p);
    cg_step1_kernel<T><<<egrid((long long)nc), 256, 0, st>>>(x.p, r.p, pv.p, q.p, n, kc, rr, pq.p);
    KLAUNCHED();
    coldot<T>(st, r.p, r.p, n, kc, part.p, rn.p);
    cg_step2_kernel<T><<<egrid((long long)nc), 256, 0, st>>>(pv.p, r.p, n, kc, rr, rn.p);
    KLAUNCHED();
    CK(cudaMemcpyAsync(rr, rn.p, kc * sizeof(double), cudaMemcpyDeviceToDevice, st));
  };
  GraphPair graphs(st);
  std::vector<double> h((size_t)2 * kc);
  int its = 0;
  for (int it = 0; it < maxit; ++it) {
    CK(cudaMemcpyAsync(h.data(), scal.p, h.size() * sizeof(double), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    bool done = true;
    for (int j = 0; j < kc; ++j)
      if (h[j] > tol * tol * h[kc + j]) done = false;
    if (done) break;
    ++its;
    if (graphs.usable && it >= 2) graphs.run(0, body);
    else body();
  }
  if (bv) copy2d<T, T>(x.p + off_r, kc, 1, xv, k, 1, n, k, st);  // gam
  if (bu) {  // lam = (bu + (I - UU') A mu) S^-2
    DBuf<T> tm((size_t)m * k);
    copy2d<T, T>(x.p + off_l, kc, 1, tn.p, k, 1, n, k, st);  // mu
    A.mul(false, k, tn.p, tm.p);
    project_out<T>(st, m, k, u, ldu, tm.p, tk.p);
    colscale_add<T>(st, tm.p, bu, s, 0, 1.0, tm.p, m, k);
    colscale_add<T>(st, xu, tm.p, s, -2, 0.0, nullptr, m, k);
  }
  return its * ns;
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
  // MIXED, n <= m: the systems in the n-dimensional coordinates of B'B (ISVD_GPU_ADJOINT_CG_A=1 keeps
  // the operator in A, for comparison).  Forming A'A costs m n^2, about as much as 2 n / k CG
  // iterations with the operator in A (2 m n k each): the form pays when n <= 128 k (64 iterations).
  const char *in_a = getenv("ISVD_GPU_ADJOINT_CG_A");
  const bool gram = A.mixed && n <= m && n % 8 == 0 && (long long)n <= 128LL * k && cg_iters > 0 && (du || dv) &&
                    !(in_a && atoi(in_a) != 0);
  const int iters = gram ? complement_gram_cg<T>(c, A, k, u, ldu, v, ldv, s, du ? ru.p : nullptr, lam.p,
                                                 dv ? rv.p : nullptr, gam.p, cg_iters, tol)
                         : complement_cg<T>(c, A, k, u, ldu, v, ldv, s, du ? ru.p : nullptr, lam.p,
                                            dv ? rv.p : nullptr, gam.p, cg_iters, tol);
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
