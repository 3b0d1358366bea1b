// Launchers of the device kernels of libisvd_gpu_b200 (all enqueue on the library stream).
#pragma once

#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cstdint>

namespace isvdb {

// ------------------------------------------------------------------ general matrix product
// C(b) = alpha * A(b) * B(b) + beta * C(b) for b < batch, with
//   A(i,k) = A[i*a_rs + k*a_cs],  B(k,j) = B[k*b_rs + j*b_cs],  C(i,j) = C[i*c_rs + j*c_cs]
// and batch offsets a_bs / b_bs / c_bs.  One of each (rs, cs) pair must be 1.
// Tout may be wider than T (double output of float products: split-K partials are
// summed in double).
template <class T, class Tout>
struct Gemm {
  int M = 0, N = 0, K = 0;
  double alpha = 1.0, beta = 0.0;
  const T *A = nullptr;
  long long a_rs = 0, a_cs = 0, a_bs = 0;
  const T *B = nullptr;
  long long b_rs = 0, b_cs = 0, b_bs = 0;
  Tout *C = nullptr;
  long long c_rs = 0, c_cs = 0, c_bs = 0;
  int batch = 1;
  int splits = 0;  // 0: choose automatically
  // C symmetric (M == N, A = B'): tiles entirely below the diagonal are not computed; the caller
  // completes C with mirror_upper
  bool upper = false;
  // FP64 tensor-core path without split-K only (dmma_gemm, splits == 1, M % 64 == 0): batch
  // pl_batch's output C(i, j) is also written as three bf16 planes of its transpose, piece q at
  // pl_t[q pl_ps + j pl_ld + i] (as split_planes(.., transpose = true) splits it)
  __nv_bfloat16 *pl_t = nullptr;
  long long pl_ld = 0, pl_ps = 0;
  int pl_batch = 0;
};

template <class T, class Tout>
void gemm(const Gemm<T, Tout> &g, cudaStream_t st);

// FP64 operands and result on the FP64 tensor-core path (mma.sync m8n8k4, k_dmma.cu); gemm()
// routes Gemm<double, double> here unless ISVD_GPU_DMMA=0.  a_kc: A has unit K stride; b_nc: B
// has unit N stride.
bool dmma_enabled();
void dmma_gemm(const Gemm<double, double> &g, bool a_kc, bool b_nc, cudaStream_t st);
// C = alpha * (sum of the `splits` partial products) + beta * C (partials: batch x splits x M x N).
void splitk_reduce(const Gemm<double, double> &g, int splits, const double *partial, cudaStream_t st);
// One product of a grouped launch over many independent products of their own shapes:
// C = alpha A B + beta C (A M x K, B K x N, element strides as in Gemm).  Its output tiles are the
// work items tile0 .. tile0 + ceil(M / BM) * tn - 1 of the launch (tn tiles along N).
struct GroupedProd {
  int M, N, K;
  const void *A;
  long long a_rs, a_cs;
  const void *B;
  long long b_rs, b_cs;
  void *C;
  long long c_rs, c_cs;
  double alpha, beta;
  int tile0, tn;
  int upper;  // C symmetric (A = B'): tiles entirely below the diagonal are skipped (mirrored by the caller)
};
// FP64 grouped products on the FP64 tensor-core path (k_dmma.cu): one persistent launch walks the
// `total` work items of prods[0 .. nprod) (device memory, tile0 ascending).  Every product has the
// same operand orientation: a_kc (a_cs == 1, else a_rs == 1) and b_nc (b_cs == 1, else b_rs == 1).
// Tile shapes: dmma_grouped_bm(shape) x dmma_grouped_bn(shape), shape < kDmmaGroupedShapes.
constexpr int kDmmaGroupedShapes = 5;
int dmma_grouped_bm(int shape);
int dmma_grouped_bn(int shape);
void dmma_grouped(const GroupedProd *prods, int nprod, int total, int shape, bool a_kc, bool b_nc, cudaStream_t st);

// ------------------------------------------------------------------ elementwise
// Omega(j, c) for j < rows, c < cols: standard normal values from Philox4x32-10 (key = seed)
// with Box-Muller, rounded to bf16; value index = offset + j * cols + c.  Written at out[j*ld + c].
// The rounding makes the Omega of every precision mode identical (the MIXED sketch consumes it
// exactly as a bf16 operand).
template <class T>
void rng_gaussian(T *out, long long rows, long long cols, long long ld, uint64_t seed, uint64_t offset,
                  cudaStream_t st);

// dst(i, j) = src(i, j) with arbitrary strides, converting type.
template <class Ts, class Td>
void copy2d(const Ts *src, long long s_rs, long long s_cs, Td *dst, long long d_rs, long long d_cs, long long rows,
            long long cols, cudaStream_t st);

// A (rows x cols, row-major, ld) := identity-padded: A(i,j) = (i == j)
template <class T>
void set_identity(T *a, long long rows, long long cols, long long ld, cudaStream_t st);

// Column scaling: dst(i, j) = f(src(i, j), s[(i / rows_per_batch) * cols + j]) with
//   kScaleMul: x * s,  kScaleDiv: x / s,  kScaleInvSqrt: x / sqrt(s),
//   kScaleHr: x / sqrt(2 (1 + s)),  kSqrtOnly: sqrt(x)  (s unused).
enum ScaleMode : int { kScaleMul = 0, kScaleDiv = 1, kScaleInvSqrt = 2, kScaleHr = 3, kSqrtOnly = 4 };
template <class Ts, class Td>
void scale_cols_batched(const Ts *src, long long lds, Td *dst, long long ldd, long long rows, long long cols,
                        long long rows_per_batch, const double *s, int mode, cudaStream_t st);

// ------------------------------------------------------------------ small dense FP64 (l x l)
// Batched symmetric eigendecomposition by parallel cyclic Jacobi, one CTA per matrix.
// A: batch x (n x n) row-major (only read), V: batch x (n x n) row-major eigenvectors (columns),
// w: batch x n eigenvalues.  order > 0: sort by |lambda| descending (gesvd of a PSD matrix);
// order < 0: ascending lambda (syev).  absval: return |lambda| in w.
struct EigDesc {  // one matrix of a grouped eigensolve: n x n row-major A -> V (columns), w
  int n;
  const double *A;
  double *V, *w;
};
// As sym_eig_batched for count matrices of different sizes (desc in device memory; max_n >= every n).
void sym_eig_grouped(const EigDesc *desc, int count, int max_n, int order, bool absval, int *status,
                     cudaStream_t st);
void sym_eig_batched(int n, int batch, const double *A, double *V, double *w, int order, bool absval,
                     int *status, cudaStream_t st);

// Batched general SVD B = U diag(s) V' by one-sided Jacobi, one CTA per matrix.
// B, U, V: batch x (n x n) row-major; s descending.
void svd_jacobi_batched(int n, int batch, const double *B, double *U, double *s, double *V, int *status,
                        cudaStream_t st);

// Kolmogorov-Nagumo l x l step (reference core/stage/@x@_integrate_kolmogorov_nagumo.c:180-234):
//   Z = Dgc - Dc^2; C = sqrt(I/2 + sqrt(I/4 - Z)); Cinv = C^-1; err = ||C - I||_F; F = C - Dc Cinv.
// Matrix square roots by coupled Newton-Schulz iterations in a cooperative multi-CTA kernel.
struct KnStep {
  int l;
  const double *Dc, *Dgc;
  double *C, *Cinv, *F, *err;
  double *work;     // kn_step: kKnWorkMatrices l^2 + 64 doubles; kn_step_fixed: 8 l^2 + 64
  int *status;      // set nonzero on failure (timeout / no convergence)
  unsigned int *bar;  // 2 words, zero
  double ns_target = 1e-18;  // Newton-Schulz steps are chosen so that rho^(2^k) <= ns_target
  // kn_step only: when set, also written as the 4l x l stack [F; Cinv * fstack_scale; F; Cinv]
  double *fstack = nullptr;
  double fstack_scale = 1.0;
};
constexpr int kKnWorkMatrices = 29;
constexpr int kSeriesLen = 64;
struct KnSeries {  // power-series coefficients of C(Z) and C(Z)^-1 (k_small.cu)
  double c[kSeriesLen], d[kSeriesLen];
};
void kn_step(const KnStep &a, cudaStream_t st);
// count independent steps (steps in device memory, each with its own buffers; max_l >= every l),
// one thread-block cluster of `cluster` CTAs per step (<= 0: eight; at most what the device
// allows).  A step's 32 x 32 product tiles are spread over its cluster: ceil(l / 32)^2 CTAs keep
// every CTA busy.
void kn_step_grouped(const KnStep *steps, int count, int max_l, int cluster, cudaStream_t st);

// ---------------------------------------------------------------- k_chol.cu
enum CholMode { kCholFactor = 0, kCholInverse = 1 };
constexpr int kStatusNotPD = 7;  // status word: a Cholesky pivot was not positive (or lost its magnitude)

// Per n x n matrix (row-major, batch stride n^2; upper triangle read):
//   A = alpha W + (shift_abs + shift_rel trace(alpha W)) I = R' R,  X = R^-1 (upper);
//   out = X (kCholFactor) or out_scale X X' = out_scale A^-1 (kCholInverse).
// A pivot not above piv_rel times its starting diagonal value sets *status = kStatusNotPD, unless
// null_mask is given (kCholFactor; batch x n ints, zero on the first use): then such a finite pivot
// marks the column as dependent (mask = 1, *null_count += 1 per newly marked column) and zeroes
// column k of X, instead of failing.  perm (batch x n ints): factor P A P' (row i = row perm[i] of
// A), X stored back at the original positions.
void chol_inv_batched(int n, int batch, const double *W, double alpha, double shift_abs, double shift_rel,
                      double piv_rel, double *out, double out_scale, int mode, int *status, cudaStream_t st,
                      int *null_mask = nullptr, int *null_count = nullptr, const int *perm = nullptr);
// One matrix of a grouped factorization: n x n row-major W (upper triangle read) -> out = R^-1
// (upper triangular, zeros below) for W = R' R.
struct CholDesc {
  int n;
  const double *W;
  double *out;
};
// chol_inv_batched in kCholFactor mode (alpha 1, no shift, piv_rel 0: a pivot that is not positive
// and finite sets *status = kStatusNotPD) for count matrices of their own sizes (desc in device
// memory, max_n >= every n).
void chol_inv_grouped(const CholDesc *desc, int count, int max_n, int *status, cudaStream_t st);
// Null columns of a TS factorization: y's columns c < cols with mask[c] set (cols = N l) are filled
// with Philox4x32-10 uniform values in [-1/2, 1/2) keyed by (seed, row_offset + row, c); perm gets,
// per block of l columns, the kept columns first and then the null ones, each in order.
template <class T>
void fill_null_columns(T *y, long long ld, long long rows, int cols, const int *mask, uint64_t seed,
                       long long row_offset, cudaStream_t st);
void kept_first_perm(const int *mask, int l, int N, int *perm, cudaStream_t st);
// X_b := X_b diag(s_b) with the Householder signs of the QR factor whose top n x n block is
// Qtop_b X_b (Qtop_b = rows 0..n-1 of Q + b q_bs, row stride q_ld).
template <class T>
void hh_sign_batched(int n, int batch, const T *Q, long long q_ld, long long q_bs, double *X, cudaStream_t st);

constexpr int kMaxDotJobs = 8;
// value = trace(a) (a n x n) when trace, else sum_i (a_i - b_i)(c_i - d_i) over n entries (b, d optional)
struct DotJob {
  const double *a = nullptr, *b = nullptr, *c = nullptr, *d = nullptr;
  long long n = 0;
  int trace = 0;
};
struct DotJobs {
  DotJob job[kMaxDotJobs];
  int count = 0;
  void dot(const double *a, const double *b, const double *c, const double *d, long long n) {
    DotJob &j = job[count++];
    j.a = a; j.b = b; j.c = c; j.d = d; j.n = n; j.trace = 0;
  }
  void trace(const double *a, long long n) {
    DotJob &j = job[count++];
    j.a = a; j.n = n; j.trace = 1;
  }
};
void dots(const DotJobs &jobs, double *out, cudaStream_t st);  // out[k] = value of job k
// out = a x + b y + c I  (rows x cols, contiguous; x or y may be null)
void lincomb(double *out, const double *x, double a, const double *y, double b, double c, long long rows,
             long long cols, cudaStream_t st);
// out[b] = the b-th l x l diagonal block of G (Nl x Nl row-major), b < N
void copy_diag_blocks(const double *G, int Nl, int l, int N, double *out, cudaStream_t st);
// d_i = num / (half max(lambda_i, 0) + add)
void recip_affine(const double *lam, int n, double num, double half, double add, double *d, cudaStream_t st);

// Launchers for the entry points that run on static scratch and must not allocate: they take the
// SM count from the caller instead of the library runtime (whose set-up allocates), and gemm_fixed
// puts split-K partial sums in the caller's buffer of `cap` elements (splitting less, or not at
// all, when it is short).
template <class T, class Tout>
void gemm_fixed(const Gemm<T, Tout> &g, int num_sms, T *partial, size_t cap, cudaStream_t st);
void kn_step_fixed(const KnStep &a, int num_sms, cudaStream_t st);
// Resolve every kernel that gemm_fixed<double, double> / kn_step_fixed can launch (all operand
// layouts and tile sizes, the split-K reduction, the cooperative step) on the current device, so
// that with lazy module loading no later launch is the first use of a kernel (which loads code and
// may allocate device memory).  Throws on a CUDA error.
void gemm_fixed_preload();
void kn_step_fixed_preload();

}  // namespace isvdb
