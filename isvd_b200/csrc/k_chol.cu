// Small dense FP64 kernels of the QR-based stages and of Wen-Yin integration: batched Cholesky
// with an in-place triangular inverse, the Householder sign rule of a QR factor, batched dot
// products and small linear combinations.  One CTA per l x l matrix, the matrix in shared memory.
#include <algorithm>
#include <cmath>

#include "kernels.h"
#include "runtime.h"

namespace isvdb {
namespace {

constexpr int kCholThreads = 512;

// Sum over the block; every thread returns the same value (same summation order).
__device__ double block_sum(double v, double *red) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  __syncthreads();
  if (lane == 0) red[warp] = v;
  __syncthreads();
  double s = 0.0;
  for (int i = 0; i < nw; ++i) s += red[i];
  return s;
}

// A = alpha W + (shift_abs + shift_rel trace(alpha W)) I from the upper triangle of W (n x n,
// row-major, batch stride n^2).  Cholesky A = R' R (R upper; right-looking), then X = R^-1 in
// place, column by column from the already inverted leading block (the order of LAPACK's trti2).
// A pivot that is not above piv_rel times its starting diagonal value (or is not finite) stops
// the CTA and sets *status = kStatusNotPD.  Output: X with zeros below the diagonal (kCholFactor)
// or out_scale X X' = out_scale A^-1 (kCholInverse).
// null_mask (kCholFactor only; n ints per matrix): a finite pivot at or below the threshold marks
// its column as numerically dependent on the ones before it instead of failing -- the column's row
// of R becomes e_k' (its Schur complement row is zero to rounding) and column k of X is zeroed, so
// Y X has an exact zero column there and the later columns are orthogonalized against the others
// only.  Each newly marked column adds 1 to *null_count.
// perm (n ints per matrix): factor P A P' instead (row / column i of the factored matrix is
// row / column perm[i] of A) and store X at the original positions, out[perm[i], perm[j]] = X[i, j].
// desc (optional): matrix blockIdx.x is desc[blockIdx.x] (its own n, W and out) instead of the
// batch entry of the uniform-size arguments.
__global__ void __launch_bounds__(kCholThreads)
    chol_inv_kernel(int n, const double *__restrict__ W, double alpha, double shift_abs, double shift_rel,
                    double piv_rel, double *__restrict__ out, double out_scale, int mode, int *status,
                    int *__restrict__ null_mask, int *__restrict__ null_count, const int *__restrict__ perm,
                    const CholDesc *__restrict__ desc) {
  extern __shared__ double sm[];
  __shared__ double red[kCholThreads / 32];
  if (desc) n = desc[blockIdx.x].n;
  const int ld = n + 1, tid = threadIdx.x, nt = blockDim.x;
  double *R = sm;                       // n x ld
  double *aux = sm + (size_t)n * ld;    // n: starting diagonal, then the column being inverted
  const double *w = desc ? desc[blockIdx.x].W : W + (size_t)blockIdx.x * n * n;
  const int *pm = perm ? perm + (size_t)blockIdx.x * n : nullptr;
  int *mask = null_mask ? null_mask + (size_t)blockIdx.x * n : nullptr;
  double tr = 0.0;
  for (int e = tid; e < n * n; e += nt) {
    const int i = e / n, j = e - i * n;
    const int pi = pm ? pm[i] : i, pj = pm ? pm[j] : j;
    const double v = alpha * ((pi <= pj) ? w[(size_t)pi * n + pj] : w[(size_t)pj * n + pi]);
    R[i * ld + j] = v;
    if (i == j) tr += v;
  }
  const double shift = shift_abs + shift_rel * block_sum(tr, red);
  for (int i = tid; i < n; i += nt) {
    R[i * ld + i] += shift;
    aux[i] = R[i * ld + i];
  }
  __syncthreads();
  for (int k = 0; k < n; ++k) {
    const double d = R[k * ld + k];
    if (!(d > piv_rel * aux[k]) || !(d > 0.0) || !(d < INFINITY)) {  // same decision in every thread
      if (mask && d == d && d < INFINITY) {  // a dependent column: null, not a failure
        __syncthreads();
        if (tid == 0) {
          R[k * ld + k] = 1.0;
          if (!mask[k]) {
            mask[k] = 1;
            atomicAdd(null_count, 1);
          }
        }
        for (int j = k + 1 + tid; j < n; j += nt) R[k * ld + j] = 0.0;
        __syncthreads();
        continue;  // row k of R is e_k': the Schur update it would make is zero
      }
      if (tid == 0) atomicExch(status, kStatusNotPD);
      return;
    }
    const double r = sqrt(d);
    __syncthreads();
    if (tid == 0) R[k * ld + k] = r;
    for (int j = k + 1 + tid; j < n; j += nt) R[k * ld + j] /= r;
    __syncthreads();
    const int mm = n - k - 1;
    for (int e = tid; e < mm * mm; e += nt) {
      const int i = k + 1 + e / mm, j = k + 1 + e % mm;
      if (j >= i) R[i * ld + j] -= R[k * ld + i] * R[k * ld + j];
    }
    __syncthreads();
  }
  // X(0:j, j) = -X(0:j, 0:j) R(0:j, j) / r_jj ;  x_jj = 1 / r_jj.  Four threads per row.
  const int quad = tid >> 2, ql = tid & 3, nq = nt >> 2;
  for (int j = 0; j < n; ++j) {
    const double inv = 1.0 / R[j * ld + j];
    for (int i = tid; i < j; i += nt) aux[i] = R[i * ld + j];
    __syncthreads();
    for (int i0 = 0; i0 < j; i0 += nq) {
      const int i = i0 + quad;
      double acc = 0.0;
      if (i < j)
        for (int k = i + ql; k < j; k += 4) acc += R[i * ld + k] * aux[k];
      acc += __shfl_xor_sync(0xffffffffu, acc, 1);
      acc += __shfl_xor_sync(0xffffffffu, acc, 2);
      if (i < j && ql == 0) R[i * ld + j] = -inv * acc;
    }
    if (tid == 0) R[j * ld + j] = inv;
    __syncthreads();
  }
  double *o = desc ? desc[blockIdx.x].out : out + (size_t)blockIdx.x * n * n;
  if (mode == kCholFactor) {
    for (int e = tid; e < n * n; e += nt) {
      const int i = e / n, j = e - i * n;
      const double v = (j >= i && !(mask && mask[j])) ? out_scale * R[i * ld + j] : 0.0;
      if (pm) o[(size_t)pm[i] * n + pm[j]] = v;
      else o[e] = v;
    }
  } else {
    for (int e = tid; e < n * n; e += nt) {
      const int i = e / n, j = e - i * n;
      double acc = 0.0;
      for (int k = (i > j ? i : j); k < n; ++k) acc += R[i * ld + k] * R[j * ld + k];
      o[e] = out_scale * acc;
    }
  }
}

// out = out_scale A^-1 for A = alpha W + shift I (upper triangle of W, n x n, one CTA per matrix) by
// the sweep operator (Goodnight, "A tutorial on the SWEEP operator", Amer. Statist. 33 (1979)):
// sweeping pivot k maps a_kk -> -1/a_kk, a_ik -> a_ik/a_kk, a_ij -> a_ij - a_ik a_kj / a_kk; after
// all pivots the matrix is -A^-1.  For a symmetric positive definite A the pivots are the Cholesky
// pivots (Schur-complement diagonals), so the elimination needs no pivoting; one pivot that is not
// above piv_rel times its starting diagonal value sets *status = kStatusNotPD.  Symmetry halves the
// per-pivot reads: row k equals column k.
constexpr int kSwThreads = 1024;

__global__ void __launch_bounds__(kSwThreads)
    spd_inverse_kernel(int n, const double *__restrict__ W, double alpha, double shift, double piv_rel,
                       double *__restrict__ out, double out_scale, int *status) {
  extern __shared__ double sm[];
  const int ld = n + 1, tid = threadIdx.x;
  double *A = sm, *col = sm + (size_t)n * ld, *diag0 = col + n;
  const double *w = W + (size_t)blockIdx.x * n * n;
  const int tx = tid & 31, ty = tid >> 5;  // element (ty + 32 a, tx + 32 b)
  for (int i = ty; i < n; i += 32)
    for (int j = tx; j < n; j += 32) {
      const double v = alpha * ((i <= j) ? w[(size_t)i * n + j] : w[(size_t)j * n + i]) + (i == j ? shift : 0.0);
      A[i * ld + j] = v;
      if (i == j) diag0[i] = v;
    }
  __syncthreads();
  for (int k = 0; k < n; ++k) {
    for (int i = tid; i < n; i += kSwThreads) col[i] = A[i * ld + k];
    __syncthreads();
    const double d = col[k];
    if (!(d > piv_rel * diag0[k]) || !(d > 0.0) || !(d < INFINITY)) {  // same decision in every thread
      if (tid == 0) atomicExch(status, kStatusNotPD);
      return;
    }
    const double inv = 1.0 / d;
    for (int i = ty; i < n; i += 32) {
      const double ci = col[i];
      for (int j = tx; j < n; j += 32) {
        double v;
        if (i == k) v = (j == k) ? -inv : col[j] * inv;
        else if (j == k) v = ci * inv;
        else v = A[i * ld + j] - ci * col[j] * inv;
        A[i * ld + j] = v;
      }
    }
    __syncthreads();
  }
  double *o = out + (size_t)blockIdx.x * n * n;
  for (int i = ty; i < n; i += 32)
    for (int j = tx; j < n; j += 32) o[(size_t)i * n + j] = -out_scale * A[i * ld + j];
}

// Householder sign rule.  P = Qtop X is the top n x n block of the next Q factor (positive-
// diagonal convention).  A Householder QR (LAPACK geqrf / gelqf) of the same matrix returns
// Q diag(s) with s_j = -sign(pivot_j) of the LU factorization of P - diag(s) carried out with
// exactly that choice of s (Ballard, Demmel, Grigori, Jacquelin, Knight, Nguyen, "Reconstructing
// Householder vectors from tall-skinny QR", J. Parallel Distrib. Comput. 85 (2015)).  X's
// columns are multiplied by s, so that Q X is the Householder factor.
template <class T>
__global__ void __launch_bounds__(kCholThreads)
    hh_sign_kernel(int n, const T *__restrict__ Q, long long q_ld, long long q_bs, double *__restrict__ X) {
  extern __shared__ double sm[];
  const int ld = n + 1, tid = threadIdx.x, nt = blockDim.x;
  double *P = sm, *sg = sm + (size_t)n * ld;
  const T *q = Q + blockIdx.x * q_bs;
  double *x = X + (size_t)blockIdx.x * n * n;
  for (int e = tid; e < n * n; e += nt) {
    const int i = e / n, j = e - i * n;
    double acc = 0.0;
    for (int k = 0; k <= j; ++k) acc += (double)q[i * q_ld + k] * x[(size_t)k * n + j];
    P[i * ld + j] = acc;
  }
  __syncthreads();
  for (int j = 0; j < n; ++j) {
    const double piv = P[j * ld + j];
    const double s = (piv >= 0.0) ? -1.0 : 1.0;
    const double u = piv - s;  // |u| >= 1
    __syncthreads();
    if (tid == 0) sg[j] = s;
    for (int i = j + 1 + tid; i < n; i += nt) P[i * ld + j] /= u;
    __syncthreads();
    const int mm = n - j - 1;
    for (int e = tid; e < mm * mm; e += nt) {
      const int i = j + 1 + e / mm, c = j + 1 + e % mm;
      P[i * ld + c] -= P[i * ld + j] * P[j * ld + c];
    }
    __syncthreads();
  }
  for (int e = tid; e < n * n; e += nt) x[e] *= sg[e % n];
}

constexpr int kDotThreads = 256;
constexpr int kDotBlocks = 64;  // CTAs per job; partial sums combined in a fixed order

// Partial sums: CTA (x, job) sums the entries x, x + kDotBlocks, ... (in units of its thread count).
__global__ void __launch_bounds__(kDotThreads) dots_kernel(DotJobs jobs, double *__restrict__ partial) {
  __shared__ double red[kDotThreads / 32];
  const DotJob jb = jobs.job[blockIdx.y];
  const long long stride = (long long)gridDim.x * blockDim.x;
  double v = 0.0;
  if (jb.trace) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < jb.n; i += stride) v += jb.a[i * jb.n + i];
  } else {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < jb.n; i += stride) {
      const double x = jb.a[i] - (jb.b ? jb.b[i] : 0.0);
      const double y = jb.c[i] - (jb.d ? jb.d[i] : 0.0);
      v += x * y;
    }
  }
  v = block_sum(v, red);
  if (threadIdx.x == 0) partial[blockIdx.y * gridDim.x + blockIdx.x] = v;
}

__global__ void dots_final_kernel(const double *__restrict__ partial, int nblocks, int count, double *__restrict__ out) {
  const int j = threadIdx.x;
  if (j < count) {
    double s = 0.0;
    for (int b = 0; b < nblocks; ++b) s += partial[j * nblocks + b];
    out[j] = s;
  }
}

// (out may alias x or y: each entry is read and written by the same thread)
__global__ void lincomb_kernel(double *out, const double *x, double a, const double *y, double b, double c,
                               long long rows, long long cols) {
  const long long total = rows * cols;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
       e += (long long)gridDim.x * blockDim.x) {
    const long long i = e / cols, j = e - i * cols;
    double v = (i == j) ? c : 0.0;
    if (x) v += a * x[e];
    if (y) v += b * y[e];
    out[e] = v;
  }
}

__global__ void copy_diag_blocks_kernel(const double *__restrict__ G, int Nl, int l, int N, double *__restrict__ out) {
  const long long total = (long long)N * l * l;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
       e += (long long)gridDim.x * blockDim.x) {
    const long long b = e / ((long long)l * l), r = e - b * l * l;
    const long long i = r / l, j = r - i * l;
    out[e] = G[(b * l + i) * Nl + b * l + j];
  }
}

// d_i = num / (half * max(lambda_i, 0) + add)
__global__ void recip_affine_kernel(const double *__restrict__ lam, int n, double num, double half, double add,
                                    double *__restrict__ d) {
  for (int i = threadIdx.x; i < n; i += blockDim.x) d[i] = num / (half * fmax(lam[i], 0.0) + add);
}

size_t chol_smem(int n) { return ((size_t)n * (n + 1) + n) * sizeof(double); }

}  // namespace

void chol_inv_batched(int n, int batch, const double *W, double alpha, double shift_abs, double shift_rel,
                      double piv_rel, double *out, double out_scale, int mode, int *status, cudaStream_t st,
                      int *null_mask, int *null_count, const int *perm) {
  if (n <= 0 || batch <= 0) return;
  if ((null_mask || perm) && mode != kCholFactor) fail(kErrArgument, "Cholesky: null columns / permutation need kCholFactor");
  if (null_mask && !null_count) fail(kErrArgument, "Cholesky: a null-column mask needs its counter");
  if (mode == kCholInverse && shift_rel == 0.0) {  // the full inverse: sweep operator, fewer dependent steps
    const size_t smem = ((size_t)n * (n + 1) + 2 * n) * sizeof(double);
    if (smem > Runtime::get().smem_optin) fail(kErrUnsupported, "SPD inverse: l = %d exceeds on-chip capacity", n);
    CK(cudaFuncSetAttribute(spd_inverse_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    spd_inverse_kernel<<<batch, kSwThreads, smem, st>>>(n, W, alpha, shift_abs, piv_rel, out, out_scale, status);
    KLAUNCHED();
    return;
  }
  const size_t smem = chol_smem(n);
  if (smem > Runtime::get().smem_optin) fail(kErrUnsupported, "Cholesky: l = %d exceeds on-chip capacity", n);
  CK(cudaFuncSetAttribute(chol_inv_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  chol_inv_kernel<<<batch, kCholThreads, smem, st>>>(n, W, alpha, shift_abs, shift_rel, piv_rel, out, out_scale,
                                                     mode, status, null_mask, null_count, perm, nullptr);
  KLAUNCHED();
}

void chol_inv_grouped(const CholDesc *desc, int count, int max_n, int *status, cudaStream_t st) {
  if (count <= 0 || max_n <= 0) return;
  const size_t smem = chol_smem(max_n);
  if (smem > Runtime::get().smem_optin) fail(kErrUnsupported, "Cholesky: l = %d exceeds on-chip capacity", max_n);
  CK(cudaFuncSetAttribute(chol_inv_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  chol_inv_kernel<<<count, kCholThreads, smem, st>>>(0, nullptr, 1.0, 0.0, 0.0, 0.0, nullptr, 1.0, kCholFactor, status,
                                                     nullptr, nullptr, nullptr, desc);
  KLAUNCHED();
}

template <class T>
void hh_sign_batched(int n, int batch, const T *Q, long long q_ld, long long q_bs, double *X, cudaStream_t st) {
  if (n <= 0 || batch <= 0) return;
  const size_t smem = chol_smem(n);
  if (smem > Runtime::get().smem_optin) fail(kErrUnsupported, "QR sign rule: l = %d exceeds on-chip capacity", n);
  CK(cudaFuncSetAttribute(hh_sign_kernel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  hh_sign_kernel<T><<<batch, kCholThreads, smem, st>>>(n, Q, q_ld, q_bs, X);
  KLAUNCHED();
}

void dots(const DotJobs &jobs, double *out, cudaStream_t st) {
  if (jobs.count <= 0) return;
  if (jobs.count > kMaxDotJobs) fail(kErrArgument, "dots: %d jobs > %d", jobs.count, kMaxDotJobs);
  DBuf<double> partial((size_t)kDotBlocks * jobs.count);
  dots_kernel<<<dim3(kDotBlocks, jobs.count), kDotThreads, 0, st>>>(jobs, partial.p);
  KLAUNCHED();
  dots_final_kernel<<<1, 32, 0, st>>>(partial.p, kDotBlocks, jobs.count, out);
  KLAUNCHED();
}

void lincomb(double *out, const double *x, double a, const double *y, double b, double c, long long rows,
             long long cols, cudaStream_t st) {
  if (rows <= 0 || cols <= 0) return;
  const long long total = rows * cols;
  const int grid = (int)std::min<long long>((total + 255) / 256, 8LL * Runtime::get().num_sms);
  lincomb_kernel<<<grid, 256, 0, st>>>(out, x, a, y, b, c, rows, cols);
  KLAUNCHED();
}

void copy_diag_blocks(const double *G, int Nl, int l, int N, double *out, cudaStream_t st) {
  const long long total = (long long)N * l * l;
  if (total <= 0) return;
  const int grid = (int)std::min<long long>((total + 255) / 256, 8LL * Runtime::get().num_sms);
  copy_diag_blocks_kernel<<<grid, 256, 0, st>>>(G, Nl, l, N, out);
  KLAUNCHED();
}

void recip_affine(const double *lam, int n, double num, double half, double add, double *d, cudaStream_t st) {
  if (n <= 0) return;
  recip_affine_kernel<<<1, 256, 0, st>>>(lam, n, num, half, add, d);
  KLAUNCHED();
}

template void hh_sign_batched<double>(int, int, const double *, long long, long long, double *, cudaStream_t);
template void hh_sign_batched<float>(int, int, const float *, long long, long long, double *, cudaStream_t);

}  // namespace isvdb
