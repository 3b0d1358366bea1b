// Small dense FP64 linear algebra on l x l matrices (l <= 160), kept on chip:
//   * batched symmetric eigendecomposition (parallel cyclic two-sided Jacobi),
//   * batched general SVD (parallel cyclic one-sided Jacobi, Hestenes),
//   * the Kolmogorov-Nagumo step C = (I/2 + (I/4 - Z)^(1/2))^(1/2) by coupled Newton-Schulz
//     iterations in one cooperative multi-CTA kernel.
// These replace LAPACK gesvd/syev (reference la/lapack/gesvd.c, syev.c) on the stages' l x l
// matrices.  Jacobi methods are used because they are accurate to working precision in the
// eigenvectors and map onto one CTA; rotation order is the round-robin tournament, so each
// round applies l/2 disjoint rotations in parallel.
#include <cooperative_groups.h>

#include <algorithm>
#include <cmath>
#include <cstdlib>

#include "kernels.h"
#include "kn_common.cuh"
#include "runtime.h"

namespace isvdb {
namespace {

constexpr int kEigThreads = 1024;
constexpr int kMaxSweeps = 60;

// Round-robin tournament: player i at round r (ne even, player 0 fixed).
__device__ __forceinline__ int rr_player(int i, int r, int ne) { return i == 0 ? 0 : 1 + (i - 1 + r) % (ne - 1); }

// Rotation (c, s) annihilating the off-diagonal of [[app, apq], [apq, aqq]] with
// R = [[c, s], [-s, c]] (Golub & Van Loan, Matrix Computations, Alg. 8.4.1 sym.schur2).
// No rotation when |apq| is below tol * max(sqrt(|app aqq|), floor): relative accuracy for the
// well-scaled pairs, and a floor (eps * ||A||_F) that guarantees termination for the pairs of
// eigenvalues that are negligible against ||A||.
__device__ __forceinline__ bool jacobi_rot(double app, double aqq, double apq, double tol, double floor_,
                                           double &c, double &s) {
  if (fabs(apq) <= tol * fmax(sqrt(fabs(app) * fabs(aqq)), floor_)) {
    c = 1.0;
    s = 0.0;
    return false;
  }
  // t = tan(theta) = sign(d) 2 apq / (|d| + sqrt(d^2 + 4 apq^2)), d = aqq - app: the smaller root of
  // t^2 + (d / apq) t - 1 = 0, with one square root, one division and one reciprocal square root
  const double d = aqq - app, e = 2.0 * apq;
  const double t = (d >= 0.0 ? e : -e) / (fabs(d) + sqrt(d * d + e * e));
  c = rsqrt(1.0 + t * t);
  s = t * c;
  return true;
}

constexpr double kEps = 2.220446049250313e-16;

// Two-sided Jacobi on a symmetric n x n matrix held packed (upper triangle, row by row) in shared
// memory, with the eigenvector matrix held transposed (row i = eigenvector i) in shared memory when
// it fits (VS = true) or in the output buffer otherwise.  Each round rotates n/2 disjoint pairs:
// the 2 x 2 blocks of A on pair rows x pair columns are updated independently (each packed entry
// belongs to exactly one block), and the rotation acts on two rows of V' (contiguous, conflict-free).
__device__ __forceinline__ int pk(int i, int j, int n) {
  if (i > j) { const int t = i; i = j; j = t; }
  return i * n - (i * (i - 1)) / 2 + (j - i);
}

// Largest n a CTA of nt threads solves: each thread keeps a fixed list of at most
// eig_max_mine(nt) of the np (np + 1) / 2 block updates of a round (np = ceil(n / 2)).
constexpr int eig_max_n(int nt) { return nt >= 1024 ? 160 : nt >= 512 ? 96 : nt >= 256 ? 64 : 32; }
constexpr int eig_max_mine(int nt) {
  return ((eig_max_n(nt) / 2) * (eig_max_n(nt) / 2 + 1) / 2 + nt - 1) / nt;
}

// One CTA of NT threads per matrix: batch b at Ag + b n^2 (uniform n), or, with desc, the matrix
// desc[b] (its own n <= eig_max_n(NT)).
template <bool VS, int NT = kEigThreads>
__global__ void __launch_bounds__(NT)
    sym_eig_kernel(int n_uniform, const double *__restrict__ Ag, double *__restrict__ Vg, double *__restrict__ wg,
                   int order, bool absval, double *__restrict__ scratch, int *status, const EigDesc *desc) {
  extern __shared__ double sm[];
  const int b = blockIdx.x, tid = threadIdx.x, nt = blockDim.x;
  const int n = desc ? desc[b].n : n_uniform;
  const double *A0 = desc ? desc[b].A : Ag + (size_t)b * n * n;
  double *V = desc ? desc[b].V : Vg + (size_t)b * n * n;
  double *w = desc ? desc[b].w : wg + (size_t)b * n;
  const int ne = n + (n & 1), np = ne / 2;
  const int npk = n * (n + 1) / 2;
  double *A = sm;                                                           // packed upper triangle
  double *Vt = VS ? (A + ((npk + 1) & ~1)) : (scratch + (size_t)b * n * n);  // V' (row i = eigenvector i)
  double *rc = VS ? (Vt + (size_t)n * n) : (A + ((npk + 1) & ~1));
  double *rs = rc + np;
  double *key = rs + np;
  int *pp = (int *)(key + n);
  int *qq = pp + np;
  int *flag = qq + np;

  __shared__ double red[NT];
  double fr = 0.0;
  for (int e = tid; e < n * n; e += nt) {
    const int i = e / n, j = e - i * n;
    if (i <= j) {
      const double v = 0.5 * (A0[i * n + j] + A0[j * n + i]);
      A[pk(i, j, n)] = v;
      fr += (i == j ? 1.0 : 2.0) * v * v;
    }
    Vt[e] = (i == j) ? 1.0 : 0.0;
  }
  red[tid] = fr;
  __syncthreads();
  for (int h = nt / 2; h > 0; h >>= 1) {
    if (tid < h) red[tid] += red[tid + h];
    __syncthreads();
  }
  const double tol = kEps * fmax(1.0, sqrt((double)n));
  const double floor_ = kEps * sqrt(red[0]);
  __syncthreads();

  const int nblk = np * (np + 1) / 2;
  const int lane = tid & 31, warp = tid >> 5, nwarp = nt >> 5;
  constexpr int kMaxMine = eig_max_mine(NT);  // n <= 160, NT = 1024: np <= 80, nblk <= 3240
  short myI[kMaxMine], myJ[kMaxMine];
  int nmy = 0;
  for (int e = tid; e < nblk && nmy < kMaxMine; e += nt) {
    int I = (int)((sqrt(8.0 * e + 1.0) - 1.0) * 0.5);
    while ((I + 1) * (I + 2) / 2 <= e) ++I;
    while (I * (I + 1) / 2 > e) --I;
    myI[nmy] = (short)I;
    myJ[nmy] = (short)(e - I * (I + 1) / 2);
    ++nmy;
  }
  int sweep = 0;
  for (; sweep < kMaxSweeps; ++sweep) {
    if (tid == 0) *flag = 0;
    __syncthreads();
    for (int r = 0; r < ne - 1; ++r) {
      for (int k = tid; k < np; k += nt) {
        int p = rr_player(k, r, ne), q = rr_player(ne - 1 - k, r, ne);
        if (p > q) { const int t = p; p = q; q = t; }
        double c = 1.0, sn = 0.0;
        if (q < n && jacobi_rot(A[pk(p, p, n)], A[pk(q, q, n)], A[pk(p, q, n)], tol, floor_, c, sn)) *flag = 1;
        pp[k] = p; qq[k] = q; rc[k] = c; rs[k] = sn;
      }
      __syncthreads();
      // A := R' A R, one 2 x 2 block (pair J rows x pair I columns, J <= I) per work item; the
      // block list of each thread is fixed (decoded once, below the sweep loop)
#pragma unroll 1
      for (int u = 0; u < nmy; ++u) {
        const int I = myI[u], J = myJ[u];
        const double si = rs[J], sj = rs[I];
        if (si == 0.0 && sj == 0.0) continue;
        const int pi = pp[J], qi = qq[J], pj = pp[I], qj = qq[I];
        const double ci = rc[J], cj = rc[I];
        const bool qiv = qi < n, qjv = qj < n;
        if (I == J) {
          if (!qiv) continue;
          const int ipp = pk(pi, pi, n), iqq = pk(qi, qi, n), ipq = pk(pi, qi, n);
          const double app = A[ipp], aqq = A[iqq], apq = A[ipq];
          const double t = si / ci;  // rotated 2 x 2 diagonal block: off-diagonal annihilated
          A[ipp] = app - t * apq;
          A[iqq] = aqq + t * apq;
          A[ipq] = 0.0;
          continue;
        }
        const int i11 = pk(pi, pj, n);
        const int i12 = qjv ? pk(pi, qj, n) : 0;
        const int i21 = qiv ? pk(qi, pj, n) : 0;
        const int i22 = (qiv && qjv) ? pk(qi, qj, n) : 0;
        const double x11 = A[i11];
        const double x12 = qjv ? A[i12] : 0.0;
        const double x21 = qiv ? A[i21] : 0.0;
        const double x22 = (qiv && qjv) ? A[i22] : 0.0;
        const double y11 = ci * x11 - si * x21, y12 = ci * x12 - si * x22;
        const double y21 = si * x11 + ci * x21, y22 = si * x12 + ci * x22;
        A[i11] = y11 * cj - y12 * sj;
        if (qjv) A[i12] = y11 * sj + y12 * cj;
        if (qiv) A[i21] = y21 * cj - y22 * sj;
        if (qiv && qjv) A[i22] = y21 * sj + y22 * cj;
      }
      // V' := R' V' : rows p and q of V'; warp w takes pairs w, w + nwarp, ..., each lane a
      // strided set of columns
      for (int k = warp; k < np; k += nwarp) {
        const double sn = rs[k];
        if (sn == 0.0) continue;
        const double c = rc[k];
        double *vp = Vt + (size_t)pp[k] * n, *vq = Vt + (size_t)qq[k] * n;
        for (int col = lane; col < n; col += 32) {
          const double v1 = vp[col], v2 = vq[col];
          vp[col] = c * v1 - sn * v2;
          vq[col] = sn * v1 + c * v2;
        }
      }
      __syncthreads();
    }
    const int f = *flag;
    __syncthreads();
    if (!f) break;
    // the next sweep would rotate nothing when every pair is below the threshold: stop here
    if (tid == 0) *flag = 0;
    __syncthreads();
    for (int i = warp; i < n; i += nwarp) {
      const double aii = fabs(A[pk(i, i, n)]);
      for (int j = i + 1 + lane; j < n; j += 32)
        if (fabs(A[pk(i, j, n)]) > tol * fmax(sqrt(aii * fabs(A[pk(j, j, n)])), floor_)) *flag = 1;
    }
    __syncthreads();
    const int g = *flag;
    __syncthreads();
    if (!g) break;
  }
  if (sweep == kMaxSweeps && tid == 0) atomicExch(status, kErrNumerical);

  // Sort eigenpairs: order > 0 by |lambda| descending, order < 0 by lambda ascending; write the
  // eigenvectors as the columns of V (row-major).
  for (int i = tid; i < n; i += nt) key[i] = A[pk(i, i, n)];
  __syncthreads();
  for (int i = tid; i < n; i += nt) {
    const double ki = key[i];
    int rank = 0;
    for (int j = 0; j < n; ++j) {
      const double kj = key[j];
      const bool before = (order > 0) ? (fabs(kj) > fabs(ki) || (fabs(kj) == fabs(ki) && j < i))
                                      : (kj < ki || (kj == ki && j < i));
      rank += before;
    }
    w[rank] = absval ? fabs(ki) : ki;
    for (int r2 = 0; r2 < n; ++r2) V[r2 * n + rank] = Vt[i * n + r2];
  }
}

// One-sided Jacobi SVD: B (row-major n x n) -> U diag(s) V'.
// Columns of B are held column-major in shared memory; V in global memory (this CTA only).
__global__ void __launch_bounds__(kEigThreads)
    svd_jacobi_kernel(int n, const double *__restrict__ Bg, double *__restrict__ Ug, double *__restrict__ sg,
                      double *__restrict__ Vg, int *status) {
  extern __shared__ double sm[];
  const int b = blockIdx.x, tid = threadIdx.x, nt = blockDim.x;
  const int lane = tid & 31, warp = tid >> 5, nwarp = nt >> 5;
  const double *B0 = Bg + (size_t)b * n * n;
  double *U = Ug + (size_t)b * n * n;
  double *V = Vg + (size_t)b * n * n;
  double *s = sg + (size_t)b * n;
  const int ne = n + (n & 1), np = ne / 2;
  double *X = sm;                  // column-major: X[j * n + i] = B(i, j)
  double *nrm = X + n * n;         // n
  int *flag = (int *)(nrm + n);

  __shared__ double red[kEigThreads];
  double fr = 0.0;
  for (int e = tid; e < n * n; e += nt) {
    const int i = e / n, j = e - i * n;
    X[j * n + i] = B0[e];
    fr += B0[e] * B0[e];
    V[e] = (i == j) ? 1.0 : 0.0;
  }
  red[tid] = fr;
  __syncthreads();
  for (int h = nt / 2; h > 0; h >>= 1) {
    if (tid < h) red[tid] += red[tid + h];
    __syncthreads();
  }
  const double tol = kEps * fmax(1.0, sqrt((double)n));
  const double floor2 = kEps * kEps * red[0];  // ||B||_F^2 eps^2
  __syncthreads();
  int sweep = 0;
  for (; sweep < kMaxSweeps; ++sweep) {
    if (tid == 0) *flag = 0;
    __syncthreads();
    for (int r = 0; r < ne - 1; ++r) {
      for (int k = warp; k < np; k += nwarp) {
        int p = rr_player(k, r, ne), q = rr_player(ne - 1 - k, r, ne);
        if (p > q) { const int t = p; p = q; q = t; }
        if (q >= n) continue;
        double al = 0.0, be = 0.0, ga = 0.0;
        for (int i = lane; i < n; i += 32) {
          const double xp = X[p * n + i], xq = X[q * n + i];
          al += xp * xp; be += xq * xq; ga += xp * xq;
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
          al += __shfl_xor_sync(0xffffffffu, al, o);
          be += __shfl_xor_sync(0xffffffffu, be, o);
          ga += __shfl_xor_sync(0xffffffffu, ga, o);
        }
        if (fabs(ga) <= tol * fmax(sqrt(al * be), floor2)) continue;
        if (lane == 0) *flag = 1;
        const double zeta = (be - al) / (2.0 * ga);
        const double t = (zeta >= 0.0 ? 1.0 : -1.0) / (fabs(zeta) + sqrt(1.0 + zeta * zeta));
        const double c = 1.0 / sqrt(1.0 + t * t), sn = t * c;
        for (int i = lane; i < n; i += 32) {
          const double xp = X[p * n + i], xq = X[q * n + i];
          X[p * n + i] = c * xp - sn * xq;
          X[q * n + i] = sn * xp + c * xq;
          const double vp = V[i * n + p], vq = V[i * n + q];
          V[i * n + p] = c * vp - sn * vq;
          V[i * n + q] = sn * vp + c * vq;
        }
      }
      __syncthreads();
    }
    const int f = *flag;
    __syncthreads();
    if (!f) break;
  }
  if (sweep == kMaxSweeps && tid == 0) atomicExch(status, kErrNumerical);
  for (int j = warp; j < n; j += nwarp) {
    double a = 0.0;
    for (int i = lane; i < n; i += 32) a += X[j * n + i] * X[j * n + i];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) a += __shfl_xor_sync(0xffffffffu, a, o);
    if (lane == 0) nrm[j] = sqrt(a);
  }
  __syncthreads();
  // sort by singular value descending; write U = X / s (row-major) and permuted V.
  for (int j = tid; j < n; j += nt) {
    const double sj = nrm[j];
    int rank = 0;
    for (int k = 0; k < n; ++k) rank += (nrm[k] > sj) || (nrm[k] == sj && k < j);
    s[rank] = sj;
    const double inv = sj > 0.0 ? 1.0 / sj : 0.0;
    for (int i = 0; i < n; ++i) U[i * n + rank] = X[j * n + i] * inv;
  }
  __syncthreads();
  // permute V columns through shared memory (X no longer needed)
  for (int j = tid; j < n; j += nt) {
    const double sj = nrm[j];
    int rank = 0;
    for (int k = 0; k < n; ++k) rank += (nrm[k] > sj) || (nrm[k] == sj && k < j);
    for (int i = 0; i < n; ++i) X[i * n + rank] = V[i * n + j];
  }
  __syncthreads();
  for (int e = tid; e < n * n; e += nt) V[e] = X[e];
}

// ------------------------------------------------------------------------------------------
// Cooperative Kolmogorov-Nagumo step.

constexpr int kKnThreads = 256;
constexpr long long kSpinLimit = 1LL << 22;  // ~0.5-2 s of polling before giving up

// Grid-wide barrier for a cooperative launch.  bar[0] counts arrivals, bar[1] is the generation.
// Every wait is bounded; on expiry the status word is set and all CTAs leave the kernel.
__device__ bool grid_barrier(unsigned int *bar, int *status) {
  __shared__ int ok;
  __syncthreads();
  if (threadIdx.x == 0) {
    volatile unsigned int *gen = bar + 1;
    const unsigned int g = *gen;
    __threadfence();
    const unsigned int t = atomicAdd(bar, 1u);
    if (t == gridDim.x - 1) {
      atomicExch(bar, 0u);
      __threadfence();
      atomicAdd(bar + 1, 1u);
    } else {
      long long spins = 0;
      while (*gen == g) {
        if (++spins > kSpinLimit) { atomicExch(status, kErrTimeout); break; }
        if (*(volatile int *)status) break;
        __nanosleep(64);
      }
    }
    __threadfence();
    ok = (*(volatile int *)status == 0);
  }
  __syncthreads();
  return ok;
}

// C = alpha * A * B + beta * Cin + diag * I over 16 x 16 tiles (row-major l x l, ld l).
// All operands may have been written by other CTAs in earlier phases: loads go through L2.
__device__ void mm_tiles(int l, int ntile_row, int tile_begin, int tile_end, double alpha, const double *A,
                         const double *B, double beta, const double *Cin, double diag, double *C) {
  __shared__ double As[16][161];
  __shared__ double Bs[160][17];
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
  // tiles are numbered globally across the products of one phase (tile ranges [tile_begin,
  // tile_end)), so that products of a phase run on different CTAs: CTA b takes tiles t = b mod grid
  const int G = gridDim.x;
  const int first = tile_begin + ((((int)blockIdx.x - tile_begin) % G) + G) % G;
  for (int t = first; t < tile_end; t += G) {
    const int tt = t - tile_begin;
    const int i0 = (tt / ntile_row) * 16, j0 = (tt % ntile_row) * 16;
    // all loads of the tile, Cin included, are issued before any is used (one L2 round trip)
    const double cin = (beta != 0.0 && i0 + ty < l && j0 + tx < l) ? __ldcg(Cin + (size_t)(i0 + ty) * l + j0 + tx)
                                                                    : 0.0;
    constexpr int kPer = (16 * 160 + kKnThreads - 1) / kKnThreads;
    double ra[kPer], rb[kPer];
#pragma unroll
    for (int u = 0; u < kPer; ++u) {
      const int e = threadIdx.x + u * kKnThreads;
      const int r = e / l, k = e - r * l;
      ra[u] = (e < 16 * l && i0 + r < l) ? __ldcg(A + (size_t)(i0 + r) * l + k) : 0.0;
      const int kb = e / 16, cb = e - kb * 16;
      rb[u] = (e < 16 * l && j0 + cb < l) ? __ldcg(B + (size_t)kb * l + j0 + cb) : 0.0;
    }
    __syncthreads();
#pragma unroll
    for (int u = 0; u < kPer; ++u) {
      const int e = threadIdx.x + u * kKnThreads;
      if (e < 16 * l) {
        const int r = e / l, k = e - r * l;
        As[r][k] = ra[u];
        const int kb = e / 16, cb = e - kb * 16;
        Bs[kb][cb] = rb[u];
      }
    }
    __syncthreads();
    const int i = i0 + ty, j = j0 + tx;
    double acc = 0.0;
    for (int k = 0; k < l; ++k) acc = fma(As[ty][k], Bs[k][tx], acc);
    if (i < l && j < l) {
      double v = alpha * acc;
      if (beta != 0.0) v += beta * cin;
      if (i == j) v += diag;
      C[(size_t)i * l + j] = v;
    }
  }
}

__global__ void __launch_bounds__(kKnThreads) kn_step_kernel(KnStep a) {
  const int l = a.l;
  const size_t ll = (size_t)l * l;
  double *Zm = a.work, *Y0 = Zm + ll, *Y1 = Y0 + ll, *Q0 = Y1 + ll, *Q1 = Q0 + ll, *T = Q1 + ll;
  double *scal = a.work + 8 * ll;  // [0] rho, [1] k
  const int nr = (l + 15) / 16, nt = nr * nr;
  __shared__ double red[kKnThreads];

  // Z = Dgc - Dc Dc (reference :184-190)
  mm_tiles(l, nr, 0, nt, -1.0, a.Dc, a.Dc, 1.0, a.Dgc, 0.0, Zm);
  if (!grid_barrier(a.bar, a.status)) return;
  // X = I - 4 Zsym (upper triangle of Z, as syev 'U' reads it); Y0 = X, Q0 = I.
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < ll; e += (size_t)gridDim.x * blockDim.x) {
    const int i = (int)(e / l), j = (int)(e % l);
    const double z = __ldcg(Zm + (size_t)min(i, j) * l + max(i, j));
    Y0[e] = (i == j ? 1.0 : 0.0) - 4.0 * z;
    Q0[e] = (i == j ? 1.0 : 0.0);
  }
  if (blockIdx.x == 0) {
    // rho = min(||4Z||_F, ||4Z||_inf): deterministic (single CTA)
    double f = 0.0;
    for (size_t e = threadIdx.x; e < ll; e += blockDim.x) {
      const int i = (int)(e / l), j = (int)(e % l);
      const double z = __ldcg(Zm + (size_t)min(i, j) * l + max(i, j));
      f += 16.0 * z * z;
    }
    red[threadIdx.x] = f;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
      if (threadIdx.x < s) red[threadIdx.x] += red[threadIdx.x + s];
      __syncthreads();
    }
    const double fro = sqrt(red[0]);
    __syncthreads();
    double rmax = 0.0;
    for (int i = threadIdx.x; i < l; i += blockDim.x) {
      double rs = 0.0;
      for (int j = 0; j < l; ++j) rs += fabs(4.0 * __ldcg(Zm + (size_t)min(i, j) * l + max(i, j)));
      rmax = fmax(rmax, rs);
    }
    red[threadIdx.x] = rmax;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
      if (threadIdx.x < s) red[threadIdx.x] = fmax(red[threadIdx.x], red[threadIdx.x + s]);
      __syncthreads();
    }
    if (threadIdx.x == 0) {
      const double rho = fmin(fro, red[0]);
      scal[0] = rho;
      scal[1] = (double)kn_ns_steps(rho, a.ns_target);
    }
  }
  if (!grid_barrier(a.bar, a.status)) return;

  // Two coupled Newton-Schulz square roots (Higham, Functions of Matrices, eq. 6.35):
  //   T = Q Y;  Y <- Y (3I - T)/2;  Q <- (3I - T) Q / 2   ->  Y -> X^(1/2), Q -> X^(-1/2).
  for (int stage = 0; stage < 2; ++stage) {
    const int k = (int)__ldcg(scal + 1);
    double *Y = Y0, *Yn = Y1, *Q = Q0, *Qn = Q1;
    for (int it = 0; it < k; ++it) {
      mm_tiles(l, nr, 0, nt, 1.0, Q, Y, 0.0, nullptr, 0.0, T);
      if (!grid_barrier(a.bar, a.status)) return;
      mm_tiles(l, nr, 0, nt, -0.5, Y, T, 1.5, Y, 0.0, Yn);
      mm_tiles(l, nr, nt, 2 * nt, -0.5, T, Q, 1.5, Q, 0.0, Qn);
      if (!grid_barrier(a.bar, a.status)) return;
      double *t1 = Y; Y = Yn; Yn = t1;
      double *t2 = Q; Q = Qn; Qn = t2;
    }
    if (stage == 0) {
      // sqrt(I/4 - Z) = Y / 2 ;  P = I/2 + Y/2 ; next: Y0 = P, Q0 = I
      for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < ll; e += (size_t)gridDim.x * blockDim.x) {
        const int i = (int)(e / l), j = (int)(e % l);
        const double p = 0.5 * __ldcg(Y + e) + (i == j ? 0.5 : 0.0);
        T[e] = p;
      }
      if (!grid_barrier(a.bar, a.status)) return;
      for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < ll; e += (size_t)gridDim.x * blockDim.x) {
        const int i = (int)(e / l), j = (int)(e % l);
        Y0[e] = __ldcg(T + e);
        Q0[e] = (i == j ? 1.0 : 0.0);
      }
      if (blockIdx.x == 0) {
        double f = 0.0;
        for (size_t e = threadIdx.x; e < ll; e += blockDim.x) {
          const int i = (int)(e / l), j = (int)(e % l);
          const double d = (i == j ? 1.0 : 0.0) - __ldcg(T + e);
          f += d * d;
        }
        red[threadIdx.x] = f;
        __syncthreads();
        for (int s = blockDim.x / 2; s > 0; s >>= 1) {
          if (threadIdx.x < s) red[threadIdx.x] += red[threadIdx.x + s];
          __syncthreads();
        }
        if (threadIdx.x == 0) scal[1] = (double)kn_ns_steps(fmin(sqrt(red[0]), 0.5), a.ns_target);
      }
      if (!grid_barrier(a.bar, a.status)) return;
    } else {
      // C = Y, Cinv = Q; F = C - Dc Cinv; err = ||C - I||_F
      for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < ll; e += (size_t)gridDim.x * blockDim.x) {
        a.C[e] = __ldcg(Y + e);
        a.Cinv[e] = __ldcg(Q + e);
      }
      if (!grid_barrier(a.bar, a.status)) return;
      mm_tiles(l, nr, 0, nt, -1.0, a.Dc, a.Cinv, 1.0, a.C, 0.0, a.F);
      if (blockIdx.x == 0) {
        double f = 0.0;
        for (size_t e = threadIdx.x; e < ll; e += blockDim.x) {
          const int i = (int)(e / l), j = (int)(e % l);
          const double d = __ldcg(a.C + e) - (i == j ? 1.0 : 0.0);
          f += d * d;
        }
        red[threadIdx.x] = f;
        __syncthreads();
        for (int s = blockDim.x / 2; s > 0; s >>= 1) {
          if (threadIdx.x < s) red[threadIdx.x] += red[threadIdx.x + s];
          __syncthreads();
        }
        if (threadIdx.x == 0) {
          const double err = sqrt(red[0]);
          *a.err = err;
          if (!(err == err)) atomicExch(a.status, kErrNumerical);
        }
      }
    }
  }
}

// ------------------------------------------------------------------------------------------
// The same two-sided Jacobi on one thread-block cluster (one matrix): the round-robin pairs are
// spread over the cluster's CTAs, each CTA holding the full rows of A and of V' (row i =
// eigenvector i) of the players of its pairs.  A round's rotation A := R' A R then touches only
// rows a CTA holds (the column rotations act within each row, the row rotations within each
// pair), so a round is local work plus one exchange: each row is stored into the shared memory
// of the CTA that holds its player in the next round, and each CTA publishes to all CTAs the
// diagonal entries of its rows and the off-diagonal entry A(p, q) of each next-round pair whose
// smaller player it holds.  Every CTA then computes all rotations of the round from the same
// table (identical results, so every CTA reaches the same convergence decision), and one
// hardware cluster barrier per round separates the exchange from its use.  No software waits.
constexpr int kEcThreads = 256;

struct EcShape {
  int n, ne, np, pp, rows;  // pairs per CTA (pp), rows per CTA (2 pp)
};

__device__ __forceinline__ EcShape ec_shape(int n, int cs) {
  EcShape e;
  e.n = n;
  e.ne = n + (n & 1);
  e.np = e.ne / 2;
  e.pp = (e.np + cs - 1) / cs;
  e.rows = 2 * e.pp;
  return e;
}

// Position -> (slot, member): positions [0, np) are the first members of slots 0..np-1, the
// others the second members of slots ne-1-i.
__device__ __forceinline__ void ec_slot(int i, int np, int ne, int &slot, int &member) {
  if (i < np) { slot = i; member = 0; } else { slot = ne - 1 - i; member = 1; }
}

__global__ void __launch_bounds__(kEcThreads, 1)
    sym_eig_cluster_kernel(int n, const double *__restrict__ A0, double *__restrict__ V, double *__restrict__ w,
                           int order, bool absval, int *status) {
  namespace cg = cooperative_groups;
  cg::cluster_group cluster = cg::this_cluster();
  const int cs = (int)cluster.num_blocks(), me = (int)cluster.block_rank();
  const EcShape sh = ec_shape(n, cs);
  const int ne = sh.ne, np = sh.np, R = sh.rows, tid = threadIdx.x, nt = blockDim.x;
  const int lane = tid & 31, warp = tid >> 5, nwarp = nt >> 5;
  extern __shared__ double sm[];
  double *rowsA = sm;                                   // [2][R][n]
  double *rowsV = rowsA + 2 * (size_t)R * n;            // [2][R][n]
  double *diag = rowsV + 2 * (size_t)R * n;             // [2][ne]
  double *off = diag + 2 * ne;                          // [2][np]
  double *rc = off + 2 * np, *rs = rc + np;             // this round's rotations
  double *red = rs + np;                                // [kEcThreads]
  int *rp = (int *)(red + kEcThreads), *rq = rp + np;   // this round's pairs (p < q)
  int *mv = rq + np;                                    // per held row: [dst, dst row, player, partner, next slot]
  int *conv = mv + 5 * R;                               // [2][16] per-CTA "a pair above the threshold" flags
  int *any = conv + 32, *exc = any + 1;
  double *keyb = red;                                   // diagonal after a round (reuses the reduction buffer, n <= 160 < 256)
  __shared__ double *peerA[16], *peerV[16], *peerD[16], *peerO[16];
  __shared__ int *peerC[16];
  if (tid < cs) {  // the same buffers in every CTA of the cluster (distributed shared memory)
    peerA[tid] = cluster.map_shared_rank(rowsA, tid);
    peerV[tid] = cluster.map_shared_rank(rowsV, tid);
    peerD[tid] = cluster.map_shared_rank(diag, tid);
    peerO[tid] = cluster.map_shared_rank(off, tid);
    peerC[tid] = cluster.map_shared_rank(conv, tid);
  }

  // symmetrised A, ||A||_F (every CTA the same sum in the same order), round-0 rows and tables
  double fr = 0.0;
  for (int e = tid; e < n * n; e += nt) {
    const int i = e / n, j = e - i * n;
    const double v = 0.5 * (A0[(size_t)i * n + j] + A0[(size_t)j * n + i]);
    fr += v * v;
  }
  red[tid] = fr;
  __syncthreads();
  for (int h = nt / 2; h > 0; h >>= 1) {
    if (tid < h) red[tid] += red[tid + h];
    __syncthreads();
  }
  const double tol = kEps * fmax(1.0, sqrt((double)n));
  const double floor_ = kEps * sqrt(red[0]);
  for (int lr = warp; lr < R; lr += nwarp) {
    const int slot = me * sh.pp + lr / 2;
    const int x = slot < np ? rr_player((lr & 1) ? ne - 1 - slot : slot, 0, ne) : ne;
    for (int j = lane; j < n; j += 32) {
      rowsA[(size_t)lr * n + j] = x < n ? 0.5 * (A0[(size_t)x * n + j] + A0[(size_t)j * n + x]) : 0.0;
      rowsV[(size_t)lr * n + j] = (x == j) ? 1.0 : 0.0;
    }
  }
  for (int x = tid; x < ne; x += nt) diag[x] = x < n ? A0[(size_t)x * n + x] : 0.0;
  for (int k = tid; k < np; k += nt) {
    int p = rr_player(k, 0, ne), q = rr_player(ne - 1 - k, 0, ne);
    if (p > q) { const int t = p; p = q; q = t; }
    off[k] = q < n ? 0.5 * (A0[(size_t)p * n + q] + A0[(size_t)q * n + p]) : 0.0;
  }
  __syncthreads();

  int cb = 0, sweep = 0, round = 0;
  bool rotated_in_sweep = false;
  for (;;) {
    double *A = rowsA + (size_t)cb * R * n, *Vt = rowsV + (size_t)cb * R * n;
    const double *dg = diag + cb * ne, *of = off + cb * np;
    const int nb = cb ^ 1, nround = (round + 1) % (ne - 1);
    // 1. all rotations of the round (every CTA alike) and where each held row goes next
    if (tid == 0) *any = 0;
    __syncthreads();
    for (int k = tid; k < np; k += nt) {
      int p = rr_player(k, round, ne), q = rr_player(ne - 1 - k, round, ne);
      if (p > q) { const int t = p; p = q; q = t; }
      double c = 1.0, sn = 0.0;
      if (q < n && jacobi_rot(dg[p], dg[q], of[k], tol, floor_, c, sn)) *any = 1;
      rp[k] = p; rq[k] = q; rc[k] = c; rs[k] = sn;
    }
    for (int lr = tid; lr < R; lr += nt) {
      const int slot = me * sh.pp + lr / 2;
      if (slot >= np) continue;
      const int i = (lr & 1) ? ne - 1 - slot : slot;  // position this round
      const int i2 = (i == 0) ? 0 : (i == 1 ? ne - 1 : i - 1);
      int s2, m2;
      ec_slot(i2, np, ne, s2, m2);
      mv[5 * lr + 0] = s2 / sh.pp;
      mv[5 * lr + 1] = 2 * (s2 % sh.pp) + m2;
      mv[5 * lr + 2] = rr_player(i, round, ne);
      mv[5 * lr + 3] = rr_player(ne - 1 - i2, nround, ne);
      mv[5 * lr + 4] = s2;
    }
    __syncthreads();
    if (*any) rotated_in_sweep = true;
    // 2. A := A R on the held rows: warp per row, lanes over the column pairs
    for (int lr = warp; lr < R; lr += nwarp) {
      double *row = A + (size_t)lr * n;
      for (int k = lane; k < np; k += 32) {
        const double sn = rs[k];
        if (sn == 0.0) continue;
        const double c = rc[k];
        const int p = rp[k], q = rq[k];
        const double xp = row[p], xq = row[q];
        row[p] = c * xp - sn * xq;
        row[q] = sn * xp + c * xq;
      }
    }
    __syncthreads();
    // 3. A := R' A and V' := R' V' on the held row pairs (warp per pair); closed form on the
    //    pair's 2 x 2 block
    for (int ls = warp; ls < sh.pp; ls += nwarp) {
      const int slot = me * sh.pp + ls;
      if (slot >= np) continue;
      const double sn = rs[slot];
      if (sn == 0.0) continue;
      const double c = rc[slot], t = sn / c;
      const int p = rp[slot], q = rq[slot];
      const bool first_is_p = mv[5 * (2 * ls) + 2] == p;  // member 0 holds the player at position `slot`
      const int lp = 2 * ls + (first_is_p ? 0 : 1), lq = 2 * ls + (first_is_p ? 1 : 0);
      double *ap = A + (size_t)lp * n, *aq = A + (size_t)lq * n;
      double *vp = Vt + (size_t)lp * n, *vq = Vt + (size_t)lq * n;
      for (int j = lane; j < n; j += 32) {
        if (j == p) { ap[p] = dg[p] - t * of[slot]; aq[p] = 0.0; }
        else if (j == q) { aq[q] = dg[q] + t * of[slot]; ap[q] = 0.0; }
        else {
          const double x1 = ap[j], x2 = aq[j];
          ap[j] = c * x1 - sn * x2;
          aq[j] = sn * x1 + c * x2;
        }
        const double v1 = vp[j], v2 = vq[j];
        vp[j] = c * v1 - sn * v2;
        vq[j] = sn * v1 + c * v2;
      }
    }
    __syncthreads();
    // 4. end of a sweep: stop when no rotation happened in it, or when every pair was found below
    //    the threshold at the end of the previous sweep (the next sweep would rotate nothing);
    //    the same decision in every CTA
    const bool last_round = (round == ne - 2);
    bool converged = false;
    if (round == 0 && sweep > 0) {
      converged = true;
      for (int c = 0; c < cs; ++c) converged &= conv[cb * 16 + c] == 0;
    }
    const bool done = (last_round && !rotated_in_sweep) || converged;
    const bool exhausted = last_round && sweep + 1 >= kMaxSweeps;
    // diagonal after this round: the table and the closed forms of step 3 (the values the rows hold)
    double *key = keyb;
    if (done || exhausted || last_round) {
      for (int y = tid; y < n; y += nt) {
        const int pos = (y == 0) ? 0 : 1 + ((y - 1 - round) % (ne - 1) + (ne - 1)) % (ne - 1);
        int sl, mb;
        ec_slot(pos, np, ne, sl, mb);
        double ky = dg[y];
        if (rs[sl] != 0.0) {
          const double t = rs[sl] / rc[sl];
          ky = (y == rp[sl]) ? dg[y] - t * of[sl] : dg[y] + t * of[sl];
        }
        key[y] = ky;
      }
      if (tid == 0) *exc = 0;
      __syncthreads();
    }
    if (done || exhausted) {
      if (exhausted && !done && me == 0 && tid == 0) atomicExch(status, kErrNumerical);
      // each CTA writes the eigenpairs of the players it holds, ranked by `order`
      for (int lr = warp; lr < R; lr += nwarp) {
        const int slot = me * sh.pp + lr / 2;
        if (slot >= np) continue;
        const int x = mv[5 * lr + 2];
        if (x >= n) continue;
        const double kx = key[x];
        int rank = 0;
        for (int y = lane; y < n; y += 32) {
          const double ky = key[y];
          rank += (order > 0) ? (fabs(ky) > fabs(kx) || (fabs(ky) == fabs(kx) && y < x))
                              : (ky < kx || (ky == kx && y < x));
        }
        for (int o = 16; o > 0; o >>= 1) rank += __shfl_xor_sync(0xffffffffu, rank, o);
        if (lane == 0) w[rank] = absval ? fabs(kx) : kx;
        const double *vrow = Vt + (size_t)lr * n;
        for (int j = lane; j < n; j += 32) V[(size_t)j * n + rank] = vrow[j];
      }
      return;
    }
    if (last_round) {  // any off-diagonal entry of a held row above the rotation threshold?
      for (int lr = warp; lr < R; lr += nwarp) {
        const int slot = me * sh.pp + lr / 2;
        if (slot >= np) continue;
        const int x = mv[5 * lr + 2];
        if (x >= n) continue;
        const double *row = A + (size_t)lr * n;
        const double kx = fabs(key[x]);
        for (int j = lane; j < n; j += 32)
          if (j != x && fabs(row[j]) > tol * fmax(sqrt(kx * fabs(key[j])), floor_)) *exc = 1;
      }
      __syncthreads();
    }
    // 5. exchange: each held row to its next-round holder (warp per row, coalesced stores into
    //    that CTA's shared memory), the diagonal and next-pair off-diagonal entries to every CTA
    for (int lr = warp; lr < R; lr += nwarp) {
      const int slot = me * sh.pp + lr / 2;
      if (slot >= np) continue;
      const int dst = mv[5 * lr + 0];
      const size_t drow = ((size_t)nb * R + mv[5 * lr + 1]) * n;
      const double *a = A + (size_t)lr * n, *v = Vt + (size_t)lr * n;
      double *ra = peerA[dst] + drow, *rv = peerV[dst] + drow;
      for (int j = lane; j < n; j += 32) {
        ra[j] = a[j];
        rv[j] = v[j];
      }
    }
    for (int e = tid; e < R * cs; e += nt) {
      const int lr = e % R, dst = e / R;
      const int slot = me * sh.pp + lr / 2;
      if (slot >= np) continue;
      const int x = mv[5 * lr + 2], partner = mv[5 * lr + 3], s2 = mv[5 * lr + 4];
      const double *row = A + (size_t)lr * n;
      peerD[dst][nb * ne + x] = x < n ? row[x] : 0.0;
      if (x < partner && partner < n) peerO[dst][nb * np + s2] = row[partner];
      else if (partner >= n && x < n) peerO[dst][nb * np + s2] = 0.0;
    }
    if (last_round && tid < cs) peerC[tid][nb * 16 + me] = *exc;
    cluster.sync();
    cb = nb;
    round = nround;
    if (round == 0) {
      ++sweep;
      rotated_in_sweep = false;
    }
  }
}

size_t eig_cluster_smem(int n, int cs) {
  const int ne = n + (n & 1), np = ne / 2, pp = (np + cs - 1) / cs, R = 2 * pp;
  return (size_t)(4 * R * n + 2 * ne + 2 * np + 2 * np + kEcThreads) * 8 + (size_t)(2 * np + 5 * R + 32 + 2) * 4;
}

size_t eig_smem(int n, bool vs) {
  const int ne = n + (n & 1), np = ne / 2;
  const size_t npk = ((size_t)n * (n + 1) / 2 + 1) & ~(size_t)1;
  return npk * 8 + (vs ? (size_t)n * n * 8 : 0) + (size_t)np * 16 + (size_t)n * 8 + (size_t)np * 8 + 16;
}
size_t svd_smem(int n) { return (size_t)n * n * 8 + (size_t)n * 8 + 16; }

}  // namespace

namespace {

// Cluster size for the one-matrix eigensolver (0: use the one-CTA kernel): the largest of 16, 8,
// 4, 2 that the device can co-schedule, for 112 <= n <= 160.  A round costs about 2.5 us on the
// cluster whatever n (barrier and exchange), against shared-memory bandwidth on one CTA, which
// grows as n^2: measured per solve on B200, 3.45 against 4.18 ms at n = 128 and 5.7 against
// 10.8 ms at n = 160, but 2.49 against 2.19 ms at n = 96.
int eig_cluster_size(int n, cudaStream_t st) {
  static int decided[2] = {-1, -1};  // per size class: n <= 128, n <= 160
  if (n < 112 || n > 160) return 0;
  // ISVD_GPU_EIG_CLUSTER: 0 off, 2..16 the largest size tried
  static const int top = [] {
    const char *e = getenv("ISVD_GPU_EIG_CLUSTER");
    return e ? std::max(0, std::min(16, atoi(e))) : 16;
  }();
  if (top < 2) return 0;
  int &d = decided[n > 128 ? 1 : 0];
  if (d >= 0) return d;
  CK(cudaFuncSetAttribute(sym_eig_cluster_kernel, cudaFuncAttributeNonPortableClusterSizeAllowed, 1));
  d = 0;
  for (int cs = top; cs >= 2; cs /= 2) {
    const size_t smem = eig_cluster_smem(n > 128 ? 160 : 128, cs);
    if (cudaFuncSetAttribute(sym_eig_cluster_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) !=
        cudaSuccess) {
      cudaGetLastError();
      continue;
    }
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(cs);
    cfg.blockDim = dim3(kEcThreads);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = cs;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    int nc = 0;
    if (cudaOccupancyMaxActiveClusters(&nc, sym_eig_cluster_kernel, &cfg) != cudaSuccess) {
      cudaGetLastError();
      continue;
    }
    if (nc >= 1) {
      d = cs;
      break;
    }
  }
  return d;
}

}  // namespace

// Kernel time under `tag` when kernel timing is on (isvd_gpu_profile_enable).
struct ProfileScope {
  const char *tag;
  cudaStream_t st;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  ProfileScope(const char *t, cudaStream_t s) : tag(t), st(s) {
    if (!profiling()) return;
    CK(cudaEventCreate(&e0));
    CK(cudaEventCreate(&e1));
    CK(cudaEventRecord(e0, st));
  }
  ~ProfileScope() {
    if (!e0) return;
    float ms = 0.f;
    if (cudaEventRecord(e1, st) == cudaSuccess && cudaEventSynchronize(e1) == cudaSuccess &&
        cudaEventElapsedTime(&ms, e0, e1) == cudaSuccess)
      profile_add(tag, ms, 0.0);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
  }
};

void sym_eig_batched(int n, int batch, const double *A, double *V, double *w, int order, bool absval, int *status,
                     cudaStream_t st) {
  if (n <= 0 || batch <= 0) return;
  ProfileScope prof("sym_eig", st);
  Runtime &rt = Runtime::get();
  if (batch == 1) {
    const int cs = eig_cluster_size(n, st);
    if (cs > 0) {
      const size_t smem = eig_cluster_smem(n, cs);
      CK(cudaFuncSetAttribute(sym_eig_cluster_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
      cudaLaunchConfig_t cfg = {};
      cfg.gridDim = dim3(cs);
      cfg.blockDim = dim3(kEcThreads);
      cfg.dynamicSmemBytes = smem;
      cfg.stream = st;
      cudaLaunchAttribute attr[1];
      attr[0].id = cudaLaunchAttributeClusterDimension;
      attr[0].val.clusterDim.x = cs;
      attr[0].val.clusterDim.y = 1;
      attr[0].val.clusterDim.z = 1;
      cfg.attrs = attr;
      cfg.numAttrs = 1;
      CK(cudaLaunchKernelEx(&cfg, sym_eig_cluster_kernel, n, A, V, w, order, absval, status));
      KLAUNCHED();
      return;
    }
  }
  const size_t smem_vs = eig_smem(n, true);
  if (smem_vs <= rt.smem_optin) {
    CK(cudaFuncSetAttribute(sym_eig_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_vs));
    sym_eig_kernel<true><<<batch, kEigThreads, smem_vs, st>>>(n, A, V, w, order, absval, nullptr, status, nullptr);
    KLAUNCHED();
    return;
  }
  const size_t smem = eig_smem(n, false);
  if (smem > rt.smem_optin) fail(kErrUnsupported, "symmetric eigensolver: l = %d exceeds on-chip capacity", n);
  DBuf<double> scratch((size_t)batch * n * n);
  CK(cudaFuncSetAttribute(sym_eig_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  sym_eig_kernel<false><<<batch, kEigThreads, smem, st>>>(n, A, V, w, order, absval, scratch.p, status,
                                                            nullptr);
  KLAUNCHED();
}

void sym_eig_grouped(const EigDesc *desc, int count, int max_n, int order, bool absval, int *status,
                     cudaStream_t st) {
  if (count <= 0 || max_n <= 0) return;
  const size_t smem = eig_smem(max_n, true);
  if (smem > Runtime::get().smem_optin)
    fail(kErrUnsupported, "symmetric eigensolver: l = %d exceeds on-chip capacity", max_n);
  // the smallest CTA that holds the largest matrix: small matrices leave room for many CTAs per SM
  auto go = [&](auto kernel, int nt) {
    CK(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    kernel<<<count, nt, smem, st>>>(0, nullptr, nullptr, nullptr, order, absval, nullptr, status, desc);
    KLAUNCHED();
  };
  if (max_n <= eig_max_n(128)) go(sym_eig_kernel<true, 128>, 128);
  else if (max_n <= eig_max_n(256)) go(sym_eig_kernel<true, 256>, 256);
  else if (max_n <= eig_max_n(512)) go(sym_eig_kernel<true, 512>, 512);
  else go(sym_eig_kernel<true, kEigThreads>, kEigThreads);
}

void svd_jacobi_batched(int n, int batch, const double *B, double *U, double *s, double *V, int *status,
                        cudaStream_t st) {
  if (n <= 0 || batch <= 0) return;
  Runtime &rt = Runtime::get();
  const size_t smem = svd_smem(n);
  if (smem > rt.smem_optin) fail(kErrUnsupported, "Jacobi SVD: l = %d exceeds on-chip capacity", n);
  CK(cudaFuncSetAttribute(svd_jacobi_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  svd_jacobi_kernel<<<batch, kEigThreads, smem, st>>>(n, B, U, s, V, status);
  KLAUNCHED();
}

void kn_step_fixed_preload() {
  cudaFuncAttributes fa;
  CK(cudaFuncGetAttributes(&fa, kn_step_kernel));
}

void kn_step_fixed(const KnStep &a, int num_sms, cudaStream_t st) {
  if (a.l > 160) fail(kErrUnsupported, "Kolmogorov-Nagumo step: l = %d > 160", a.l);
  const int nr = (a.l + 15) / 16;
  int blocks = 0;
  CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, kn_step_kernel, kKnThreads, 0));
  int grid = std::min(2 * nr * nr, blocks * num_sms);
  grid = std::max(1, std::min(grid, num_sms));
  KnStep arg = a;
  void *args[] = {&arg};
  CK(cudaLaunchCooperativeKernel((void *)kn_step_kernel, dim3(grid), dim3(kKnThreads), args, 0, st));
  KLAUNCHED();
}

}  // namespace isvdb
