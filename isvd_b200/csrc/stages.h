// Device-level iSVD stages at one MPI rank.  All pointers are device pointers; matrices keep
// the reference layouts (yst m x Nl row-major, qt m x l row-major, ut/vt row-major, A per ordera).
#pragma once

#include <cstdint>

#include <cuda_runtime.h>

namespace isvdb {

struct MixedCache;    // bf16 planes of A kept between the sketch and the postprocess (mixed.h)
struct PlaneHandoff;  // bf16 planes of one stage's output handed to the next stage (mixed.h)

struct StageCtx {
  cudaStream_t st;
  int precision;   // kNative / kMixed
  int *status;     // device status word (zeroed by the caller)
  MixedCache *cache = nullptr;
  // MIXED driver: the second (polar) pass of the Gramian orthogonalization is left to the
  // integration, which re-orthonormalizes the blocks in the coordinates of G (coeff_orthonormalize)
  bool deferred_orth = false;
  // Gramian orthogonalization may return any orthonormal basis of each span(Y_i) (Cholesky factor
  // instead of the eigenbasis): set by the driver when the rest of the pipeline is basis-invariant
  bool chol_basis = false;
  // rows of the whole matrix when this process holds a row block of it (multi-rank; 0: the
  // stage's own rows are all of them), and the first of this process's rows
  long long m_total = 0;
  long long row_begin = 0;
  // column blocks (dista 'C') on several ranks: this process holds all m_total rows of A and its
  // columns [col_begin, col_begin + a_cols) (a_cols 0: A holds every column of its rows); the sketch
  // draws the rows of Omega from col_begin on
  long long col_begin = 0;
  long long a_cols = 0;
  // the stage's matrix is whole and the same on every rank (an n x l factor formed after a sum over
  // the ranks): no exchange between ranks, and every rank computes the same result
  bool replicated = false;
  // out-of-core A: a host A is streamed through the device in row panels of this many rows by the
  // sketch and the projection (0: A is on the device, or copied there whole)
  long long a_panel_rows = 0;
  // MIXED driver, GP / GR / (KN or WY): the sketch and the Gramian apply write the bf16 planes of
  // their output here instead of its values, and the next stage reads them instead of splitting
  PlaneHandoff *handoff = nullptr;
};

struct IterResult {
  int iterations = 0;
  double error = 0.0;
};

struct WyArgs {
  int maxit = 256;
  double tol = 1e-3, tau0 = 1.0, taumax = 1e14, taumin = 1e-14;
  int taumaxit = 20;
  double beta = 0.5, sigma = 1e-4, eta = 0.85;
};

// Y = A * Omega (reference core/stage/@x@_sketch.h:92-146).  omega == nullptr: drawn from seed.
template <class T>
void sketch_dev(const StageCtx &c, int m, int n, int Nl, char ordera, const T *a, long long lda, const T *omega,
                long long ldom, uint64_t seed, T *y, long long ldy);

// In-place Gramian orthogonalization of the N blocks of yst (reference @x@_orthogonalize_gramian.c).
template <class T>
void orth_gramian_dev(const StageCtx &c, int m, int l, int N, T *y, long long ldy);

// In-place TSQR orthogonalization (reference @x@_orthogonalize_tall_skinny_qr.c), Householder QR per block.
template <class T>
void orth_tsqr_dev(const StageCtx &c, int m, int l, int N, T *y, long long ldy);

template <class T>
IterResult integrate_kn_dev(const StageCtx &c, int m, int l, int N, const T *qs, long long ldq, T *qt,
                            long long ldqt, int maxit, double tol);

// Kolmogorov-Nagumo integration in FP64 on the static device scratch of noalloc.cu: no device
// allocation, operands in device memory, enqueued on `st`; returns once the work has completed.
IterResult integrate_kn_static(cudaStream_t st, int m, int l, int N, const double *qs, long long ldq, double *qt,
                               long long ldqt, int maxit, double tol);

template <class T>
IterResult integrate_wy_dev(const StageCtx &c, int m, int l, int N, const T *qs, long long ldq, T *qt,
                            long long ldqt, const WyArgs &w);

template <class T>
void integrate_hr_dev(const StageCtx &c, int m, int l, int N, T *qs, long long ldq, T *qt, long long ldqt);

// Postprocessing.  s has l entries; ut (m x k, ldut), vt (n x k or n x l for TS, ldvt) when wanted.
// MIXED driver, after a Gramian orthogonalization without its second pass: with R_i' R_i = G_ii
// (Cholesky) and X = diag(R_i^-1), the blocks of Qs X are orthonormal with respect to G to FP64
// rounding.  G (Nl x Nl, row-major) becomes X' G X in place; X (N blocks of l x l) is returned, and
// a coefficient matrix M of Qs X is M' = X M for Qs (coeff_unorthonormalize).
void coeff_orthonormalize(const StageCtx &c, int Nl, int l, int N, double *G, double *X);
// out (Nl x l, ld l) = diag(X_i) M  for M with row stride ldm
void coeff_unorthonormalize(const StageCtx &c, int Nl, int l, int N, const double *X, const double *M, long long ldm,
                            double *out);

// Adjoint of the truncated SVD A ~ U diag(s) V' (adjoint.cu): dA from dU (m x k), ds (k), dV (n x k),
// any of them null.  A and dA stored per ordera; U, V, dU, dV row-major.  cg_iters bounds the
// conjugate-gradient iterations of the orthogonal-complement terms (0: rank-k formula).  Returns
// the iterations used (both complement systems).
template <class T>
int svd_adjoint_dev(const StageCtx &c, int m, int n, int k, char ordera, const T *a, long long lda, const T *u,
                    long long ldu, const T *s, const T *v, long long ldv, const T *du, long long lddu, const T *ds,
                    const T *dv, long long lddv, T *da, long long ldda, int cg_iters, double tol);

// Z = A' Qbar (n x l, row-major, ld l) for A m x n stored per ordera.
template <class T>
void project(const StageCtx &c, int m, int n, int l, char ordera, const T *a, long long lda, const T *qt,
             long long ldqt, T *z);

// Z = A' Qbar (n x l) summed over the ranks, the whole of it on every rank: m and qt are this
// rank's rows of Qbar; with row blocks A holds the same m rows, with column blocks (a_cols > 0) all
// m_total rows and a_cols columns.
template <class T>
void project_sum(const StageCtx &c, int m, int n, int l, char ordera, const T *a, long long lda, const T *qt,
                 long long ldqt, T *z);

template <class T>
void post_gramian_dev(const StageCtx &c, int m, int n, int k, int l, char ordera, const T *a, long long lda,
                      const T *qt, long long ldqt, T *s, T *ut, long long ldut, T *vt, long long ldvt, bool wu,
                      bool wv);
template <class T>
void post_tsqr_dev(const StageCtx &c, int m, int n, int k, int l, char ordera, const T *a, long long lda,
                   const T *qt, long long ldqt, T *s, T *ut, long long ldut, T *vt, long long ldvt, bool wu, bool wv);
template <class T>
void post_symmetric_dev(const StageCtx &c, int m, int n, int k, int l, char ordera, const T *a, long long lda,
                        const T *qt, long long ldqt, T *s, T *ut, long long ldut, bool wu);

}  // namespace isvdb
