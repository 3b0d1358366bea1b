// Batched iSVD of many independent matrices of uneven sizes (batched.cu).
#pragma once

#include <cuda_runtime.h>

namespace isvdb {

// Workspace, device-side work lists and captured graphs of one batch shape.
struct BatchPlan {
  virtual ~BatchPlan() = default;
  int elem = 0;  // sizeof the element type (4: float, 8: double)
};

int plan_count(const BatchPlan *plan);

// count matrices m_i x n_i (row-major), rank k_i, oversampling p_i, N sketches each.
template <class T>
BatchPlan *batch_plan_create(int count, const int *m, const int *n, const int *k, const int *p, int N);

// GP / GR / KN / GR solve of every matrix of the plan: a[i] (device, row-major, lda[i]) ->
// s[i] (l_i values), ut[i] (m_i x l_i, leading dimension ldut[i], k_i valid columns), vt[i]
// (n_i x l_i); seeds[i] draws the Gaussian test matrix exactly as a single solve with that seed.
// KN stops each matrix at its own tolerance (maxit, tol: as isvd_?IntegrateKolmogorovNagumo);
// iters[i], errs[i] receive its iteration count and final error.
template <class T>
void batch_solve(BatchPlan *plan, const T *const *a, const long long *lda, T *const *s, T *const *ut,
                 const long long *ldut, T *const *vt, const long long *ldvt, const unsigned long long *seeds, int maxit,
                 double tol, int *iters, double *errs);

}  // namespace isvdb
