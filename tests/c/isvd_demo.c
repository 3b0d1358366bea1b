/*
 * A C caller of the iSVD API, written against include/isvd.h only: the same calls a program
 * written for the reference library makes (environment, parameters, the isvd_dIsvd driver with
 * the GP / GR / KN / GR stages), linked with -lisvd_gpu_b200 instead of the reference's
 * -lisvd_core -lisvd_la_* -lisvd_gpu_*.  Prints the leading singular values and stage times.
 *
 *   usage: isvd_demo [m n k p N]
 */
#include <isvd.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>

int main(int argc, char **argv) {
  int m = 1200, n = 800, k = 10, p = 6, N = 8;
  if (argc == 6) { m = atoi(argv[1]); n = atoi(argv[2]); k = atoi(argv[3]); p = atoi(argv[4]); N = atoi(argv[5]); }
  isvd_Init(&argc, &argv, MPI_COMM_WORLD);
  const int l = k + p;

  /* A = sum_i sigma_i u_i v_i' with sigma_i = 0.8^i on a deterministic pattern (row-major). */
  double *a = isvd_dMalloc((size_t)m * n);
  for (int i = 0; i < m; ++i)
    for (int j = 0; j < n; ++j) {
      double v = 0.0;
      for (int r = 0; r < 12; ++r) v += pow(0.8, r) * cos(0.37 * (r + 1) * (i + 1)) * sin(0.53 * (r + 1) * (j + 1));
      a[(size_t)i * n + j] = v;
    }
  isvd_Param param = isvd_createParam(m, n, k, p, N, 0, MPI_COMM_WORLD);
  double *s = isvd_dMalloc(l), *ut = isvd_dMalloc((size_t)m * l), *vt = isvd_dMalloc((size_t)n * l);
  const double argv_i[2] = {256, 1e-4};
  const double *args[4] = {NULL, NULL, argv_i, NULL};
  const isvd_int_t argcs[4] = {0, 0, 2, 0};
  double ret_i[2];
  double *rets[4] = {NULL, NULL, ret_i, NULL};
  const isvd_int_t retcs[4] = {0, 0, 2, 0};
  double time[4];
  isvd_dIsvd(param, "GP_gpu", "GR", "KN", "GR_gpu", args, argcs, rets, retcs, time, stdout, 'R', 'R', a, n, s, ut, l,
             vt, l, 0, -1, -1);
  const int err = isvd_gpu_get_last_error();
  if (err) {
    fprintf(stderr, "isvd_dIsvd failed: %s\n", isvd_gpu_get_error_string());
    return 1;
  }
  printf("KN iterations %d, error %.3e\n", (int)ret_i[0], ret_i[1]);
  printf("sigma:");
  for (int i = 0; i < k; ++i) printf(" %.6f", s[i]);
  printf("\ntimes: sketch %.4f s, orthogonalize %.4f s, integrate %.4f s, postprocess %.4f s\n", time[0], time[1],
         time[2], time[3]);
  isvd_Free(a);
  isvd_Free(s);
  isvd_Free(ut);
  isvd_Free(vt);
  isvd_Finalize();
  return 0;
}
