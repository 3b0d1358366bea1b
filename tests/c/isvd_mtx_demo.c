/*
 * A Matrix Market demo written the way the reference's demo/cdemo.c is: A is read with the mmio
 * routines (here the header-only include/mmio_shim/mmio.h) and one isvd_dFget per value
 * (column-major "array real general"), the driver runs GP / GR / KN / GR on the row block of this
 * rank with dista 'R', ordera 'C' (lda = m), and the stage times are printed.  It then reads A a
 * second time with isvd_dMtxRead and checks that both readers agree, and writes the results with
 * isvd_dMtxWrite: S (l x 1), U (m x k), V (n x k).
 *
 *   usage: isvd_mtx_demo <A-mtx-file> <S-mtx-file> <U-mtx-file> <V-mtx-file>
 */
#include <isvd.h>
#include <mmio.h>
#include <stdio.h>
#include <stdlib.h>

int main(int argc, char **argv) {
  isvd_Init(&argc, &argv, MPI_COMM_WORLD);
  const mpi_int_t mpi_rank = isvd_getMpiRank(MPI_COMM_WORLD), mpi_root = 0;
  if (argc < 5) {
    printf("Usage: %s <A-mtx-file> <S-mtx-file> <U-mtx-file> <V-mtx-file>\n\n", argv[0]);
    return 1;
  }
  if (mpi_rank == mpi_root) {
    printf("iSVD C demo (Matrix Market)\n");
    isvd_PrintEnvironment(MPI_COMM_WORLD);
  }

  /* read A: banner, size, then one value at a time */
  FILE *file = fopen(argv[1], "r");
  if (!file) {
    fprintf(stderr, "cannot open %s\n", argv[1]);
    return 1;
  }
  MM_typecode matcode;
  int m = 0, n = 0;
  if (mm_read_banner(file, &matcode) != 0 || !mm_is_array(matcode) || !mm_is_real(matcode) ||
      !mm_is_general(matcode)) {
    char *t = mm_typecode_to_str(matcode);
    fprintf(stderr, "Sorry, this application does not support Matrix Market type: [%s]\n", t ? t : "?");
    free(t);
    return 1;
  }
  if (mm_read_mtx_array_size(file, &m, &n) != 0) {
    fprintf(stderr, "no size line in %s\n", argv[1]);
    return 1;
  }
  double *a = isvd_dMalloc((size_t)m * n);
  const isvd_int_t lda = m;
  for (isvd_int_t j = 0; j < n; ++j)
    for (isvd_int_t i = 0; i < m; ++i) isvd_dFget(file, &a[i + j * lda]);
  fclose(file);
  if (isvd_gpu_get_last_error()) {
    fprintf(stderr, "reading %s: %s\n", argv[1], isvd_gpu_get_error_string());
    return 1;
  }

  /* the parallel reader gives the same matrix */
  isvd_int_t m2 = 0, n2 = 0;
  if (isvd_dMtxRead(argv[1], &m2, &n2, NULL, 1, 'C') != ISVD_GPU_SUCCESS || m2 != m || n2 != n) {
    fprintf(stderr, "isvd_dMtxRead size: %s\n", isvd_gpu_get_error_string());
    return 1;
  }
  double *a2 = isvd_dMalloc((size_t)m * n);
  if (isvd_dMtxRead(argv[1], &m2, &n2, a2, m, 'C') != ISVD_GPU_SUCCESS) {
    fprintf(stderr, "isvd_dMtxRead: %s\n", isvd_gpu_get_error_string());
    return 1;
  }
  size_t differ = 0;
  for (size_t e = 0; e < (size_t)m * n; ++e) differ += a[e] != a2[e];
  printf("readers agree: %s (%zu of %zu values differ)\n", differ ? "no" : "yes", differ, (size_t)m * n);
  isvd_Free(a2);

  /* solve */
  const isvd_int_t k = 20, p = 12, N = 16;
  const isvd_Param param = isvd_createParam(m, n, k, p, N, mpi_root, MPI_COMM_WORLD);
  const isvd_int_t mb = param.nrow_each, Pmb = param.nrow_total, Pnb = param.ncol_total, l = param.dim_sketch;
  double *s = isvd_dMalloc(l);
  double *ut = isvd_dMalloc((size_t)l * Pmb);
  double *vt = isvd_dMalloc((size_t)l * Pnb);
  double time[4];
  isvd_dIsvd(param, "GP_gpu", "GR", "KN", "GR_gpu", NULL, NULL, NULL, NULL, time, stdout, 'R', 'C',
             a + mb * mpi_rank, lda, s, ut, l, vt, l, 0, mpi_root, mpi_root);
  if (isvd_gpu_get_last_error()) {
    fprintf(stderr, "isvd_dIsvd failed: %s\n", isvd_gpu_get_error_string());
    return 1;
  }
  if (mpi_rank == mpi_root) {
    printf("\n");
    printf("Average total computing time:   %8.6f seconds.\n", time[0] + time[1] + time[2] + time[3]);
    printf("Average sketching time:         %8.6f seconds.\n", time[0]);
    printf("Average orthogonalizing time:   %8.6f seconds.\n", time[1]);
    printf("Average integrating time:       %8.6f seconds.\n", time[2]);
    printf("Average postprocessing time:    %8.6f seconds.\n", time[3]);
    printf("\n");
    if (isvd_dMtxWrite(argv[2], l, 1, s, l, 'C') || isvd_dMtxWrite(argv[3], m, k, ut, l, 'R') ||
        isvd_dMtxWrite(argv[4], n, k, vt, l, 'R')) {
      fprintf(stderr, "writing the results: %s\n", isvd_gpu_get_error_string());
      return 1;
    }
  }
  isvd_Free(a);
  isvd_Free(s);
  isvd_Free(ut);
  isvd_Free(vt);
  isvd_Finalize();
  return 0;
}
