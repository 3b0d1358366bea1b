/*
 * Host-only check of the Matrix Market readers (no GPU work): reads the banner and size of
 * argv[1] with the mmio routines of include/mmio_shim/mmio.h, the values with one isvd_dFget
 * each (column-major, as the reference's demo/cdemo.c:51-64), and the whole file again with
 * isvd_dMtxRead; prints the typecode, the size, the number of differing values and the sum.
 *
 *   usage: mtx_read_check <mtx-file>
 */
#include <isvd.h>
#include <mmio.h>
#include <stdio.h>
#include <stdlib.h>

int main(int argc, char **argv) {
  if (argc < 2) return 2;
  FILE *f = fopen(argv[1], "r");
  if (!f) return 2;
  MM_typecode tc;
  int m = 0, n = 0;
  const int rb = mm_read_banner(f, &tc);
  char *ts = mm_typecode_to_str(tc);
  printf("banner %d [%s] valid %d\n", rb, ts ? ts : "", mm_is_valid(tc));
  free(ts);
  if (rb != 0 || !mm_is_array(tc)) return 3;
  if (mm_read_mtx_array_size(f, &m, &n) != 0) return 4;
  double *a = isvd_dMalloc((size_t)m * n), *b = isvd_dMalloc((size_t)m * n);
  for (isvd_int_t j = 0; j < n; ++j)
    for (isvd_int_t i = 0; i < m; ++i) isvd_dFget(f, &a[i + j * (isvd_int_t)m]);
  fclose(f);
  const int fget_err = isvd_gpu_get_last_error();
  isvd_int_t m2 = 0, n2 = 0;
  const int st = isvd_dMtxRead(argv[1], &m2, &n2, b, m, 'C');
  size_t differ = 0;
  double sum = 0.0;
  for (size_t e = 0; e < (size_t)m * n; ++e) {
    differ += a[e] != b[e];
    sum += a[e];
  }
  printf("size %d %d read %d %d status %d fget %d differ %zu sum %.17g\n", m, n, (int)m2, (int)n2, st, fget_err,
         differ, sum);
  isvd_Free(a);
  isvd_Free(b);
  return 0;
}
