// The C headers compile as C++ (extern "C" linkage, no C-only constructs) and link against the
// library; the mmio routines of include/mmio_shim/mmio.h write a banner and size that read back.
#include <isvd.h>
#include <mmio.h>

#include <cstdio>
#include <cstring>

int main(int argc, char **argv) {
  if (argc < 2) return 2;
  FILE *f = std::fopen(argv[1], "w+");
  if (!f) return 2;
  MM_typecode tc;
  mm_initialize_typecode(&tc);
  mm_set_matrix(&tc);
  mm_set_array(&tc);
  mm_set_real(&tc);
  mm_set_general(&tc);
  if (mm_write_banner(f, tc) != 0 || mm_write_mtx_array_size(f, 3, 2) != 0) return 3;
  for (int e = 0; e < 6; ++e) std::fprintf(f, "%d.5\n", e);
  std::rewind(f);
  MM_typecode rd;
  int m = 0, n = 0;
  if (mm_read_banner(f, &rd) != 0 || std::memcmp(rd, tc, 4) != 0) return 4;
  if (mm_read_mtx_array_size(f, &m, &n) != 0 || m != 3 || n != 2) return 5;
  double v = 0.0, sum = 0.0;
  for (int e = 0; e < 6; ++e) {
    isvd_dFget(f, &v);
    sum += v;
  }
  std::fclose(f);
  const isvd_Param p = isvd_createParam(40, 30, 4, 2, 3, 0, MPI_COMM_WORLD);
  std::printf("sum %.1f dim_sketch %d omp %d error %d\n", sum, (int)p.dim_sketch, (int)isvd_getOmpMaxSize(),
              isvd_gpu_get_last_error());
  return 0;
}
