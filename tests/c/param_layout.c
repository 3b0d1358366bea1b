/* Prints the size of isvd_Param and the offset and size of each of its fields, one per line, for
 * whichever <isvd/core/param.h> and <mpi.h> the include path selects (the library's or the
 * reference's, under the same mpi.h): the layout of the struct every entry point takes by value. */
#include <stddef.h>
#include <stdio.h>
#include <isvd/core/param.h>

#define FIELD(f) printf("%s %zu %zu\n", #f, offsetof(isvd_Param, f), sizeof(((isvd_Param *)0)->f))

int main(void) {
  printf("sizeof %zu %zu\n", sizeof(isvd_Param), _Alignof(isvd_Param));
  FIELD(mpi_comm);
  FIELD(mpi_size);
  FIELD(mpi_root);
  FIELD(mpi_rank);
  FIELD(nrow);
  FIELD(ncol);
  FIELD(nrow_proc);
  FIELD(ncol_proc);
  FIELD(nrow_each);
  FIELD(ncol_each);
  FIELD(nrow_total);
  FIELD(ncol_total);
  FIELD(rowidxbegin);
  FIELD(rowidxend);
  FIELD(colidxbegin);
  FIELD(colidxend);
  FIELD(rank);
  FIELD(over_rank);
  FIELD(dim_sketch);
  FIELD(dim_sketch_total);
  FIELD(num_sketch);
  return 0;
}
