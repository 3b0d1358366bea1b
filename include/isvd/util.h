/* Utilities (reference src/include/c/isvd/util.h). */
#ifndef ISVD_UTIL_H_
#define ISVD_UTIL_H_

#include <isvd/util/io.h>
#include <isvd/util/memory.h>
#include <isvd/util/mpi.h>
#include <isvd/util/omp.h>

#endif  /* ISVD_UTIL_H_ */
