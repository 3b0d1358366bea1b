/* OpenMP utilities (reference src/include/c/isvd/util/omp.h:19-21; la/util/omp.c:20-63).  This
 * library runs no OpenMP team on the caller's behalf (its host work is the GPU's launch path), so
 * these return the reference's values for a build without OpenMP: max size 1, size 1, rank 0. */
#ifndef ISVD_UTIL_OMP_H_
#define ISVD_UTIL_OMP_H_

#include <isvd/def.h>

#if defined(__cplusplus)
extern "C" {
#endif

omp_int_t isvd_getOmpMaxSize( void );
omp_int_t isvd_getOmpSize( void );
omp_int_t isvd_getOmpRank( void );

#if defined(__cplusplus)
}
#endif

#endif  /* ISVD_UTIL_OMP_H_ */
