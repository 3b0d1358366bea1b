/* MPI helpers (reference src/include/c/isvd/util/mpi.h:20-32; util/mpi.c:21-35). */
#ifndef ISVD_UTIL_MPI_H_
#define ISVD_UTIL_MPI_H_

#include <isvd/def.h>

#if defined(__cplusplus)
extern "C" {
#endif

#if !defined(ISVD_USE_ILP64)
#define MPI_ISVD_INT_T    MPI_INTEGER4
#else
#define MPI_ISVD_INT_T    MPI_INTEGER8
#endif
#define MPI_ISVD_S_VAL_T  MPI_REAL4
#define MPI_ISVD_D_VAL_T  MPI_REAL8

/* Replaces isvd_getMpiSize (reference util/mpi.c:21). */
mpi_int_t isvd_getMpiSize( const isvd_MpiComm comm );
/* Replaces isvd_getMpiRank (reference util/mpi.c:33). */
mpi_int_t isvd_getMpiRank( const isvd_MpiComm comm );

#if defined(__cplusplus)
}
#endif

#endif  /* ISVD_UTIL_MPI_H_ */
