/* Environment routines (reference src/include/c/isvd/core/env.h:20-54; core/env.c:21-48). */
#ifndef ISVD_CORE_ENV_H_
#define ISVD_CORE_ENV_H_

#include <isvd/def.h>
#include <isvd/gpu/env.h>

#if defined(__cplusplus)
extern "C" {
#endif

/* Replaces isvd_Init_cpu (reference core/env.c:21): MPI_Init. */
void isvd_Init_cpu( int *argcp, char ***argvp, const isvd_MpiComm mpi_comm );
/* Replaces isvd_Finalize_cpu (reference core/env.c:34): MPI_Finalize. */
void isvd_Finalize_cpu( void );
/* Replaces isvd_PrintEnvironment_cpu (reference core/env.c:42). */
void isvd_PrintEnvironment_cpu( const isvd_MpiComm comm );

static inline void isvd_Init( int *argcp, char ***argvp, const isvd_MpiComm mpi_comm ) {
  isvd_Init_cpu(argcp, argvp, mpi_comm);
  isvd_Init_gpu(argcp, argvp, mpi_comm);
}

static inline void isvd_Finalize( void ) {
  isvd_Finalize_cpu();
  isvd_Finalize_gpu();
}

static inline void isvd_PrintEnvironment( const isvd_MpiComm mpi_comm ) {
  isvd_PrintEnvironment_cpu(mpi_comm);
  isvd_PrintEnvironment_gpu(mpi_comm);
}

#if defined(__cplusplus)
}
#endif

#endif  /* ISVD_CORE_ENV_H_ */
