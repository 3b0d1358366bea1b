/*
 * Basic types of the iSVD API (reference src/include/c/isvd/def.h:84-131).
 *
 * isvd_int_t is int32_t unless ISVD_USE_ILP64 is defined.  <mpi.h> is either a
 * real MPI or the single-rank shim in include/mpi_shim (add -Iinclude/mpi_shim).
 */
#ifndef ISVD_DEF_H_
#define ISVD_DEF_H_

#include <assert.h>
#include <stdio.h>
#include <stdint.h>
#include <stddef.h>
#include <mpi.h>
#include <isvd/config.h>

#if defined(__cplusplus)
extern "C" {
#endif

#if !defined(ISVD_USE_ILP64)
typedef int32_t  isvd_int_t;   /* index type (LP64 build) */
typedef uint32_t isvd_uint_t;
#else
typedef int64_t  isvd_int_t;   /* index type (ILP64 build) */
typedef uint64_t isvd_uint_t;
#endif

typedef float  isvd_s_val_t;   /* real single */
typedef double isvd_d_val_t;   /* real double */

typedef int mpi_int_t;         /* MPI rank / size type */
typedef int omp_int_t;         /* OpenMP thread index type */

typedef MPI_Comm isvd_MpiComm; /* MPI communicator */

#if defined(__cplusplus)
}
#endif

#endif  /* ISVD_DEF_H_ */
