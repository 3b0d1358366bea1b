/*
 * Problem parameters (reference src/include/c/isvd/core/param.h:27-100; core/param.c:14-83).
 *
 * Field order and types are part of the ABI: the struct is passed by value to
 * every driver and stage routine.
 */
#ifndef ISVD_CORE_PARAM_H_
#define ISVD_CORE_PARAM_H_

#include <isvd/def.h>

#if defined(__cplusplus)
extern "C" {
#endif

typedef struct {
  const isvd_MpiComm mpi_comm;         /* MPI communicator */
  const mpi_int_t    mpi_size;         /* P, number of ranks */
  const mpi_int_t    mpi_root;         /* root rank */
  const mpi_int_t    mpi_rank;         /* j, this rank */
  const isvd_int_t   nrow;             /* m */
  const isvd_int_t   ncol;             /* n */
  const isvd_int_t   nrow_proc;        /* m^(j), rows on this rank */
  const isvd_int_t   ncol_proc;        /* n^(j), columns on this rank */
  const isvd_int_t   nrow_each;        /* m_b = ceil(m / P) */
  const isvd_int_t   ncol_each;        /* n_b = ceil(n / P) */
  const isvd_int_t   nrow_total;       /* P m_b */
  const isvd_int_t   ncol_total;       /* P n_b */
  const isvd_int_t   rowidxbegin;      /* first row of this rank */
  const isvd_int_t   rowidxend;        /* one past the last row */
  const isvd_int_t   colidxbegin;      /* first column of this rank */
  const isvd_int_t   colidxend;        /* one past the last column */
  const isvd_int_t   rank;             /* k, target rank */
  const isvd_int_t   over_rank;        /* p, oversampling */
  const isvd_int_t   dim_sketch;       /* l = k + p */
  const isvd_int_t   dim_sketch_total; /* N l */
  const isvd_int_t   num_sketch;       /* N, number of sketches */
} isvd_Param;

/* Replaces isvd_createParam (reference core/param.c:14).  Unlike the reference,
 * tall matrices (nrow > ncol) are accepted. */
isvd_Param isvd_createParam(
    const isvd_int_t nrow, const isvd_int_t ncol, const isvd_int_t rank, const isvd_int_t over_rank,
    const isvd_int_t num_sketch, const mpi_int_t mpi_root, const isvd_MpiComm mpi_comm
);

#if defined(__cplusplus)
}
#endif

#endif  /* ISVD_CORE_PARAM_H_ */
