/*
 * Test stand-in for an MPI whose communicator handle is a pointer, as in Open MPI (MPICH and the
 * single-rank stand-in in include/mpi_shim use an int).  It exists to check that the library,
 * built against such an mpi.h (isvd_b200/build.py --mpi-include), lays out isvd_Param as the
 * reference does under the same header and calls "MPI" through it.
 *
 * A communicator points to a struct isvd_test_comm that the test fills: its size and rank, and an
 * optional in-place sum used by MPI_Allreduce (called with the element count and the element size
 * in bytes).  A null communicator has one rank.  No MPI symbol is exported (static inline only).
 */
#ifndef ISVD_TEST_MPI_PTR_H_
#define ISVD_TEST_MPI_PTR_H_

#include <stddef.h>
#include <string.h>

#if defined(__cplusplus)
extern "C" {
#endif

struct isvd_test_comm {
  int size;
  int rank;
  void (*allreduce)(void *buf, int count, int elem_bytes, void *user);
  void *user;
};
typedef struct isvd_test_comm *MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;

#define MPI_SUCCESS       0
#define MPI_ERR_OTHER     15
#define MPI_COMM_NULL     ((MPI_Comm)0)
#define MPI_IN_PLACE      ((void *)-1)

#define MPI_INT           ((MPI_Datatype)0x0304)
#define MPI_INTEGER4      ((MPI_Datatype)0x0404)
#define MPI_INTEGER8      ((MPI_Datatype)0x0508)
#define MPI_FLOAT         ((MPI_Datatype)0x0604)
#define MPI_DOUBLE        ((MPI_Datatype)0x0708)
#define MPI_REAL4         ((MPI_Datatype)0x0804)
#define MPI_REAL8         ((MPI_Datatype)0x0908)
#define MPI_INT64_T       ((MPI_Datatype)0x0c08)
#define MPI_SUM           ((MPI_Op)1)

static inline int MPI_Init(int *argc, char ***argv) { (void)argc; (void)argv; return MPI_SUCCESS; }
static inline int MPI_Finalize(void) { return MPI_SUCCESS; }
static inline int MPI_Comm_size(MPI_Comm c, int *size) { *size = c ? c->size : 1; return MPI_SUCCESS; }
static inline int MPI_Comm_rank(MPI_Comm c, int *rank) { *rank = c ? c->rank : 0; return MPI_SUCCESS; }

static inline int MPI_Allreduce(const void *send, void *recv, int count, MPI_Datatype t, MPI_Op op, MPI_Comm c) {
  const int esz = t & 0xff;
  if (op != MPI_SUM || count < 0) return MPI_ERR_OTHER;
  if (send != MPI_IN_PLACE) memmove(recv, send, (size_t)count * (size_t)esz);
  if (c && c->size > 1) {
    if (!c->allreduce) return MPI_ERR_OTHER;
    c->allreduce(recv, count, esz, c->user);
  }
  return MPI_SUCCESS;
}

#if defined(__cplusplus)
}
#endif

#endif  /* ISVD_TEST_MPI_PTR_H_ */
