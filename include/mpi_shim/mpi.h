/*
 * Single-process stand-in for <mpi.h>.
 *
 * The iSVD C API embeds an MPI communicator in `isvd_Param` and its stages call
 * a handful of MPI collectives.  This header lets the API compile and run
 * without an MPI installation: every communicator has exactly one rank (rank 0),
 * so each collective reduces to a local copy (or nothing for MPI_IN_PLACE).
 *
 * Only the subset of MPI that the iSVD stage routines use is provided:
 *   MPI_Init / MPI_Finalize / MPI_Initialized / MPI_Comm_size / MPI_Comm_rank,
 *   MPI_Bcast, MPI_Allreduce, MPI_Reduce_scatter_block, MPI_Allgather,
 *   MPI_Gather, MPI_Sendrecv, MPI_Wtime.
 * Everything is `static inline`, so no MPI symbol is exported from any
 * library compiled against this header (a real MPI can still be linked into
 * the same process without symbol clashes).
 *
 * Datatype handles encode their element size in the low byte.
 */
#ifndef ISVD_MPI_SHIM_H_
#define ISVD_MPI_SHIM_H_

#include <string.h>
#include <time.h>

#if defined(__cplusplus)
extern "C" {
#endif

#define ISVD_MPI_SHIM 1

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
typedef struct { int MPI_SOURCE; int MPI_TAG; int MPI_ERROR; } MPI_Status;

#define MPI_SUCCESS       0
#define MPI_COMM_WORLD    ((MPI_Comm)0x44000000)
#define MPI_COMM_SELF     ((MPI_Comm)0x44000001)
#define MPI_IN_PLACE      ((void *)-1)
#define MPI_STATUS_IGNORE ((MPI_Status *)0)

#define MPI_BYTE          ((MPI_Datatype)0x0101)
#define MPI_CHAR          ((MPI_Datatype)0x0201)
#define MPI_INT           ((MPI_Datatype)0x0304)
#define MPI_INTEGER4      ((MPI_Datatype)0x0404)
#define MPI_INTEGER8      ((MPI_Datatype)0x0508)
#define MPI_FLOAT         ((MPI_Datatype)0x0604)
#define MPI_DOUBLE        ((MPI_Datatype)0x0708)
#define MPI_REAL4         ((MPI_Datatype)0x0804)
#define MPI_REAL8         ((MPI_Datatype)0x0908)
#define MPI_COMPLEX8      ((MPI_Datatype)0x0a08)
#define MPI_COMPLEX16     ((MPI_Datatype)0x0b10)
#define MPI_INT64_T       ((MPI_Datatype)0x0c08)

#define MPI_SUM           ((MPI_Op)1)
#define MPI_MAX           ((MPI_Op)2)
#define MPI_MIN           ((MPI_Op)3)

static inline size_t isvd_mpi_shim_size_(MPI_Datatype t) { return (size_t)(t & 0xff); }

static inline void isvd_mpi_shim_copy_(void *dst, const void *src, int count, MPI_Datatype t) {
  if (src == MPI_IN_PLACE || dst == NULL || src == NULL || dst == src || count <= 0) return;
  memmove(dst, src, (size_t)count * isvd_mpi_shim_size_(t));
}

static inline int MPI_Init(int *argc, char ***argv) { (void)argc; (void)argv; return MPI_SUCCESS; }
static inline int MPI_Finalize(void) { return MPI_SUCCESS; }
static inline int MPI_Initialized(int *flag) { if (flag) *flag = 1; return MPI_SUCCESS; }
static inline int MPI_Comm_size(MPI_Comm c, int *size) { (void)c; *size = 1; return MPI_SUCCESS; }
static inline int MPI_Comm_rank(MPI_Comm c, int *rank) { (void)c; *rank = 0; return MPI_SUCCESS; }

static inline int MPI_Bcast(void *buf, int count, MPI_Datatype t, int root, MPI_Comm c) {
  (void)buf; (void)count; (void)t; (void)root; (void)c; return MPI_SUCCESS;
}

static inline int MPI_Allreduce(const void *send, void *recv, int count, MPI_Datatype t, MPI_Op op, MPI_Comm c) {
  (void)op; (void)c; isvd_mpi_shim_copy_(recv, send, count, t); return MPI_SUCCESS;
}

static inline int MPI_Reduce_scatter_block(const void *send, void *recv, int count, MPI_Datatype t, MPI_Op op,
                                           MPI_Comm c) {
  (void)op; (void)c; isvd_mpi_shim_copy_(recv, send, count, t); return MPI_SUCCESS;
}

static inline int MPI_Allgather(const void *send, int scount, MPI_Datatype st, void *recv, int rcount,
                                MPI_Datatype rt, MPI_Comm c) {
  (void)rcount; (void)rt; (void)c; isvd_mpi_shim_copy_(recv, send, scount, st); return MPI_SUCCESS;
}

static inline int MPI_Gather(const void *send, int scount, MPI_Datatype st, void *recv, int rcount,
                             MPI_Datatype rt, int root, MPI_Comm c) {
  (void)rcount; (void)rt; (void)root; (void)c; isvd_mpi_shim_copy_(recv, send, scount, st); return MPI_SUCCESS;
}

static inline int MPI_Sendrecv(const void *send, int scount, MPI_Datatype st, int dest, int stag, void *recv,
                               int rcount, MPI_Datatype rt, int src, int rtag, MPI_Comm c, MPI_Status *status) {
  (void)dest; (void)stag; (void)rcount; (void)rt; (void)src; (void)rtag; (void)c; (void)status;
  isvd_mpi_shim_copy_(recv, send, scount, st); return MPI_SUCCESS;
}

static inline double MPI_Wtime(void) {
  struct timespec ts;
  clock_gettime(CLOCK_MONOTONIC, &ts);
  return (double)ts.tv_sec + 1e-9 * (double)ts.tv_nsec;
}

#if defined(__cplusplus)
}
#endif

#endif  /* ISVD_MPI_SHIM_H_ */
