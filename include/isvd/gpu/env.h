/* GPU environment (reference src/include/c/isvd/gpu/env.h:19-25; gpu/env.c:19-58). */
#ifndef ISVD_GPU_ENV_H_
#define ISVD_GPU_ENV_H_

#include <isvd/def.h>

#if defined(__cplusplus)
extern "C" {
#endif

/* Replaces the global of reference gpu/env.c:19.  0 = no limit.  When A does not fit
 * under the limit next to the sketch, A is streamed through the device in column
 * panels as the reference does (gpu/stage/@x@_sketch_gpu.h:65-77). */
extern size_t isvd_gpu_memory_limit;

/* Replaces isvd_Init_gpu (reference gpu/env.c:27): selects device (rank % device count). */
void isvd_Init_gpu( int *argcp, char ***argvp, const isvd_MpiComm mpi_comm );
/* Replaces isvd_Finalize_gpu (reference gpu/env.c:45): releases the device context. */
void isvd_Finalize_gpu( void );
/* Replaces isvd_PrintEnvironment_gpu (reference gpu/env.c:54). */
void isvd_PrintEnvironment_gpu( const isvd_MpiComm comm );

#if defined(__cplusplus)
}
#endif

#endif  /* ISVD_GPU_ENV_H_ */
