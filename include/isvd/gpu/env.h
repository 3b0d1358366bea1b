/* GPU environment (reference src/include/c/isvd/gpu/env.h:19-25; gpu/env.c:19-58). */
#ifndef ISVD_GPU_ENV_H_
#define ISVD_GPU_ENV_H_

#include <isvd/def.h>

#if defined(__cplusplus)
extern "C" {
#endif

/* Replaces the global of reference gpu/env.c:19.  0 = no limit.  Device memory is planned
 * against min(free device memory, this limit): a host A that does not fit beside the solve's
 * other buffers is streamed through the device in row panels, by the sketch and again by the
 * postprocessing projection, each copy overlapped with the previous panel's products (the
 * reference streams column panels sized the same way, gpu/stage/@x@_sketch_gpu.h:65-135). */
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
