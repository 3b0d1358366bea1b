/* GPU-named API (reference src/include/c/isvd/gpu.h). */
#ifndef ISVD_GPU_H_
#define ISVD_GPU_H_

#include <isvd/gpu/env.h>
#include <isvd/gpu/s_stage.h>
#include <isvd/gpu/d_stage.h>

#endif  /* ISVD_GPU_H_ */
