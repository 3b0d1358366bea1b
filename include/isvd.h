/*
 * iSVD C API, B200 implementation (libisvd_gpu_b200).
 *
 * Drop-in for the headers of emfomy/isvd v1.3.2 (src/include/c/isvd.h:13-16):
 * the same types, the same isvd_Param, the same driver / stage / environment /
 * memory entry points with the same argument meaning and layouts.  Every stage
 * runs on the GPU; the CPU-named stages and their `_gpu` twins are the same
 * implementation.  B200-only extensions live in <isvd/b200.h>.
 */
#ifndef ISVD_H_
#define ISVD_H_

#include <isvd/core.h>
#include <isvd/gpu.h>
#include <isvd/util.h>
#include <isvd/b200.h>

#endif  /* ISVD_H_ */
