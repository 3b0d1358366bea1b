// Device helpers of the bf16 plane representation x = x0 + x1 + x2 (+ O(2^-24 |x|)), shared by
// the kernels that write planes (splits, GEMM epilogues).
#pragma once

#include <cuda_bf16.h>

#include <cstdint>

namespace isvdb {

// Piece q of x: x0 = bf16(x), x1 = bf16(x - x0), x2 = bf16(x - x0 - x1) (round to nearest).
template <class T>
__device__ __forceinline__ void split3(T x, __nv_bfloat16 *o, int np) {
  double r = (double)x;
#pragma unroll
  for (int q = 0; q < 3; ++q) {
    if (q >= np) break;
    const __nv_bfloat16 h = __double2bfloat16(r);
    o[q] = h;
    r -= (double)__bfloat162float(h);
  }
}

__device__ __forceinline__ uint4 pack8(const __nv_bfloat16 *v) {
  uint4 u;
  u.x = (uint32_t)__bfloat16_as_ushort(v[0]) | ((uint32_t)__bfloat16_as_ushort(v[1]) << 16);
  u.y = (uint32_t)__bfloat16_as_ushort(v[2]) | ((uint32_t)__bfloat16_as_ushort(v[3]) << 16);
  u.z = (uint32_t)__bfloat16_as_ushort(v[4]) | ((uint32_t)__bfloat16_as_ushort(v[5]) << 16);
  u.w = (uint32_t)__bfloat16_as_ushort(v[6]) | ((uint32_t)__bfloat16_as_ushort(v[7]) << 16);
  return u;
}

}  // namespace isvdb
