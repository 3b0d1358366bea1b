// Elementwise kernels: Gaussian test matrix (Philox4x32-10 + Box-Muller), strided copies,
// identity fill, column scaling.
#include <cuda_bf16.h>

#include <algorithm>

#include "kernels.h"
#include "runtime.h"

namespace isvdb {
namespace {

inline int grid_for(long long n, int threads) {
  const long long cap = 16LL * Runtime::get().num_sms;
  return (int)std::max<long long>(1, std::min<long long>((n + threads - 1) / threads, cap));
}

// Philox4x32-10 (Salmon, Moraes, Dror, Shaw, "Parallel random numbers: as easy as 1, 2, 3", SC'11).
__device__ __forceinline__ uint4 philox4x32_10(uint4 c, uint32_t k0, uint32_t k1) {
  const uint32_t M0 = 0xD2511F53u, M1 = 0xCD9E8D57u, W0 = 0x9E3779B9u, W1 = 0xBB67AE85u;
#pragma unroll
  for (int r = 0; r < 10; ++r) {
    const uint32_t hi0 = __umulhi(M0, c.x), lo0 = M0 * c.x;
    const uint32_t hi1 = __umulhi(M1, c.z), lo1 = M1 * c.z;
    c = make_uint4(hi1 ^ c.y ^ k0, lo1, hi0 ^ c.w ^ k1, lo0);
    k0 += W0;
    k1 += W1;
  }
  return c;
}

// Two standard normals from one Philox block: u1 in (0,1], u2 in [0,1) with 53-bit resolution,
// z0 = r cos(2 pi u2), z1 = r sin(2 pi u2), r = sqrt(-2 ln u1)  (Box & Muller, 1958).
__device__ __forceinline__ double2 normal_pair(uint64_t pair, uint64_t seed) {
  const uint4 x = philox4x32_10(make_uint4((uint32_t)pair, (uint32_t)(pair >> 32), 0u, 0u), (uint32_t)seed,
                                (uint32_t)(seed >> 32));
  const uint64_t a = ((((uint64_t)x.x) << 32) | x.y) >> 11;
  const uint64_t b = ((((uint64_t)x.z) << 32) | x.w) >> 11;
  const double u1 = (double)(a + 1) * 0x1.0p-53;
  const double u2 = (double)b * 0x1.0p-53;
  const double r = sqrt(-2.0 * log(u1));
  double s, c;
  sincospi(2.0 * u2, &s, &c);
  return make_double2(r * c, r * s);
}

template <class T>
__global__ void rng_gaussian_kernel(T *__restrict__ out, long long rows, long long cols, long long ld,
                                    uint64_t seed, uint64_t offset) {
  const long long total = rows * cols;
  // value index v = offset + e (e = j * cols + c); pairs are (2p, 2p+1) in v-space.
  const long long p_begin = (long long)(offset >> 1);
  const long long p_end = (long long)((offset + (uint64_t)total + 1) >> 1);
  for (long long p = p_begin + blockIdx.x * (long long)blockDim.x + threadIdx.x; p < p_end;
       p += (long long)gridDim.x * blockDim.x) {
    const double2 z = normal_pair((uint64_t)p, seed);
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const long long v = 2 * p + h;
      const long long e = v - (long long)offset;
      if (e < 0 || e >= total) continue;
      const long long j = e / cols, c = e - j * cols;
      // rounded to bf16 (8 significant bits) so that every precision mode draws the same Omega
      out[j * ld + c] = (T)__bfloat162float(__double2bfloat16(h ? z.y : z.x));
    }
  }
}

template <class Ts, class Td>
__global__ void copy2d_kernel(const Ts *__restrict__ src, long long s_rs, long long s_cs, Td *__restrict__ dst,
                              long long d_rs, long long d_cs, long long rows, long long cols) {
  const long long total = rows * cols;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
       e += (long long)gridDim.x * blockDim.x) {
    long long i, j;
    if (d_cs == 1 || s_cs == 1) { i = e / cols; j = e - i * cols; }
    else { j = e / rows; i = e - j * rows; }
    dst[i * d_rs + j * d_cs] = (Td)src[i * s_rs + j * s_cs];
  }
}

template <class T>
__global__ void set_identity_kernel(T *__restrict__ a, long long rows, long long cols, long long ld) {
  const long long total = rows * cols;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
       e += (long long)gridDim.x * blockDim.x) {
    const long long i = e / cols, j = e - i * cols;
    a[i * ld + j] = (T)(i == j ? 1 : 0);
  }
}

template <class Ts, class Td>
__global__ void scale_cols_kernel(const Ts *__restrict__ src, long long lds, Td *__restrict__ dst, long long ldd,
                                  long long rows, long long cols, long long rpb, const double *__restrict__ s,
                                  int mode) {
  const long long total = rows * cols;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
       e += (long long)gridDim.x * blockDim.x) {
    const long long i = e / cols, j = e - i * cols;
    const double x = (double)src[i * lds + j];
    double v;
    if (mode == kSqrtOnly) {
      v = sqrt(x);
    } else {
      const double f = s[(i / rpb) * cols + j];
      switch (mode) {
        case kScaleMul: v = x * f; break;
        case kScaleDiv: v = x / f; break;
        case kScaleInvSqrt: v = x / sqrt(f); break;
        default: v = x / sqrt(2.0 * (1.0 + f)); break;
      }
    }
    dst[i * ldd + j] = (Td)v;
  }
}

// Null columns of a TS factorization get values uniform in [-1/2, 1/2): one Philox block per
// element, counter (row, column), key seed.
template <class T>
__global__ void fill_null_columns_kernel(T *__restrict__ y, long long ld, long long rows, int cols,
                                         const int *__restrict__ mask, uint64_t seed, long long row_offset) {
  const long long total = rows * cols;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
       e += (long long)gridDim.x * blockDim.x) {
    const long long i = e / cols;
    const int c = (int)(e - i * cols);
    if (!mask[c]) continue;
    const uint64_t row = (uint64_t)(row_offset + i);
    const uint4 x = philox4x32_10(make_uint4((uint32_t)row, (uint32_t)(row >> 32), (uint32_t)c, 0u), (uint32_t)seed,
                                  (uint32_t)(seed >> 32));
    y[i * ld + c] = (T)((double)(x.x >> 8) * 0x1.0p-24 - 0.5);
  }
}

// Per block of l columns: kept columns first, then the null ones, each in increasing order.
__global__ void kept_first_perm_kernel(const int *__restrict__ mask, int l, int N, int *__restrict__ perm) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= N) return;
  const int *m = mask + (size_t)b * l;
  int *p = perm + (size_t)b * l;
  int pos = 0;
  for (int j = 0; j < l; ++j)
    if (!m[j]) p[pos++] = j;
  for (int j = 0; j < l; ++j)
    if (m[j]) p[pos++] = j;
}

}  // namespace

template <class T>
void fill_null_columns(T *y, long long ld, long long rows, int cols, const int *mask, uint64_t seed,
                       long long row_offset, cudaStream_t st) {
  if (rows <= 0 || cols <= 0) return;
  fill_null_columns_kernel<T><<<grid_for(rows * cols, 256), 256, 0, st>>>(y, ld, rows, cols, mask, seed, row_offset);
  KLAUNCHED();
}

void kept_first_perm(const int *mask, int l, int N, int *perm, cudaStream_t st) {
  if (l <= 0 || N <= 0) return;
  kept_first_perm_kernel<<<(N + 127) / 128, 128, 0, st>>>(mask, l, N, perm);
  KLAUNCHED();
}

template void fill_null_columns<double>(double *, long long, long long, int, const int *, uint64_t, long long,
                                        cudaStream_t);
template void fill_null_columns<float>(float *, long long, long long, int, const int *, uint64_t, long long,
                                       cudaStream_t);

template <class T>
void rng_gaussian(T *out, long long rows, long long cols, long long ld, uint64_t seed, uint64_t offset,
                  cudaStream_t st) {
  if (rows <= 0 || cols <= 0) return;
  rng_gaussian_kernel<T><<<grid_for((rows * cols + 1) / 2 + 1, 256), 256, 0, st>>>(out, rows, cols, ld, seed, offset);
  KLAUNCHED();
}

template <class Ts, class Td>
void copy2d(const Ts *src, long long s_rs, long long s_cs, Td *dst, long long d_rs, long long d_cs, long long rows,
            long long cols, cudaStream_t st) {
  if (rows <= 0 || cols <= 0) return;
  copy2d_kernel<Ts, Td><<<grid_for(rows * cols, 256), 256, 0, st>>>(src, s_rs, s_cs, dst, d_rs, d_cs, rows, cols);
  KLAUNCHED();
}

template <class T>
void set_identity(T *a, long long rows, long long cols, long long ld, cudaStream_t st) {
  if (rows <= 0 || cols <= 0) return;
  set_identity_kernel<T><<<grid_for(rows * cols, 256), 256, 0, st>>>(a, rows, cols, ld);
  KLAUNCHED();
}

template <class Ts, class Td>
void scale_cols_batched(const Ts *src, long long lds, Td *dst, long long ldd, long long rows, long long cols,
                        long long rows_per_batch, const double *s, int mode, cudaStream_t st) {
  if (rows <= 0 || cols <= 0) return;
  scale_cols_kernel<Ts, Td><<<grid_for(rows * cols, 256), 256, 0, st>>>(src, lds, dst, ldd, rows, cols,
                                                                         rows_per_batch, s, mode);
  KLAUNCHED();
}

template void rng_gaussian<double>(double *, long long, long long, long long, uint64_t, uint64_t, cudaStream_t);
template void rng_gaussian<float>(float *, long long, long long, long long, uint64_t, uint64_t, cudaStream_t);
template void copy2d<double, double>(const double *, long long, long long, double *, long long, long long, long long,
                                     long long, cudaStream_t);
template void copy2d<float, float>(const float *, long long, long long, float *, long long, long long, long long,
                                   long long, cudaStream_t);
template void copy2d<float, double>(const float *, long long, long long, double *, long long, long long, long long,
                                    long long, cudaStream_t);
template void copy2d<double, float>(const double *, long long, long long, float *, long long, long long, long long,
                                    long long, cudaStream_t);
template void set_identity<double>(double *, long long, long long, long long, cudaStream_t);
template void set_identity<float>(float *, long long, long long, long long, cudaStream_t);
template void scale_cols_batched<double, double>(const double *, long long, double *, long long, long long,
                                                 long long, long long, const double *, int, cudaStream_t);
template void scale_cols_batched<double, float>(const double *, long long, float *, long long, long long,
                                                long long, long long, const double *, int, cudaStream_t);
template void scale_cols_batched<float, float>(const float *, long long, float *, long long, long long,
                                               long long, long long, const double *, int, cudaStream_t);

}  // namespace isvdb
