// General strided matrix product on CUDA cores (FP64 / FP32), used by the NATIVE precision path
// and for the small (Nl x l, l x l) products of the integration loop.
//
// Tiling: BM x BN output tile per 256-thread CTA, BK-deep K slices staged in shared memory
// with register prefetch of the next slice; each thread owns a (BM/16) x (BN/16) register
// block at rows ty + 16 i, cols tx + 16 j (conflict-free shared reads, coalesced stores).
// Tall-skinny products (K >> M N) are split along K; partials are summed in FP64.
#include <algorithm>
#include <type_traits>

#include "kernels.h"
#include "runtime.h"

namespace isvdb {
namespace {

constexpr int kThreads = 256;

template <class T, class Tout, int BM, int BN, int BK, bool A_KC, bool B_NC>
__global__ void __launch_bounds__(kThreads)
    gemm_kernel(const Gemm<T, Tout> g, const int splits, const int kchunk, T *__restrict__ partial) {
  constexpr int TM = BM / 16, TN = BN / 16;
  constexpr int LA = BM * BK / kThreads, LB = BK * BN / kThreads;
  __shared__ T As[BK][BM + 1];
  __shared__ T Bs[BK][BN + 1];

  const int tid = threadIdx.x, tx = tid & 15, ty = tid >> 4;
  const int m0 = blockIdx.x * BM, n0 = blockIdx.y * BN;
  if (g.upper && n0 + BN <= m0) return;  // tile strictly below the diagonal: mirrored by the caller
  const int b = blockIdx.z / splits, sp = blockIdx.z % splits;
  const int kb = sp * kchunk;
  const int ke = min(g.K, kb + kchunk);
  const T *__restrict__ A = g.A + (long long)b * g.a_bs;
  const T *__restrict__ B = g.B + (long long)b * g.b_bs;

  T acc[TM][TN];
#pragma unroll
  for (int i = 0; i < TM; ++i)
#pragma unroll
    for (int j = 0; j < TN; ++j) acc[i][j] = T(0);

  T ra[LA], rb[LB];
  auto a_idx = [](int e, int &mm, int &kk) {
    if (A_KC) { kk = e % BK; mm = e / BK; } else { mm = e % BM; kk = e / BM; }
  };
  auto b_idx = [](int e, int &kk, int &nn) {
    if (B_NC) { nn = e % BN; kk = e / BN; } else { kk = e % BK; nn = e / BK; }
  };
  auto load = [&](int k0) {
#pragma unroll
    for (int r = 0; r < LA; ++r) {
      int mm, kk;
      a_idx(tid + r * kThreads, mm, kk);
      const int gm = m0 + mm, gk = k0 + kk;
      ra[r] = (gm < g.M && gk < ke) ? A[(long long)gm * g.a_rs + (long long)gk * g.a_cs] : T(0);
    }
#pragma unroll
    for (int r = 0; r < LB; ++r) {
      int kk, nn;
      b_idx(tid + r * kThreads, kk, nn);
      const int gn = n0 + nn, gk = k0 + kk;
      rb[r] = (gn < g.N && gk < ke) ? B[(long long)gk * g.b_rs + (long long)gn * g.b_cs] : T(0);
    }
  };
  auto store = [&]() {
#pragma unroll
    for (int r = 0; r < LA; ++r) {
      int mm, kk;
      a_idx(tid + r * kThreads, mm, kk);
      As[kk][mm] = ra[r];
    }
#pragma unroll
    for (int r = 0; r < LB; ++r) {
      int kk, nn;
      b_idx(tid + r * kThreads, kk, nn);
      Bs[kk][nn] = rb[r];
    }
  };

  if (kb < ke) load(kb);
  for (int k0 = kb; k0 < ke; k0 += BK) {
    store();
    __syncthreads();
    if (k0 + BK < ke) load(k0 + BK);
#pragma unroll
    for (int kk = 0; kk < BK; ++kk) {
      T av[TM], bv[TN];
#pragma unroll
      for (int i = 0; i < TM; ++i) av[i] = As[kk][ty + 16 * i];
#pragma unroll
      for (int j = 0; j < TN; ++j) bv[j] = Bs[kk][tx + 16 * j];
#pragma unroll
      for (int i = 0; i < TM; ++i)
#pragma unroll
        for (int j = 0; j < TN; ++j) acc[i][j] = fma(av[i], bv[j], acc[i][j]);
    }
    __syncthreads();
  }

  if (splits == 1) {
    Tout *__restrict__ C = g.C + (long long)b * g.c_bs;
#pragma unroll
    for (int i = 0; i < TM; ++i) {
      const int gm = m0 + ty + 16 * i;
      if (gm >= g.M) continue;
#pragma unroll
      for (int j = 0; j < TN; ++j) {
        const int gn = n0 + tx + 16 * j;
        if (gn >= g.N) continue;
        Tout *c = C + (long long)gm * g.c_rs + (long long)gn * g.c_cs;
        double v = g.alpha * (double)acc[i][j];
        if (g.beta != 0.0) v += g.beta * (double)(*c);
        *c = (Tout)v;
      }
    }
  } else {
    T *__restrict__ P = partial + ((long long)blockIdx.z * g.M) * g.N;
#pragma unroll
    for (int i = 0; i < TM; ++i) {
      const int gm = m0 + ty + 16 * i;
      if (gm >= g.M) continue;
#pragma unroll
      for (int j = 0; j < TN; ++j) {
        const int gn = n0 + tx + 16 * j;
        if (gn < g.N) P[(long long)gm * g.N + gn] = acc[i][j];
      }
    }
  }
}

// C = alpha * (sum of the split partials) + beta * C.  Eight lanes per output: lane u adds the
// partials of splits u, u + 8, u + 16, ... in increasing order (eight loads in flight per output
// across the lanes, several outputs per warp), then the eight sums are combined by shuffles as
// ((s0 + s1) + (s2 + s3)) + ((s4 + s5) + (s6 + s7)) -- a fixed order, the same in every launch.
template <class T, class Tout>
__global__ void splitk_reduce_kernel(const Gemm<T, Tout> g, const int splits, const T *__restrict__ partial) {
  const long long MN = (long long)g.M * g.N;
  const long long total = MN * g.batch;
  const int u = threadIdx.x & 7;
  const long long groups0 = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 3;
  const long long gstride = ((long long)gridDim.x * blockDim.x) >> 3;
  // every lane of a warp runs the same number of loop trips (the shuffles need all 32)
  const long long trips = (total + gstride - 1) / gstride;
  for (long long t = 0; t < trips; ++t) {
    const long long e = groups0 + t * gstride;
    const bool live = e < total;
    double acc = 0.0;
    long long r = 0;
    int b = 0;
    if (live) {
      b = (int)(e / MN);
      r = e - (long long)b * MN;
      const T *p = partial + ((long long)b * splits) * MN + r;
      for (int sp = u; sp < splits; sp += 8) acc += (double)p[(long long)sp * MN];
    }
    acc += __shfl_down_sync(0xffffffffu, acc, 1);
    acc += __shfl_down_sync(0xffffffffu, acc, 2);
    acc += __shfl_down_sync(0xffffffffu, acc, 4);
    if (live && u == 0) {
      const int gm = (int)(r / g.N), gn = (int)(r - (long long)gm * g.N);
      Tout *c = g.C + (long long)b * g.c_bs + (long long)gm * g.c_rs + (long long)gn * g.c_cs;
      double v = g.alpha * acc;
      if (g.beta != 0.0) v += g.beta * (double)(*c);
      *c = (Tout)v;
    }
  }
}

template <class T, class Tout, int BM, int BN, int BK>
void launch(const Gemm<T, Tout> &g, bool a_kc, bool b_nc, cudaStream_t st) {
  Runtime &rt = Runtime::get();
  const int gx = (g.M + BM - 1) / BM, gy = (g.N + BN - 1) / BN;
  const long long tiles = (long long)gx * gy * g.batch;
  int splits = g.splits;
  if (splits <= 0) {
    const long long target = 2LL * rt.num_sms;
    splits = 1;
    if (tiles < target) {
      long long s = (target + tiles - 1) / tiles;
      long long smax = std::max<long long>(1, g.K / (8 * BK));
      splits = (int)std::min<long long>(s, smax);
    }
  }
  int kchunk = (g.K + splits - 1) / splits;
  kchunk = ((kchunk + BK - 1) / BK) * BK;
  if (kchunk <= 0) kchunk = BK;
  splits = std::max(1, (g.K + kchunk - 1) / kchunk);
  DBuf<T> part;
  if (splits > 1) part.alloc((size_t)g.batch * splits * g.M * g.N);
  dim3 grid(gx, gy, g.batch * splits);
#define ISVD_GEMM_CASE(AK, BN_)                                                                   \
  if (a_kc == AK && b_nc == BN_) {                                                                \
    gemm_kernel<T, Tout, BM, BN, BK, AK, BN_><<<grid, kThreads, 0, st>>>(g, splits, kchunk, part.p); \
    KLAUNCHED();                                                                                  \
  }
  ISVD_GEMM_CASE(true, true)
  ISVD_GEMM_CASE(true, false)
  ISVD_GEMM_CASE(false, true)
  ISVD_GEMM_CASE(false, false)
#undef ISVD_GEMM_CASE
  if (splits > 1) {
    const long long total = (long long)g.M * g.N * g.batch;
    int blocks = (int)std::min<long long>((8 * total + 255) / 256, 16LL * rt.num_sms);  // 8 lanes per output
    splitk_reduce_kernel<T, Tout><<<blocks, 256, 0, st>>>(g, splits, part.p);
    KLAUNCHED();
  }
}

// As launch(), for callers that cannot allocate: the SM count comes from the caller and the
// split-K partial sums go to the caller's buffer of `cap` elements (fewer splits when it is short).
template <class T, class Tout, int BM, int BN, int BK>
void launch_fixed(const Gemm<T, Tout> &g, bool a_kc, bool b_nc, int sms, T *partial, size_t cap, cudaStream_t st) {
  const int gx = (g.M + BM - 1) / BM, gy = (g.N + BN - 1) / BN;
  const long long tiles = (long long)gx * gy * g.batch;
  int splits = g.splits;
  if (splits <= 0) {
    const long long target = 2LL * sms;
    splits = 1;
    if (tiles < target) {
      long long s = (target + tiles - 1) / tiles;
      long long smax = std::max<long long>(1, g.K / (8 * BK));
      splits = (int)std::min<long long>(s, smax);
    }
  }
  const long long per_split = (long long)g.batch * g.M * g.N;
  const long long fit = partial ? (long long)(cap / (size_t)per_split) : 1;
  splits = (int)std::max<long long>(1, std::min<long long>(splits, fit));
  int kchunk = (g.K + splits - 1) / splits;
  kchunk = ((kchunk + BK - 1) / BK) * BK;
  if (kchunk <= 0) kchunk = BK;
  splits = std::max(1, (g.K + kchunk - 1) / kchunk);
  T *part = splits > 1 ? partial : nullptr;
  dim3 grid(gx, gy, g.batch * splits);
#define ISVD_GEMM_CASE(AK, BN_)                                                                   \
  if (a_kc == AK && b_nc == BN_) {                                                                \
    gemm_kernel<T, Tout, BM, BN, BK, AK, BN_><<<grid, kThreads, 0, st>>>(g, splits, kchunk, part); \
    KLAUNCHED();                                                                                  \
  }
  ISVD_GEMM_CASE(true, true)
  ISVD_GEMM_CASE(true, false)
  ISVD_GEMM_CASE(false, true)
  ISVD_GEMM_CASE(false, false)
#undef ISVD_GEMM_CASE
  if (splits > 1) {
    const long long total = (long long)g.M * g.N * g.batch;
    int blocks = (int)std::min<long long>((8 * total + 255) / 256, 16LL * sms);  // 8 lanes per output
    splitk_reduce_kernel<T, Tout><<<blocks, 256, 0, st>>>(g, splits, part);
    KLAUNCHED();
  }
}

}  // namespace

void splitk_reduce(const Gemm<double, double> &g, int splits, const double *partial, cudaStream_t st) {
  const long long total = (long long)g.M * g.N * g.batch;
  const int blocks = (int)std::min<long long>((8 * total + 255) / 256, 16LL * Runtime::get().num_sms);
  splitk_reduce_kernel<double, double><<<blocks, 256, 0, st>>>(g, splits, partial);
  KLAUNCHED();
}

template <class T, class Tout>
void gemm(const Gemm<T, Tout> &g, cudaStream_t st) {
  if (g.M <= 0 || g.N <= 0 || g.batch <= 0) return;
  if (g.K <= 0) {
    if (g.beta == 1.0) return;
    fail(kErrArgument, "gemm: empty inner dimension with beta != 1");
  }
  const bool a_kc = (g.a_cs == 1);
  const bool b_nc = (g.b_cs == 1);
  if (!a_kc && g.a_rs != 1) fail(kErrArgument, "gemm: operand A has no unit stride");
  if (!b_nc && g.b_rs != 1) fail(kErrArgument, "gemm: operand B has no unit stride");
  if constexpr (std::is_same<T, double>::value && std::is_same<Tout, double>::value) {
    if (dmma_enabled()) {  // FP64 operands: the FP64 tensor-core path (k_dmma.cu)
      dmma_gemm(g, a_kc, b_nc, st);
      return;
    }
  }
  if (g.pl_t) fail(kErrArgument, "gemm: plane output only on the FP64 tensor-core path");
  // 128 x 128 tiles when they fill the GPU, or when a long inner dimension lets split-K fill it
  // (8 x 8 register blocks: half the shared-memory reads per FMA of 64 x 64 tiles); otherwise
  // 64 x 64 tiles (4x more CTAs)
  const long long tiles128 = (long long)((g.M + 127) / 128) * ((g.N + 127) / 128) * g.batch;
  const int sms = Runtime::get().num_sms;
  const bool long_k = g.splits <= 0 && (long long)g.K >= 2048 && tiles128 * (g.K / 1024) >= 2LL * sms;
  if (g.M <= 64 || g.N <= 64 || (tiles128 < 2LL * sms && !long_k))
    launch<T, Tout, 64, 64, 16>(g, a_kc, b_nc, st);
  else
    launch<T, Tout, 128, 128, 16>(g, a_kc, b_nc, st);
}

template <class T, class Tout>
void gemm_fixed(const Gemm<T, Tout> &g, int num_sms, T *partial, size_t cap, cudaStream_t st) {
  if (g.M <= 0 || g.N <= 0 || g.batch <= 0) return;
  if (g.K <= 0) {
    if (g.beta == 1.0) return;
    fail(kErrArgument, "gemm: empty inner dimension with beta != 1");
  }
  const bool a_kc = (g.a_cs == 1);
  const bool b_nc = (g.b_cs == 1);
  if (!a_kc && g.a_rs != 1) fail(kErrArgument, "gemm: operand A has no unit stride");
  if (!b_nc && g.b_rs != 1) fail(kErrArgument, "gemm: operand B has no unit stride");
  const long long tiles128 = (long long)((g.M + 127) / 128) * ((g.N + 127) / 128) * g.batch;
  if (g.M <= 64 || g.N <= 64 || tiles128 < 2LL * num_sms)
    launch_fixed<T, Tout, 64, 64, 16>(g, a_kc, b_nc, num_sms, partial, cap, st);
  else
    launch_fixed<T, Tout, 128, 128, 16>(g, a_kc, b_nc, num_sms, partial, cap, st);
}

template void gemm_fixed<double, double>(const Gemm<double, double> &, int, double *, size_t, cudaStream_t);

void gemm_fixed_preload() {
  cudaFuncAttributes fa;
#define ISVD_PRELOAD(BM_, BN_, AK, BNC)                                                         \
  CK(cudaFuncGetAttributes(&fa, gemm_kernel<double, double, BM_, BN_, 16, AK, BNC>));
  ISVD_PRELOAD(64, 64, true, true)
  ISVD_PRELOAD(64, 64, true, false)
  ISVD_PRELOAD(64, 64, false, true)
  ISVD_PRELOAD(64, 64, false, false)
  ISVD_PRELOAD(128, 128, true, true)
  ISVD_PRELOAD(128, 128, true, false)
  ISVD_PRELOAD(128, 128, false, true)
  ISVD_PRELOAD(128, 128, false, false)
#undef ISVD_PRELOAD
  CK(cudaFuncGetAttributes(&fa, splitk_reduce_kernel<double, double>));
}

template void gemm<double, double>(const Gemm<double, double> &, cudaStream_t);
template void gemm<float, float>(const Gemm<float, float> &, cudaStream_t);
template void gemm<float, double>(const Gemm<float, double> &, cudaStream_t);

}  // namespace isvdb
