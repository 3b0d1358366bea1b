// FP64 matrix product on the FP64 tensor-core path (mma.sync m8n8k4 .f64: the only tensor-core
// instruction with FP64 operands on sm_100a; tcgen05 has no FP64 kind).  Same contract as the
// CUDA-core gemm<double, double> (arbitrary strides with one unit stride per operand, batch,
// split-K, alpha / beta); every product term is an IEEE FP64 fused multiply-add, so results
// differ from the CUDA-core kernel only in the order of the K summation.
//
// Tiling: BM x BN output tile per CTA of WM x WN warps, each warp a (BM / WM) x (BN / WN) block
// of 8 x 8 mma tiles held in registers.  BK = 16 deep K slices are copied global -> shared by
// cp.async (8-byte elements, zero-filled outside the matrix) in a 3-stage ring.  Each operand is
// staged in the orientation of its unit stride (K-contiguous rows of BK + 4, or MN-contiguous
// rows of BM + 4 / BN + 4 doubles), which makes both the copies and the fragment reads free of
// shared-memory bank conflicts.
#include <algorithm>
#include <cstdlib>

#include "kernels.h"
#include "planes.cuh"
#include "runtime.h"

namespace isvdb {
namespace {

constexpr int kBK = 16, kStages = 3, kPad = 4;

__device__ __forceinline__ void cp_async8(void *smem, const void *gmem, bool valid) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(s), "l"(gmem), "r"(valid ? 8 : 0));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N)); }

// D = A B + D for one 8 x 8 x 4 tile: a = A(lane / 4, lane % 4), b = B(lane % 4, lane / 4),
// d = D(lane / 4, 2 (lane % 4) + {0, 1}).
__device__ __forceinline__ void dmma884(double (&d)[2], double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
               : "+d"(d[0]), "+d"(d[1])
               : "d"(a), "d"(b));
}

template <int BM, int BN, bool A_KC, bool B_NC>
struct DmmaLayout {
  static constexpr int a_elems = A_KC ? BM * (kBK + kPad) : kBK * (BM + kPad);
  static constexpr int b_elems = B_NC ? kBK * (BN + kPad) : BN * (kBK + kPad);
  static constexpr int stage = a_elems + b_elems;
  __device__ static int a_at(int m, int k) { return A_KC ? m * (kBK + kPad) + k : k * (BM + kPad) + m; }
  __device__ static int b_at(int k, int n) { return B_NC ? k * (BN + kPad) + n : n * (kBK + kPad) + k; }
};

// acc += A[m0 .. m0 + BM, kb .. ke) B[kb .. ke, n0 .. n0 + BN) for one output tile, with A(i, k) =
// A[i a_rs + k a_cs] and B(k, j) = B[k b_rs + j b_cs]; rows >= M, columns >= N read as zero.  K
// slices flow through the kStages-deep cp.async ring in smem.  On return every copy has landed,
// but warps may still read the ring: a caller that refills it must synchronise the block first.
template <int BM, int BN, int WM, int WN, bool A_KC, bool B_NC>
__device__ __forceinline__ void dmma_tile(double *smem, const double *__restrict__ A, long long a_rs, long long a_cs,
                                          const double *__restrict__ B, long long b_rs, long long b_cs, int M, int N,
                                          int kb, int ke, int m0, int n0,
                                          double (&acc)[BM / WM / 8][BN / WN / 8][2]) {
  using L = DmmaLayout<BM, BN, A_KC, B_NC>;
  constexpr int NT = WM * WN * 32;
  constexpr int TM = BM / WM / 8, TN = BN / WN / 8;  // 8 x 8 tiles per warp
  constexpr int LA = BM * kBK / NT, LB = BN * kBK / NT;
  static_assert(LA * NT == BM * kBK && LB * NT == BN * kBK, "tile / thread mismatch");
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int wm0 = (warp / WN) * (BM / WM), wn0 = (warp % WN) * (BN / WN);
  const int nk = ke > kb ? (ke - kb + kBK - 1) / kBK : 0;

  auto issue = [&](int kt) {  // k slice kt into stage kt % kStages
    double *As = smem + (kt % kStages) * L::stage, *Bs = As + L::a_elems;
    const int k0 = kb + kt * kBK;
#pragma unroll
    for (int r = 0; r < LA; ++r) {
      const int e = tid + r * NT;
      const int mm = A_KC ? e / kBK : e % BM, kk = A_KC ? e % kBK : e / BM;
      const int gm = m0 + mm, gk = k0 + kk;
      const bool ok = gm < M && gk < ke;
      cp_async8(As + L::a_at(mm, kk), ok ? A + (long long)gm * a_rs + (long long)gk * a_cs : A, ok);
    }
#pragma unroll
    for (int r = 0; r < LB; ++r) {
      const int e = tid + r * NT;
      const int nn = B_NC ? e % BN : e / kBK, kk = B_NC ? e / BN : e % kBK;
      const int gn = n0 + nn, gk = k0 + kk;
      const bool ok = gn < N && gk < ke;
      cp_async8(Bs + L::b_at(kk, nn), ok ? B + (long long)gk * b_rs + (long long)gn * b_cs : B, ok);
    }
  };

#pragma unroll
  for (int s = 0; s < kStages - 1; ++s) {
    if (s < nk) issue(s);
    cp_async_commit();
  }
  const int fr = lane >> 2, fc = lane & 3;  // fragment row / column within an 8 x 4 (4 x 8) tile
  for (int kt = 0; kt < nk; ++kt) {
    cp_async_wait<kStages - 2>();
    __syncthreads();  // slice kt visible to all; slice kt - 1 no longer read (its stage is refilled)
    if (kt + kStages - 1 < nk) issue(kt + kStages - 1);
    cp_async_commit();
    const double *As = smem + (kt % kStages) * L::stage, *Bs = As + L::a_elems;
#pragma unroll
    for (int k4 = 0; k4 < kBK; k4 += 4) {
      double av[TM], bv[TN];
#pragma unroll
      for (int i = 0; i < TM; ++i) av[i] = As[L::a_at(wm0 + 8 * i + fr, k4 + fc)];
#pragma unroll
      for (int j = 0; j < TN; ++j) bv[j] = Bs[L::b_at(k4 + fc, wn0 + 8 * j + fr)];
#pragma unroll
      for (int i = 0; i < TM; ++i)
#pragma unroll
        for (int j = 0; j < TN; ++j) dmma884(acc[i][j], av[i], bv[j]);
    }
  }
  cp_async_wait<0>();
}

template <int BM, int BN, int WM, int WN, bool A_KC, bool B_NC>
__global__ void __launch_bounds__(WM * WN * 32)
    dmma_gemm_kernel(const Gemm<double, double> g, const int splits, const int kchunk, double *__restrict__ partial) {
  constexpr int TM = BM / WM / 8, TN = BN / WN / 8;  // 8 x 8 tiles per warp
  extern __shared__ double smem[];

  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int wm0 = (warp / WN) * (BM / WM), wn0 = (warp % WN) * (BN / WN);
  const int m0 = blockIdx.x * BM, n0 = blockIdx.y * BN;
  if (g.upper && n0 + BN <= m0) return;  // tile strictly below the diagonal: mirrored by the caller
  const int b = blockIdx.z / splits, sp = blockIdx.z % splits;
  const int kb = sp * kchunk, ke = min(g.K, kb + kchunk);

  double acc[TM][TN][2];
#pragma unroll
  for (int i = 0; i < TM; ++i)
#pragma unroll
    for (int j = 0; j < TN; ++j) acc[i][j][0] = acc[i][j][1] = 0.0;
  dmma_tile<BM, BN, WM, WN, A_KC, B_NC>(smem, g.A + (long long)b * g.a_bs, g.a_rs, g.a_cs, g.B + (long long)b * g.b_bs,
                                        g.b_rs, g.b_cs, g.M, g.N, kb, ke, m0, n0, acc);

  const int fr = lane >> 2, fc = lane & 3;
  const bool direct = splits == 1;
  double *__restrict__ C = direct ? g.C + (long long)b * g.c_bs : partial + ((long long)blockIdx.z * g.M) * g.N;
#pragma unroll
  for (int i = 0; i < TM; ++i) {
    const int gm = m0 + wm0 + 8 * i + fr;
    if (gm >= g.M) continue;
#pragma unroll
    for (int j = 0; j < TN; ++j)
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int gn = n0 + wn0 + 8 * j + 2 * fc + h;
        if (gn >= g.N) continue;
        if (direct) {
          double *c = C + (long long)gm * g.c_rs + (long long)gn * g.c_cs;
          double v = g.alpha * acc[i][j][h];
          if (g.beta != 0.0) v += g.beta * *c;
          *c = v;
          acc[i][j][h] = v;  // the stored value, for the plane output below
        } else {
          C[(long long)gm * g.N + gn] = acc[i][j][h];
        }
      }
  }
  using L = DmmaLayout<BM, BN, A_KC, B_NC>;
  if constexpr (BN * (BM + 1) <= kStages * L::stage) {
    if (direct && g.pl_t && b == g.pl_batch) {
      // bf16 planes of this tile's transpose: the values go through the (now idle) cp.async ring
      // as a BN x BM tile, then each thread splits 8 consecutive rows of one output column and
      // stores 16 bytes per plane (plane row gn, columns gm .. gm + 7)
      constexpr int TLD = BM + 1;
      __syncthreads();
#pragma unroll
      for (int i = 0; i < TM; ++i)
#pragma unroll
        for (int j = 0; j < TN; ++j)
#pragma unroll
          for (int h = 0; h < 2; ++h)
            smem[(wn0 + 8 * j + 2 * fc + h) * TLD + (wm0 + 8 * i + fr)] = acc[i][j][h];
      __syncthreads();
      constexpr int NT = WM * WN * 32;
      for (int t = tid; t < BN * (BM / 8); t += NT) {
        const int cl = t / (BM / 8), seg = t - cl * (BM / 8);
        const int gn = n0 + cl;
        if (gn >= g.N) continue;
        __nv_bfloat16 o[3][8];
#pragma unroll
        for (int e = 0; e < 8; ++e) {
          __nv_bfloat16 pc[3];
          split3<double>(smem[cl * TLD + 8 * seg + e], pc, 3);
#pragma unroll
          for (int q = 0; q < 3; ++q) o[q][e] = pc[q];
        }
        const long long po = (long long)gn * g.pl_ld + m0 + 8 * seg;
#pragma unroll
        for (int q = 0; q < 3; ++q) *(uint4 *)(g.pl_t + q * g.pl_ps + po) = pack8(o[q]);
      }
    }
  }
}

// Grouped products (dmma_grouped): each CTA walks the work items blockIdx.x, blockIdx.x + gridDim.x,
// ...; a work item is one BM x BN output tile of the product that owns it (binary search on tile0).
template <int BM, int BN, int WM, int WN, bool A_KC, bool B_NC>
__global__ void __launch_bounds__(WM * WN * 32)
    dmma_grouped_kernel(const GroupedProd *__restrict__ prods, int nprod, int total) {
  constexpr int TM = BM / WM / 8, TN = BN / WN / 8;
  extern __shared__ double smem[];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int wm0 = (warp / WN) * (BM / WM), wn0 = (warp % WN) * (BN / WN);
  const int fr = lane >> 2, fc = lane & 3;
  for (int t = blockIdx.x; t < total; t += gridDim.x) {
    int lo = 0, hi = nprod - 1;
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (prods[mid].tile0 <= t) lo = mid;
      else hi = mid - 1;
    }
    const GroupedProd g = prods[lo];
    const int tt = t - g.tile0, m0 = (tt / g.tn) * BM, n0 = (tt % g.tn) * BN;
    if (g.upper && n0 + BN <= m0) continue;  // strictly below the diagonal (uniform in the CTA)
    double acc[TM][TN][2];
#pragma unroll
    for (int i = 0; i < TM; ++i)
#pragma unroll
      for (int j = 0; j < TN; ++j) acc[i][j][0] = acc[i][j][1] = 0.0;
    __syncthreads();  // the previous work item's reads of the ring are done before it is refilled
    dmma_tile<BM, BN, WM, WN, A_KC, B_NC>(smem, static_cast<const double *>(g.A), g.a_rs, g.a_cs,
                                          static_cast<const double *>(g.B), g.b_rs, g.b_cs, g.M, g.N, 0, g.K, m0, n0,
                                          acc);
    double *__restrict__ C = static_cast<double *>(g.C);
#pragma unroll
    for (int i = 0; i < TM; ++i) {
      const int gm = m0 + wm0 + 8 * i + fr;
      if (gm >= g.M) continue;
#pragma unroll
      for (int j = 0; j < TN; ++j)
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          const int gn = n0 + wn0 + 8 * j + 2 * fc + h;
          if (gn >= g.N) continue;
          double *c = C + (long long)gm * g.c_rs + (long long)gn * g.c_cs;
          double v = g.alpha * acc[i][j][h];
          if (g.beta != 0.0) v += g.beta * *c;
          *c = v;
        }
    }
  }
}

template <int BM, int BN, int WM, int WN, bool A_KC, bool B_NC>
void dmma_grouped_launch(const GroupedProd *prods, int nprod, int total, cudaStream_t st) {
  auto *k = dmma_grouped_kernel<BM, BN, WM, WN, A_KC, B_NC>;
  constexpr int NT = WM * WN * 32;
  const int bytes = kStages * DmmaLayout<BM, BN, A_KC, B_NC>::stage * (int)sizeof(double);
  static int per_sm = 0;  // resident CTAs per SM, resolved on first use
  if (per_sm == 0) {
    CK(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, NT, bytes));
    per_sm = std::max(1, per_sm);
  }
  const int grid = std::max(1, std::min(total, per_sm * Runtime::get().num_sms));
  k<<<grid, NT, bytes, st>>>(prods, nprod, total);
  KLAUNCHED();
}

template <int BM, int BN, int WM, int WN>
void dmma_launch(const Gemm<double, double> &g, bool a_kc, bool b_nc, cudaStream_t st) {
  Runtime &rt = Runtime::get();
  const int gx = (g.M + BM - 1) / BM, gy = (g.N + BN - 1) / BN;
  const long long tiles = (long long)gx * gy * g.batch;
  int splits = g.splits;
  if (splits <= 0) {
    // split-K by a time model: the busiest SM runs ceil(tiles s / SMs) CTAs of BM BN (K / s) FMAs
    // (about 0.23 TFLOP/s per SM on mma.sync f64) plus a fixed 2 us each, and s > 1 adds the
    // partial sums' round trip (s + 1) M N 8 bytes at about 4 TB/s; the smallest s within 3 % of
    // the best, with at least 64 of K per split and at most 512 MB of partials
    const double rate = 0.23e12, fixed = 2e-6, bw = 4e12;
    const long long mnb = (long long)g.M * g.N * g.batch;
    auto model = [&](long long s) {
      const long long per_sm = (tiles * s + rt.num_sms - 1) / rt.num_sms;
      const double kc = (double)((g.K + s - 1) / s);
      return per_sm * (2.0 * BM * BN * kc / rate + fixed) + (s > 1 ? (double)(s + 1) * mnb * 8.0 / bw : 0.0);
    };
    const long long smax = std::max<long long>(
        1, std::min<long long>({64, (long long)g.K / 64, (512LL << 20) / std::max<long long>(1, mnb * 8)}));
    double best = model(1);
    for (long long s = 2; s <= smax; ++s) best = std::min(best, model(s));
    splits = 1;
    for (long long s = 1; s <= smax; ++s)
      if (model(s) <= 1.03 * best) {
        splits = (int)s;
        break;
      }
  }
  int kchunk = (g.K + splits - 1) / splits;
  kchunk = ((kchunk + kBK - 1) / kBK) * kBK;
  if (kchunk <= 0) kchunk = kBK;
  splits = std::max(1, (g.K + kchunk - 1) / kchunk);
  DBuf<double> part;
  if (splits > 1) part.alloc((size_t)g.batch * splits * g.M * g.N);
  const dim3 grid(gx, gy, g.batch * splits);
  constexpr int NT = WM * WN * 32;
#define ISVD_DMMA_CASE(AK, BNC)                                                                        \
  if (a_kc == AK && b_nc == BNC) {                                                                     \
    auto *k = dmma_gemm_kernel<BM, BN, WM, WN, AK, BNC>;                                               \
    const int bytes = kStages * DmmaLayout<BM, BN, AK, BNC>::stage * (int)sizeof(double);              \
    CK(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));                   \
    k<<<grid, NT, bytes, st>>>(g, splits, kchunk, part.p);                                             \
    KLAUNCHED();                                                                                       \
  }
  ISVD_DMMA_CASE(true, true)
  ISVD_DMMA_CASE(true, false)
  ISVD_DMMA_CASE(false, true)
  ISVD_DMMA_CASE(false, false)
#undef ISVD_DMMA_CASE
  if (splits > 1) splitk_reduce(g, splits, part.p, st);
}

}  // namespace

bool dmma_enabled() {
  static const bool on = [] {
    const char *e = getenv("ISVD_GPU_DMMA");
    return !(e && atoi(e) == 0);
  }();
  return on;
}

void dmma_gemm(const Gemm<double, double> &g, bool a_kc, bool b_nc, cudaStream_t st) {
  // 128 x 128 tiles when they fill the GPU or a long K lets split-K fill it; otherwise 64 x 64
  const long long tiles128 = (long long)((g.M + 127) / 128) * ((g.N + 127) / 128) * g.batch;
  const int sms = Runtime::get().num_sms;
  const bool long_k = g.splits <= 0 && (long long)g.K >= 2048 && tiles128 * (g.K / 1024) >= 2LL * sms;
  if (g.pl_t && (g.splits != 1 || g.M % 64 || g.pl_ld % 8 || ((uintptr_t)g.pl_t & 15) || g.pl_ps % 8 ||
                 g.pl_batch < 0 || g.pl_batch >= g.batch))
    fail(kErrArgument, "dmma_gemm: plane output needs splits = 1, M %% 64 == 0 and 16-byte aligned plane rows");
  // plane output: 64 x 64 tiles (their epilogue stages a tile's transpose through the cp.async
  // ring; without split-K the tile shape does not change the results)
  if (g.pl_t || g.M <= 64 || g.N <= 64 || (tiles128 < 2LL * sms && !long_k))
    dmma_launch<64, 64, 2, 2>(g, a_kc, b_nc, st);
  else
    dmma_launch<128, 128, 2, 4>(g, a_kc, b_nc, st);
}

int dmma_grouped_bm(int shape) { return shape == 2 ? 128 : shape == 4 ? 32 : 64; }
int dmma_grouped_bn(int shape) { return (shape == 0 || shape >= 3) ? 32 : 64; }

void dmma_grouped(const GroupedProd *prods, int nprod, int total, int shape, bool a_kc, bool b_nc, cudaStream_t st) {
  if (nprod <= 0 || total <= 0) return;
#define ISVD_DMMA_GROUPED(BM, BN, WM, WN)                                                              \
  if (a_kc && b_nc) dmma_grouped_launch<BM, BN, WM, WN, true, true>(prods, nprod, total, st);          \
  else if (a_kc) dmma_grouped_launch<BM, BN, WM, WN, true, false>(prods, nprod, total, st);            \
  else if (b_nc) dmma_grouped_launch<BM, BN, WM, WN, false, true>(prods, nprod, total, st);            \
  else dmma_grouped_launch<BM, BN, WM, WN, false, false>(prods, nprod, total, st);
  switch (shape) {  // warp tiles of 32 x 32 outputs (4 x 4 mma tiles), or 32 x 16 (shape 3)
    case 0: ISVD_DMMA_GROUPED(64, 32, 2, 1) break;
    case 1: ISVD_DMMA_GROUPED(64, 64, 2, 2) break;
    case 2: ISVD_DMMA_GROUPED(128, 64, 4, 2) break;
    case 3: ISVD_DMMA_GROUPED(64, 32, 2, 2) break;
    default: ISVD_DMMA_GROUPED(32, 32, 1, 1) break;
  }
#undef ISVD_DMMA_GROUPED
}

}  // namespace isvdb
