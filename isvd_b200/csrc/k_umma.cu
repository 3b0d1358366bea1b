// tcgen05 GEMM engine over bf16 planes (see umma.h), plus the plane split and bf16 Omega kernels.
//
// CTA = 10 warps: warp 0 issues TMA loads into a ring of shared-memory stages, warp 1 allocates
// tensor memory and issues tcgen05.mma (one thread), warps 2-9 drain the accumulator.
//
// Accumulation is chunked: the tensor core adds products into its FP32 accumulator with an error
// that grows with the length of the accumulation chain (measured on B200: ~1e-9 relative per
// unit of K, i.e. 2e-5 at K = 2e4 in one chain).  So the MMAs accumulate only kChunkK-deep
// chunks in tensor memory, alternating between two 128 x BN TMEM buffers; while the tensor core
// fills one buffer, the epilogue warps add the other into FP32 registers (round to nearest) and
// release it.  Each epilogue warp owns one TMEM lane quarter (warp % 4) and one half of the
// columns.  Every mbarrier wait is bounded; on expiry the CTA records ISVD_GPU_ERROR_TIMEOUT in
// the status word, drains its outstanding copies / MMAs (bounded) and frees its tensor memory
// before returning.
#include <cuda.h>
#include <cuda_bf16.h>

#include <algorithm>
#include <cstdlib>
#include <cstring>

#include "runtime.h"
#include "umma.h"

namespace isvdb {
namespace {

constexpr int BM = 128;
constexpr int kThreads = 320;
constexpr int kEpiWarps = 8;
constexpr int kChunkK = 128;  // K depth of one tensor-memory accumulation chunk
constexpr long long kWaitLimit = 1LL << 23;

struct KParams {
  int M, N, K;
  int na, nb, nprod;
  int pa[8], pb[8];
  int batch;
  long long a_mn_step, b_mn_step, c_step;
  long long a_k_step, b_k_step;  // per-batch K offsets (elements)
  void *C;
  int c_double;
  long long c_rs, c_cs;
  double alpha;
  int splits, kbps, total_kb;
  float *partial;
  int upper;  // only tiles intersecting the upper triangle (symmetric output)
  int *status;
};

__device__ __forceinline__ uint32_t su32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(su32(bar)), "r"(count));
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(su32(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try(uint64_t *bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}\n"
      : "=r"(ok)
      : "r"(su32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
// Bounded wait; false on expiry or when another role has aborted.
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity, volatile int *abort_flag) {
  for (long long i = 0; i < kWaitLimit; ++i) {
    if (mbar_try(bar, parity)) return true;
    if ((i & 255) == 255 && *abort_flag) return false;
  }
  return false;
}

__device__ __forceinline__ void tma_load_3d(void *dst, const CUtensorMap *map, uint64_t *bar, int x, int y, int z) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4, %5}], [%2];" ::
          "r"(su32(dst)),
      "l"((uint64_t)map), "r"(su32(bar)), "r"(x), "r"(y), "r"(z)
      : "memory");
}

// Shared-memory matrix descriptor (sm100 layout: start>>4 [0,14), LBO>>4 [16,30), SBO>>4 [32,46),
// version 1 at bit 46, swizzle mode [61,64)).
__device__ __forceinline__ uint64_t sdesc(uint32_t saddr, uint32_t lbo, uint32_t sbo, uint32_t layout) {
  return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | ((uint64_t)1 << 46) | ((uint64_t)layout << 61);
}

// Instruction descriptor, kind::f16: FP32 accumulate, BF16 A and B, operand majors per flags.
__host__ __device__ constexpr uint32_t idesc_bf16(int M, int N, bool a_mn, bool b_mn) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((a_mn ? 1u : 0u) << 15) | ((b_mn ? 1u : 0u) << 16) |
         ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ void umma_bf16(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t idesc, uint32_t acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\ttcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::
          "r"(tmem_d),
      "l"(da), "l"(db), "r"(idesc), "r"(acc));
}
__device__ __forceinline__ void umma_commit(uint64_t *bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(su32(bar))
               : "memory");
}
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

__device__ __forceinline__ void tmem_ld8(uint32_t taddr, float *v) {
  uint32_t r[8];
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
               : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 8; ++i) v[i] = __uint_as_float(r[i]);
}

template <int BN, int BK, bool AMN, bool BMN>
struct Cfg {
  static constexpr int A_TILE = BM * BK * 2;  // bytes per A plane tile
  static constexpr int B_TILE = BN * BK * 2;  // bytes per B plane tile
  static constexpr uint32_t A_LAYOUT = (BK == 64) ? 2u : 4u;   // SWIZZLE_128B / SWIZZLE_64B
  static constexpr uint32_t A_SBO = (BK == 64) ? 1024u : 512u;  // 8 rows of BK bf16
  static constexpr int TMEM_COLS = (2 * BN <= 64) ? 64 : (2 * BN <= 128) ? 128 : (2 * BN <= 256) ? 256 : 512;
  static constexpr int CHUNK = (kChunkK / BK) > 0 ? (kChunkK / BK) : 1;  // k-blocks per chunk
  static constexpr int HALF = BN / 2;                                      // columns per epilogue warp
};

template <int BN, int BK, bool AMN, bool BMN>
__global__ void __launch_bounds__(kThreads, 1)
    umma_gemm_kernel(const __grid_constant__ CUtensorMap mapA, const __grid_constant__ CUtensorMap mapB,
                     const KParams p, const int stages) {
  using C = Cfg<BN, BK, AMN, BMN>;
  extern __shared__ __align__(1024) uint8_t smem_raw[];
  uint8_t *smem = (uint8_t *)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  const int stage_bytes = p.na * C::A_TILE + p.nb * C::B_TILE;
  uint64_t *full = (uint64_t *)(smem + (size_t)stages * stage_bytes);
  uint64_t *empty = full + stages;
  uint64_t *tfull = empty + stages;  // [2] chunk in TMEM buffer b complete
  uint64_t *tempty = tfull + 2;      // [2] TMEM buffer b drained by the epilogue
  uint32_t *tslot = (uint32_t *)(tempty + 2);
  volatile int *abort_flag = (volatile int *)(tslot + 1);

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int nt = blockIdx.x, mt = blockIdx.y;
  const int b = blockIdx.z / p.splits, split = blockIdx.z % p.splits;
  const int m0 = mt * BM, n0 = nt * BN;
  if (p.upper && n0 + BN <= m0) return;  // tile strictly below the diagonal: mirrored later
  const int kb0 = split * p.kbps;
  const int nkb = max(0, min(p.total_kb, kb0 + p.kbps) - kb0);

  if (threadIdx.x == 0) {
    for (int s = 0; s < stages; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
    }
    for (int b2 = 0; b2 < 2; ++b2) {
      mbar_init(&tfull[b2], 1);
      mbar_init(&tempty[b2], kEpiWarps);
    }
    *abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 1) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(su32(tslot)),
                 "r"((uint32_t)C::TMEM_COLS));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tslot;

  if (warp == 0 && lane == 0) {
    // ---------------------------------------------------------------- TMA producer
    const int a_row = (int)(b * p.a_mn_step) + m0;
    const int b_row = (int)(b * p.b_mn_step) + n0;
    int issued = 0;
    for (int kb = 0; kb < nkb; ++kb) {
      const int s = kb % stages;
      if (kb >= stages && !mbar_wait(&empty[s], ((kb / stages) & 1) ^ 1, abort_flag)) {
        *abort_flag = 1;
        break;
      }
      uint8_t *st = smem + (size_t)s * stage_bytes;
      mbar_expect_tx(&full[s], (uint32_t)stage_bytes);
      const int k0 = (kb0 + kb) * BK;
      const int ka = k0 + (int)(b * p.a_k_step), kbb = k0 + (int)(b * p.b_k_step);
      for (int q = 0; q < p.na; ++q) {
        if (!AMN) {
          tma_load_3d(st + q * C::A_TILE, &mapA, &full[s], ka, a_row, q);
        } else {
#pragma unroll
          for (int j = 0; j < BM / 64; ++j)
            tma_load_3d(st + q * C::A_TILE + j * (BK * 128), &mapA, &full[s], a_row + 64 * j, ka, q);
        }
      }
      uint8_t *bt = st + p.na * C::A_TILE;
      for (int q = 0; q < p.nb; ++q) {
        if (!BMN) {
          tma_load_3d(bt + q * C::B_TILE, &mapB, &full[s], kbb, b_row, q);
        } else {
#pragma unroll
          for (int j = 0; j < BN / 64; ++j)
            tma_load_3d(bt + q * C::B_TILE + j * (BK * 128), &mapB, &full[s], b_row + 64 * j, kbb, q);
        }
      }
      ++issued;
    }
    // Drain: every issued load has landed before the CTA can exit (bounded).
    for (int kb = max(0, issued - stages); kb < issued; ++kb) {
      const int s = kb % stages;
      long long i = 0;
      while (!mbar_try(&full[s], (kb / stages) & 1) && ++i < kWaitLimit) {
      }
    }
  } else if (warp == 1 && lane == 0) {
    // ---------------------------------------------------------------- MMA issuer
    const uint32_t idesc = idesc_bf16(BM, BN, AMN, BMN);
    int chunk = 0;
    uint32_t tacc = tmem;
    bool first = true;
    for (int kb = 0; kb < nkb; ++kb) {
      if (kb % C::CHUNK == 0) {
        const int b2 = chunk & 1;
        if (chunk >= 2 && !mbar_wait(&tempty[b2], ((chunk >> 1) & 1) ^ 1, abort_flag)) {
          *abort_flag = 1;
          break;
        }
        tc_fence_after();
        tacc = tmem + (uint32_t)(b2 * BN);
        first = true;
      }
      const int s = kb % stages;
      if (!mbar_wait(&full[s], (kb / stages) & 1, abort_flag)) {
        *abort_flag = 1;
        break;
      }
      tc_fence_after();
      const uint32_t st = su32(smem + (size_t)s * stage_bytes);
      for (int i = 0; i < p.nprod; ++i) {
        const uint32_t a_base = st + p.pa[i] * C::A_TILE;
        const uint32_t b_base = st + p.na * C::A_TILE + p.pb[i] * C::B_TILE;
#pragma unroll
        for (int kk = 0; kk < BK / 16; ++kk) {
          const uint64_t da = AMN ? sdesc(a_base + kk * 2048, BK * 128, 1024, 2u)
                                  : sdesc(a_base + kk * 32, 16, C::A_SBO, C::A_LAYOUT);
          const uint64_t db = BMN ? sdesc(b_base + kk * 2048, BK * 128, 1024, 2u)
                                  : sdesc(b_base + kk * 32, 16, C::A_SBO, C::A_LAYOUT);
          umma_bf16(tacc, da, db, idesc, first ? 0u : 1u);
          first = false;
        }
      }
      umma_commit(&empty[s]);
      if (kb % C::CHUNK == C::CHUNK - 1 || kb == nkb - 1) {
        umma_commit(&tfull[chunk & 1]);  // arrives when this chunk's MMAs have completed
        ++chunk;
      }
    }
  } else if (warp >= 2) {
    // ---------------------------------------------------------------- epilogue
    const int q = warp & 3;                 // TMEM lane quarter accessible to this warp
    const int h = (warp - 2) >> 2;          // column half
    const int row = q * 32 + lane;
    const int nchunks = (nkb + C::CHUNK - 1) / C::CHUNK;
    float acc[C::HALF];
#pragma unroll
    for (int j = 0; j < C::HALF; ++j) acc[j] = 0.f;
    bool ok = true;
    for (int c = 0; c < nchunks; ++c) {
      const int b2 = c & 1;
      int okw = 0;
      if (lane == 0) okw = mbar_wait(&tfull[b2], (c >> 1) & 1, abort_flag) ? 1 : 0;
      ok = __shfl_sync(0xffffffffu, okw, 0) != 0;
      if (!ok) {
        if (lane == 0) *abort_flag = 1;
        break;
      }
      tc_fence_after();
      const uint32_t tbase = tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)(b2 * BN + h * C::HALF);
#pragma unroll
      for (int j = 0; j < C::HALF; j += 8) {
        float v[8];
        tmem_ld8(tbase + (uint32_t)j, v);
#pragma unroll
        for (int i = 0; i < 8; ++i) acc[j + i] += v[i];
      }
      tc_fence_before();
      __syncwarp();
      if (lane == 0) asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(su32(&tempty[b2])) : "memory");
    }
    const int gm = m0 + row;
    if (ok && gm < p.M) {
      const bool upper_tile = p.upper != 0;
#pragma unroll
      for (int j = 0; j < C::HALF; ++j) {
        const int gn = n0 + h * C::HALF + j;
        if (gn >= p.N) break;
        if (upper_tile && gn < gm) continue;
        if (p.splits == 1) {
          const long long off = (long long)b * p.c_step + (long long)gm * p.c_rs + (long long)gn * p.c_cs;
          if (p.c_double) ((double *)p.C)[off] = p.alpha * (double)acc[j];
          else ((float *)p.C)[off] = (float)(p.alpha * (double)acc[j]);
        } else {
          p.partial[(((long long)b * p.splits + split) * p.M + gm) * p.N + gn] = acc[j];
        }
      }
    }
  }
  __syncthreads();
  if (*abort_flag && threadIdx.x == 0) atomicExch(p.status, (int)kErrTimeout);
  if (warp == 1) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"((uint32_t)C::TMEM_COLS));
  }
}

// C(b, r, c) = alpha * sum_s partial(b, s, r, c) (FP64 sum); upper: only c >= r.
__global__ void umma_reduce_kernel(const KParams p) {
  const long long MN = (long long)p.M * p.N;
  const long long total = MN * p.batch;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
       e += (long long)gridDim.x * blockDim.x) {
    const long long b = e / MN, r = (e % MN) / p.N, c = e % p.N;
    if (p.upper && c < r) continue;
    // eight independent partial sums, so that eight loads are in flight
    const float *q = p.partial + ((b * p.splits) * p.M + r) * p.N + c;
    const long long stride = (long long)p.M * p.N;
    double acc[8] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
    int sp = 0;
    for (; sp + 8 <= p.splits; sp += 8) {
#pragma unroll
      for (int u = 0; u < 8; ++u) acc[u] += (double)q[(sp + u) * stride];
    }
    for (int u = 0; sp < p.splits; ++sp, ++u) acc[u] += (double)q[sp * stride];
    const double s = ((acc[0] + acc[1]) + (acc[2] + acc[3])) + ((acc[4] + acc[5]) + (acc[6] + acc[7]));
    const long long off = b * p.c_step + r * p.c_rs + c * p.c_cs;
    if (p.c_double) ((double *)p.C)[off] = p.alpha * s;
    else ((float *)p.C)[off] = (float)(p.alpha * s);
  }
}

// Symmetric completion: C(c, r) = C(r, c) for c > r.
template <class T>
__global__ void mirror_upper_kernel(T *C, long long n, long long ld) {
  const long long total = n * n;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
       e += (long long)gridDim.x * blockDim.x) {
    const long long r = e / n, c = e % n;
    if (c < r) C[r * ld + c] = C[c * ld + r];
  }
}

// ------------------------------------------------------------------------------ splits
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

// Non-transposed: plane(r, c) for r < rows_pad, c < ld (zero outside rows x cols); each thread
// converts 8 consecutive columns and writes one 16-byte vector per plane.
template <class T>
__global__ void split_kernel(const T *__restrict__ src, long long s_rs, long long s_cs, long long rows,
                             long long cols, long long rows_pad, int np, __nv_bfloat16 *__restrict__ dst,
                             long long ld, long long ps) {
  const long long gpr = ld / 8;
  const long long total = rows_pad * gpr;
  for (long long g = blockIdx.x * (long long)blockDim.x + threadIdx.x; g < total;
       g += (long long)gridDim.x * blockDim.x) {
    const long long r = g / gpr, c0 = (g - r * gpr) * 8;
    __nv_bfloat16 o[3][8];
#pragma unroll
    for (int i = 0; i < 8; ++i) {
      const long long c = c0 + i;
      const T x = (r < rows && c < cols) ? src[r * s_rs + c * s_cs] : T(0);
      __nv_bfloat16 t[3];
      split3<T>(x, t, 3);
#pragma unroll
      for (int q = 0; q < 3; ++q) o[q][i] = t[q];
    }
    for (int q = 0; q < np; ++q) *(uint4 *)(dst + q * ps + r * ld + c0) = pack8(o[q]);
  }
}

// Transposed: plane(c, r) = piece(src(r, c)) through a 64 (r) x 32 (c) shared tile; each thread
// writes 8 consecutive r of one output row c (16-byte vectors).  Plane rows beyond cols and
// columns beyond rows are zeroed separately.
template <class T>
__global__ void split_t_kernel(const T *__restrict__ src, long long s_rs, long long s_cs, long long rows,
                               long long cols, long long rows_pad, int np, __nv_bfloat16 *__restrict__ dst,
                               long long ld, long long ps) {
  __shared__ T tile[64][33];
  const long long r0 = (long long)blockIdx.x * 64, c0 = (long long)blockIdx.y * 32;
  const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;  // 32 x 8 threads
  for (int j = ty; j < 64; j += 8) {
    const long long r = r0 + j, c = c0 + tx;
    tile[j][tx] = (r < rows && c < cols) ? src[r * s_rs + c * s_cs] : T(0);
  }
  __syncthreads();
  const int cl = threadIdx.x >> 3, seg = threadIdx.x & 7;  // output row c0 + cl, columns r0 + 8 seg ..
  const long long c = c0 + cl, rr = r0 + 8 * seg;
  if (c < rows_pad && rr < ld) {
    __nv_bfloat16 o[3][8];
#pragma unroll
    for (int i = 0; i < 8; ++i) {
      __nv_bfloat16 t[3];
      split3<T>(tile[8 * seg + i][cl], t, 3);
#pragma unroll
      for (int q = 0; q < 3; ++q) o[q][i] = t[q];
    }
    for (int q = 0; q < np; ++q) *(uint4 *)(dst + q * ps + c * ld + rr) = pack8(o[q]);
  }
}

// Philox4x32-10 + Box-Muller (same stream as rng_gaussian in k_misc.cu), rounded to bf16 and
// written transposed: dst(c, j) = bf16(Omega(j, c)), value index j * Nl + c.
__device__ __forceinline__ uint4 philox(uint4 c, uint32_t k0, uint32_t k1) {
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

__global__ void rng_bf16_t_kernel(__nv_bfloat16 *__restrict__ dst, long long n, long long Nl, long long ld,
                                  long long rows_pad, uint64_t seed) {
  // one thread per (c, j-pair): value indices j*Nl + c; pairs in value space (2p, 2p + 1) hold
  // consecutive c for even Nl, so each thread produces one pair and writes two rows of dst.
  const long long total_pairs = (n * Nl + 1) / 2;
  for (long long pi = blockIdx.x * (long long)blockDim.x + threadIdx.x; pi < total_pairs;
       pi += (long long)gridDim.x * blockDim.x) {
    const uint4 x = philox(make_uint4((uint32_t)pi, (uint32_t)(pi >> 32), 0u, 0u), (uint32_t)seed,
                           (uint32_t)(seed >> 32));
    const uint64_t a = ((((uint64_t)x.x) << 32) | x.y) >> 11;
    const uint64_t bb = ((((uint64_t)x.z) << 32) | x.w) >> 11;
    const double u1 = (double)(a + 1) * 0x1.0p-53, u2 = (double)bb * 0x1.0p-53;
    const double rr = sqrt(-2.0 * log(u1));
    double s, c;
    sincospi(2.0 * u2, &s, &c);
    const double z[2] = {rr * c, rr * s};
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const long long v = 2 * pi + h;
      if (v >= n * Nl) break;
      const long long j = v / Nl, col = v % Nl;
      dst[col * ld + j] = __double2bfloat16(z[h]);
    }
  }
  (void)rows_pad;
}

// ------------------------------------------------------------------------------ host side
typedef CUresult (*EncodeTiledFn)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                  const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiledFn encode_fn() {
  static EncodeTiledFn fn = nullptr;
  if (!fn) {
    void *ptr = nullptr;
    cudaDriverEntryPointQueryResult q;
    CK(cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &ptr, cudaEnableDefault, &q));
    if (!ptr || q != cudaDriverEntryPointSuccess) fail(kErrCuda, "cuTensorMapEncodeTiled unavailable");
    fn = (EncodeTiledFn)ptr;
  }
  return fn;
}

// 3-D tensor map over bf16 planes: dims {inner, outer, planes}, box {bx, by, 1}.
CUtensorMap make_map(const Planes &P, int bx, int by, CUtensorMapSwizzle sw) {
  CUtensorMap m;
  memset(&m, 0, sizeof(m));
  const cuuint64_t inner = (cuuint64_t)std::max<long long>(P.cols, bx);
  const cuuint64_t outer = (cuuint64_t)std::max<long long>(P.rows, by);
  cuuint64_t dims[3] = {inner, outer, (cuuint64_t)P.np};
  cuuint64_t strides[2] = {(cuuint64_t)P.ld * 2, (cuuint64_t)P.plane_stride * 2};
  cuuint32_t box[3] = {(cuuint32_t)bx, (cuuint32_t)by, 1};
  cuuint32_t es[3] = {1, 1, 1};
  if ((P.ld * 2) % 16 || (P.plane_stride * 2) % 16 || ((uintptr_t)P.ptr) % 16)
    fail(kErrArgument, "tensor map: planes must be 16-byte aligned");
  if ((long long)inner > P.ld) fail(kErrArgument, "tensor map: inner extent exceeds the row stride");
  CUresult r = encode_fn()(&m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 3, (void *)P.ptr, dims, strides, box, es,
                           CU_TENSOR_MAP_INTERLEAVE_NONE, sw, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                           CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) fail(kErrCuda, "cuTensorMapEncodeTiled failed (%d)", (int)r);
  return m;
}

template <int BN, int BK, bool AMN, bool BMN>
void launch_t(const UmmaGemm &g, cudaStream_t st, int *status) {
  using C = Cfg<BN, BK, AMN, BMN>;
  Runtime &rt = Runtime::get();
  KParams p;
  memset(&p, 0, sizeof(p));
  p.M = g.M; p.N = g.N; p.K = g.K;
  p.na = g.A.np; p.nb = g.B.np; p.nprod = g.nprod;
  for (int i = 0; i < g.nprod; ++i) { p.pa[i] = g.pa[i]; p.pb[i] = g.pb[i]; }
  p.batch = g.batch;
  p.a_mn_step = g.a_mn_step; p.b_mn_step = g.b_mn_step; p.c_step = g.c_step;
  p.a_k_step = g.a_k_step; p.b_k_step = g.b_k_step;
  if ((g.a_k_step | g.b_k_step) % 8 || ((g.a_k_step || g.b_k_step) && g.K % BK))
    fail(kErrArgument, "tcgen05 GEMM: per-batch K offsets need K %% %d == 0 and 8-element alignment", BK);
  // TMA requires the innermost coordinate of every box to start on a 16-byte boundary: for an
  // MN-major operand that coordinate is the MN offset (batch step + tile origin), for a K-major
  // operand the K offset (checked above).  Tile origins are multiples of 64.
  if ((AMN && g.a_mn_step % 8) || (BMN && g.b_mn_step % 8))
    fail(kErrArgument, "tcgen05 GEMM: MN-major operand batch steps must be multiples of 8 elements");
  p.C = g.C; p.c_double = g.c_double;
  p.c_rs = g.c_rs; p.c_cs = g.c_cs;
  p.alpha = g.alpha;
  p.upper = g.upper ? 1 : 0;
  p.status = status;
  p.total_kb = (g.K + BK - 1) / BK;
  const int gx = (g.N + BN - 1) / BN, gy = (g.M + BM - 1) / BM;
  const long long tiles = (long long)gx * gy * g.batch;
  int splits = g.splits;
  if (const char *e = getenv("ISVD_UMMA_SPLITS")) splits = atoi(e);  // diagnostic override
  if (splits <= 0) {
    splits = 1;
    if (tiles < rt.num_sms) splits = (int)std::min<long long>((rt.num_sms + tiles - 1) / tiles, std::max(1, p.total_kb / 8));
  }
  splits = std::max(1, std::min(splits, p.total_kb));
  p.kbps = (p.total_kb + splits - 1) / splits;
  p.splits = (p.total_kb + p.kbps - 1) / p.kbps;
  DBuf<float> part;
  if (p.splits > 1) {
    part.alloc((size_t)g.batch * p.splits * g.M * g.N);
    p.partial = part.p;
  }
  const CUtensorMapSwizzle swa = (BK == 64) ? CU_TENSOR_MAP_SWIZZLE_128B : CU_TENSOR_MAP_SWIZZLE_64B;
  CUtensorMap ma = AMN ? make_map(g.A, 64, BK, CU_TENSOR_MAP_SWIZZLE_128B) : make_map(g.A, BK, BM, swa);
  CUtensorMap mb = BMN ? make_map(g.B, 64, BK, CU_TENSOR_MAP_SWIZZLE_128B) : make_map(g.B, BK, BN, swa);
  const int stage_bytes = g.A.np * C::A_TILE + g.B.np * C::B_TILE;
  const int budget = (int)rt.smem_optin - 1024 - 256;
  int stages = std::min(8, budget / stage_bytes);
  if (stages < 2) fail(kErrUnsupported, "tcgen05 GEMM: %d planes do not fit in shared memory", g.A.np + g.B.np);
  const size_t smem = (size_t)stages * stage_bytes + 1024 + 256;
  static_assert(kThreads == 64 + 32 * kEpiWarps, "warp roles");
  auto kern = umma_gemm_kernel<BN, BK, AMN, BMN>;
  CK(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  dim3 grid(gx, gy, g.batch * p.splits);
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  if (profiling()) {
    CK(cudaEventCreate(&e0));
    CK(cudaEventCreate(&e1));
    CK(cudaEventRecord(e0, st));
  }
  kern<<<grid, kThreads, smem, st>>>(ma, mb, p, stages);
  KLAUNCHED();
  if (profiling()) {
    CK(cudaEventRecord(e1, st));
    CK(cudaEventSynchronize(e1));
    float ms = 0.f;
    CK(cudaEventElapsedTime(&ms, e0, e1));
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    profile_add(g.tag, ms, 2.0 * g.M * (double)g.N * g.K * g.batch * g.nprod);
  }
  if (p.splits > 1) {
    const long long total = (long long)g.M * g.N * g.batch;
    const int blocks = (int)std::min<long long>((total + 255) / 256, 16LL * rt.num_sms);
    umma_reduce_kernel<<<blocks, 256, 0, st>>>(p);
    KLAUNCHED();
  }
}

}  // namespace

template <class T>
void split_planes(const T *src, long long s_rs, long long s_cs, long long rows, long long cols, int np,
                  bool transpose, __nv_bfloat16 *dst, long long ld, long long plane_stride, cudaStream_t st) {
  Runtime &rt = Runtime::get();
  const long long out_rows = transpose ? cols : rows;
  const long long rows_pad = plane_stride / ld;
  if (rows_pad < out_rows || ld < (transpose ? rows : cols)) fail(kErrArgument, "split_planes: plane too small");
  if (!transpose) {
    if (ld % 8) fail(kErrArgument, "split_planes: ld must be a multiple of 8");
    const long long total = rows_pad * (ld / 8);
    const int blocks = (int)std::min<long long>((total + 255) / 256, 32LL * rt.num_sms);
    split_kernel<T><<<blocks, 256, 0, st>>>(src, s_rs, s_cs, rows, cols, rows_pad, np, dst, ld, plane_stride);
    KLAUNCHED();
  } else {
    // zero the padding (rows beyond cols, columns beyond rows), then transpose-split
    for (int q = 0; q < np; ++q) {
      __nv_bfloat16 *pl = dst + (size_t)q * plane_stride;
      if (rows_pad > cols)
        CK(cudaMemsetAsync(pl + (size_t)cols * ld, 0, (size_t)(rows_pad - cols) * ld * sizeof(__nv_bfloat16), st));
      if (ld > rows)
        CK(cudaMemset2DAsync(pl + rows, ld * sizeof(__nv_bfloat16), 0, (ld - rows) * sizeof(__nv_bfloat16), cols,
                             st));
    }
    if (ld % 8) fail(kErrArgument, "split_planes: ld must be a multiple of 8");
    dim3 grid((unsigned)((rows + 63) / 64), (unsigned)((cols + 31) / 32));
    split_t_kernel<T><<<grid, 256, 0, st>>>(src, s_rs, s_cs, rows, cols, rows_pad, np, dst, ld, plane_stride);
    KLAUNCHED();
  }
}

template <class T>
void split_rows(const T *src, long long s_rs, long long s_cs, long long rows, long long cols, int np, bool transpose,
                __nv_bfloat16 *dst, long long ld, long long plane_stride, cudaStream_t st) {
  Runtime &rt = Runtime::get();
  if (ld % 8) fail(kErrArgument, "split_rows: ld must be a multiple of 8");
  if (!transpose) {
    if (ld < cols) fail(kErrArgument, "split_rows: plane too narrow");
    const long long total = rows * (ld / 8);
    const int blocks = (int)std::min<long long>((total + 255) / 256, 32LL * rt.num_sms);
    split_kernel<T><<<blocks, 256, 0, st>>>(src, s_rs, s_cs, rows, cols, rows, np, dst, ld, plane_stride);
    KLAUNCHED();
  } else {
    // output rows = cols of src, output columns = rows of src; the grid covers ld when
    // ld == roundup(rows, 64)
    if (ld != (rows + 63) / 64 * 64) fail(kErrArgument, "split_rows: transposed rows need ld = roundup(rows, 64)");
    dim3 grid((unsigned)((rows + 63) / 64), (unsigned)((cols + 31) / 32));
    split_t_kernel<T><<<grid, 256, 0, st>>>(src, s_rs, s_cs, rows, cols, cols, np, dst, ld, plane_stride);
    KLAUNCHED();
  }
}
template void split_rows<float>(const float *, long long, long long, long long, long long, int, bool, __nv_bfloat16 *,
                                long long, long long, cudaStream_t);
template void split_rows<double>(const double *, long long, long long, long long, long long, int, bool,
                                 __nv_bfloat16 *, long long, long long, cudaStream_t);

void rng_gaussian_bf16_t(__nv_bfloat16 *dst, long long n, long long Nl, long long ld, long long rows_pad,
                         uint64_t seed, cudaStream_t st) {
  Runtime &rt = Runtime::get();
  if (rows_pad > Nl)
    CK(cudaMemsetAsync(dst + (size_t)Nl * ld, 0, (size_t)(rows_pad - Nl) * ld * sizeof(__nv_bfloat16), st));
  if (ld > n)
    CK(cudaMemset2DAsync(dst + n, ld * sizeof(__nv_bfloat16), 0, (ld - n) * sizeof(__nv_bfloat16), Nl, st));
  const long long pairs = (n * Nl + 1) / 2;
  const int blocks = (int)std::min<long long>((pairs + 255) / 256, 32LL * rt.num_sms);
  rng_bf16_t_kernel<<<blocks, 256, 0, st>>>(dst, n, Nl, ld, Nl, seed);
  KLAUNCHED();
}

void umma_gemm(const UmmaGemm &g, cudaStream_t st) {
  if (g.M <= 0 || g.N <= 0 || g.K <= 0) return;
  if (g.nprod < 1 || g.nprod > 8) fail(kErrArgument, "tcgen05 GEMM: 1..8 plane products");
  Runtime &rt = Runtime::get();
  if (rt.cc_major != 10) fail(kErrUnsupported, "tcgen05 GEMM needs an sm_100 device (found sm_%d%d)", rt.cc_major,
                              rt.cc_minor);
  int *status = g.status ? g.status : reinterpret_cast<int *>(rt.ctl + 32);
  if (!g.status) CK(cudaMemsetAsync(status, 0, sizeof(int), st));
  const bool amn = g.A.mn_major, bmn = g.B.mn_major;
  const int stage64 = g.A.np * BM * 64 * 2 + g.B.np * 256 * 64 * 2;
  const bool small_n = g.N <= 128;
  if (amn && bmn) {
    launch_t<128, 64, true, true>(g, st, status);
  } else if (amn) {
    fail(kErrUnsupported, "tcgen05 GEMM: MN-major A needs MN-major B");
  } else if (bmn) {
    launch_t<128, 64, false, true>(g, st, status);
  } else if (small_n) {
    launch_t<128, 64, false, false>(g, st, status);
  } else if (3 * stage64 <= (int)rt.smem_optin - 2048) {
    launch_t<256, 64, false, false>(g, st, status);
  } else {
    launch_t<256, 32, false, false>(g, st, status);
  }
  if (g.status) return;  // the caller checks the status word (no host synchronisation here)
  int h = 0;
  CK(cudaMemcpyAsync(&h, status, sizeof(int), cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  if (h) fail(kErrTimeout, "tcgen05 GEMM: a pipeline wait timed out");
}

template void split_planes<float>(const float *, long long, long long, long long, long long, int, bool,
                                  __nv_bfloat16 *, long long, long long, cudaStream_t);
template void split_planes<double>(const double *, long long, long long, long long, long long, int, bool,
                                   __nv_bfloat16 *, long long, long long, cudaStream_t);

void mirror_upper(double *C, long long n, long long ld, cudaStream_t st) {
  const long long total = n * n;
  const int blocks = (int)std::min<long long>((total + 255) / 256, 16LL * Runtime::get().num_sms);
  mirror_upper_kernel<double><<<blocks, 256, 0, st>>>(C, n, ld);
  KLAUNCHED();
}

}  // namespace isvdb
