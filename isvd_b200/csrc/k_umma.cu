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

#include "planes.cuh"
#include "runtime.h"
#include "umma.h"

namespace isvdb {
namespace {

constexpr int BM = 128;
constexpr int kThreads = 320;
constexpr int kEpiWarps = 8;
constexpr int kChunkK = 128;  // K depth of one tensor-memory accumulation chunk
constexpr long long kWaitLimit = 1LL << 23;       // iterations of an unsuspended poll (drains)
constexpr unsigned long long kWaitNs = 4000000000ull;  // wall-clock bound of one pipeline wait
constexpr uint32_t kSuspendNs = 1000000;             // suspension cap of one try_wait

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
  int chunk_kb;   // k-blocks per tensor-memory accumulation chunk
  int stage_out;  // epilogue stages its rows through shared memory (C rows contiguous)
  int bloop;      // one CTA runs every batch of its tile in turn (grid z = 1, no split-K)
  int vec_out;    // direct epilogue stores as 16-byte vectors (C rows contiguous and aligned)
  __nv_bfloat16 *pl;  // optional bf16 planes of the output (UmmaGemm::planes)
  long long pl_ld, pl_ps;
  int n_group;  // N tiles per column group of the tile order (0: row-major tile order)
  int l2_hint;  // bit 0: B loads evict-last, A loads evict-first; bit 1: A loads evict-last
};

__device__ __forceinline__ uint32_t su32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

// The three bf16 planes of an output value v = alpha acc, split as split_planes splits the stored
// value: FP32 pieces of the FP32-rounded value, or FP64 pieces of the FP64 value.
__device__ __forceinline__ void out_pieces(double v, int c_double, __nv_bfloat16 *o) {
  if (c_double) {
    double r = v;
#pragma unroll
    for (int q = 0; q < 3; ++q) {
      const __nv_bfloat16 h = __double2bfloat16(r);
      o[q] = h;
      r -= (double)__bfloat162float(h);
    }
  } else {
    const float x = (float)v;
    const __nv_bfloat16 h0 = __float2bfloat16_rn(x);
    const float r1 = x - __bfloat162float(h0);
    const __nv_bfloat16 h1 = __float2bfloat16_rn(r1);
    o[0] = h0;
    o[1] = h1;
    o[2] = __float2bfloat16_rn(r1 - __bfloat162float(h1));
  }
}
__device__ __forceinline__ void store_pieces(const KParams &p, long long off, double v) {
  __nv_bfloat16 o[3];
  out_pieces(v, p.c_double, o);
#pragma unroll
  for (int q = 0; q < 3; ++q) p.pl[q * p.pl_ps + off] = o[q];
}

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
// try_wait that suspends the thread (up to kSuspendNs) until the phase completes, so that waiting
// warps take no issue slots from the MMA and TMA threads that share their sub-partition.
__device__ __forceinline__ bool mbar_try_susp(uint64_t *bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n\tselp.u32 %0, 1, 0, p;\n\t}\n"
      : "=r"(ok)
      : "r"(su32(bar)), "r"(parity), "r"(kSuspendNs)
      : "memory");
  return ok != 0;
}
__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}
// Bounded wait (kWaitNs of wall clock); false on expiry or when another role has aborted.
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity, volatile int *abort_flag) {
  if (mbar_try_susp(bar, parity)) return true;
  const unsigned long long t0 = global_ns();
  for (;;) {
    if (mbar_try_susp(bar, parity)) return true;
    if (*abort_flag || global_ns() - t0 > kWaitNs) return false;
  }
}

__device__ __forceinline__ void tma_load_3d(void *dst, const CUtensorMap *map, uint64_t *bar, int x, int y, int z) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4, %5}], [%2];" ::
          "r"(su32(dst)),
      "l"((uint64_t)map), "r"(su32(bar)), "r"(x), "r"(y), "r"(z)
      : "memory");
}
// The same load with an L2 cache policy (createpolicy): evict-first for streamed operands,
// evict-last for the operand that the other resident CTAs read again.
__device__ __forceinline__ void tma_load_3d_pol(void *dst, const CUtensorMap *map, uint64_t *bar, int x, int y, int z,
                                                uint64_t pol) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes.L2::cache_hint [%0], [%1, {%3, "
      "%4, %5}], [%2], %6;" ::"r"(su32(dst)),
      "l"((uint64_t)map), "r"(su32(bar)), "r"(x), "r"(y), "r"(z), "l"(pol)
      : "memory");
}
__device__ __forceinline__ uint64_t l2_policy_evict_first() {
  uint64_t pol;
  asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(pol));
  return pol;
}
__device__ __forceinline__ uint64_t l2_policy_evict_normal() {
  uint64_t pol;
  asm volatile("createpolicy.fractional.L2::evict_normal.b64 %0, 1.0;" : "=l"(pol));
  return pol;
}
__device__ __forceinline__ uint64_t l2_policy_evict_last() {
  uint64_t pol;
  asm volatile("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(pol));
  return pol;
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

// 32 consecutive columns of this warp's 32 lanes; completes at the caller's tmem_wait().
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, uint32_t *r) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, "
      "%16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]), "=r"(r[16]),
        "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]),
        "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr));
}
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, uint32_t *r) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, "
      "[%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
}
__device__ __forceinline__ void tmem_wait() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

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
  int nt = blockIdx.x, mt = blockIdx.y;
  if (p.n_group > 0 && p.n_group < (int)gridDim.x) {
    // column-grouped tile order: the linear block index walks group g's n_group N tiles (fastest)
    // for every M tile, then group g + 1; the last group may be narrower
    const unsigned L = blockIdx.y * gridDim.x + blockIdx.x, span = (unsigned)p.n_group * gridDim.y;
    const unsigned g = L / span, r = L - g * span;
    const unsigned w = min((unsigned)p.n_group, gridDim.x - g * (unsigned)p.n_group);
    mt = (int)(r / w);
    nt = (int)(g * (unsigned)p.n_group + r % w);
  }
  // segments: the batches this CTA accumulates one after the other (bloop), else its one batch
  // (batch loops and vector stores serve the skinny N <= 128 shapes; the 256-wide sketch tiles keep
  // their registers for the 128-column accumulators)
  const bool bloop = BN <= 128 && p.bloop;
  const int nseg = bloop ? p.batch : 1;
  const int bz = bloop ? 0 : blockIdx.z / p.splits, split = bloop ? 0 : blockIdx.z % p.splits;
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
    int issued = 0, s = 0;
    uint32_t ph = 1;  // parity of the empty phase to wait for (first pass: none)
    const bool hint = p.l2_hint != 0;
    const uint64_t pol_a = (p.l2_hint & 2) ? l2_policy_evict_last() : (p.l2_hint & 1) ? l2_policy_evict_first() : 0;
    const uint64_t pol_b = (p.l2_hint & 1) ? l2_policy_evict_last() : l2_policy_evict_normal();
    for (int seg = 0; seg < nseg && !*abort_flag; ++seg) {
    const int b = bloop ? seg : bz;
    const int a_row = (int)(b * p.a_mn_step) + m0;
    const int b_row = (int)(b * p.b_mn_step) + n0;
    for (int kb = 0; kb < nkb; ++kb) {
      if (issued >= stages && !mbar_try(&empty[s], ph) && !mbar_wait(&empty[s], ph, abort_flag)) {
        *abort_flag = 1;
        break;
      }
      uint8_t *st = smem + (size_t)s * stage_bytes;
      mbar_expect_tx(&full[s], (uint32_t)stage_bytes);
      const int k0 = (kb0 + kb) * BK;
      const int ka = k0 + (int)(b * p.a_k_step), kbb = k0 + (int)(b * p.b_k_step);
      for (int q = 0; q < p.na; ++q) {
        if (!AMN) {
          if (hint) tma_load_3d_pol(st + q * C::A_TILE, &mapA, &full[s], ka, a_row, q, pol_a);
          else tma_load_3d(st + q * C::A_TILE, &mapA, &full[s], ka, a_row, q);
        } else {
#pragma unroll
          for (int j = 0; j < BM / 64; ++j)
            tma_load_3d(st + q * C::A_TILE + j * (BK * 128), &mapA, &full[s], a_row + 64 * j, ka, q);
        }
      }
      uint8_t *bt = st + p.na * C::A_TILE;
      for (int q = 0; q < p.nb; ++q) {
        if (!BMN) {
          if (hint) tma_load_3d_pol(bt + q * C::B_TILE, &mapB, &full[s], kbb, b_row, q, pol_b);
          else tma_load_3d(bt + q * C::B_TILE, &mapB, &full[s], kbb, b_row, q);
        } else {
#pragma unroll
          for (int j = 0; j < BN / 64; ++j)
            tma_load_3d(bt + q * C::B_TILE + j * (BK * 128), &mapB, &full[s], b_row + 64 * j, kbb, q);
        }
      }
      ++issued;
      if (++s == stages) {
        s = 0;
        ph ^= 1u;
      }
    }
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
    // The tensor core queues about one MMA ahead of this thread, so everything between two MMAs
    // stalls the pipe: descriptors are precomputed (start-address field + byte offset / 16),
    // stage and chunk positions are counters, and the full-barrier wait tries once inline first.
    const uint32_t idesc = idesc_bf16(BM, BN, AMN, BMN);
    const uint64_t dA = AMN ? sdesc(0, BK * 128, 1024, 2u) : sdesc(0, 16, C::A_SBO, C::A_LAYOUT);
    const uint64_t dB = BMN ? sdesc(0, BK * 128, 1024, 2u) : sdesc(0, 16, C::A_SBO, C::A_LAYOUT);
    constexpr uint32_t kStepA = AMN ? 2048 / 16 : 32 / 16;  // one K = 16 step, in 16-byte units
    constexpr uint32_t kStepB = BMN ? 2048 / 16 : 32 / 16;
    const int nprod = p.nprod;
    uint32_t aoff[8], boff[8];
#pragma unroll
    for (int i = 0; i < 8; ++i) {
      aoff[i] = (i < nprod) ? (uint32_t)(p.pa[i] * C::A_TILE) >> 4 : 0u;
      boff[i] = (i < nprod) ? (uint32_t)(p.na * C::A_TILE + p.pb[i] * C::B_TILE) >> 4 : 0u;
    }
    const uint32_t smem16 = su32(smem) >> 4, stage16 = (uint32_t)stage_bytes >> 4;
    const int chunk_kb = p.chunk_kb;
    int chunk = 0, cleft = 0, s = 0;
    uint32_t ph = 0, tacc = tmem, accf = 0;
    for (int seg = 0; seg < nseg && !*abort_flag; ++seg)
    for (int kb = 0; kb < nkb; ++kb) {
      if (cleft == 0) {
        const int b2 = chunk & 1;
        if (chunk >= 2 && !mbar_wait(&tempty[b2], ((chunk >> 1) & 1) ^ 1, abort_flag)) {
          *abort_flag = 1;
          break;
        }
        tc_fence_after();
        tacc = tmem + (uint32_t)(b2 * BN);
        accf = 0;
        cleft = chunk_kb;
      }
      if (!mbar_try(&full[s], ph) && !mbar_wait(&full[s], ph, abort_flag)) {
        *abort_flag = 1;
        break;
      }
      tc_fence_after();
      const uint64_t so = (uint64_t)(smem16 + (uint32_t)s * stage16);
#pragma unroll
      for (int i = 0; i < 8; ++i) {
        if (i < nprod) {
          const uint64_t da = dA + so + aoff[i], db = dB + so + boff[i];
#pragma unroll
          for (int kk = 0; kk < BK / 16; ++kk) {
            umma_bf16(tacc, da + kk * kStepA, db + kk * kStepB, idesc, accf);
            accf = 1u;
          }
        }
      }
      umma_commit(&empty[s]);
      if (--cleft == 0 || kb == nkb - 1) {
        umma_commit(&tfull[chunk & 1]);  // arrives when this chunk's MMAs have completed
        ++chunk;
        cleft = 0;
      }
      if (++s == stages) {
        s = 0;
        ph ^= 1u;
      }
    }
  } else if (warp >= 2) {
    // ---------------------------------------------------------------- epilogue
    const int q = warp & 3;                 // TMEM lane quarter accessible to this warp
    const int h = (warp - 2) >> 2;          // column half
    const int row = q * 32 + lane;
    const int nchunks = (nkb + p.chunk_kb - 1) / p.chunk_kb;  // per segment
    const int gm = m0 + row;
    bool ok = true;
    int c = 0;  // chunks drained so far (all segments)
    for (int seg = 0; seg < nseg && ok; ++seg) {
    const int b = bloop ? seg : bz;
    float acc[C::HALF];
#pragma unroll
    for (int j = 0; j < C::HALF; ++j) acc[j] = 0.f;
    for (int cc = 0; cc < nchunks; ++cc, ++c) {
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
      for (int j = 0; j < C::HALF; j += 16) {
        uint32_t v[16];
        tmem_ld16(tbase + (uint32_t)j, v);
        tmem_wait();
#pragma unroll
        for (int i = 0; i < 16; ++i) acc[j + i] += __uint_as_float(v[i]);
      }
      tc_fence_before();
      __syncwarp();
      if (lane == 0) asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(su32(&tempty[b2])) : "memory");
    }
    if (ok && p.stage_out) {
      // every MMA has completed (last tfull), so every load has landed and the pipeline buffers
      // are free: each warp transposes its 32 x HALF block through them and writes whole rows
      constexpr int SROW = C::HALF + 1;
      float *stg = (float *)smem + (size_t)(warp - 2) * 32 * SROW;
#pragma unroll
      for (int j = 0; j < C::HALF; ++j) stg[lane * SROW + j] = acc[j];
      __syncwarp();
      // plane output (no value output): two consecutive columns per lane, one 4-byte store per plane
      const bool pairs = p.pl && !p.C && p.splits == 1 && !p.upper && (p.N & 1) == 0 && (C::HALF % 64) == 0 &&
                         ((p.c_step | p.pl_ld) & 1) == 0 && ((uintptr_t)p.pl & 3) == 0;
      for (int r = 0; pairs && r < 32; ++r) {
        const int gr = m0 + q * 32 + r;
        if (gr >= p.M) break;
#pragma unroll
        for (int t = 0; t < C::HALF / 64; ++t) {
          const int gn = n0 + h * C::HALF + t * 64 + 2 * lane;
          if (gn >= p.N) continue;
          __nv_bfloat16 o0[3], o1[3];
          out_pieces(p.alpha * (double)stg[r * SROW + t * 64 + 2 * lane], p.c_double, o0);
          out_pieces(p.alpha * (double)stg[r * SROW + t * 64 + 2 * lane + 1], p.c_double, o1);
          const long long po = (long long)b * p.c_step + (long long)gr * p.pl_ld + gn;
#pragma unroll
          for (int qq = 0; qq < 3; ++qq)
            *(uint32_t *)(p.pl + qq * p.pl_ps + po) =
                (uint32_t)__bfloat16_as_ushort(o0[qq]) | ((uint32_t)__bfloat16_as_ushort(o1[qq]) << 16);
        }
      }
      for (int r = 0; !pairs && r < 32; ++r) {
        const int gr = m0 + q * 32 + r;
        if (gr >= p.M) break;
#pragma unroll
        for (int t = 0; t < C::HALF / 32; ++t) {
          const int gn = n0 + h * C::HALF + t * 32 + lane;
          if (gn >= p.N || (p.upper && gn < gr)) continue;
          const float v = stg[r * SROW + t * 32 + lane];
          if (p.splits == 1) {
            if (p.pl) store_pieces(p, (long long)b * p.c_step + (long long)gr * p.pl_ld + gn, p.alpha * (double)v);
            if (!p.C) continue;
            const long long off = (long long)b * p.c_step + (long long)gr * p.c_rs + (long long)gn * p.c_cs;
            if (p.c_double) ((double *)p.C)[off] = p.alpha * (double)v;
            else ((float *)p.C)[off] = (float)(p.alpha * (double)v);
          } else {
            p.partial[(((long long)b * p.splits + split) * p.M + gr) * p.N + gn] = v;
          }
        }
      }
    } else if (BN <= 128 && ok && gm < p.M && p.vec_out && p.splits == 1) {
      // this thread's row: 16-byte stores of 4 (FP32) or 2 (FP64) consecutive columns
      const int gn0 = n0 + h * C::HALF;
      const long long off0 = (long long)b * p.c_step + (long long)gm * p.c_rs + gn0;
      if (p.pl) {  // eight consecutive columns: one 16-byte store per plane (N, ld, steps multiples of 8)
        const long long po0 = (long long)b * p.c_step + (long long)gm * p.pl_ld + gn0;
#pragma unroll
        for (int j = 0; j < C::HALF; j += 8) {
          if (gn0 + j >= p.N) break;
          __nv_bfloat16 o[8][3];
#pragma unroll
          for (int u = 0; u < 8; ++u) out_pieces(p.alpha * (double)acc[j + u], p.c_double, o[u]);
#pragma unroll
          for (int q = 0; q < 3; ++q) {
            uint4 w;
            w.x = (uint32_t)__bfloat16_as_ushort(o[0][q]) | ((uint32_t)__bfloat16_as_ushort(o[1][q]) << 16);
            w.y = (uint32_t)__bfloat16_as_ushort(o[2][q]) | ((uint32_t)__bfloat16_as_ushort(o[3][q]) << 16);
            w.z = (uint32_t)__bfloat16_as_ushort(o[4][q]) | ((uint32_t)__bfloat16_as_ushort(o[5][q]) << 16);
            w.w = (uint32_t)__bfloat16_as_ushort(o[6][q]) | ((uint32_t)__bfloat16_as_ushort(o[7][q]) << 16);
            *(uint4 *)(p.pl + q * p.pl_ps + po0 + j) = w;
          }
        }
      }
#pragma unroll
      for (int j = 0; j < C::HALF; j += 4) {
        if (!p.C || gn0 + j >= p.N) break;  // N % 4 == 0: a group is either whole or outside
        if (p.c_double) {
          double2 *o = (double2 *)((double *)p.C + off0 + j);
          o[0] = make_double2(p.alpha * (double)acc[j], p.alpha * (double)acc[j + 1]);
          o[1] = make_double2(p.alpha * (double)acc[j + 2], p.alpha * (double)acc[j + 3]);
        } else {
          *(float4 *)((float *)p.C + off0 + j) =
              make_float4((float)(p.alpha * (double)acc[j]), (float)(p.alpha * (double)acc[j + 1]),
                          (float)(p.alpha * (double)acc[j + 2]), (float)(p.alpha * (double)acc[j + 3]));
        }
      }
    } else if (ok && gm < p.M) {
      const bool upper_tile = p.upper != 0;
#pragma unroll
      for (int j = 0; j < C::HALF; ++j) {
        const int gn = n0 + h * C::HALF + j;
        if (gn >= p.N) break;
        if (upper_tile && gn < gm) continue;
        if (p.splits == 1) {
          if (p.pl) store_pieces(p, (long long)b * p.c_step + (long long)gm * p.pl_ld + gn, p.alpha * (double)acc[j]);
          if (!p.C) continue;
          const long long off = (long long)b * p.c_step + (long long)gm * p.c_rs + (long long)gn * p.c_cs;
          if (p.c_double) ((double *)p.C)[off] = p.alpha * (double)acc[j];
          else ((float *)p.C)[off] = (float)(p.alpha * (double)acc[j]);
        } else {
          p.partial[(((long long)b * p.splits + split) * p.M + gm) * p.N + gn] = acc[j];
        }
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

// ------------------------------------------------------------------ CTA-pair (cta_group::2) GEMM
// K-major A and B, no batch / split-K / triangle.  The two CTAs of a cluster compute one 256 x 256
// tile: CTA r (rank in the pair) stages A rows [m0 + 128 r, +128) and B rows [n0 + 128 r, +128) of
// every plane in its own shared memory, and CTA 0 issues tcgen05.mma.cta_group::2 (M = 256), which
// reads the A half and both B halves of each CTA.  Each SM thus loads half a B tile per k-block
// instead of a whole one, which halves the L2-to-SM traffic of B (what limits the many-plane Gram
// products; the sketch, with one B plane, is not limited by it).
// Barriers: full[s] lives in CTA 0 and receives the bytes of both CTAs' loads; empty[s] and
// tfull[b] exist in both CTAs and receive one tcgen05.commit each from CTA 0; tempty[b] lives in
// CTA 0 and counts the epilogue warps of both CTAs (remote arrivals from CTA 1).  The epilogue
// stages each warp's 32 x 128 FP32 block through the (then idle) pipeline buffers, so the final
// store writes whole 128-byte rows.
__device__ __forceinline__ uint32_t cluster_ctarank() {
  uint32_t r;
  asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
  return r;
}
// shared::cluster address of the variable at shared::cta address `saddr` in CTA `rank` of the cluster
__device__ __forceinline__ uint32_t mapa_shared(uint32_t saddr, uint32_t rank) {
  uint32_t r;
  asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(r) : "r"(saddr), "r"(rank));
  return r;
}
__device__ __forceinline__ void cluster_sync_all() {
  asm volatile("barrier.cluster.arrive.release.aligned;\n\tbarrier.cluster.wait.acquire.aligned;" ::: "memory");
}
__device__ __forceinline__ bool mbar_try_cluster(uint64_t *bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.acquire.cluster.shared::cta.b64 p, [%1], %2, %3;\n\tselp.u32 "
      "%0, 1, 0, p;\n\t}\n"
      : "=r"(ok)
      : "r"(su32(bar)), "r"(parity), "r"(kSuspendNs)
      : "memory");
  return ok != 0;
}
__device__ __forceinline__ bool mbar_wait_cluster(uint64_t *bar, uint32_t parity, volatile int *abort_flag) {
  if (mbar_try_cluster(bar, parity)) return true;
  const unsigned long long t0 = global_ns();
  for (;;) {
    if (mbar_try_cluster(bar, parity)) return true;
    if (*abort_flag || global_ns() - t0 > kWaitNs) return false;
  }
}
__device__ __forceinline__ void mbar_arrive_remote(uint32_t bar_cluster) {
  asm volatile("mbarrier.arrive.release.cluster.shared::cluster.b64 _, [%0];" ::"r"(bar_cluster) : "memory");
}
// TMA load into this CTA's shared memory whose completion is counted on a barrier of either CTA of
// the pair (bar_cluster: a shared::cluster address); no multicast.
__device__ __forceinline__ void tma_load_3d_pair(void *dst, const CUtensorMap *map, uint32_t bar_cluster, int x,
                                                 int y, int z) {
  asm volatile(
      "cp.async.bulk.tensor.3d.cta_group::2.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4, "
      "%5}], [%2];" ::"r"(su32(dst)),
      "l"((uint64_t)map), "r"(bar_cluster), "r"(x), "r"(y), "r"(z)
      : "memory");
}
__device__ __forceinline__ void umma_bf16_pair(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t idesc,
                                               uint32_t acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\ttcgen05.mma.cta_group::2.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::
          "r"(tmem_d),
      "l"(da), "l"(db), "r"(idesc), "r"(acc));
}
// Arrives on the barrier at shared::cluster address bar_cluster once this thread's earlier
// cta_group::2 MMAs have completed.
__device__ __forceinline__ void umma_commit_pair(uint32_t bar_cluster) {
  asm volatile("tcgen05.commit.cta_group::2.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar_cluster)
               : "memory");
}

// MN: both operands MN-major (stored K x M and K x N, M / N contiguous; BK = 64 only), e.g. the
// Gram matrix Q'Q of a row-major Q; `upper` then skips pairs strictly below the diagonal.
template <int BK, bool MN>
__global__ void __launch_bounds__(kThreads, 1)
    umma_pair_kernel(const __grid_constant__ CUtensorMap mapA, const __grid_constant__ CUtensorMap mapB,
                     const KParams p, const int stages) {
  static_assert(!MN || BK == 64, "MN-major pair tiles use 64-deep k-blocks");
  constexpr int HT = BM * BK * 2;  // bytes of one 128-row plane tile (A, or half of B)
  constexpr uint32_t LAYOUT = (BK == 64) ? 2u : 4u;
  constexpr uint32_t SBO = (BK == 64) ? 1024u : 512u;
  const int CHUNK = p.chunk_kb;
  constexpr int BN2 = 256;         // tile columns (both halves of B)
  constexpr int HALF = BN2 / 2;    // columns per epilogue warp
  constexpr int TMEM_COLS = 512;   // two 256-column accumulators
  constexpr int SROW = HALF + 1;   // staging row stride (floats), conflict-free both ways
  extern __shared__ __align__(1024) uint8_t smem_raw[];
  uint8_t *smem = (uint8_t *)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  const int stage_bytes = (p.na + p.nb) * HT;
  uint64_t *full = (uint64_t *)(smem + (size_t)stages * stage_bytes);
  uint64_t *empty = full + stages;
  uint64_t *tfull = empty + stages;
  uint64_t *tempty = tfull + 2;
  uint64_t *mdone = tempty + 2;
  uint32_t *tslot = (uint32_t *)(mdone + 1);
  volatile int *abort_flag = (volatile int *)(tslot + 1);

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const uint32_t rank = cluster_ctarank();
  const int nt = blockIdx.x >> 1, pt = blockIdx.y;
  const int m0 = pt * (2 * BM) + (int)rank * BM, n0 = nt * BN2;
  const int nkb = p.total_kb;
  if (p.upper && n0 + BN2 <= pt * (2 * BM)) return;  // both CTAs: pair strictly below the diagonal

  if (threadIdx.x == 0) {
    for (int s = 0; s < stages; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
    }
    for (int b2 = 0; b2 < 2; ++b2) {
      mbar_init(&tfull[b2], 1);
      mbar_init(&tempty[b2], 2 * kEpiWarps);
    }
    mbar_init(mdone, 1);
    *abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 1) {
    asm volatile("tcgen05.alloc.cta_group::2.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(su32(tslot)),
                 "r"((uint32_t)TMEM_COLS));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::2.sync.aligned;");
  }
  tc_fence_before();
  __syncthreads();
  cluster_sync_all();  // barriers of CTA 0 initialised before CTA 1 loads into them
  tc_fence_after();
  const uint32_t tmem = *tslot;

  if (warp == 0 && lane == 0) {
    // ---------------------------------------------------------------- TMA producer (both CTAs)
    const int b_row = n0 + (int)rank * BM;
    const uint32_t full0 = mapa_shared(su32(full), 0);  // CTA 0's full barriers
    int issued = 0, s = 0;
    uint32_t ph = 1;
    for (int kb = 0; kb < nkb; ++kb) {
      if (kb >= stages && !mbar_try(&empty[s], ph) && !mbar_wait(&empty[s], ph, abort_flag)) {
        *abort_flag = 1;
        break;
      }
      uint8_t *st = smem + (size_t)s * stage_bytes;
      const uint32_t fb = full0 + 8u * (uint32_t)s;
      if (rank == 0) mbar_expect_tx(&full[s], (uint32_t)(2 * stage_bytes));
      const int k0 = kb * BK;
      if (!MN) {
        for (int q = 0; q < p.na; ++q) tma_load_3d_pair(st + q * HT, &mapA, fb, k0, m0, q);
        for (int q = 0; q < p.nb; ++q) tma_load_3d_pair(st + (p.na + q) * HT, &mapB, fb, k0, b_row, q);
      } else {
        // two 64-wide MN atoms of BK K-rows each per 128-row half
        for (int q = 0; q < p.na; ++q)
          for (int j = 0; j < 2; ++j) tma_load_3d_pair(st + q * HT + j * (BK * 128), &mapA, fb, m0 + 64 * j, k0, q);
        for (int q = 0; q < p.nb; ++q)
          for (int j = 0; j < 2; ++j)
            tma_load_3d_pair(st + (p.na + q) * HT + j * (BK * 128), &mapB, fb, b_row + 64 * j, k0, q);
      }
      ++issued;
      if (++s == stages) {
        s = 0;
        ph ^= 1u;
      }
    }
    // Drain (CTA 0 holds the barriers): every issued load has landed before the pair can exit.
    if (rank == 0) {
      for (int kb = max(0, issued - stages); kb < issued; ++kb) {
        const int s = kb % stages;
        long long i = 0;
        while (!mbar_try(&full[s], (kb / stages) & 1) && ++i < kWaitLimit) {
        }
      }
    }
  } else if (warp == 1 && lane == 0 && rank == 0) {
    // ---------------------------------------------------------------- MMA issuer (CTA 0)
    const uint32_t idesc = idesc_bf16(2 * BM, BN2, MN, MN);
    const uint64_t d0 = MN ? sdesc(0, BK * 128, 1024, 2u) : sdesc(0, 16, SBO, LAYOUT);
    constexpr uint32_t kStep = MN ? 2048 / 16 : 32 / 16;  // one K = 16 step, in 16-byte units
    const int nprod = p.nprod;
    uint32_t aoff[8], boff[8];
#pragma unroll
    for (int i = 0; i < 8; ++i) {
      aoff[i] = (i < nprod) ? (uint32_t)(p.pa[i] * HT) >> 4 : 0u;
      boff[i] = (i < nprod) ? (uint32_t)((p.na + p.pb[i]) * HT) >> 4 : 0u;
    }
    const uint32_t smem16 = su32(smem) >> 4, stage16 = (uint32_t)stage_bytes >> 4;
    // shared::cluster addresses of both CTAs' barrier arrays (each CTA's window is contiguous)
    const uint32_t empty0 = mapa_shared(su32(empty), 0), empty1 = mapa_shared(su32(empty), 1);
    const uint32_t tfull0 = mapa_shared(su32(tfull), 0), tfull1 = mapa_shared(su32(tfull), 1);
    int chunk = 0, cleft = 0, s = 0;
    uint32_t ph = 0, tacc = tmem, accf = 0;
    for (int kb = 0; kb < nkb; ++kb) {
      if (cleft == 0) {
        const int b2 = chunk & 1;
        if (chunk >= 2 && !mbar_wait_cluster(&tempty[b2], ((chunk >> 1) & 1) ^ 1, abort_flag)) {
          *abort_flag = 1;
          break;
        }
        tc_fence_after();
        tacc = tmem + (uint32_t)(b2 * BN2);
        accf = 0;
        cleft = CHUNK;
      }
      if (!mbar_try(&full[s], ph) && !mbar_wait(&full[s], ph, abort_flag)) {
        *abort_flag = 1;
        break;
      }
      tc_fence_after();
      const uint64_t so = (uint64_t)(smem16 + (uint32_t)s * stage16);
#pragma unroll
      for (int i = 0; i < 8; ++i) {
        if (i < nprod) {
          const uint64_t da = d0 + so + aoff[i], db = d0 + so + boff[i];
#pragma unroll
          for (int kk = 0; kk < BK / 16; ++kk) {
            umma_bf16_pair(tacc, da + kk * kStep, db + kk * kStep, idesc, accf);
            accf = 1u;
          }
        }
      }
      umma_commit_pair(empty0 + 8u * (uint32_t)s);
      umma_commit_pair(empty1 + 8u * (uint32_t)s);
      if (--cleft == 0 || kb == nkb - 1) {
        const int b2 = chunk & 1;
        umma_commit_pair(tfull0 + 8u * (uint32_t)b2);
        umma_commit_pair(tfull1 + 8u * (uint32_t)b2);
        ++chunk;
        cleft = 0;
      }
      if (++s == stages) {
        s = 0;
        ph ^= 1u;
      }
    }
    // every MMA (they write both CTAs' tensor memory) has completed before the pair frees it
    umma_commit_pair(mapa_shared(su32(mdone), 0));
    long long i = 0;
    while (!mbar_try(mdone, 0) && ++i < kWaitLimit) {
    }
  } else if (warp >= 2) {
    // ---------------------------------------------------------------- epilogue (both CTAs)
    const int q = warp & 3;
    const int h = (warp - 2) >> 2;
    const int nchunks = (nkb + CHUNK - 1) / CHUNK;
    float acc[HALF];
#pragma unroll
    for (int j = 0; j < HALF; ++j) acc[j] = 0.f;
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
      const uint32_t tbase = tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)(b2 * BN2 + h * HALF);
#pragma unroll
      for (int j = 0; j < HALF; j += 32) {
        uint32_t v[32];
        tmem_ld32(tbase + (uint32_t)j, v);
        tmem_wait();
#pragma unroll
        for (int i = 0; i < 32; ++i) acc[j + i] += __uint_as_float(v[i]);
      }
      tc_fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive_remote(mapa_shared(su32(&tempty[b2]), 0));
    }
    if (ok) {
      // all MMAs have completed (last tfull), so every load has landed: the pipeline buffers are free
      float *stg = (float *)smem + (size_t)(warp - 2) * 32 * SROW;
#pragma unroll
      for (int j = 0; j < HALF; ++j) stg[lane * SROW + j] = acc[j];
      __syncwarp();
      const int gn0 = n0 + h * HALF;
      for (int r = 0; r < 32; ++r) {
        const int gm = m0 + q * 32 + r;
        if (gm >= p.M) break;
#pragma unroll
        for (int t = 0; t < HALF / 32; ++t) {
          const int gn = gn0 + t * 32 + lane;
          if (gn < p.N && !(p.upper && gn < gm)) {
            const float v = stg[r * SROW + t * 32 + lane];
            const long long off = (long long)gm * p.c_rs + (long long)gn * p.c_cs;
            if (p.c_double) ((double *)p.C)[off] = p.alpha * (double)v;
            else ((float *)p.C)[off] = (float)(p.alpha * (double)v);
          }
        }
      }
    }
  }
  __syncthreads();
  if (*abort_flag && threadIdx.x == 0) atomicExch(p.status, (int)kErrTimeout);
  tc_fence_before();
  cluster_sync_all();  // CTA 0's MMAs are complete before either CTA frees tensor memory
  if (warp == 1) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::2.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"((uint32_t)TMEM_COLS));
  }
}

// C(b, r, c) = alpha * sum_s partial(b, s, r, c) (FP64 sum); upper: only c >= r.
__global__ void umma_reduce_kernel(const KParams p) {
  // one thread per 4 consecutive columns of a row; the partial of split sp is added into
  // accumulator sp % 8 and the eight are summed pairwise (a fixed order)
  const int n4 = (p.N + 3) >> 2;
  const unsigned groups = (unsigned)p.M * (unsigned)n4 * (unsigned)p.batch;  // < 2^31 (host check)
  const long long stride = (long long)p.M * p.N;
  const bool vec = (p.N & 3) == 0;
  for (unsigned g = blockIdx.x * blockDim.x + threadIdx.x; g < groups; g += gridDim.x * blockDim.x) {
    const unsigned c4 = g % (unsigned)n4, rb = g / (unsigned)n4;
    const unsigned r = rb % (unsigned)p.M, b = rb / (unsigned)p.M;
    const int c0 = (int)c4 * 4;
    const float *q = p.partial + (((long long)b * p.splits) * p.M + r) * p.N + c0;
    double acc[8][4];
#pragma unroll
    for (int u = 0; u < 8; ++u)
#pragma unroll
      for (int j = 0; j < 4; ++j) acc[u][j] = 0.0;
    for (int sp0 = 0; sp0 < p.splits; sp0 += 8) {
#pragma unroll
      for (int u = 0; u < 8; ++u) {
        if (sp0 + u < p.splits) {
          const float *qs = q + (sp0 + u) * stride;
          float v[4];
          if (vec) {
            const float4 t = __ldg((const float4 *)qs);
            v[0] = t.x; v[1] = t.y; v[2] = t.z; v[3] = t.w;
          } else {
#pragma unroll
            for (int j = 0; j < 4; ++j) v[j] = (c0 + j < p.N) ? qs[j] : 0.f;
          }
#pragma unroll
          for (int j = 0; j < 4; ++j) acc[u][j] += (double)v[j];
        }
      }
    }
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const int c = c0 + j;
      if (c >= p.N || (p.upper && c < (int)r)) continue;
      const double sum = ((acc[0][j] + acc[1][j]) + (acc[2][j] + acc[3][j])) + ((acc[4][j] + acc[5][j]) + (acc[6][j] + acc[7][j]));
      if (p.pl) store_pieces(p, (long long)b * p.c_step + (long long)r * p.pl_ld + c, p.alpha * sum);
      if (!p.C) continue;
      const long long off = (long long)b * p.c_step + (long long)r * p.c_rs + (long long)c * p.c_cs;
      if (p.c_double) ((double *)p.C)[off] = p.alpha * sum;
      else ((float *)p.C)[off] = (float)(p.alpha * sum);
    }
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

// Pieces of an FP32 value in FP32 arithmetic: x - bf16(x) is exact in FP32 (the rounding error of
// an 8-bit rounding of a 24-bit significand), and so is the next remainder.
__device__ __forceinline__ void split3f(float x, __nv_bfloat16 *o) {
  const __nv_bfloat16 h0 = __float2bfloat16_rn(x);
  const float r1 = x - __bfloat162float(h0);
  const __nv_bfloat16 h1 = __float2bfloat16_rn(r1);
  const float r2 = r1 - __bfloat162float(h1);
  o[0] = h0;
  o[1] = h1;
  o[2] = __float2bfloat16_rn(r2);
}

// Non-transposed: plane(r, c) for r < rows_pad, c < ld (zero outside rows x cols).  Grid: x over
// 8-column groups of a row (one 16-byte vector per plane per thread), y striding over rows; rows
// with unit column stride and 16-byte aligned starts are read as vectors.
template <class T>
__global__ void split_kernel(const T *__restrict__ src, long long s_rs, long long s_cs, long long rows,
                             long long cols, long long rows_pad, int np, __nv_bfloat16 *__restrict__ dst,
                             long long ld, long long ps) {
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  const long long c0 = 8LL * g;
  if (c0 >= ld) return;
  for (long long r = blockIdx.y; r < rows_pad; r += gridDim.y) {
    T x[8];
    const T *row = src + r * s_rs;
    if (r < rows && c0 + 8 <= cols && s_cs == 1 && ((uintptr_t)(row + c0) & 15) == 0) {
      if (sizeof(T) == 4) {
        const float4 u = __ldg((const float4 *)(row + c0)), v = __ldg((const float4 *)(row + c0) + 1);
        x[0] = (T)u.x; x[1] = (T)u.y; x[2] = (T)u.z; x[3] = (T)u.w;
        x[4] = (T)v.x; x[5] = (T)v.y; x[6] = (T)v.z; x[7] = (T)v.w;
      } else {
#pragma unroll
        for (int i = 0; i < 4; ++i) {
          const double2 u = __ldg((const double2 *)(row + c0) + i);
          x[2 * i] = (T)u.x;
          x[2 * i + 1] = (T)u.y;
        }
      }
    } else {
#pragma unroll
      for (int i = 0; i < 8; ++i) {
        const long long c = c0 + i;
        x[i] = (r < rows && c < cols) ? src[r * s_rs + c * s_cs] : T(0);
      }
    }
    __nv_bfloat16 o[3][8];
#pragma unroll
    for (int i = 0; i < 8; ++i) {
      __nv_bfloat16 t[3];
      if (sizeof(T) == 4) split3f((float)x[i], t);
      else split3<T>(x[i], t, 3);
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
                                  long long rows_pad, uint64_t seed, long long pair0) {
  // one thread per (c, j-pair): value indices offset + j*Nl + c (offset = 2 pair0); pairs in value
  // space (2p, 2p + 1) hold consecutive c for even Nl, so each thread produces one pair and writes
  // two rows of dst.
  const long long total_pairs = (n * Nl + 1) / 2;
  for (long long pi = blockIdx.x * (long long)blockDim.x + threadIdx.x; pi < total_pairs;
       pi += (long long)gridDim.x * blockDim.x) {
    const long long gp = pair0 + pi;
    const uint4 x = philox(make_uint4((uint32_t)gp, (uint32_t)(gp >> 32), 0u, 0u), (uint32_t)seed,
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

// k-blocks per accumulation chunk: chunk_k deep (0: kChunkK; ISVD_UMMA_CHUNK_K overrides)
int chunk_kblocks(int bk, int chunk_k) {
  int ck = chunk_k > 0 ? chunk_k : kChunkK;
  if (const char *e = getenv("ISVD_UMMA_CHUNK_K")) ck = std::max(bk, atoi(e));
  return std::max(1, ck / bk);
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
  p.pl = g.planes; p.pl_ld = g.p_ld; p.pl_ps = g.p_ps;
  if (g.planes && (g.c_cs != 1 || g.upper)) fail(kErrArgument, "tcgen05 GEMM: plane output needs unit column stride");
  p.n_group = std::max(0, g.n_group);
  p.l2_hint = (g.l2_hint ? 1 : 0) | (g.a_keep ? 2 : 0);
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
    // split-K by a time model (one CTA per SM): the busiest SM runs ceil(tiles s / SMs) CTAs of
    // ceil(k-blocks / s) k-blocks (BM BN BK 2 nprod flops each at about 9.5 TFLOP/s of bf16 per
    // SM) plus a fixed 3 us (TMEM, pipeline fill, epilogue), and s > 1 adds the FP32 partials'
    // round trip, (s + 1) M N 4 bytes at about 3 TB/s; the smallest s within 3 % of the best
    // (s <= 16, at least 8 k-blocks per split; only below four waves, beyond which quantisation
    // costs under 6 % and partial sums add traffic)
    const int smax = tiles < 4LL * rt.num_sms ? (int)std::max(1, std::min(16, p.total_kb / 8)) : 1;
    const double t_kb = (double)BM * BN * BK * 2.0 * g.nprod / 9.5e12, t_fixed = 3e-6, bw = 3e12;
    const double mnb = (double)g.M * g.N * g.batch;
    auto model = [&](int sp) {
      const long long per_sm = (tiles * sp + rt.num_sms - 1) / rt.num_sms;
      const long long kb = (p.total_kb + sp - 1) / sp;
      return per_sm * (kb * t_kb + t_fixed) + (sp > 1 ? (sp + 1) * mnb * 4.0 / bw : 0.0);
    };
    double best = 1e30;
    for (int sp = 1; sp <= smax; ++sp) best = std::min(best, model(sp));
    splits = 1;
    for (int sp = 1; sp <= smax; ++sp)
      if (model(sp) <= 1.03 * best) {
        splits = sp;
        break;
      }
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
  p.chunk_kb = chunk_kblocks(BK, g.chunk_k);
  // rows of C contiguous (or a split-K partial): stage the epilogue through shared memory when the
  // pipeline buffers can hold the 8 warps' 32 x (BN/2 + 1) blocks
  // many short batches (e.g. N block products of K = l): one CTA per tile runs all of them in turn,
  // each one accumulation segment, instead of one CTA per (tile, batch) that would mostly set up
  p.bloop = (BN <= 128 && g.batch > 1 && p.splits == 1 && p.total_kb <= 16) ? 1 : 0;
  p.stage_out = (!p.bloop && (p.splits > 1 || g.c_cs == 1) && stages * stage_bytes >= 8 * 32 * (C::HALF + 1) * 4) ? 1 : 0;
  if (g.planes_in_place && !p.bloop) fail(kErrUnsupported, "tcgen05 GEMM: in-place plane output needs the batch loop");
  p.vec_out = (BN <= 128 && g.c_cs == 1 && !g.upper && g.N % 4 == 0 && g.c_rs % 4 == 0 && g.c_step % 4 == 0 &&
               (!g.planes || (g.N % 8 == 0 && g.p_ld % 8 == 0 && g.c_step % 8 == 0 && ((uintptr_t)g.planes % 16) == 0)) &&
               ((uintptr_t)g.C % 16) == 0) ? 1 : 0;
  if (stages < 2) fail(kErrUnsupported, "tcgen05 GEMM: %d planes do not fit in shared memory", g.A.np + g.B.np);
  const size_t smem = (size_t)stages * stage_bytes + 1024 + 256;
  static_assert(kThreads == 64 + 32 * kEpiWarps, "warp roles");
  auto kern = umma_gemm_kernel<BN, BK, AMN, BMN>;
  CK(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  dim3 grid(gx, gy, p.bloop ? 1 : g.batch * p.splits);
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
    const long long groups = (long long)g.M * ((g.N + 3) / 4) * g.batch;
    if (groups >= (1LL << 31)) fail(kErrUnsupported, "tcgen05 GEMM: split-K output too large");
    const int blocks = (int)std::min<long long>((groups + 255) / 256, 16LL * rt.num_sms);
    umma_reduce_kernel<<<blocks, 256, 0, st>>>(p);
    KLAUNCHED();
  }
}

// Pair kernel: K-major A and B, one batch, no split-K, no triangle; grid (2 x N tiles, M pairs),
// clusters of two CTAs along x.
template <int BK, bool MN>
void launch_pair(const UmmaGemm &g, cudaStream_t st, int *status) {
  Runtime &rt = Runtime::get();
  KParams p;
  memset(&p, 0, sizeof(p));
  p.M = g.M; p.N = g.N; p.K = g.K;
  p.na = g.A.np; p.nb = g.B.np; p.nprod = g.nprod;
  for (int i = 0; i < g.nprod; ++i) { p.pa[i] = g.pa[i]; p.pb[i] = g.pb[i]; }
  p.batch = 1; p.splits = 1;
  p.C = g.C; p.c_double = g.c_double;
  if (g.planes) fail(kErrUnsupported, "tcgen05 CTA-pair GEMM: no plane output");
  p.c_rs = g.c_rs; p.c_cs = g.c_cs;
  p.alpha = g.alpha;
  p.upper = g.upper ? 1 : 0;
  p.status = status;
  p.total_kb = (g.K + BK - 1) / BK;
  p.kbps = p.total_kb;
  p.chunk_kb = chunk_kblocks(BK, g.chunk_k);
  const CUtensorMapSwizzle sw = (BK == 64) ? CU_TENSOR_MAP_SWIZZLE_128B : CU_TENSOR_MAP_SWIZZLE_64B;
  CUtensorMap ma = MN ? make_map(g.A, 64, BK, CU_TENSOR_MAP_SWIZZLE_128B) : make_map(g.A, BK, BM, sw);
  // 128-row halves of the 256-row B tile
  CUtensorMap mb = MN ? make_map(g.B, 64, BK, CU_TENSOR_MAP_SWIZZLE_128B) : make_map(g.B, BK, BM, sw);
  const int stage_bytes = (g.A.np + g.B.np) * BM * BK * 2;
  const int budget = (int)rt.smem_optin - 1024 - 256;
  const int stages = std::min(8, budget / stage_bytes);
  // the epilogue stages 8 warps x 32 rows x 129 floats in the pipeline buffers
  if (stages < 2 || stages * stage_bytes < 8 * 32 * 129 * 4)
    fail(kErrUnsupported, "tcgen05 pair GEMM: %d planes do not fit in shared memory", g.A.np + g.B.np);
  const size_t smem = (size_t)stages * stage_bytes + 1024 + 256;
  auto kern = umma_pair_kernel<BK, MN>;
  CK(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  const int gx = (g.N + 255) / 256, gy = (g.M + 2 * BM - 1) / (2 * BM);
  cudaLaunchConfig_t cfg;
  memset(&cfg, 0, sizeof(cfg));
  cfg.gridDim = dim3((unsigned)(2 * gx), (unsigned)gy, 1);
  cfg.blockDim = dim3(kThreads, 1, 1);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = 2;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  if (profiling()) {
    CK(cudaEventCreate(&e0));
    CK(cudaEventCreate(&e1));
    CK(cudaEventRecord(e0, st));
  }
  CK(cudaLaunchKernelEx(&cfg, kern, ma, mb, p, stages));
  KLAUNCHED();
  if (profiling()) {
    CK(cudaEventRecord(e1, st));
    CK(cudaEventSynchronize(e1));
    float ms = 0.f;
    CK(cudaEventElapsedTime(&ms, e0, e1));
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    profile_add(g.tag, ms, 2.0 * g.M * (double)g.N * g.K * g.nprod);
  }
}

}  // namespace

template <class T>
void split_planes(const T *src, long long s_rs, long long s_cs, long long rows, long long cols, int np,
                  bool transpose, __nv_bfloat16 *dst, long long ld, long long plane_stride, cudaStream_t st) {
  const long long out_rows = transpose ? cols : rows;
  const long long rows_pad = plane_stride / ld;
  if (rows_pad < out_rows || ld < (transpose ? rows : cols)) fail(kErrArgument, "split_planes: plane too small");
  if (!transpose) {
    if (ld % 8) fail(kErrArgument, "split_planes: ld must be a multiple of 8");
    const dim3 grid((unsigned)((ld / 8 + 255) / 256), (unsigned)std::min<long long>(rows_pad, 65535));
    split_kernel<T><<<grid, 256, 0, st>>>(src, s_rs, s_cs, rows, cols, rows_pad, np, dst, ld, plane_stride);
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
  if (ld % 8) fail(kErrArgument, "split_rows: ld must be a multiple of 8");
  if (!transpose) {
    if (ld < cols) fail(kErrArgument, "split_rows: plane too narrow");
    const dim3 grid((unsigned)((ld / 8 + 255) / 256), (unsigned)std::min<long long>(std::max(rows, 1LL), 65535));
    split_kernel<T><<<grid, 256, 0, st>>>(src, s_rs, s_cs, rows, cols, rows, np, dst, ld, plane_stride);
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
                         uint64_t seed, cudaStream_t st, long long offset) {
  if (offset % 2) fail(kErrUnsupported, "bf16 Omega: an odd value offset (odd rows x odd Nl)");
  Runtime &rt = Runtime::get();
  if (rows_pad > Nl)
    CK(cudaMemsetAsync(dst + (size_t)Nl * ld, 0, (size_t)(rows_pad - Nl) * ld * sizeof(__nv_bfloat16), st));
  if (ld > n)
    CK(cudaMemset2DAsync(dst + n, ld * sizeof(__nv_bfloat16), 0, (ld - n) * sizeof(__nv_bfloat16), Nl, st));
  const long long pairs = (n * Nl + 1) / 2;
  const int blocks = (int)std::min<long long>((pairs + 255) / 256, 32LL * rt.num_sms);
  rng_bf16_t_kernel<<<blocks, 256, 0, st>>>(dst, n, Nl, ld, Nl, seed, offset / 2);
  KLAUNCHED();
}

// The CTA-pair kernel serves K-major products with enough 256 x 256 tiles to fill the GPU when
// ISVD_UMMA_PAIR=1 (ISVD_UMMA_PAIR_BK=32 selects 32-deep k-blocks).  Off by default: on the
// sketch shape it measures 2 % slower than the one-CTA kernel, whose tensor pipe is not limited by
// shared-memory bandwidth once its issue loop is tight.
static bool pair_ok(const UmmaGemm &g) {
  const char *e = getenv("ISVD_UMMA_PAIR");
  if (!e || atoi(e) == 0) return false;
  const long long tiles = (long long)((g.N + 255) / 256) * ((g.M + 255) / 256);
  return tiles >= Runtime::get().num_sms / 2 && g.K >= 1024;
}
// MN-major pairs (Gram matrices Q'Q of row-major panels; ISVD_UMMA_PAIR_MN=0 turns them off): each
// SM stages half of the B tile, which halves the L2 traffic of these shared-operand products (the
// Gram Qs'Qs of a 200000 x 4096 Qs, as 2 x 2 planes: 13.3 -> 8.0 ms).
static bool pair_mn_ok(const UmmaGemm &g) {
  const char *e = getenv("ISVD_UMMA_PAIR_MN");
  if (e && atoi(e) == 0) return false;
  const long long tiles = (long long)((g.N + 255) / 256) * ((g.M + 255) / 256);
  return tiles >= Runtime::get().num_sms / 2 && g.K >= 1024 && g.A.np + g.B.np <= 4;
}
// ISVD_UMMA_WIDE_MN=0: MN-major B products keep 128-wide tiles (for comparison)
static bool wide_mn_off() {
  const char *e = getenv("ISVD_UMMA_WIDE_MN");
  return e && atoi(e) == 0;
}
// ISVD_UMMA_SMALLN_BK=64 / 32: the k-block depth of the N <= 128 products with five or more planes
// (0: by the tile count, below)
static int smalln_bk() {
  const char *e = getenv("ISVD_UMMA_SMALLN_BK");
  return e ? atoi(e) : 0;
}
static bool bk32_forced() {
  const char *e = getenv("ISVD_UMMA_BK");
  return e && atoi(e) == 32;
}
static int pair_bk() {
  const char *e = getenv("ISVD_UMMA_PAIR_BK");
  return (e && atoi(e) == 32) ? 32 : 64;
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
    if (g.batch == 1 && g.splits <= 0 && !g.planes && pair_mn_ok(g)) launch_pair<64, true>(g, st, status);
    else launch_t<128, 64, true, true>(g, st, status);
  } else if (amn) {
    fail(kErrUnsupported, "tcgen05 GEMM: MN-major A needs MN-major B");
  } else if (bmn) {
    // wide MN-major B against at most 128 rows of A (the projection Z' = Qbar' A, n columns): 256-wide
    // tiles read the A operand half as often from L2 (32-deep k-blocks keep four pipeline stages)
    if (g.M <= BM && g.N >= 2048 && !g.upper && !wide_mn_off()) launch_t<256, 32, false, true>(g, st, status);
    else launch_t<128, 64, false, true>(g, st, status);
  } else if (g.N <= 64) {
    // narrow outputs (N <= 64, e.g. products with k or l columns): 64-wide tiles, no half-empty MMAs
    launch_t<64, 64, false, false>(g, st, status);
  } else if (small_n) {
    // six or more planes: 32-deep k-blocks give four pipeline stages instead of two, which pays
    // when there are many tiles; for a few split-K tiles (the Kolmogorov-Nagumo G B product,
    // 4096 x 128 x 4096) 64-deep k-blocks halve the per-k-block overhead (19.4 against 20.7 ms
    // for 107 iterations)
    const long long tiles128 = (long long)((g.N + 127) / 128) * ((g.M + BM - 1) / BM) * g.batch;
    const bool few_tiles = tiles128 < Runtime::get().num_sms;
    const int sbk = smalln_bk();
    if (g.A.np + g.B.np >= 5 && (sbk == 32 || (sbk != 64 && !few_tiles))) launch_t<128, 32, false, false>(g, st, status);
    else launch_t<128, 64, false, false>(g, st, status);
  } else if (g.batch == 1 && g.splits <= 0 && !g.upper && !g.planes && pair_ok(g)) {
    if (pair_bk() == 32) launch_pair<32, false>(g, st, status);
    else launch_pair<64, false>(g, st, status);
  } else if (3 * stage64 <= (int)rt.smem_optin - 2048 && !bk32_forced()) {
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
