// tcgen05 (5th-generation tensor core) GEMM engine over bf16 "planes".
//
// A matrix X held in FP32/FP64 is represented by np bf16 planes X = X0 + X1 + X2 (+ O(2^-24 |X|)).
// The engine computes C = alpha * sum_{(p, q) in products} A_p * B_q' with FP32 accumulation in
// tensor memory, where A_p is M x K and B_q is N x K (both "K-major": K contiguous), or B_q is
// stored K x N ("MN-major": N contiguous).  Tiles are moved by TMA (no multicast) into 128B/64B
// swizzled shared memory; one thread issues tcgen05.mma; four warps drain TMEM in the epilogue.
#pragma once

#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cstdint>

namespace isvdb {

struct Planes {
  const __nv_bfloat16 *ptr = nullptr;  // plane p starts at ptr + p * plane_stride
  int np = 0;                          // number of planes
  long long rows = 0;                  // K-major: MN extent; MN-major: K extent
  long long cols = 0;                  // K-major: K extent;  MN-major: MN extent
  long long ld = 0;                    // row stride in elements (multiple of 8)
  long long plane_stride = 0;          // elements
  bool mn_major = false;
};

struct UmmaGemm {
  int M = 0, N = 0, K = 0;  // per batch
  Planes A, B;
  int nprod = 0;
  int pa[8] = {0}, pb[8] = {0};  // plane pairs accumulated into C
  // batching: batch b reads A rows from b * a_mn_step, B rows from b * b_mn_step and writes
  // C at c + b * c_step.
  int batch = 1;
  long long a_mn_step = 0, b_mn_step = 0, c_step = 0;
  long long a_k_step = 0, b_k_step = 0;  // per-batch K offsets (multiples of 8, with K % BK == 0)
  // output
  void *C = nullptr;          // C(i, j) at C[i * c_rs + j * c_cs] (+ b * c_step)
  bool c_double = false;
  long long c_rs = 0, c_cs = 1;
  double alpha = 1.0;
  int splits = 0;      // split-K (0: automatic); partial sums are added in FP64
  bool upper = false;  // symmetric output: only tiles touching the upper triangle, j >= i written
  int chunk_k = 0;     // K depth of one tensor-memory accumulation chunk (0: 128)
  const char *tag = "gemm";  // name under which launches are recorded when profiling is enabled
  int *status = nullptr;     // device status word: set, the call returns without a host synchronisation
  // Optional output as three bf16 planes: element (i, j) of batch b, in the output type (FP32, or
  // FP64 with c_double), split as split_planes splits it, at planes + q p_ps + i p_ld + b c_step + j.
  // Needs c_cs == 1; C may then be null (no value output).  planes_in_place: the planes
  // overwrite the A operand's own planes (block applies: every CTA runs its batches in order, so a
  // batch's output columns are written after the last read of them); the call fails otherwise.
  __nv_bfloat16 *planes = nullptr;
  long long p_ld = 0, p_ps = 0;
  bool planes_in_place = false;
  // Tile order (long-K products whose B operand is larger than L2, e.g. the sketch's Omega'):
  // n_group > 0 runs the output tiles in column groups of n_group N tiles, every M tile of a group
  // before the next group, so that the CTAs resident at one time read one group's B rows;
  // l2_hint loads B with the L2 evict-last policy and A with evict-first.
  int n_group = 0;
  bool l2_hint = false;
  // A loads with the L2 evict-last policy (B unchanged): an A operand that later launches read
  // again and that fits in L2 (the Kolmogorov-Nagumo G planes, read once per iteration)
  bool a_keep = false;
};

// Geometry of a plane buffer for a rows x cols matrix: ld = cols rounded up to 64, rows padded to
// a multiple of 256 (every TMA box stays inside the buffer; the padding is zero).
inline long long plane_ld(long long cols) { return (cols + 63) / 64 * 64; }
inline long long plane_rows(long long rows) { return (rows + 255) / 256 * 256; }

// Split src (rows x cols, element (r, c) at src[r * s_rs + c * s_cs]) into np bf16 planes.
// transpose: plane p holds the cols x rows transpose.  dst must hold np * plane_stride elements.
template <class T>
void split_planes(const T *src, long long s_rs, long long s_cs, long long rows, long long cols, int np,
                  bool transpose, __nv_bfloat16 *dst, long long ld, long long plane_stride, cudaStream_t st);

// Planes for a block of rows only (no padding rows written): rows x cols of src (transpose:
// cols x rows output, requiring ld == roundup(rows, 64)) into dst (already offset to the first row).
template <class T>
void split_rows(const T *src, long long s_rs, long long s_cs, long long rows, long long cols, int np, bool transpose,
                __nv_bfloat16 *dst, long long ld, long long plane_stride, cudaStream_t st);

// Omega' drawn directly in bf16: plane(c, j) = bf16(N(0,1) value with index offset + j * Nl + c)
// so that Omega(j, c) matches rng_gaussian's value index convention (rounded); offset even (the
// first of this process's rows of Omega times Nl).
void rng_gaussian_bf16_t(__nv_bfloat16 *dst, long long n, long long Nl, long long ld, long long rows_pad,
                         uint64_t seed, cudaStream_t st, long long offset = 0);

void umma_gemm(const UmmaGemm &g, cudaStream_t st);

// C(c, r) = C(r, c) for c > r (completes a symmetric n x n matrix written by an `upper` GEMM).
void mirror_upper(double *C, long long n, long long ld, cudaStream_t st);

}  // namespace isvdb
