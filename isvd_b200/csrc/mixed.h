// MIXED precision engine: bf16 split products on tcgen05 tensor cores with FP32 accumulation.
// Each FP32/FP64 operand x is split into bf16 pieces x = x0 + x1 + x2 (+ residual); a product
// keeps the piece pairs whose combined magnitude is above the FP32 rounding level.
#pragma once

#include <cstdint>

#include "runtime.h"
#include "stages.h"
#include "umma.h"

namespace isvdb {

// An owned set of bf16 planes.
struct PlaneBuf {
  DBuf<__nv_bfloat16> buf;
  Planes P;
};

// Planes of the rows x cols matrix src (element (r, c) at src[r * s_rs + c]), optionally transposed.
template <class T>
void make_planes(PlaneBuf &pb, const T *src, long long s_rs, long long rows, long long cols, int np, bool transpose,
                 cudaStream_t st);

// Kolmogorov-Nagumo products with a fixed Nl x Nl FP64 matrix G on the tensor cores:
// Bgc = alpha * G * Bc (Bc: Nl x l FP64 row-major), G held as 3 bf16 planes, Bc split per call.
struct MixedGProduct {
  PlaneBuf g, b;
  int Nl = 0;
  void prepare(const StageCtx &c, int Nl_, const double *G);
  // Bgc = alpha G Bc (Nl x l, row strides ldb and ldo)
  void apply(const StageCtx &c, int l, const double *Bc, long long ldb, double alpha, double *Bgc, long long ldo);
};

// A's bf16 planes (m x n, K-major along n), made by the sketch and reused by the postprocess.
struct MixedCache {
  const void *src = nullptr;
  long long m = 0, n = 0;
  char ordera = 0;
  DBuf<__nv_bfloat16> buf;
  Planes A;
};

// Y = A * Omega (m x Nl, row-major ldy).  omega == nullptr: Omega is drawn exactly in bf16
// (Philox + Box-Muller, rounded), so only A is split (2 products, one per A plane).  Otherwise
// Omega is split too.
// bf16 planes of A the MIXED sketch keeps per element (2; 3 with ISVD_GPU_SKETCH_PLANES=3).
int sketch_planes();

template <class T>
void mixed_sketch(const StageCtx &c, int m, int n, int Nl, char ordera, const T *a, long long lda, const T *omega,
                  long long ldom, uint64_t seed, T *y, long long ldy);

// The next four take bf16 planes `yp` of an m x Nl row-major matrix (split without transpose,
// make_planes(.., false)) and the matrix itself (`y`, used when the block width rules out the
// plane path: l % 8 != 0 for MN-major operands, l % 64 != 0 for per-block K offsets).

// W_i = Y_i' Y_i for the N column blocks (W: N x l x l, FP64), as an MN-major x MN-major product.
template <class T>
void mixed_block_gram(const StageCtx &c, const Planes &yp, int m, int l, int N, const T *y, long long ldy,
                      double *W);

// Q_i = Y_i Wp_i (Wp: N x l x l in T) -> out (m x Nl, ld ldo).
template <class T>
void mixed_block_apply(const StageCtx &c, const Planes &yp, int m, int l, int N, const T *y, long long ldy,
                       const T *Wp, T *out, long long ldo);

// G = Qs' Qs (Nl x Nl, FP64 out; symmetric, computed on the upper triangle and mirrored).
// all_pairs: every plane product (p, q < np), so that G is the Gram of the planes' sum itself (to
// FP32 accumulation), instead of the products above the FP32 rounding level of the matrix.
template <class T>
void mixed_gram_full(const StageCtx &c, const Planes &qp, int m, int Nl, const T *qs, long long ldq, double *G,
                     int np = 2, bool all_pairs = false);

// Qbar = Qs M (M: Nl x l FP64, row-major) -> qt (m x l, ld ldqt).
template <class T>
void mixed_apply_coeff(const StageCtx &c, const Planes &qp, int m, int Nl, int l, const T *qs, long long ldq,
                       const double *M, T *qt, long long ldqt);

// Z = A' Qbar (n x l row-major).
template <class T>
void mixed_project(const StageCtx &c, int m, int n, int l, char ordera, const T *a, long long lda, const T *qt,
                   long long ldqt, T *z);

}  // namespace isvdb
