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

// The three bf16 planes (rows x cols, ld = cols, padding rows zero) that stand for the matrix at
// `of` (row stride ld_of) between two stages: its values there are not written.  `of` null: empty.
struct PlaneHandoff {
  PlaneBuf pb;
  const void *of = nullptr;
  long long ld_of = 0;
  bool holds(const void *p, long long ld) const { return of && of == p && ld_of == ld; }
  // the planes of a rows x cols matrix at p (row stride ld), to be written: allocated, padding zeroed
  void prepare(const void *p, long long ld, long long rows, long long cols, cudaStream_t st);
};
// Whether a stage of this shape can hand its output over as planes: cols a multiple of 64 (no
// padding columns), so that plane_ld(cols) == cols.
inline bool handoff_shape_ok(long long cols) { return cols > 0 && cols % 64 == 0; }

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
  // Bgc = alpha G Bc (Nl x l, row strides ldb and ldo).  split == false: Bc's planes (b) were
  // written by the producer of Bc (the previous iteration's update), Bc itself is not read.
  void apply(const StageCtx &c, int l, const double *Bc, long long ldb, double alpha, double *Bgc, long long ldo,
             bool split = true);
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

// Y = A Omega (m x Nl, row stride ldy).  hand (Nl a multiple of 64): Y's three bf16 planes are
// written into it instead of Y's values.
template <class T>
void mixed_sketch(const StageCtx &c, int m, int n, int Nl, char ordera, const T *a, long long lda, const T *omega,
                  long long ldom, uint64_t seed, T *y, long long ldy, PlaneHandoff *hand = nullptr);

// The next four take bf16 planes `yp` of an m x Nl row-major matrix (split without transpose,
// make_planes(.., false)) and the matrix itself (`y`, used when the block width rules out the
// plane path: l % 8 != 0 for MN-major operands, l % 64 != 0 for per-block K offsets).

// W_i = Y_i' Y_i for the N column blocks (W: N x l x l, FP64), as an MN-major x MN-major product.
template <class T>
void mixed_block_gram(const StageCtx &c, const Planes &yp, int m, int l, int N, const T *y, long long ldy,
                      double *W);

// Q_i = Y_i Wp_i (Wp: N x l x l in T) -> out (m x Nl, ld ldo).  hand (l a multiple of 64): the
// output's three bf16 planes go into it instead of its values -- over yp in place when yp are the
// hand-off's own planes.
template <class T>
void mixed_block_apply(const StageCtx &c, const Planes &yp, int m, int l, int N, const T *y, long long ldy,
                       const T *Wp, T *out, long long ldo, PlaneHandoff *hand = nullptr);

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
