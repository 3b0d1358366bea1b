// Kolmogorov-Nagumo l x l step (reference @x@_integrate_kolmogorov_nagumo.c:184-226) on one
// thread-block cluster.
//
// With g(z) = 1/2 + (1/4 - z)^(1/2) = 1 - sum_{n>=1} Cat(n-1) z^n (Cat: Catalan numbers), the step
// needs C = g(Z)^(1/2) and C^-1 = g(Z)^(-1/2) for Z = Dgc - Dc Dc.  Both are power series in Z with
// radius of convergence 1/4 (coefficients from J. C. P. Miller's recurrence for powers of a
// series).  When rho >= ||4 Z||_2 is small, as in all but the first iterations, a series of degree
// d evaluated by the Paterson-Stockmeyer scheme (powers Z^2..Z^s by doubling, then Horner in Z^s)
// needs ceil(log2 s) + d / s dependent products, against about twenty for two coupled
// Newton-Schulz square roots; d is the smallest degree whose tail bound
// sum_{n>d} max(|c_n|, |d_n|) (rho / 4)^n is below the target.  When no degree up to the table
// size reaches it (rho close to 1), the step runs the Newton-Schulz iteration instead.
//
// The cost of the step is the chain of dependent l x l products, not their flops (2 l^3 = 4 MFLOP
// at l = 128).  All phases run in one cluster of up to 16 CTAs: operands stay in L2, a product is
// split in 32 x 32 output tiles spread over the CTAs, and phases are separated by the hardware
// cluster barrier (release / acquire at cluster scope), which costs a fraction of a microsecond
// where a grid-wide barrier through global atomics costs several.  Every CTA follows the same
// control flow (degrees and step counts are read from memory after a barrier), and there is no
// software spin-wait.
#include <cooperative_groups.h>

#include <algorithm>
#include <cmath>

#include "kernels.h"
#include "kn_common.cuh"
#include "runtime.h"

namespace cg = cooperative_groups;

namespace isvdb {
namespace {

constexpr int kKsThreads = 1024;  // one output of a 32 x 32 tile per thread
constexpr int kKsMaxL = 160;
// shared-memory row strides of the A tile (32 x l) and the B tile (l x 32), both 4 (mod 16) doubles:
// the mma.sync fragment reads (8 rows x 4 inner indices, or 4 x 8) hit 16 distinct bank pairs
constexpr int kAld = kKsMaxL + 4;
constexpr int kBld = 36;
constexpr int kKsPer = (32 * kKsMaxL + kKsThreads - 1) / kKsThreads;

struct Ks {
  int l, nr, cs, rank;
  double *As, *Bs, *part;
  // one-CTA steps (cs == 1) with l <= kKsFullL: both operands of a product staged whole in shared
  // memory (A: roundup(l, 32) rows of row stride ald, B: l4 rows of row stride bld), so that the
  // CTA's nr^2 tiles read L2 once per product instead of once per tile
  bool full;
  int ald, bld;
};
constexpr int kKsFullL = 96;
__host__ __device__ constexpr int ks_full_ld(int l) { return (l + 31) / 32 * 32 + 4; }  // 4 (mod 16) doubles
// dynamic shared memory of the whole-operand layout: A, B and the two halves' 32 x 32 partial sums
__host__ __device__ constexpr size_t ks_full_smem(int l) {
  return ((size_t)((l + 31) / 32 * 32) * ks_full_ld(l) + (size_t)((l + 3) & ~3) * ks_full_ld(l) + 2 * 1024) *
         sizeof(double);
}

// C = alpha A B + beta Cin + diag I on the 32 x 32 output tiles [tile_begin, tile_end) of a phase
// (tiles numbered across the products of the phase); CTA r takes the tiles t = r mod cs.
// Row-major l x l operands; every load goes through L2 (__ldcg), as they are written by other CTAs.
// Tile product on the FP64 tensor-core path (mma.sync m8n8k4 f64): 16 tiles of 8 x 8, two warps
// per tile (halves of the inner dimension, zero-padded to a multiple of 4); the halves' partial
// sums meet in shared memory and are added in a fixed order.
// C2, C3 (optional) receive copies of C.
__device__ void ks_mm(const Ks &k, int tile_begin, int tile_end, double alpha, const double *A, const double *B,
                      double beta, const double *Cin, double diag, double *C, double *C2 = nullptr,
                      double *C3 = nullptr) {
  const int l = k.l, tid = threadIdx.x;
  const int ty = tid >> 5, tx = tid & 31;  // output (ty, tx) of the tile in the epilogue
  const int lane = tid & 31, half = ty >> 4, mt = ty & 15, ti = mt >> 2, tj = mt & 3;  // warp: 8 x 8 tile, half
  const int l4 = (l + 3) & ~3, kh = ((l4 >> 1) + 3) & ~3;
  const int kb = half * kh, ke = min(l4, kb + kh);
  if (k.full) {  // cs == 1: every tile of [tile_begin, tile_end) in this CTA, operands staged once
    const int lr = (l + 31) & ~31;
    __syncthreads();  // the previous product's reads of the staged operands are done
    for (int e = tid; e < lr * k.ald; e += kKsThreads) {  // A rows [0, lr) x columns [0, ald), zero outside l x l
      const int r = e / k.ald, cc = e - r * k.ald;
      k.As[e] = (r < l && cc < l) ? __ldcg(A + (size_t)r * l + cc) : 0.0;
    }
    for (int e = tid; e < l4 * k.bld; e += kKsThreads) {  // B rows [0, l4) x columns [0, bld)
      const int r = e / k.bld, cc = e - r * k.bld;
      k.Bs[e] = (r < l && cc < l) ? __ldcg(B + (size_t)r * l + cc) : 0.0;
    }
    __syncthreads();
    for (int t = tile_begin; t < tile_end; ++t) {
      const int tt = t - tile_begin;
      const int i0 = (tt / k.nr) * 32, j0 = (tt % k.nr) * 32;
      const int i = i0 + ty, j = j0 + tx;
      const double cin = (beta != 0.0 && i < l && j < l) ? __ldcg(Cin + (size_t)i * l + j) : 0.0;
      double d[2] = {0.0, 0.0};
      const double *ap = k.As + (i0 + ti * 8 + (lane >> 2)) * k.ald + (lane & 3);
      const double *bq = k.Bs + (lane & 3) * k.bld + j0 + tj * 8 + (lane >> 2);
      for (int kk = kb; kk < ke; kk += 4)
        asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
                     : "+d"(d[0]), "+d"(d[1])
                     : "d"(ap[kk]), "d"(bq[kk * k.bld]));
      double *part = k.part + half * 1024;
      const int orow = ti * 8 + (lane >> 2), ocol = tj * 8 + 2 * (lane & 3);
      __syncthreads();  // the previous tile's epilogue reads of the partial sums are done
      part[orow * 32 + ocol] = d[0];
      part[orow * 32 + ocol + 1] = d[1];
      __syncthreads();
      const int o = ty * 32 + tx;
      const double acc = k.part[o] + k.part[1024 + o];
      if (i < l && j < l) {
        const double v = alpha * acc + beta * cin + (i == j ? diag : 0.0);
        C[(size_t)i * l + j] = v;
        if (C2) C2[(size_t)i * l + j] = v;
        if (C3) C3[(size_t)i * l + j] = v;
      }
    }
    return;
  }
  const int first = tile_begin + (((k.rank - tile_begin) % k.cs) + k.cs) % k.cs;
  for (int t = first; t < tile_end; t += k.cs) {
    const int tt = t - tile_begin;
    const int i0 = (tt / k.nr) * 32, j0 = (tt % k.nr) * 32;
    const int i = i0 + ty, j = j0 + tx;
    const double cin = (beta != 0.0 && i < l && j < l) ? __ldcg(Cin + (size_t)i * l + j) : 0.0;
    double ra[kKsPer], rb[kKsPer];
#pragma unroll
    for (int u = 0; u < kKsPer; ++u) {
      const int e = tid + u * kKsThreads;
      const int r = e / l, kk = e - r * l;  // A tile: 32 rows x l
      ra[u] = (e < 32 * l && i0 + r < l) ? __ldcg(A + (size_t)(i0 + r) * l + kk) : 0.0;
      const int kr = e >> 5, cb = e & 31;   // B tile: l rows x 32
      rb[u] = (e < 32 * l && j0 + cb < l) ? __ldcg(B + (size_t)kr * l + j0 + cb) : 0.0;
    }
    __syncthreads();  // the previous tile's shared memory reads are done
#pragma unroll
    for (int u = 0; u < kKsPer; ++u) {
      const int e = tid + u * kKsThreads;
      if (e < 32 * l) {
        const int r = e / l, kk = e - r * l;
        k.As[r * kAld + kk] = ra[u];
        k.Bs[(e >> 5) * kBld + (e & 31)] = rb[u];
      }
    }
    for (int e = tid; e < 32 * 4; e += kKsThreads) {  // zero the inner-dimension padding [l, l4)
      const int r = e >> 2, kk = l + (e & 3);
      if (kk < l4) {
        k.As[r * kAld + kk] = 0.0;
        k.Bs[kk * kBld + r] = 0.0;
      }
    }
    __syncthreads();
    double d[2] = {0.0, 0.0};
    const double *ap = k.As + (ti * 8 + (lane >> 2)) * kAld + (lane & 3);
    const double *bq = k.Bs + (lane & 3) * kBld + tj * 8 + (lane >> 2);
    for (int kk = kb; kk < ke; kk += 4)
      asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
                   : "+d"(d[0]), "+d"(d[1])
                   : "d"(ap[kk]), "d"(bq[kk * kBld]));
    double *part = k.part + half * 1024;  // 32 x 32 partial sums of this half
    const int orow = ti * 8 + (lane >> 2), ocol = tj * 8 + 2 * (lane & 3);
    part[orow * 32 + ocol] = d[0];
    part[orow * 32 + ocol + 1] = d[1];
    __syncthreads();
    const int o = ty * 32 + tx;
    const double acc = k.part[o] + k.part[1024 + o];
    if (i < l && j < l) {
      const double v = alpha * acc + beta * cin + (i == j ? diag : 0.0);
      C[(size_t)i * l + j] = v;
      if (C2) C2[(size_t)i * l + j] = v;
      if (C3) C3[(size_t)i * l + j] = v;
    }
  }
}

// Block-wide sum or max; every thread gets the result.
__device__ double ks_block_reduce(double v, bool is_max, double *red) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    const double w = __shfl_xor_sync(0xffffffffu, v, o);
    v = is_max ? fmax(v, w) : v + w;
  }
  __syncthreads();
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
  __syncthreads();
  double s = red[0];
  for (int i = 1; i < (int)(blockDim.x >> 5); ++i) s = is_max ? fmax(s, red[i]) : s + red[i];
  return s;
}

// Cluster-wide sum: every CTA adds its value into partial slot base + rank, the cluster
// synchronises, and each CTA sums the slots in rank order (the same value in every CTA).
__device__ double ks_cluster_sum(const Ks &k, cg::cluster_group &cluster, double v, double *slots, double *red) {
  v = ks_block_reduce(v, false, red);
  if (threadIdx.x == 0) slots[k.rank] = v;
  cluster.sync();
  double s = 0.0;
  for (int r = 0; r < k.cs; ++r) s += __ldcg(slots + r);
  return s;
}

// Series degree for rho >= ||4 Z||_2: the smallest d whose tail bound
//   tail(d) = sum_{d < n < 64} max(|c_n|, |d_n|) (rho / 4)^n + (table remainder)
// is below the target, or -1 (the remainder beyond the table is bounded by the last term times
// rho / (1 - rho)).  Evaluated by one warp: lane j holds the terms 2j and 2j + 1, suffix sums by
// shuffles, and tail is decreasing in d, so the degree is the first d whose bound passes.
__device__ int ks_degree_warp(const KnSeries &ser, double rho, double target) {
  if (!(rho < 0.9)) return -1;
  const unsigned full = 0xffffffffu;
  const int lane = threadIdx.x & 31, n0 = 2 * lane;
  const double x = 0.25 * rho;
  double xn = 1.0, b = x;  // x^(2 lane) by repeated squaring
  for (int e = n0; e; e >>= 1, b *= b)
    if (e & 1) xn *= b;
  const double t0 = fmax(fabs(ser.c[n0]), fabs(ser.d[n0])) * xn;
  const double t1 = fmax(fabs(ser.c[n0 + 1]), fabs(ser.d[n0 + 1])) * (xn * x);
  const double rem = __shfl_sync(full, t1, 31) * rho / (1.0 - rho);
  if (rem > target) return -1;
  // suf = sum of the pairs of lanes lane..31
  double suf = t0 + t1;
  for (int o = 1; o < 32; o <<= 1) {
    const double v = __shfl_down_sync(full, suf, o);
    if (lane + o < 32) suf += v;
  }
  const double after = __shfl_down_sync(full, suf, 1);  // pairs of lanes lane+1..31
  const double tail_odd = rem + (lane < 31 ? after : 0.0);  // d = 2 lane + 1
  const double tail_even = tail_odd + t1;                     // d = 2 lane
  const unsigned ok_even = __ballot_sync(full, tail_even <= target);
  const unsigned ok_odd = __ballot_sync(full, tail_odd <= target);
  const int le = ok_even ? __ffs(ok_even) - 1 : 64, lo = ok_odd ? __ffs(ok_odd) - 1 : 64;
  const int d = min(2 * le, 2 * lo + 1);
  return d < 64 ? d : 63;
}

// Block size s of the Paterson-Stockmeyer scheme: fewest dependent products, then the smallest.
__device__ int ks_block_size(int deg) {
  if (deg < 1) return 1;
  int sb = 1, best = 1 << 30;
  for (int cand = 1; cand <= 8; ++cand) {
    int lg = 0;
    while ((1 << lg) < cand) ++lg;
    const int cost = lg + deg / cand;
    if (cost < best) { best = cost; sb = cand; }
  }
  if (deg / sb > 7) sb = 8;  // at most 8 blocks B_0..B_7
  return sb;
}

__device__ __forceinline__ void kn_cluster_body(const KnStep &a, const KnSeries &ser, bool full = false) {
  extern __shared__ double sm[];
  __shared__ double red[kKsThreads / 32];
  __shared__ int plan[3];  // degree (-1: Newton-Schulz), block size, Newton-Schulz steps
  cg::cluster_group cluster = cg::this_cluster();
  const int l = a.l;
  const size_t ll = (size_t)l * l;
  Ks k{l, (l + 31) / 32, (int)cluster.num_blocks(), (int)cluster.block_rank(), sm, sm + 32 * kAld,
         sm + 32 * kAld + (kKsMaxL + 4) * kBld, false, kAld, kBld};
  if (full) {  // the whole-operand layout (the launch sized the dynamic shared memory for it)
    k.full = true;
    k.ald = k.bld = ks_full_ld(l);
    k.As = sm;
    k.Bs = sm + (size_t)((l + 31) / 32 * 32) * k.ald;
    k.part = k.Bs + (size_t)((l + 3) & ~3) * k.bld;
  }
  const int nt = k.nr * k.nr;
  const int gtid = k.rank * kKsThreads + threadIdx.x, gstride = k.cs * kKsThreads;
  // work: Z | P_1..P_8 | accC x2 | accCi x2 | BC_0..BC_7 | BI_0..BI_7 (Newton-Schulz: P_1..P_5), then
  // partial sums of the cluster reductions (3 x 16 slots)
  double *Zm = a.work, *P = Zm + ll, *AC = P + 8 * ll, *AI = AC + 2 * ll, *BC = AI + 2 * ll, *BI = BC + 8 * ll;
  double *slots = a.work + (size_t)kKnWorkMatrices * ll;

  ks_mm(k, 0, nt, -1.0, a.Dc, a.Dc, 1.0, a.Dgc, 0.0, Zm);  // Z = Dgc - Dc Dc (:184-190)
  cluster.sync();
  // P_1 = Zsym from the upper triangle (as syev 'U' reads Z); rho = ||4 Zsym||_F >= ||4 Z||_2
  double f = 0.0;
  for (int e = gtid; e < (int)ll; e += gstride) {
    const int i = e / l, j = e - i * l;
    const double z = __ldcg(Zm + (size_t)min(i, j) * l + max(i, j));
    P[e] = z;
    f += 16.0 * z * z;
  }
  const double rho = sqrt(ks_cluster_sum(k, cluster, f, slots, red));
  if (threadIdx.x < 32) {
    const int d = ks_degree_warp(ser, rho, a.ns_target);
    if (threadIdx.x == 0) {
      plan[0] = d;
      plan[1] = ks_block_size(d);
      plan[2] = d < 0 ? kn_ns_steps(rho, a.ns_target) : 0;
    }
  }
  __syncthreads();
  const int deg = plan[0];
  const double *C, *Ci;
  if (deg >= 0) {
    const int sb = plan[1];
    for (int h = 1; h < sb; h *= 2) {  // P_j = P_h P_(j-h), h < j <= min(2h, sb)
      const int hi = min(2 * h, sb);
      for (int j = h + 1; j <= hi; ++j) {
        const int slot = j - h - 1;
        ks_mm(k, slot * nt, (slot + 1) * nt, 1.0, P + (h - 1) * ll, P + (j - h - 1) * ll, 0.0, nullptr, 0.0,
              P + (j - 1) * ll);
      }
      cluster.sync();
    }
    // Paterson-Stockmeyer: B_b = sum_{t<sb} coef[b sb + t] Z^t (b = 0..q); acc = B_q; acc = acc Z^sb + B_b
    const int q = deg / sb;
    for (int e = gtid; e < (int)ll; e += gstride) {
      const int i = e / l, j = e - i * l;
      for (int b = 0; b <= q; ++b) {
        double vc = (i == j) ? ser.c[b * sb] : 0.0, vd = (i == j) ? ser.d[b * sb] : 0.0;
        for (int t = 1; t < sb && b * sb + t <= deg; ++t) {
          const double p = __ldcg(P + (t - 1) * ll + e);
          vc += ser.c[b * sb + t] * p;
          vd += ser.d[b * sb + t] * p;
        }
        BC[b * ll + e] = vc;
        BI[b * ll + e] = vd;
      }
    }
    cluster.sync();
    const double *accC = BC + q * ll, *accI = BI + q * ll;
    int cur = 0;
    for (int b = q - 1; b >= 0; --b) {
      ks_mm(k, 0, nt, 1.0, accC, P + (sb - 1) * ll, 1.0, BC + b * ll, 0.0, AC + cur * ll);
      ks_mm(k, nt, 2 * nt, 1.0, accI, P + (sb - 1) * ll, 1.0, BI + b * ll, 0.0, AI + cur * ll);
      cluster.sync();
      accC = AC + cur * ll;
      accI = AI + cur * ll;
      cur = 1 - cur;
    }
    C = accC;
    Ci = accI;
  } else {
    // Two coupled Newton-Schulz square roots (Higham, Functions of Matrices, eq. 6.35):
    //   T = Q Y;  Y <- Y (3I - T)/2;  Q <- (3I - T) Q / 2   ->  Y -> X^(1/2), Q -> X^(-1/2),
    // first of X = I - 4 Zsym (sqrt(I/4 - Z) = Y/2), then of P = I/2 + Y/2.
    double *Y = P, *Yn = P + ll, *Q = P + 2 * ll, *Qn = P + 3 * ll, *T = P + 4 * ll;
    for (int e = gtid; e < (int)ll; e += gstride) {
      const int i = e / l, j = e - i * l;
      Y[e] = (i == j ? 1.0 : 0.0) - 4.0 * __ldcg(P + e);  // Y is P_1: each entry read, then written
      Q[e] = (i == j ? 1.0 : 0.0);
    }
    cluster.sync();
    int steps = plan[2];
    for (int stage = 0; stage < 2; ++stage) {
      for (int it = 0; it < steps; ++it) {
        ks_mm(k, 0, nt, 1.0, Q, Y, 0.0, nullptr, 0.0, T);
        cluster.sync();
        ks_mm(k, 0, nt, -0.5, Y, T, 1.5, Y, 0.0, Yn);
        ks_mm(k, nt, 2 * nt, -0.5, T, Q, 1.5, Q, 0.0, Qn);
        cluster.sync();
        double *t1 = Y; Y = Yn; Yn = t1;
        double *t2 = Q; Q = Qn; Qn = t2;
      }
      if (stage == 0) {
        double d2 = 0.0;
        for (int e = gtid; e < (int)ll; e += gstride) {
          const int i = e / l, j = e - i * l;
          const double pv = 0.5 * __ldcg(Y + e) + (i == j ? 0.5 : 0.0);
          Yn[e] = pv;
          Qn[e] = (i == j ? 1.0 : 0.0);
          const double d = (i == j ? 1.0 : 0.0) - pv;
          d2 += d * d;
        }
        steps = kn_ns_steps(fmin(sqrt(ks_cluster_sum(k, cluster, d2, slots + 16, red)), 0.5), a.ns_target);
        double *t1 = Y; Y = Yn; Yn = t1;
        double *t2 = Q; Q = Qn; Qn = t2;
      }
    }
    C = Y;
    Ci = Q;
  }
  // C, C^-1, F = C - Dc C^-1 (:218), the stacked copies, err = ||C - I||_F (:230-234)
  double e2 = 0.0;
  for (int e = gtid; e < (int)ll; e += gstride) {
    const int i = e / l, j = e - i * l;
    const double cv = __ldcg(C + e), ci = __ldcg(Ci + e);
    a.C[e] = cv;
    a.Cinv[e] = ci;
    if (a.fstack) {
      a.fstack[ll + e] = a.fstack_scale * ci;
      a.fstack[3 * ll + e] = ci;
    }
    const double d = cv - (i == j ? 1.0 : 0.0);
    e2 += d * d;
  }
  // F once, written to F and to both F slots of the stack
  ks_mm(k, 0, nt, -1.0, a.Dc, Ci, 1.0, C, 0.0, a.F, a.fstack, a.fstack ? a.fstack + 2 * ll : nullptr);
  const double err = sqrt(ks_cluster_sum(k, cluster, e2, slots + 32, red));
  if (k.rank == 0 && threadIdx.x == 0) {
    *a.err = err;
    if (!(err == err)) atomicExch(a.status, kErrNumerical);
  }
}

__global__ void __launch_bounds__(kKsThreads, 1) kn_cluster_kernel(KnStep a, KnSeries ser) { kn_cluster_body(a, ser); }

// One cluster per step of steps[] (grid = count x cluster size): many independent problems.
// full: one-CTA clusters with the whole-operand product layout (every l <= kKsFullL).
__global__ void __launch_bounds__(kKsThreads, 1) kn_cluster_grouped_kernel(const KnStep *steps, KnSeries ser,
                                                                         int full) {
  const KnStep a = steps[blockIdx.x / cg::this_cluster().num_blocks()];
  kn_cluster_body(a, ser, full != 0);
}

// Coefficients of g(z)^(1/2) and g(z)^(-1/2), g(z) = 1 - sum_{n>=1} Cat(n-1) z^n: for h = f^alpha
// with f_0 = 1, h_0 = 1 and h_n = (1/n) sum_{k=1..n} (alpha k - (n - k)) f_k h_(n-k).
KnSeries make_series() {
  KnSeries s;
  double f[kSeriesLen], cat = 1.0;  // Cat(0) = 1, Cat(n) = Cat(n-1) 2 (2n - 1) / (n + 1)
  f[0] = 1.0;
  for (int n = 1; n < kSeriesLen; ++n) {
    f[n] = -cat;
    cat = cat * 2.0 * (2.0 * n - 1.0) / (n + 1.0);
  }
  const double alpha[2] = {0.5, -0.5};
  double *out[2] = {s.c, s.d};
  for (int w = 0; w < 2; ++w) {
    double *h = out[w];
    h[0] = 1.0;
    for (int n = 1; n < kSeriesLen; ++n) {
      double acc = 0.0;
      for (int kk = 1; kk <= n; ++kk) acc += (alpha[w] * kk - (n - kk)) * f[kk] * h[n - kk];
      h[n] = acc / n;
    }
  }
  return s;
}

constexpr size_t kKsSmem = (size_t)(32 * kAld + (kKsMaxL + 4) * kBld + 4 * 1024) * sizeof(double);
int g_cluster_size = -1;  // -1: not decided yet; 0: no cluster launch possible

int choose_cluster_size(const KnStep &a, cudaStream_t st) {
  if (g_cluster_size >= 0) return g_cluster_size;
  CK(cudaFuncSetAttribute(kn_cluster_kernel, cudaFuncAttributeNonPortableClusterSizeAllowed, 1));
  CK(cudaFuncSetAttribute(kn_cluster_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kKsSmem));
  g_cluster_size = 0;
  for (int cs = 16; cs >= 2; cs /= 2) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(cs);
    cfg.blockDim = dim3(kKsThreads);
    cfg.dynamicSmemBytes = kKsSmem;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = cs;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    int n = 0;
    const cudaError_t e = cudaOccupancyMaxActiveClusters(&n, kn_cluster_kernel, &cfg);
    if (e != cudaSuccess) {
      cudaGetLastError();
      continue;
    }
    if (n >= 1) {
      g_cluster_size = cs;
      break;
    }
  }
  (void)a;
  return g_cluster_size;
}

}  // namespace

void kn_step_grouped(const KnStep *steps, int count, int max_l, int cluster, cudaStream_t st) {
  if (count <= 0) return;
  if (max_l > kKsMaxL) fail(kErrUnsupported, "Kolmogorov-Nagumo step: l = %d > %d", max_l, kKsMaxL);
  KnStep probe;
  probe.l = max_l;
  int cs = choose_cluster_size(probe, st);
  if (cs == 0) fail(kErrUnsupported, "grouped Kolmogorov-Nagumo step: no thread-block cluster launch on this device");
  const size_t smem_max = std::max(kKsSmem, ks_full_smem(kKsFullL));
  static bool attr = false;
  if (!attr) {
    CK(cudaFuncSetAttribute(kn_cluster_grouped_kernel, cudaFuncAttributeNonPortableClusterSizeAllowed, 1));
    CK(cudaFuncSetAttribute(kn_cluster_grouped_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_max));
    attr = true;
  }
  // many clusters run side by side: `cluster` CTAs each (default eight)
  cs = std::min(cs, cluster > 0 ? cluster : 8);
  const int full = (cs == 1 && max_l <= kKsFullL) ? 1 : 0;
  static const KnSeries series = make_series();
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(count * cs);
  cfg.blockDim = dim3(kKsThreads);
  cfg.dynamicSmemBytes = full ? std::max(kKsSmem, ks_full_smem(max_l)) : kKsSmem;
  cfg.stream = st;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeClusterDimension;
  at[0].val.clusterDim.x = cs;
  at[0].val.clusterDim.y = 1;
  at[0].val.clusterDim.z = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  CK(cudaLaunchKernelEx(&cfg, kn_cluster_grouped_kernel, steps, series, full));
  KLAUNCHED();
}

void kn_step(const KnStep &a, cudaStream_t st) {
  if (a.l > kKsMaxL) fail(kErrUnsupported, "Kolmogorov-Nagumo step: l = %d > %d", a.l, kKsMaxL);
  const int cs = choose_cluster_size(a, st);
  if (cs == 0) {  // no cluster launch on this device: the grid-barrier kernel (work 8 l^2 + 64 fits)
    CK(cudaMemsetAsync(a.bar, 0, 8, st));  // its barrier counters
    kn_step_fixed(a, Runtime::get().num_sms, st);
    return;
  }
  static const KnSeries series = make_series();
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(cs);
  cfg.blockDim = dim3(kKsThreads);
  cfg.dynamicSmemBytes = kKsSmem;
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = cs;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  CK(cudaLaunchKernelEx(&cfg, kn_cluster_kernel, a, series));
  KLAUNCHED();
}

}  // namespace isvdb
