// MIXED precision stages: bf16 planes + tcgen05 (umma.h) for the products whose cost scales with
// the large dimensions; FP64 for every l x l step (done by the callers in stages.cu).
//
// Plane counts per product (relative error of one product term, before FP32 accumulation):
//   sketch       A: 2 planes (16 significant bits; ISVD_GPU_SKETCH_PLANES=3 keeps FP32 A exact)
//                x  Omega: 1 exact bf16 plane, or 3 when passed in.  Two planes leave a relative
//                error of at most 2^-17 per element of A (TF32 keeps 2^-11); its effect on each
//                entry of Y = A Omega averages over the n-long inner products to about that of an
//                FP32 GEMM's own rounding at n ~ 1e4, and the sketch only fixes the subspace, whose
//                Rayleigh-Ritz values (the postprocess) move by the square of a subspace
//                perturbation.
//   block Gram   Y': 3 x 3 planes, 6 products  (W feeds the orthogonalizing eigensolve)
//   G = Qs' Qs   2 x 2 planes, 3 products      (errors average over the m-long inner products)
//   Z = A' Qbar  Qbar': 2 planes x A: 2 planes, 3 products
#include <algorithm>
#include <cstdlib>

#include "kernels.h"
#include "mixed.h"
#include "panels.h"
#include "runtime.h"

namespace isvdb {
template <class T>
void make_planes(PlaneBuf &pb, const T *src, long long s_rs, long long rows, long long cols, int np, bool transpose,
                 cudaStream_t st) {
  const long long orows = transpose ? cols : rows, ocols = transpose ? rows : cols;
  const long long ld = plane_ld(ocols), rp = plane_rows(orows), ps = rp * ld;
  pb.buf.ensure((size_t)np * ps);
  split_planes<T>(src, s_rs, 1, rows, cols, np, transpose, pb.buf.p, ld, ps, st);
  pb.P.ptr = pb.buf.p;
  pb.P.np = np;
  pb.P.rows = orows;
  pb.P.cols = ocols;
  pb.P.ld = ld;
  pb.P.plane_stride = ps;
  pb.P.mn_major = false;
}
template void make_planes<float>(PlaneBuf &, const float *, long long, long long, long long, int, bool, cudaStream_t);
template void make_planes<double>(PlaneBuf &, const double *, long long, long long, long long, int, bool,
                                  cudaStream_t);

namespace {

void set_products(UmmaGemm &g, int na, int nb) {
  // keep (p, q) with p + q < max(na, nb): the terms above the FP32 rounding level
  const int order = (na > nb ? na : nb);
  g.nprod = 0;
  for (int s = 0; s < order; ++s)
    for (int p = 0; p <= s; ++p) {
      const int q = s - p;
      if (p < na && q < nb) { g.pa[g.nprod] = p; g.pb[g.nprod] = q; ++g.nprod; }
    }
}

template <class T>
constexpr bool is_double() { return sizeof(T) == 8; }

}  // namespace

// Rows per streamed panel of A: about 1 GiB of A, a multiple of 128 rows (environment override
// ISVD_GPU_PANEL_ROWS, rounded to 128).
static long long panel_rows(long long m, long long n, size_t elem) {
  long long p = (long long)((1ll << 30) / ((long long)n * (long long)elem));
  if (const char *e = getenv("ISVD_GPU_PANEL_ROWS")) p = atoll(e);
  p = std::max<long long>(128, p / 128 * 128);
  return std::min<long long>(p, m);
}

// bf16 planes of A used by the sketch (2, or 3 with ISVD_GPU_SKETCH_PLANES=3); the postprocess
// reads the first two.
int sketch_planes() {
  static const int np = [] {
    const char *e = getenv("ISVD_GPU_SKETCH_PLANES");
    return (e && atoi(e) == 3) ? 3 : 2;
  }();
  return np;
}

// Tile order of the sketch GEMM.  Every CTA runs the whole K = n, so the CTAs resident at one time
// read all of Omega' that their N tiles cover.  When Omega' (Nl x n bf16 planes) is larger than L2,
// the tiles run in two column groups (each group's M tiles one after the other), so that the
// resident CTAs share half of Omega' and A is read twice.  Measured on the 200000 x 20000 x 4096
// sketch (164 MB of Omega'): two groups of eight 256-wide N tiles cut the DRAM reads by 12 % and
// the kernel time by about 2 % against the row-major order; four groups (A read four times) gain
// less, eight lose 5 %, and the L2 evict-last policy on Omega' gains nothing.
// ISVD_GPU_SKETCH_NGROUP overrides the group width (0: row-major order), ISVD_GPU_SKETCH_L2HINT=1
// adds the evict-last / evict-first policies.
static void sketch_tile_order(UmmaGemm &g, long long n, long long Nl, int bn) {
  static const long long l2 = [] {
    int dev = 0, v = 0;
    CK(cudaGetDevice(&dev));
    CK(cudaDeviceGetAttribute(&v, cudaDevAttrL2CacheSize, dev));
    return (long long)v;
  }();
  const long long gx = (Nl + bn - 1) / bn;
  const long long bbytes = Nl * n * 2LL * g.B.np;
  g.n_group = (l2 > 0 && bbytes > l2 && gx > 1) ? (int)((gx + 1) / 2) : 0;
  const char *e = getenv("ISVD_GPU_SKETCH_NGROUP");
  if (e) g.n_group = std::max(0, atoi(e));
  e = getenv("ISVD_GPU_SKETCH_L2HINT");
  g.l2_hint = e && atoi(e) == 1;
}

// Sketch Y = A Omega with A processed in row panels: each panel is split into A's bf16 planes
// (kept for the postprocess) and multiplied by Omega' on the tensor cores.  When A is in host
// memory, panel p + 1 is copied to the device on the copy stream while panel p is split and
// multiplied, so that the PCIe transfer overlaps the tensor-core work (the reference streams A in
// column panels through the GPU for the same reason, gpu/stage/@x@_sketch_gpu.h:238-254).  The
// FP32 A is never resident on the device in this mode.  Out of core (c.a_panel_rows > 0, host A):
// only one panel's planes exist at a time and none are kept; the projection streams A again.
template <class T>
void mixed_sketch(const StageCtx &c, int m, int n, int Nl, char ordera, const T *a, long long lda, const T *omega,
                  long long ldom, uint64_t seed, T *y, long long ldy, PlaneHandoff *hand) {
  if (hand && !handoff_shape_ok(Nl)) hand = nullptr;
  if (hand) hand->prepare(y, ldy, m, Nl, c.st);
  const bool a_dev = is_device_pointer(a);
  const bool ooc = !a_dev && c.a_panel_rows > 0;
  const long long P = ooc ? c.a_panel_rows : panel_rows(m, n, sizeof(T));
  const long long held = ooc ? P : m;  // rows of planes held at once
  const long long ld = plane_ld(n), rp = plane_rows(held), ps = rp * ld;
  MixedCache local;
  MixedCache *mc = (c.cache && !ooc) ? c.cache : &local;
  if (ooc && c.cache) {
    c.cache->buf.release();
    c.cache->src = nullptr;
  }
  const int na = sketch_planes();
  mc->buf.alloc((size_t)na * ps);
  auto zero_rows_from = [&](long long r) {  // TMA boxes of the last tile read rows [r, rp)
    for (int q = 0; q < na; ++q)
      if (rp > r)
        CK(cudaMemsetAsync(mc->buf.p + (size_t)q * ps + (size_t)r * ld, 0, (size_t)(rp - r) * ld * 2, c.st));
  };
  zero_rows_from(held);
  Planes all;
  all.ptr = mc->buf.p; all.np = na; all.rows = m; all.cols = n; all.ld = ld; all.plane_stride = ps;
  PlaneBuf om;
  if (!omega) {
    const long long old = plane_ld(n), orp = plane_rows(Nl);
    om.buf.alloc((size_t)orp * old);
    rng_gaussian_bf16_t(om.buf.p, n, Nl, old, orp, seed, c.st, c.col_begin * (long long)Nl);
    om.P.ptr = om.buf.p; om.P.np = 1; om.P.rows = Nl; om.P.cols = n; om.P.ld = old; om.P.plane_stride = orp * old;
  } else {
    make_planes<T>(om, omega, ldom, n, Nl, 3, true, c.st);  // Omega' planes (Nl x n)
  }
  UmmaGemm g;
  g.N = Nl; g.K = n;
  g.B = om.P;
  set_products(g, na, om.P.np);
  g.c_double = is_double<T>(); g.c_rs = ldy; g.c_cs = 1;
  g.status = c.status;
  g.chunk_k = 512;  // 5e-7 relative tensor-core chain error per chunk, below the 2^-17 split level
  g.tag = "sketch";
  sketch_tile_order(g, n, Nl, Nl > 128 ? 256 : 128);
  if (hand) { g.p_ld = hand->pb.P.ld; g.p_ps = hand->pb.P.plane_stride; }
  if (a_dev) {
    // A on the device: split every row, then one launch over all m rows (no per-panel wave tail)
    for (long long r0 = 0; r0 < m; r0 += P) {
      const long long rows = std::min<long long>(P, m - r0);
      __nv_bfloat16 *dst = mc->buf.p + (size_t)r0 * ld;
      if (ordera == 'R') split_rows<T>(a + r0 * lda, lda, 1, rows, n, na, false, dst, ld, ps, c.st);
      else split_rows<T>(a + r0, lda, 1, n, rows, na, true, dst, ld, ps, c.st);  // A' rows r0.. as n x rows
    }
    g.M = m;
    g.A = all;
    g.C = hand ? nullptr : y;
    if (hand) g.planes = hand->pb.buf.p;
    umma_gemm(g, c.st);
  } else {
    // A in host memory: panel p + 1 is copied while panel p is split and multiplied
    for_each_host_panel<T>(c, a, lda, ordera, m, n, P, [&](long long r0, long long rows, const T *ap, long long ldp) {
      __nv_bfloat16 *dst = ooc ? mc->buf.p : mc->buf.p + (size_t)r0 * ld;
      if (ooc && rows < P) zero_rows_from(rows);  // the last panel: rows of the previous one
      if (ordera == 'R') split_rows<T>(ap, ldp, 1, rows, n, na, false, dst, ld, ps, c.st);
      else split_rows<T>(ap, ldp, 1, n, rows, na, true, dst, ld, ps, c.st);
      Planes pp = all;
      pp.ptr = dst;
      pp.rows = rows;
      g.M = (int)rows;
      g.A = pp;
      g.C = hand ? nullptr : y + r0 * ldy;
      if (hand) g.planes = hand->pb.buf.p + (size_t)r0 * hand->pb.P.ld;
      umma_gemm(g, c.st);
    });
  }
  if (!ooc) {
    mc->src = a; mc->m = m; mc->n = n; mc->ordera = ordera;
    mc->A = all;
  }
}

template <class T>
void mixed_block_gram(const StageCtx &c, const Planes &yp, int m, int l, int N, const T *y, long long ldy,
                      double *W) {
  UmmaGemm g;
  g.M = l; g.N = l; g.K = m;
  if (l % 8 == 0) {
    Planes a = yp;
    a.mn_major = true;  // stored m x Nl: as the l x m operand Y_i' it is MN-major
    g.A = a; g.B = a;
    set_products(g, a.np, a.np);
    g.batch = N; g.a_mn_step = l; g.b_mn_step = l; g.c_step = (long long)l * l;
    g.C = W; g.c_double = true; g.c_rs = l; g.c_cs = 1;
    g.status = c.status;
  g.tag = "block_gram";
    umma_gemm(g, c.st);
    return;
  }
  PlaneBuf yt;
  make_planes<T>(yt, y, ldy, m, (long long)N * l, 3, true, c.st);  // Y' planes (Nl x m)
  g.A = yt.P; g.B = yt.P;
  set_products(g, 3, 3);
  g.batch = N; g.a_mn_step = l; g.b_mn_step = l; g.c_step = (long long)l * l;
  g.C = W; g.c_double = true; g.c_rs = l; g.c_cs = 1;
  g.status = c.status;
  g.tag = "block_gram";
  umma_gemm(g, c.st);
}

template <class T>
void mixed_block_apply(const StageCtx &c, const Planes &yp, int m, int l, int N, const T *y, long long ldy,
                       const T *Wp, T *out, long long ldo, PlaneHandoff *hand) {
  if (hand && l % 64 != 0) fail(kErrUnsupported, "plane hand-off of the block applies needs l %% 64 == 0");
  if (l % 64 == 0) {
    PlaneBuf wt;
    make_planes<T>(wt, Wp, l, (long long)N * l, l, 3, true, c.st);  // [Wp_0' .. Wp_N-1'] (l x Nl)
    UmmaGemm g;
    g.M = m; g.N = l; g.K = l;
    g.A = yp; g.B = wt.P;
    set_products(g, yp.np, 3);
    g.batch = N; g.a_k_step = l; g.b_k_step = l; g.c_step = l;
    g.C = out; g.c_double = is_double<T>(); g.c_rs = ldo; g.c_cs = 1;
    g.status = c.status;
    g.tag = "block_apply";
    if (hand) {
      const bool in_place = hand->of && yp.ptr == hand->pb.buf.p;
      if (!in_place) hand->prepare(out, ldo, m, (long long)N * l, c.st);
      g.C = nullptr;
      g.planes = hand->pb.buf.p; g.p_ld = hand->pb.P.ld; g.p_ps = hand->pb.P.plane_stride;
      g.planes_in_place = in_place;
      hand->of = out;
      hand->ld_of = ldo;
    }
    umma_gemm(g, c.st);
    return;
  }
  Gemm<T, T> g;
  g.M = m; g.N = l; g.K = l; g.batch = N;
  g.A = y; g.a_rs = ldy; g.a_cs = 1; g.a_bs = l;
  g.B = Wp; g.b_rs = l; g.b_cs = 1; g.b_bs = (long long)l * l;
  g.C = out; g.c_rs = ldo; g.c_cs = 1; g.c_bs = l;
  gemm(g, c.st);
}

template <class T>
void mixed_gram_full(const StageCtx &c, const Planes &qp, int m, int Nl, const T *qs, long long ldq, double *G,
                     int np, bool all_pairs) {
  UmmaGemm g;
  g.M = Nl; g.N = Nl; g.K = m;
  PlaneBuf qt;
  if (Nl % 8 == 0) {
    Planes a = qp;
    a.np = np;
    a.mn_major = true;
    g.A = a; g.B = a;
  } else {
    make_planes<T>(qt, qs, ldq, m, Nl, np, true, c.st);  // Qs' planes (Nl x m)
    g.A = qt.P; g.B = qt.P;
  }
  set_products(g, np, np);
  if (all_pairs) {
    g.nprod = 0;
    for (int p = 0; p < np; ++p)
      for (int q = 0; q < np; ++q) { g.pa[g.nprod] = p; g.pb[g.nprod] = q; ++g.nprod; }
  }
  g.C = G; g.c_double = true; g.c_rs = Nl; g.c_cs = 1;
  g.upper = true;
  g.status = c.status;
  g.tag = "gram_full";
  umma_gemm(g, c.st);
  mirror_upper(G, Nl, Nl, c.st);
}

template <class T>
void mixed_apply_coeff(const StageCtx &c, const Planes &qp, int m, int Nl, int l, const T *qs, long long ldq,
                       const double *M, T *qt, long long ldqt) {
  (void)qs; (void)ldq;
  PlaneBuf mt;
  make_planes<double>(mt, M, l, Nl, l, 3, true, c.st);  // M' planes (l x Nl)
  UmmaGemm g;
  g.M = m; g.N = l; g.K = Nl;
  g.A = qp; g.B = mt.P;
  set_products(g, qp.np, 3);
  g.C = qt; g.c_double = is_double<T>(); g.c_rs = ldqt; g.c_cs = 1;
  g.status = c.status;
  g.tag = "coeff_apply";
  umma_gemm(g, c.st);
}

// Out-of-core projection: Z = sum over row panels of A_p' Qbar_p, each panel of the host A split
// into two bf16 planes on arrival and multiplied on the tensor cores, the panel sums added in FP64.
template <class T>
void mixed_project_streamed(const StageCtx &c, int m, int n, int l, char ordera, const T *a, long long lda,
                            const T *qt, long long ldqt, T *z) {
  const long long P = c.a_panel_rows, ld = plane_ld(n), rp = plane_rows(P), ps = rp * ld;
  DBuf<__nv_bfloat16> pl((size_t)2 * ps);
  auto zero_rows_from = [&](long long r) {
    for (int q = 0; q < 2; ++q)
      if (rp > r) CK(cudaMemsetAsync(pl.p + (size_t)q * ps + (size_t)r * ld, 0, (size_t)(rp - r) * ld * 2, c.st));
  };
  zero_rows_from(P);
  DBuf<double> zacc((size_t)n * l), zp((size_t)n * l);
  for_each_host_panel<T>(c, a, lda, ordera, m, n, P, [&](long long r0, long long rows, const T *ap, long long ldp) {
    if (rows < P) zero_rows_from(rows);
    if (ordera == 'R') split_rows<T>(ap, ldp, 1, rows, n, 2, false, pl.p, ld, ps, c.st);
    else split_rows<T>(ap, ldp, 1, n, rows, 2, true, pl.p, ld, ps, c.st);
    PlaneBuf qp;
    make_planes<T>(qp, qt + r0 * ldqt, ldqt, rows, l, 2, true, c.st);  // Qbar_p' planes (l x rows)
    Planes b;  // the panel's planes, rows x n (n contiguous): as the N x K = n x rows operand, MN-major
    b.ptr = pl.p; b.np = 2; b.rows = rows; b.cols = n; b.ld = ld; b.plane_stride = ps; b.mn_major = true;
    UmmaGemm g;
    g.M = l; g.N = n; g.K = (int)rows;
    g.A = qp.P; g.B = b;
    set_products(g, 2, 2);
    g.C = r0 == 0 ? zacc.p : zp.p; g.c_double = true; g.c_rs = 1; g.c_cs = l;
    g.status = c.status;
    g.tag = "project";
    umma_gemm(g, c.st);
    if (r0 > 0) lincomb(zacc.p, zacc.p, 1.0, zp.p, 1.0, 0.0, n, l, c.st);
  });
  copy2d<double, T>(zacc.p, l, 1, z, l, 1, n, l, c.st);
}

template <class T>
void mixed_project(const StageCtx &c, int m, int n, int l, char ordera, const T *a, long long lda, const T *qt,
                   long long ldqt, T *z) {
  PlaneBuf qp;
  make_planes<T>(qp, qt, ldqt, m, l, 2, true, c.st);  // Qbar' planes (l x m)
  PlaneBuf local;
  Planes ap;
  MixedCache *mc = c.cache;
  if (mc && mc->src == a && mc->m == m && mc->n == n && mc->ordera == ordera && mc->buf.p) {
    ap = mc->A;
  } else if (!is_device_pointer(a) && c.a_panel_rows > 0) {
    mixed_project_streamed<T>(c, m, n, l, ordera, a, lda, qt, ldqt, z);
    return;
  } else {
    if (!is_device_pointer(a)) fail(kErrArgument, "mixed postprocess: A is not on the device and not cached");
    if (ordera == 'R') make_planes<T>(local, a, lda, m, n, 2, false, c.st);
    else make_planes<T>(local, a, lda, n, m, 2, true, c.st);
    ap = local.P;
  }
  // A planes are stored m x n (n contiguous): as the N x K = n x m operand they are MN-major.
  Planes b = ap;
  b.np = 2;
  b.mn_major = true;
  UmmaGemm g;
  g.M = l; g.N = n; g.K = m;
  g.A = qp.P; g.B = b;
  set_products(g, 2, 2);
  g.C = z; g.c_double = is_double<T>(); g.c_rs = 1; g.c_cs = l;  // Z' tile written into Z (n x l)
  g.status = c.status;
  g.tag = "project";
  umma_gemm(g, c.st);
}

void MixedGProduct::prepare(const StageCtx &c, int Nl_, const double *G) {
  Nl = Nl_;
  make_planes<double>(g, G, Nl, Nl, Nl, 3, false, c.st);  // G is symmetric: rows (M) x K
}

void MixedGProduct::apply(const StageCtx &c, int l, const double *Bc, long long ldb, double alpha, double *Bgc,
                          long long ldo, bool split) {
  if (split) make_planes<double>(b, Bc, ldb, Nl, l, 3, true, c.st);  // Bc' planes (l x Nl): N x K
  else if (!b.buf.p || b.P.rows != l || b.P.cols != Nl) fail(kErrArgument, "KN G product: Bc planes not prepared");
  UmmaGemm gg;
  gg.M = Nl; gg.N = l; gg.K = Nl;
  gg.A = g.P; gg.B = b.P;
  set_products(gg, 3, 3);
  gg.C = Bgc; gg.c_double = true; gg.c_rs = ldo; gg.c_cs = 1;
  gg.alpha = alpha;
  gg.status = c.status;
  gg.tag = "kn_product";
  // G's planes (3 Nl^2 bf16) are read again by every iteration: evict-last keeps them in L2 when
  // they fit (ISVD_GPU_KN_L2KEEP=0: default policy)
  static const long long l2 = [] {
    int dev = 0, v = 0;
    CK(cudaGetDevice(&dev));
    CK(cudaDeviceGetAttribute(&v, cudaDevAttrL2CacheSize, dev));
    return (long long)v;
  }();
  gg.a_keep = 3LL * Nl * Nl * 2 <= l2 * 85 / 100 && [] {
    const char *e = getenv("ISVD_GPU_KN_L2KEEP");
    return !(e && atoi(e) == 0);
  }();
  umma_gemm(gg, c.st);
}

void PlaneHandoff::prepare(const void *p, long long ld, long long rows, long long cols, cudaStream_t st) {
  const long long pld = plane_ld(cols), rp = plane_rows(rows), ps = rp * pld;
  pb.buf.ensure((size_t)3 * ps);
  for (int q = 0; q < 3; ++q) {  // padding rows and columns: zero (TMA boxes of the last tiles read them)
    __nv_bfloat16 *pl = pb.buf.p + (size_t)q * ps;
    if (rp > rows) CK(cudaMemsetAsync(pl + (size_t)rows * pld, 0, (size_t)(rp - rows) * pld * 2, st));
    if (pld > cols) CK(cudaMemset2DAsync(pl + cols, pld * 2, 0, (pld - cols) * 2, rows, st));
  }
  pb.P.ptr = pb.buf.p; pb.P.np = 3; pb.P.rows = rows; pb.P.cols = cols; pb.P.ld = pld; pb.P.plane_stride = ps;
  pb.P.mn_major = false;
  of = p;
  ld_of = ld;
}

#define ISVD_INST(T)                                                                                        \
  template void mixed_sketch<T>(const StageCtx &, int, int, int, char, const T *, long long, const T *,      \
                                long long, uint64_t, T *, long long, PlaneHandoff *);                      \
  template void mixed_block_gram<T>(const StageCtx &, const Planes &, int, int, int, const T *, long long,    \
                                    double *);                                                             \
  template void mixed_block_apply<T>(const StageCtx &, const Planes &, int, int, int, const T *, long long,   \
                                     const T *, T *, long long, PlaneHandoff *);                           \
  template void mixed_gram_full<T>(const StageCtx &, const Planes &, int, int, const T *, long long,          \
                                   double *, int, bool);                                                        \
  template void mixed_apply_coeff<T>(const StageCtx &, const Planes &, int, int, int, const T *, long long,   \
                                     const double *, T *, long long);                                      \
  template void mixed_project<T>(const StageCtx &, int, int, int, char, const T *, long long, const T *,     \
                                 long long, T *);
ISVD_INST(float)
ISVD_INST(double)

}  // namespace isvdb
