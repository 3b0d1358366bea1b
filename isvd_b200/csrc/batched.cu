// Batched iSVD: many independent matrices of uneven sizes and ranks (GP / GR / KN / GR, one MPI
// rank, products in the matrices' own type, FP64 l x l steps).
//
// Every stage runs as grouped launches over all matrices instead of one launch per matrix:
//   * products: one persistent GEMM kernel walks a list of (product, output tile) work items --
//     the sketches, Gram matrices, applies, G = Qs'Qs products and Kolmogorov-Nagumo coefficient
//     products of every matrix in one launch; FP64 lists on the FP64 tensor cores (k_dmma.cu),
//     the others on CUDA cores.  Its tile shape is chosen per product list by measurement on first
//     use (the fastest candidate is kept and remembered by a signature of the list);
//   * orthogonalization: block i of a matrix is Q_i = Y_i R_i^-1 with Y_i' Y_i = R_i' R_i (grouped
//     Cholesky, one CTA per block), where the reference's Gramian orthogonalization takes the
//     eigenbasis, Q_i = Y_i V_i S_i^-1.  The two bases span the same space and differ by an
//     orthogonal l x l factor; the Kolmogorov-Nagumo iteration only sees the projectors Q_i Q_i'
//     and the starting block Q_1 (whose rotation rotates every iterate alike, leaving the error
//     norm, the iteration count and the postprocessed U, s, V unchanged), so the results are those
//     of single solves to rounding, at a fraction of the eigensolves' cost;
//   * small dense steps: the Jacobi eigensolver with one CTA per l x l matrix of its own size
//     (postprocessing), and the Kolmogorov-Nagumo step with one thread-block cluster per matrix;
//   * the Kolmogorov-Nagumo iterations of all matrices advance together; a matrix leaves the
//     active set at its own convergence test, so its iteration count and error are those of a
//     single solve.
// A plan holds the workspace and the device-side work lists of one batch shape.  The work before
// and after the iterations is captured as two CUDA graphs on the second solve with the same
// buffers (the first one runs eagerly and measures the tile shapes) and replayed afterwards.
#include <algorithm>
#include <cmath>
#include <map>
#include <memory>
#include <string>
#include <type_traits>
#include <vector>

#include "batched.h"
#include "kernels.h"
#include "runtime.h"

namespace isvdb {
namespace {

// ------------------------------------------------------------------------- grouped GEMM
using GProd = GroupedProd;  // C = alpha A B + beta C, its work items from tile0 (kernels.h)

constexpr int kGThreads = 256;

// V consecutive elements from 16-byte aligned shared memory as one or two vector loads.
template <int V, class T>
__device__ __forceinline__ void lds_vec(const T *p, T (&out)[V]) {
  constexpr int kPer16 = 16 / (int)sizeof(T);  // elements of one 16-byte load
  static_assert(V % 2 == 0 && (V <= kPer16 || V % kPer16 == 0), "vector width");
  if (V >= kPer16) {
#pragma unroll
    for (int v = 0; v < V; v += kPer16) {
      const float4 w = *reinterpret_cast<const float4 *>(p + v);
      const T *e = reinterpret_cast<const T *>(&w);
#pragma unroll
      for (int u = 0; u < kPer16; ++u) out[v + u] = e[u];
    }
  } else {  // two floats (8 bytes)
    const float2 w = *reinterpret_cast<const float2 *>(p);
    const T *e = reinterpret_cast<const T *>(&w);
#pragma unroll
    for (int u = 0; u < V; ++u) out[u] = e[u];
  }
}

// cp.async of one element (4 or 8 bytes) global -> shared, zero-filled when !valid.
template <class T>
__device__ __forceinline__ void cp_async_elem(T *smem, const T *gmem, bool valid) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(smem);
  if (sizeof(T) == 8)
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(d), "l"(gmem), "r"(valid ? 8 : 0));
  else
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;\n" ::"r"(d), "l"(gmem), "r"(valid ? 4 : 0));
}
__device__ __forceinline__ void cp_async_commit_group() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_async_wait_group() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N)); }

constexpr int kGStages = 3, kGBK = 16;
template <class T, int BM, int BN>
constexpr int ggemm_smem() {  // bytes of the kGStages ring of A (BK x BM) and B (BK x BN) slices
  return kGStages * kGBK * (BM + BN + 2 * (16 / (int)sizeof(T))) * (int)sizeof(T);
}

// Grouped products on CUDA cores: each CTA walks the work items blockIdx.x, blockIdx.x + gridDim.x,
// ...; a work item is one BM x BN output tile of the product that owns it.  K slices of 16 flow
// through a kGStages-deep cp.async ring in shared memory (A stored k-major as As[k][m], B as
// Bs[k][n]).  256 threads in a 16 x 16 grid, each accumulating TM x TN outputs: rows
// ty * TM/2 + [0, TM/2) of both halves of the tile (and columns likewise), so that a thread's
// operands of one k are two vector loads from shared memory per operand.  Each output is one FMA
// chain in ascending k.
template <class T, class Tout, int BM, int BN>
__global__ void __launch_bounds__(kGThreads) ggemm_kernel(const GProd *__restrict__ prods, int nprod, int total) {
  constexpr int BK = kGBK, TM = BM / 16, TN = BN / 16, HM = TM / 2, HN = TN / 2;
  constexpr int LA = BM * BK / kGThreads, LB = BK * BN / kGThreads;
  constexpr int kPad = 16 / (int)sizeof(T);  // rows stay 16-byte aligned; transposing stores spread over banks
  constexpr int ALD = BM + kPad, BLD = BN + kPad, STAGE = BK * (ALD + BLD);
  extern __shared__ __align__(16) unsigned char gsm[];
  T *ring = reinterpret_cast<T *>(gsm);
  const int tid = threadIdx.x, tx = tid & 15, ty = tid >> 4;
  for (int t = blockIdx.x; t < total; t += gridDim.x) {
    int lo = 0, hi = nprod - 1;  // the product owning work item t
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (prods[mid].tile0 <= t) lo = mid;
      else hi = mid - 1;
    }
    const GProd g = prods[lo];
    const int tt = t - g.tile0, m0 = (tt / g.tn) * BM, n0 = (tt % g.tn) * BN;
    if (g.upper && n0 + BN <= m0) continue;  // strictly below the diagonal (uniform in the CTA)
    const T *__restrict__ A = static_cast<const T *>(g.A);
    const T *__restrict__ B = static_cast<const T *>(g.B);
    const bool akc = (g.a_cs == 1), bnc = (g.b_cs == 1);
    const int nk = (g.K + BK - 1) / BK;
    T acc[TM][TN];
#pragma unroll
    for (int i = 0; i < TM; ++i)
#pragma unroll
      for (int j = 0; j < TN; ++j) acc[i][j] = T(0);
    auto issue = [&](int kt) {  // K slice kt into stage kt % kGStages
      T *As = ring + (kt % kGStages) * STAGE, *Bs = As + BK * ALD;
      const int k0 = kt * BK;
#pragma unroll
      for (int r = 0; r < LA; ++r) {
        const int e = tid + r * kGThreads;
        const int mm = akc ? e / BK : e % BM, kk = akc ? e % BK : e / BM;
        const int gm = m0 + mm, gk = k0 + kk;
        const bool ok = gm < g.M && gk < g.K;
        cp_async_elem(As + kk * ALD + mm, ok ? A + (long long)gm * g.a_rs + (long long)gk * g.a_cs : A, ok);
      }
#pragma unroll
      for (int r = 0; r < LB; ++r) {
        const int e = tid + r * kGThreads;
        const int nn = bnc ? e % BN : e / BK, kk = bnc ? e / BN : e % BK;
        const int gn = n0 + nn, gk = k0 + kk;
        const bool ok = gn < g.N && gk < g.K;
        cp_async_elem(Bs + kk * BLD + nn, ok ? B + (long long)gk * g.b_rs + (long long)gn * g.b_cs : B, ok);
      }
    };
    __syncthreads();  // the previous work item's reads of the ring are done before it is refilled
#pragma unroll
    for (int s0 = 0; s0 < kGStages - 1; ++s0) {
      if (s0 < nk) issue(s0);
      cp_async_commit_group();
    }
    for (int kt = 0; kt < nk; ++kt) {
      cp_async_wait_group<kGStages - 2>();
      __syncthreads();  // slice kt visible to all; slice kt - 1 no longer read (its stage is refilled)
      if (kt + kGStages - 1 < nk) issue(kt + kGStages - 1);
      cp_async_commit_group();
      const T *As = ring + (kt % kGStages) * STAGE, *Bs = As + BK * ALD;
#pragma unroll
      for (int kk = 0; kk < BK; ++kk) {
        T av[TM], bv[TN];
        T (&a0)[HM] = *reinterpret_cast<T(*)[HM]>(av), (&a1)[HM] = *reinterpret_cast<T(*)[HM]>(av + HM);
        T (&b0)[HN] = *reinterpret_cast<T(*)[HN]>(bv), (&b1)[HN] = *reinterpret_cast<T(*)[HN]>(bv + HN);
        lds_vec<HM>(As + kk * ALD + ty * HM, a0);
        lds_vec<HM>(As + kk * ALD + BM / 2 + ty * HM, a1);
        lds_vec<HN>(Bs + kk * BLD + tx * HN, b0);
        lds_vec<HN>(Bs + kk * BLD + BN / 2 + tx * HN, b1);
#pragma unroll
        for (int i = 0; i < TM; ++i)
#pragma unroll
          for (int j = 0; j < TN; ++j) acc[i][j] = fma(av[i], bv[j], acc[i][j]);
      }
    }
    cp_async_wait_group<0>();
    Tout *__restrict__ C = static_cast<Tout *>(g.C);
#pragma unroll
    for (int i = 0; i < TM; ++i) {
      const int gm = m0 + (i < HM ? ty * HM + i : BM / 2 + ty * HM + (i - HM));
      if (gm >= g.M) continue;
#pragma unroll
      for (int j = 0; j < TN; ++j) {
        const int gn = n0 + (j < HN ? tx * HN + j : BN / 2 + tx * HN + (j - HN));
        if (gn >= g.N) continue;
        Tout *c = C + (long long)gm * g.c_rs + (long long)gn * g.c_cs;
        double v = g.alpha * (double)acc[i][j];
        if (g.beta != 0.0) v += g.beta * (double)(*c);
        *c = (Tout)v;
      }
    }
  }
}

template <class T, class Tout, int BM, int BN>
void ggemm_launch(const GProd *prods, int nprod, int total, cudaStream_t st) {
  auto *k = ggemm_kernel<T, Tout, BM, BN>;
  constexpr int bytes = ggemm_smem<T, BM, BN>();
  static int per_sm = 0;  // resident CTAs per SM, resolved on first use
  if (per_sm == 0) {
    CK(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, kGThreads, bytes));
    per_sm = std::max(1, per_sm);
  }
  const int grid = std::max(1, std::min(total, per_sm * Runtime::get().num_sms));
  k<<<grid, kGThreads, bytes, st>>>(prods, nprod, total);
  KLAUNCHED();
}

// ---------------------------------------------------------------- grouped elementwise
struct GMap {  // dst(r, c) = f(src(r, c), w[c]) over rows x cols
  const void *src;
  long long s_rs, s_cs;
  void *dst;
  long long d_rs, d_cs;
  int rows, cols;
  const double *w;
  int mode;
};
// kMapMirror: the strictly lower triangle from the upper one, dst(r, c) = src(c, r) for r > c
enum { kMapCopy = 0, kMapInvSqrt = 1, kMapSqrt = 2, kMapIdentity = 3, kMapMirror = 4 };

template <class Ts, class Td>
__global__ void gmap_kernel(const GMap *__restrict__ maps) {
  const GMap g = maps[blockIdx.y];
  const long long total = (long long)g.rows * g.cols;
  const Ts *src = static_cast<const Ts *>(g.src);
  Td *dst = static_cast<Td *>(g.dst);
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
       e += (long long)gridDim.x * blockDim.x) {
    const long long r = e / g.cols, c = e - r * g.cols;
    double v;
    if (g.mode == kMapIdentity) {
      v = (r == c) ? 1.0 : 0.0;
    } else if (g.mode == kMapMirror) {
      if (r <= c) continue;
      v = (double)src[c * g.s_rs + r * g.s_cs];
    } else {
      const double x = (double)src[r * g.s_rs + c * g.s_cs];
      v = g.mode == kMapInvSqrt ? x / sqrt(g.w[c]) : g.mode == kMapSqrt ? sqrt(x) : x;
    }
    dst[r * g.d_rs + c * g.d_cs] = (Td)v;
  }
}

// ----------------------------------------------------------------------- device lists
template <class X>
struct DevList {
  DBuf<X> d;
  int count = 0;
  void upload(const std::vector<X> &h, cudaStream_t st) {
    count = (int)h.size();
    d.ensure(std::max<size_t>(1, h.size()));
    if (!h.empty()) CK(cudaMemcpyAsync(d.p, h.data(), h.size() * sizeof(X), cudaMemcpyHostToDevice, st));
  }
};

constexpr int kConfigs = 3;
constexpr int kBM[kConfigs] = {64, 128, 128}, kBN[kConfigs] = {64, 64, 128};
std::map<std::string, int> g_tuned;  // product-list signature -> tile shape

// A grouped product list: host descriptors, the device copy for the chosen tile shape.  FP64
// lists whose products share one operand orientation run on the FP64 tensor cores
// (dmma_grouped, tile shapes dmma_grouped_bm / _bn); other lists on the CUDA-core ggemm_kernel.
template <class T, class Tout>
struct GemmList {
  static constexpr bool kFp64 = std::is_same<T, double>::value && std::is_same<Tout, double>::value;
  std::vector<GProd> host;
  DevList<GProd> dev;
  int config = -1, total = 0, uploaded = -1;
  bool dmma = false, a_kc = false, b_nc = false;  // orientation of the tensor-core launch

  void clear() {
    host.clear();
    uploaded = -1;
  }
  // dmma, a_kc, b_nc from the current products
  void orient() {
    dmma = false;
    if (!kFp64 || host.empty() || !dmma_enabled()) return;
    auto all = [&](auto pred) {
      for (const auto &g : host)
        if (!pred(g)) return false;
      return true;
    };
    const bool akc = all([](const GProd &g) { return g.a_cs == 1; }), amc = all([](const GProd &g) { return g.a_rs == 1; });
    const bool bnc = all([](const GProd &g) { return g.b_cs == 1; }), bkc = all([](const GProd &g) { return g.b_rs == 1; });
    if ((akc || amc) && (bnc || bkc)) {
      dmma = true;
      a_kc = akc;
      b_nc = bnc;
    }
  }
  int bm(int cfg) const { return dmma ? dmma_grouped_bm(cfg) : kBM[cfg]; }
  int bn(int cfg) const { return dmma ? dmma_grouped_bn(cfg) : kBN[cfg]; }
  std::string signature() const {
    int bm = 0, bn = 0, bk = 0;
    for (const auto &g : host) {
      bm = std::max(bm, g.M);
      bn = std::max(bn, g.N);
      bk = std::max(bk, g.K);
    }
    auto lg = [](int v) {
      int b = 0;
      while ((1 << b) < v) ++b;
      return b;
    };
    return std::to_string(sizeof(T)) + std::to_string(sizeof(Tout)) + (dmma ? "t" : "c") + ":" +
           std::to_string(host.size()) + ":" +
           std::to_string(lg(bm)) + "," + std::to_string(lg(bn)) + "," + std::to_string(lg(bk));
  }
  void finalize(int cfg, cudaStream_t st) {  // work items for tile shape cfg, uploaded
    int tot = 0;
    for (auto &g : host) {
      g.tn = (g.N + bn(cfg) - 1) / bn(cfg);
      g.tile0 = tot;
      tot += ((g.M + bm(cfg) - 1) / bm(cfg)) * g.tn;
    }
    total = tot;
    dev.upload(host, st);
    uploaded = cfg;
  }
  void launch(int cfg, cudaStream_t st) {  // kernels only (capturable)
    if (host.empty() || total == 0) return;
    if (dmma) {
      dmma_grouped(static_cast<const GroupedProd *>(dev.d.p), dev.count, total, cfg, a_kc, b_nc, st);
      return;
    }
    switch (cfg) {
      case 0: ggemm_launch<T, Tout, 64, 64>(dev.d.p, dev.count, total, st); break;
      case 1: ggemm_launch<T, Tout, 128, 64>(dev.d.p, dev.count, total, st); break;
      default: ggemm_launch<T, Tout, 128, 128>(dev.d.p, dev.count, total, st); break;
    }
  }
  // Choose the tile shape (measuring every candidate on first sight of the signature when all
  // products overwrite their outputs) and upload the work items.  May run the products.
  void prepare(cudaStream_t st, bool may_measure) {
    if (host.empty()) return;
    const bool was = dmma;
    orient();
    if (dmma != was) {  // another kernel family: its tile shape is chosen afresh
      config = -1;
      uploaded = -1;
    }
    if (config < 0) {
      const std::string key = signature();
      auto it = g_tuned.find(key);
      bool idempotent = true;
      for (const auto &g : host) idempotent = idempotent && g.beta == 0.0;
      if (it != g_tuned.end()) {
        config = it->second;
      } else if (may_measure && idempotent) {
        cudaEvent_t e0, e1;
        CK(cudaEventCreate(&e0));
        CK(cudaEventCreate(&e1));
        float best = 1e30f;
        int bestc = 0;
        for (int cfg = 0; cfg < (dmma ? kDmmaGroupedShapes : kConfigs); ++cfg) {
          finalize(cfg, st);
          launch(cfg, st);  // untimed: a kernel's first launch sets its attributes on the host
          CK(cudaEventRecord(e0, st));
          launch(cfg, st);
          CK(cudaEventRecord(e1, st));
          CK(cudaEventSynchronize(e1));
          float ms = 0.f;
          CK(cudaEventElapsedTime(&ms, e0, e1));
          if (ms < best) {
            best = ms;
            bestc = cfg;
          }
        }
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        config = bestc;
        g_tuned[key] = bestc;
      } else {
        config = 0;
      }
    }
    if (uploaded != config) finalize(config, st);
  }
  void run(cudaStream_t st, bool may_measure) {
    prepare(st, may_measure);
    launch(config, st);
  }
};

template <class Ts, class Td>
struct MapList {
  std::vector<GMap> host;
  DevList<GMap> dev;
  int gx = 1;
  void prepare(cudaStream_t st) {
    dev.upload(host, st);
    long long mx = 1;
    for (const auto &g : host) mx = std::max<long long>(mx, (long long)g.rows * g.cols);
    gx = (int)std::min<long long>((mx + 255) / 256, 64);
  }
  void launch(cudaStream_t st) {
    if (host.empty()) return;
    gmap_kernel<Ts, Td><<<dim3(gx, (unsigned)host.size()), 256, 0, st>>>(dev.d.p);
    KLAUNCHED();
  }
};

inline GProd prod(int M, int N, int K, const void *A, long long a_rs, long long a_cs, const void *B, long long b_rs,
                  long long b_cs, void *C, long long c_rs, long long c_cs, double alpha = 1.0) {
  GProd g;
  g.M = M; g.N = N; g.K = K;
  g.A = A; g.a_rs = a_rs; g.a_cs = a_cs;
  g.B = B; g.b_rs = b_rs; g.b_cs = b_cs;
  g.C = C; g.c_rs = c_rs; g.c_cs = c_cs;
  g.alpha = alpha; g.beta = 0.0;
  g.tile0 = 0; g.tn = 1;
  g.upper = 0;
  return g;
}

inline GMap gm(const void *src, long long s_rs, long long s_cs, void *dst, long long d_rs, long long d_cs, int rows,
               int cols, int mode, const double *w = nullptr) {
  GMap g;
  g.src = src; g.s_rs = s_rs; g.s_cs = s_cs;
  g.dst = dst; g.d_rs = d_rs; g.d_cs = d_cs;
  g.rows = rows; g.cols = cols; g.w = w; g.mode = mode;
  return g;
}

// ---------------------------------------------------------------------------- the plan
template <class T>
struct Plan : BatchPlan {
  int count = 0, N = 0, max_l = 0;
  std::vector<int> m, n, k, l, Nl;
  struct Mat {  // workspace of one matrix
    DBuf<T> om, y, qs, wp, mt, qbar, z, wk, vk;
    DBuf<double> wg, xr, G, W, DD, C, Ci, F, Fs, work, wz, vz, lz;
  };
  std::vector<std::unique_ptr<Mat>> mats;
  DBuf<double> errs;
  DBuf<int> status;
  // bound user buffers
  std::vector<const T *> a;
  std::vector<long long> lda, ldut, ldvt;
  std::vector<T *> s, ut, vt;
  std::vector<unsigned long long> seeds;
  bool bound = false;
  int solves = 0;
  // work lists
  GemmList<T, T> sketch, apply, qbar_l, proj, ul, vl;
  GemmList<T, double> gram, gfull, wzl;
  GemmList<double, double> l1, l2, l4;
  MapList<double, T> m_x, m_mt, m_s, m_wk, m_vk;
  MapList<double, double> m_init, m_mirror;
  DevList<CholDesc> chol;        // the orthogonalization's block factors
  DevList<EigDesc> eig2;         // the postprocessing's eigensolves, sorted by n, descending
  std::vector<std::pair<int, int>> eig2_cls;  // (first, largest n) of each size class
  DevList<KnStep> steps;
  // graphs of the work before and after the iterations
  cudaGraphExec_t pre = nullptr, post = nullptr;
  unsigned long long pre_k = 0, post_k = 0;

  // side streams on which the step launches of several size classes run beside each other
  cudaStream_t side[2] = {nullptr, nullptr};
  cudaEvent_t fork = nullptr, join[2] = {nullptr, nullptr};

  ~Plan() override {
    drop_graphs();
    for (int i = 0; i < 2; ++i) {
      if (side[i]) cudaStreamDestroy(side[i]);
      if (join[i]) cudaEventDestroy(join[i]);
    }
    if (fork) cudaEventDestroy(fork);
  }
  void make_side_streams() {
    if (fork) return;
    CK(cudaEventCreateWithFlags(&fork, cudaEventDisableTiming));
    for (int i = 0; i < 2; ++i) {
      CK(cudaStreamCreateWithFlags(&side[i], cudaStreamNonBlocking));
      CK(cudaEventCreateWithFlags(&join[i], cudaEventDisableTiming));
    }
  }
  void drop_graphs() {
    if (pre) cudaGraphExecDestroy(pre);
    if (post) cudaGraphExecDestroy(post);
    pre = post = nullptr;
  }
};

template <class T>
void build_lists(Plan<T> &P, cudaStream_t st) {
  const int B = P.count, N = P.N;
  P.sketch.clear(); P.apply.clear(); P.qbar_l.clear(); P.proj.clear(); P.ul.clear(); P.vl.clear();
  P.gram.clear(); P.gfull.clear(); P.wzl.clear();
  P.m_x.host.clear(); P.m_s.host.clear(); P.m_mirror.host.clear(); P.m_wk.host.clear(); P.m_vk.host.clear(); P.m_init.host.clear();
  std::vector<CholDesc> c1;
  std::vector<EigDesc> e2;
  for (int b = 0; b < B; ++b) {
    auto &M = *P.mats[b];
    const int m = P.m[b], n = P.n[b], k = P.k[b], l = P.l[b], Nl = P.Nl[b];
    const size_t ll = (size_t)l * l;
    P.sketch.host.push_back(prod(m, Nl, n, P.a[b], P.lda[b], 1, M.om.p, Nl, 1, M.y.p, Nl, 1));
    for (int i = 0; i < N; ++i) {
      P.gram.host.push_back(prod(l, l, m, M.y.p + i * l, 1, Nl, M.y.p + i * l, Nl, 1, M.wg.p + i * ll, l, 1));
      c1.push_back(CholDesc{l, M.wg.p + i * ll, M.xr.p + i * ll});
      P.m_x.host.push_back(gm(M.xr.p + i * ll, l, 1, M.wp.p + i * ll, l, 1, l, l, kMapCopy));
      P.apply.host.push_back(prod(m, l, l, M.y.p + i * l, Nl, 1, M.wp.p + i * ll, l, 1, M.qs.p + i * l, Nl, 1));
    }
    P.gfull.host.push_back(prod(Nl, Nl, m, M.qs.p, 1, Nl, M.qs.p, Nl, 1, M.G.p, Nl, 1));
    P.gfull.host.back().upper = 1;  // G = Qs'Qs symmetric: the upper triangle's tiles, then mirrored
    P.m_mirror.host.push_back(gm(M.G.p, Nl, 1, M.G.p, Nl, 1, Nl, Nl, kMapMirror));
    // iterate [M | B | Bgc] in W[0]: Bc = G[:, 0:l], M = [I; 0]
    P.m_init.host.push_back(gm(M.G.p, Nl, 1, M.W.p + l, 3 * l, 1, Nl, l, kMapCopy));
    P.m_init.host.push_back(gm(nullptr, 0, 0, M.W.p, 3 * l, 1, Nl, l, kMapIdentity));
    // after the iterations: Qbar = Qs M, Z = A' Qbar, W = Z'Z, eig, s, U, V
    P.qbar_l.host.push_back(prod(m, l, Nl, M.qs.p, Nl, 1, M.mt.p, l, 1, M.qbar.p, l, 1));
    P.proj.host.push_back(prod(n, l, m, P.a[b], 1, P.lda[b], M.qbar.p, l, 1, M.z.p, l, 1));
    P.wzl.host.push_back(prod(l, l, n, M.z.p, 1, l, M.z.p, l, 1, M.wz.p, l, 1));
    e2.push_back(EigDesc{l, M.wz.p, M.vz.p, M.lz.p});
    P.m_s.host.push_back(gm(M.lz.p, 1, 0, P.s[b], 1, 0, l, 1, kMapSqrt));
    P.m_wk.host.push_back(gm(M.vz.p, l, 1, M.wk.p, k, 1, l, k, kMapCopy));
    P.m_vk.host.push_back(gm(M.vz.p, l, 1, M.vk.p, k, 1, l, k, kMapInvSqrt, M.lz.p));
    P.ul.host.push_back(prod(m, k, l, M.qbar.p, l, 1, M.wk.p, k, 1, P.ut[b], P.ldut[b], 1));
    P.vl.host.push_back(prod(n, k, l, M.z.p, l, 1, M.vk.p, k, 1, P.vt[b], P.ldvt[b], 1));
  }
  // each eigensolve list sorted by size, largest first, and cut into the size classes of the
  // eigensolver's CTA shapes (n <= 32, <= 64, <= 96): one launch per class
  auto classes = [](std::vector<EigDesc> &e, std::vector<std::pair<int, int>> &cls) {
    std::stable_sort(e.begin(), e.end(), [](const EigDesc &x, const EigDesc &y) { return x.n > y.n; });
    auto cl = [](int n) { return n <= 32 ? 0 : n <= 64 ? 1 : 2; };
    cls.clear();
    for (int i = 0; i < (int)e.size(); ++i)
      if (i == 0 || cl(e[i].n) != cl(e[i - 1].n)) cls.emplace_back(i, e[i].n);
  };
  classes(e2, P.eig2_cls);
  P.chol.upload(c1, st);
  P.eig2.upload(e2, st);
  P.m_x.prepare(st); P.m_s.prepare(st); P.m_mirror.prepare(st); P.m_wk.prepare(st); P.m_vk.prepare(st); P.m_init.prepare(st);
}

// The grouped eigensolves of list d (classes cls: first index and largest n), one launch per class.
inline void eig_classes(const DevList<EigDesc> &d, const std::vector<std::pair<int, int>> &cls, int *status,
                        cudaStream_t st) {
  for (size_t c = 0; c < cls.size(); ++c) {
    const int first = cls[c].first, end = c + 1 < cls.size() ? cls[c + 1].first : d.count;
    sym_eig_grouped(d.d.p + first, end - first, cls[c].second, +1, true, status, st);
  }
}

template <class T>
void run_pre(Plan<T> &P, cudaStream_t st, bool measure) {
  for (int b = 0; b < P.count; ++b)
    rng_gaussian<T>(P.mats[b]->om.p, P.n[b], P.Nl[b], P.Nl[b], P.seeds[b], 0, st);
  P.sketch.run(st, measure);
  P.gram.run(st, measure);
  chol_inv_grouped(P.chol.d.p, P.chol.count, P.max_l, P.status.p, st);
  P.m_x.launch(st);
  P.apply.run(st, measure);
  P.gfull.run(st, measure);
  P.m_mirror.launch(st);
  P.m_init.launch(st);
}

template <class T>
void run_post(Plan<T> &P, cudaStream_t st, bool measure) {
  P.qbar_l.run(st, measure);
  P.proj.run(st, measure);
  P.wzl.run(st, measure);
  eig_classes(P.eig2, P.eig2_cls, P.status.p, st);
  P.m_s.launch(st);
  P.m_wk.launch(st);
  P.m_vk.launch(st);
  P.ul.run(st, measure);
  P.vl.run(st, measure);
}

// Runs body eagerly (first solve, which measures tile shapes), or captures it once and replays it.
template <class F>
void graphed(cudaGraphExec_t &exec, unsigned long long &nk, bool capture, cudaStream_t st, F &&body) {
  if (!capture) {
    body();
    return;
  }
  if (!exec) {
    CK(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
    try {
      body();
    } catch (...) {
      cudaGraph_t g = nullptr;
      cudaStreamEndCapture(st, &g);
      if (g) cudaGraphDestroy(g);
      throw;
    }
    cudaGraph_t g = nullptr;
    CK(cudaStreamEndCapture(st, &g));
    nk = count_kernel_nodes(g);
    const cudaError_t e = cudaGraphInstantiate(&exec, g, 0);
    cudaGraphDestroy(g);
    CK(e);
  }
  CK(cudaGraphLaunch(exec, st));
  g_launches.fetch_add(nk);
}

}  // namespace

int plan_count(const BatchPlan *plan) {
  return plan->elem == 4 ? static_cast<const Plan<float> *>(plan)->count : static_cast<const Plan<double> *>(plan)->count;
}

template <class T>
BatchPlan *batch_plan_create(int count, const int *m, const int *n, const int *k, const int *p, int N) {
  if (count <= 0) fail(kErrArgument, "batched iSVD: count = %d", count);
  if (N <= 0) fail(kErrArgument, "batched iSVD: N = %d", N);
  std::unique_ptr<Plan<T>> P(new Plan<T>());
  P->elem = sizeof(T);
  P->count = count;
  P->N = N;
  P->mats.resize(count);
  for (int b = 0; b < count; ++b) {
    const int l = k[b] + p[b], Nl = N * l;
    if (m[b] <= 0 || n[b] <= 0 || k[b] <= 0 || p[b] < 0 || l > n[b] || l > m[b])
      fail(kErrArgument, "batched iSVD: matrix %d: m = %d, n = %d, k = %d, p = %d", b, m[b], n[b], k[b], p[b]);
    if (l > 96) fail(kErrUnsupported, "batched iSVD: matrix %d: l = %d > 96", b, l);
    P->m.push_back(m[b]); P->n.push_back(n[b]); P->k.push_back(k[b]); P->l.push_back(l); P->Nl.push_back(Nl);
    P->max_l = std::max(P->max_l, l);
    auto M = std::make_unique<typename Plan<T>::Mat>();
    const size_t ll = (size_t)l * l, nl = (size_t)Nl * l;
    M->om.alloc((size_t)n[b] * Nl);
    M->y.alloc((size_t)m[b] * Nl);
    M->qs.alloc((size_t)m[b] * Nl);
    M->wp.alloc(N * ll);
    M->mt.alloc(nl);
    M->qbar.alloc((size_t)m[b] * l);
    M->z.alloc((size_t)n[b] * l);
    M->wk.alloc((size_t)l * k[b]);
    M->vk.alloc((size_t)l * k[b]);
    M->wg.alloc(N * ll); M->xr.alloc(N * ll);
    M->G.alloc((size_t)Nl * Nl);
    M->W.alloc(6 * nl);
    M->DD.alloc(2 * ll); M->C.alloc(ll); M->Ci.alloc(ll); M->F.alloc(ll); M->Fs.alloc(4 * ll);
    M->work.alloc(kKnWorkMatrices * ll + 64);
    M->wz.alloc(ll); M->vz.alloc(ll); M->lz.alloc(l);
    P->mats[b] = std::move(M);
  }
  P->errs.alloc(count);
  P->status.alloc(1);
  return P.release();
}

template <class T>
void batch_solve(BatchPlan *plan, const T *const *a, const long long *lda, T *const *s, T *const *ut,
                 const long long *ldut, T *const *vt, const long long *ldvt, const unsigned long long *seeds, int maxit,
                 double tol, int *iters, double *errs) {
  if (!plan || plan->elem != (int)sizeof(T)) fail(kErrArgument, "batched iSVD: plan of another element type");
  Plan<T> &P = *static_cast<Plan<T> *>(plan);
  Runtime &rt = Runtime::get();
  cudaStream_t st = rt.stream;
  const int B = P.count, N = P.N;
  // bind the caller's buffers; a change rebuilds the work lists and the graphs
  bool same = P.bound;
  for (int b = 0; b < B && same; ++b)
    same = P.a[b] == a[b] && P.lda[b] == lda[b] && P.s[b] == s[b] && P.ut[b] == ut[b] && P.ldut[b] == ldut[b] &&
           P.vt[b] == vt[b] && P.ldvt[b] == ldvt[b] && P.seeds[b] == seeds[b];
  if (!same) {
    for (int b = 0; b < B; ++b) {
      if (lda[b] < P.n[b] || ldut[b] < P.l[b] || ldvt[b] < P.l[b])
        fail(kErrArgument, "batched iSVD: matrix %d: leading dimension too small", b);
      if (!is_device_pointer(a[b]) || !is_device_pointer(s[b]) || !is_device_pointer(ut[b]) ||
          !is_device_pointer(vt[b]))
        fail(kErrArgument, "batched iSVD: matrix %d: a, s, ut and vt must be device memory", b);
    }
    P.a.assign(a, a + B); P.lda.assign(lda, lda + B); P.s.assign(s, s + B); P.ut.assign(ut, ut + B);
    P.ldut.assign(ldut, ldut + B); P.vt.assign(vt, vt + B); P.ldvt.assign(ldvt, ldvt + B);
    P.seeds.assign(seeds, seeds + B);
    P.drop_graphs();
    build_lists(P, st);
    P.bound = true;
    P.solves = 0;
  }
  const bool capture = P.solves > 0 && st != nullptr && !profiling();
  CK(cudaMemsetAsync(P.status.p, 0, sizeof(int), st));
  graphed(P.pre, P.pre_k, capture, st, [&] { run_pre(P, st, !capture); });

  // ---- Kolmogorov-Nagumo iterations of the active matrices (reference :153-266)
  const double invN = 1.0 / N;
  const int cap = maxit > 0 ? maxit : 1000000;
  std::vector<int> active(B), cur(B, 0), it_of(B, 0);
  for (int b = 0; b < B; ++b) active[b] = b;
  std::vector<double> herr(B, 0.0);
  std::vector<KnStep> hsteps;
  for (int iter = 1; !active.empty(); ++iter) {
    P.l1.clear(); P.l2.clear(); P.l4.clear();
    hsteps.clear();
    for (int b : active) {
      auto &M = *P.mats[b];
      const int l = P.l[b], Nl = P.Nl[b];
      const size_t ll = (size_t)l * l, nl3 = (size_t)Nl * 3 * l;
      double *Wc = M.W.p + cur[b] * nl3, *Wn = M.W.p + (1 - cur[b]) * nl3;
      const long long lw = 3LL * l;
      P.l1.host.push_back(prod(Nl, l, Nl, M.G.p, Nl, 1, Wc + l, lw, 1, Wc + 2 * l, lw, 1, invN));
      P.l2.host.push_back(prod(l, l, Nl, Wc + l, 1, lw, Wc + l, lw, 1, M.DD.p, l, 1, invN));
      P.l2.host.push_back(prod(l, l, Nl, Wc + l, 1, lw, Wc + 2 * l, lw, 1, M.DD.p + ll, l, 1, invN));
      P.l4.host.push_back(prod(Nl, l, 2 * l, Wc, lw, 1, M.Fs.p, l, 1, Wn, lw, 1));
      P.l4.host.push_back(prod(Nl, l, 2 * l, Wc + l, lw, 1, M.Fs.p + 2 * ll, l, 1, Wn + l, lw, 1));
      KnStep s;
      s.l = l; s.Dc = M.DD.p; s.Dgc = M.DD.p + ll; s.C = M.C.p; s.Cinv = M.Ci.p; s.F = M.F.p;
      s.err = P.errs.p + b; s.work = M.work.p; s.status = P.status.p; s.bar = nullptr;
      s.ns_target = 1e-18;
      s.fstack = M.Fs.p; s.fstack_scale = invN;
      hsteps.push_back(s);
    }
    P.l1.run(st, true);
    P.l2.run(st, true);
    // the steps grouped by their number of 32 x 32 product tiles, nt = ceil(l / 32)^2, one launch
    // per group with the cluster size c that minimises waves x tiles per CTA,
    // ceil(count c / SMs) ceil(nt / c) (one 1024-thread CTA per SM); the groups (at most three for
    // l <= 96) run side by side, the largest on the library stream, the others on side streams
    auto tiles_of = [](const KnStep &s) { return ((s.l + 31) / 32) * ((s.l + 31) / 32); };
    std::stable_sort(hsteps.begin(), hsteps.end(),
                     [&](const KnStep &x, const KnStep &y) { return tiles_of(x) > tiles_of(y); });
    P.steps.upload(hsteps, st);
    P.make_side_streams();
    CK(cudaEventRecord(P.fork, st));
    int group = 0;
    const int sms = rt.num_sms;
    for (size_t g0 = 0; g0 < hsteps.size(); ++group) {
      const int nt = tiles_of(hsteps[g0]);
      size_t g1 = g0;
      int lmax = 0;
      while (g1 < hsteps.size() && tiles_of(hsteps[g1]) == nt) lmax = std::max(lmax, hsteps[g1++].l);
      const long long cnt = (long long)(g1 - g0);
      int best_c = 1;
      long long best = -1;
      for (int c = 1; c <= 8 && c <= nt; c *= 2) {
        const long long cost = ((cnt * c + sms - 1) / sms) * ((nt + c - 1) / c);
        if (best < 0 || cost < best) { best = cost; best_c = c; }
      }
      cudaStream_t gs = st;
      if (group > 0 && group <= 2) {
        gs = P.side[group - 1];
        CK(cudaStreamWaitEvent(gs, P.fork, 0));
      }
      kn_step_grouped(P.steps.d.p + g0, (int)cnt, lmax, best_c, gs);
      if (gs != st) {
        CK(cudaEventRecord(P.join[group - 1], gs));
        CK(cudaStreamWaitEvent(st, P.join[group - 1], 0));
      }
      g0 = g1;
    }
    P.l4.run(st, true);
    int hstatus = 0;
    CK(cudaMemcpyAsync(herr.data(), P.errs.p, B * sizeof(double), cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(&hstatus, P.status.p, sizeof(int), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    if (hstatus) fail(kErrNumerical, "batched iSVD: small dense solver reported status %d", hstatus);
    std::vector<int> next;
    for (int b : active) {
      cur[b] = 1 - cur[b];  // the iterate just written
      if (herr[b] <= tol) {                 // (:235-237)
        it_of[b] = iter;
      } else if (iter == cap) {             // (:238-241)
        it_of[b] = iter + 1;
      } else {
        next.push_back(b);
      }
    }
    active.swap(next);
  }
  // M of each matrix (in its final iterate) to the element type
  {
    MapList<double, T> mt;
    for (int b = 0; b < B; ++b) {
      auto &M = *P.mats[b];
      const size_t nl3 = (size_t)P.Nl[b] * 3 * P.l[b];
      mt.host.push_back(gm(M.W.p + cur[b] * nl3, 3LL * P.l[b], 1, M.mt.p, P.l[b], 1, P.Nl[b], P.l[b], kMapCopy));
    }
    mt.prepare(st);
    mt.launch(st);
    graphed(P.post, P.post_k, capture, st, [&] { run_post(P, st, !capture); });
    int hstatus = 0;
    CK(cudaMemcpyAsync(&hstatus, P.status.p, sizeof(int), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    if (hstatus) fail(kErrNumerical, "batched iSVD: small dense solver reported status %d", hstatus);
  }
  for (int b = 0; b < B; ++b) {
    if (iters) iters[b] = it_of[b];
    if (errs) errs[b] = herr[b];
  }
  ++P.solves;
}

template BatchPlan *batch_plan_create<float>(int, const int *, const int *, const int *, const int *, int);
template BatchPlan *batch_plan_create<double>(int, const int *, const int *, const int *, const int *, int);
template void batch_solve<float>(BatchPlan *, const float *const *, const long long *, float *const *, float *const *,
                                 const long long *, float *const *, const long long *, const unsigned long long *, int,
                                 double, int *, double *);
template void batch_solve<double>(BatchPlan *, const double *const *, const long long *, double *const *,
                                  double *const *, const long long *, double *const *, const long long *,
                                  const unsigned long long *, int, double, int *, double *);

}  // namespace isvdb
