// Kolmogorov-Nagumo integration on a statically allocated device scratch array.
//
// Some callers cannot let a library allocate device memory while it runs: a serving process
// that has handed the whole device to its own pool allocator (a cudaMalloc then fails, or
// blocks until other streams drain), a real-time loop where an allocation's implicit device
// synchronisation breaks a latency budget, or an application that reserves all of its memory
// up front and treats any later allocation as a leak.  The ordinary stage (integrate_kn_dev)
// takes its buffers from the stream-ordered pool and its control words from the library
// runtime, whose set-up allocates.  This variant does neither: every intermediate lives in
// g_kn_scratch, a file-scope __device__ array that the module loader places once per device.
//
// The computation is the NATIVE FP64 path of integrate_kn_dev (reference
// @x@_integrate_kolmogorov_nagumo.c:153-266 in the coordinates of Qs) with the same kernels;
// only the launchers differ (SM count passed in, split-K partial sums in the scratch).
//
// Scratch contents, each region starting on a 256-byte boundary:
//   control block (32 doubles: status int, 2 grid-barrier words, error estimate),
//   G (Nl x Nl), Bc, B+ , Mc, M+ , Bgc (Nl x l each), Dc, Dgc, C, C^-1, F (l x l each),
//   the step's work area (8 l^2 + 64), then split-K partial sums in whatever is left.
// Nothing in it must be zero on entry: the control block is cleared at the start of each call
// and the barrier words again before each step, on the caller's stream.
//
// Calls that overlapped on one device would share these intermediates and corrupt each other.
// The exported entry point holds the library's process-wide lock for the whole call and
// synchronises its stream before returning, so calls from any thread or stream run one after
// the other.
#include <cuda_runtime.h>

#include <algorithm>
#include <mutex>
#include <utility>

#include "kernels.h"
#include "runtime.h"
#include "stages.h"

namespace isvdb {

constexpr size_t kKnScratchDoubles = size_t(1) << 20;  // 8 MiB per device
static __device__ __align__(256) double g_kn_scratch[kKnScratchDoubles];

namespace {

constexpr int kMaxDevices = 64;

struct ScratchSlot {
  double *base = nullptr;
  int sms = 0;
};

std::mutex g_slot_mu;
ScratchSlot g_slot[kMaxDevices];

__global__ void kn_start_kernel(const double *__restrict__ G, int Nl, int l, double *__restrict__ Bc,
                                double *__restrict__ Mc);

// First use on a device (that device current): the array's address (looking it up loads the
// module that holds it, when modules load lazily), the SM count, and every kernel this entry point
// can launch resolved once, so that with lazy module loading no later call (another shape, another
// tile size, split-K) is the first launch of a kernel, which would load code and could allocate.
// Later calls reuse all of it.
ScratchSlot slot_for_current_device(int dev) {
  if (dev < 0 || dev >= kMaxDevices) fail(kErrUnsupported, "static scratch: device ordinal %d out of range", dev);
  std::lock_guard<std::mutex> lk(g_slot_mu);
  ScratchSlot &s = g_slot[dev];
  if (!s.base) {
    void *p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_kn_scratch);
    if (e != cudaSuccess || p == nullptr)
      fail(kErrCuda, "static scratch: cudaGetSymbolAddress failed on device %d: %s", dev, cudaGetErrorString(e));
    int sms = 0;
    CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    cudaFuncAttributes fa;
    CK(cudaFuncGetAttributes(&fa, kn_start_kernel));
    gemm_fixed_preload();
    kn_step_fixed_preload();
    s.sms = sms;
    s.base = static_cast<double *>(p);
  }
  return s;
}

void require_device_memory(const void *p, int dev, const char *name) {
  cudaPointerAttributes at;
  CK(cudaPointerGetAttributes(&at, p));
  const bool ok = (at.type == cudaMemoryTypeDevice && at.device == dev) || at.type == cudaMemoryTypeManaged;
  if (!ok)
    fail(kErrArgument, "Kolmogorov-Nagumo on static scratch: %s must be device or managed memory of device %d",
         name, dev);
}

// Region offsets in doubles; every region is rounded up to 32 doubles (256 bytes).
struct ScratchLayout {
  size_t used = 0;
  size_t take(size_t n) {
    const size_t at = used;
    used += (n + 31) & ~size_t(31);
    return at;
  }
};

// Bc = G[:, 0:l] (= Qs' Q0) and Mc = [I; 0] (Q0 = the first block of Qs).
__global__ void kn_start_kernel(const double *__restrict__ G, int Nl, int l, double *__restrict__ Bc,
                                double *__restrict__ Mc) {
  const long long total = (long long)Nl * l;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
       e += (long long)gridDim.x * blockDim.x) {
    const long long i = e / l, j = e - i * l;
    Bc[e] = G[i * Nl + j];
    Mc[e] = (i == j) ? 1.0 : 0.0;
  }
}

inline Gemm<double, double> gmd(int M, int N, int K) {
  Gemm<double, double> g;
  g.M = M; g.N = N; g.K = K;
  return g;
}

}  // namespace

IterResult integrate_kn_static(cudaStream_t st, int m, int l, int N, const double *qs, long long ldq, double *qt,
                               long long ldqt, int maxit, double tol) {
  if (m <= 0 || l <= 0 || N <= 0) fail(kErrArgument, "Kolmogorov-Nagumo on static scratch: m, l, N must be positive");
  if (l > 160) fail(kErrArgument, "Kolmogorov-Nagumo on static scratch: l = %d > 160", l);
  const int Nl = N * l;
  const size_t nl = (size_t)Nl * l, ll = (size_t)l * l;
  ScratchLayout lay;
  const size_t o_ctl = lay.take(32), o_g = lay.take((size_t)Nl * Nl);
  const size_t o_bc = lay.take(nl), o_bp = lay.take(nl), o_mc = lay.take(nl), o_mp = lay.take(nl);
  const size_t o_bgc = lay.take(nl), o_dc = lay.take(ll), o_dgc = lay.take(ll), o_c = lay.take(ll);
  const size_t o_ci = lay.take(ll), o_f = lay.take(ll), o_work = lay.take(8 * ll + 64);
  if (lay.used > kKnScratchDoubles)
    fail(kErrArgument,
         "Kolmogorov-Nagumo on static scratch: N*l = %d, l = %d need %zu doubles of scratch; the static "
         "scratch holds %zu (8 MiB)",
         Nl, l, lay.used, kKnScratchDoubles);
  int dev = 0;
  CK(cudaGetDevice(&dev));
  const ScratchSlot slot = slot_for_current_device(dev);
  require_device_memory(qs, dev, "yst");
  require_device_memory(qt, dev, "qt");
  double *const base = slot.base;
  const int sms = slot.sms;
  int *const status = reinterpret_cast<int *>(base + o_ctl);
  unsigned int *const bar = reinterpret_cast<unsigned int *>(base + o_ctl + 1);
  double *const err = base + o_ctl + 4;
  double *const G = base + o_g;
  double *Bc = base + o_bc, *Bp = base + o_bp, *Mc = base + o_mc, *Mp = base + o_mp;
  double *const Bgc = base + o_bgc, *const Dc = base + o_dc, *const Dgc = base + o_dgc;
  double *const C = base + o_c, *const Ci = base + o_ci, *const F = base + o_f, *const work = base + o_work;
  double *const partial = base + lay.used;
  const size_t pcap = kKnScratchDoubles - lay.used;
  const double invN = 1.0 / N;
  IterResult res;
  try {
    CK(cudaMemsetAsync(base + o_ctl, 0, 32 * sizeof(double), st));
    {  // G = Qs' Qs
      Gemm<double, double> g = gmd(Nl, Nl, m);
      g.A = qs; g.a_rs = 1; g.a_cs = ldq;
      g.B = qs; g.b_rs = ldq; g.b_cs = 1;
      g.C = G; g.c_rs = Nl; g.c_cs = 1;
      gemm_fixed(g, sms, partial, pcap, st);
    }
    kn_start_kernel<<<(int)std::min<long long>(((long long)nl + 255) / 256, 4LL * sms), 256, 0, st>>>(G, Nl, l,
                                                                                                        Bc, Mc);
    KLAUNCHED();
    double herr = 0.0;
    const int cap = maxit > 0 ? maxit : 1000000;
    int iter = 1;
    for (;; ++iter) {
      {  // Bgc = G Bc / N
        Gemm<double, double> g = gmd(Nl, l, Nl);
        g.alpha = invN;
        g.A = G; g.a_rs = Nl; g.a_cs = 1;
        g.B = Bc; g.b_rs = l; g.b_cs = 1;
        g.C = Bgc; g.c_rs = l; g.c_cs = 1;
        gemm_fixed(g, sms, partial, pcap, st);
      }
      {  // Dc = Bc' Bc / N ; Dgc = Bc' Bgc / N
        Gemm<double, double> g = gmd(l, l, Nl);
        g.alpha = invN;
        g.A = Bc; g.a_rs = 1; g.a_cs = l;
        g.B = Bc; g.b_rs = l; g.b_cs = 1;
        g.C = Dc; g.c_rs = l; g.c_cs = 1;
        gemm_fixed(g, sms, partial, pcap, st);
        g.B = Bgc;
        g.C = Dgc;
        gemm_fixed(g, sms, partial, pcap, st);
      }
      CK(cudaMemsetAsync(bar, 0, 2 * sizeof(unsigned int), st));
      KnStep s;
      s.l = l; s.Dc = Dc; s.Dgc = Dgc; s.C = C; s.Cinv = Ci; s.F = F; s.err = err;
      s.work = work; s.status = status; s.bar = bar;
      s.ns_target = 1e-18;
      kn_step_fixed(s, sms, st);
      {  // M+ = Mc F + (Bc / N) C^-1 ;  B+ = Bc F + Bgc C^-1
        Gemm<double, double> g = gmd(Nl, l, l);
        g.A = Mc; g.a_rs = l; g.a_cs = 1;
        g.B = F; g.b_rs = l; g.b_cs = 1;
        g.C = Mp; g.c_rs = l; g.c_cs = 1;
        gemm_fixed(g, sms, partial, pcap, st);
        g.A = Bc; g.B = Ci; g.alpha = invN; g.beta = 1.0;
        gemm_fixed(g, sms, partial, pcap, st);
        g.A = Bc; g.B = F; g.C = Bp; g.alpha = 1.0; g.beta = 0.0;
        gemm_fixed(g, sms, partial, pcap, st);
        g.A = Bgc; g.B = Ci; g.beta = 1.0;
        gemm_fixed(g, sms, partial, pcap, st);
      }
      int h = 0;
      CK(cudaMemcpyAsync(&herr, err, sizeof(double), cudaMemcpyDeviceToHost, st));
      CK(cudaMemcpyAsync(&h, status, sizeof(int), cudaMemcpyDeviceToHost, st));
      CK(cudaStreamSynchronize(st));
      if (h == kErrTimeout) fail(kErrTimeout, "Kolmogorov-Nagumo integration: a device-side wait timed out");
      if (h) fail(kErrNumerical, "Kolmogorov-Nagumo integration: small dense solver reported status %d", h);
      if (herr <= tol) break;
      if (iter == cap) { ++iter; break; }
      std::swap(Bc, Bp);
      std::swap(Mc, Mp);
    }
    res.iterations = iter;
    res.error = herr;
    {  // Qbar = Qs M+
      Gemm<double, double> g = gmd(m, l, Nl);
      g.A = qs; g.a_rs = ldq; g.a_cs = 1;
      g.B = Mp; g.b_rs = l; g.b_cs = 1;
      g.C = qt; g.c_rs = ldqt; g.c_cs = 1;
      gemm_fixed(g, sms, partial, pcap, st);
    }
    CK(cudaStreamSynchronize(st));
  } catch (...) {
    cudaStreamSynchronize(st);  // the scratch must be idle before another call can use it
    throw;
  }
  return res;
}

}  // namespace isvdb
