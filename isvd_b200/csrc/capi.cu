// C ABI of libisvd_gpu_b200: the iSVD entry points of emfomy/isvd v1.3.2 (include/isvd.h) plus
// the B200 extensions (include/isvd/b200.h).  This file is host code only: argument checking
// with the reference's semantics, host <-> device marshalling, stage dispatch and the driver.
#include <cuda_runtime.h>

#include <cctype>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "batched.h"
#include "kernels.h"
#include "mixed.h"
#include "mtx.h"
#include "panels.h"
#include "runtime.h"
#include "stages.h"

// The library is built with -fvisibility=hidden; only the C ABI is exported.
#pragma GCC visibility push(default)
extern "C" {
#include <isvd.h>
}
#pragma GCC visibility pop

using namespace isvdb;

// ============================================================================ error state
namespace {

thread_local int t_last_error = 0;
thread_local std::string t_last_msg;
std::recursive_mutex g_api_mu;  // the API is not re-entrant (as the reference); calls are serialised

void record_error(int code, const std::string &msg) {
  t_last_error = code;
  t_last_msg = msg;
  fprintf(stderr, "isvd: %s\n", msg.c_str());
}

// Print-and-return argument failure (reference util/arg.h:40-48 prints and returns 0).
struct ArgFail {};

template <class F>
int api_call(F &&f) {
  std::lock_guard<std::recursive_mutex> lk(g_api_mu);
  try {
    f();
    return kSuccess;
  } catch (const ArgFail &) {
    return t_last_error;
  } catch (const Error &e) {
    record_error(e.code, e.what());
    return e.code;
  } catch (const std::exception &e) {
    record_error(kErrCuda, e.what());
    return kErrCuda;
  }
}

[[noreturn]] void arg_error(const char *fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  t_last_error = kErrArgument;
  t_last_msg = buf;
  fputs(buf, stderr);
  throw ArgFail();
}

// Reference isvd_assert_* failures abort; here they become an argument error.
#define REQUIRE(cond)                                                                        \
  do {                                                                                       \
    if (!(cond)) ::isvdb::fail(kErrArgument, "argument check failed: %s", #cond);            \
  } while (0)

// Case-insensitive single-character option (reference util/arg.h:22-49).
char arg2char(const char *name, char arg, const char *opts) {
  for (const char *o = opts; *o; ++o)
    if (toupper((unsigned char)arg) == toupper((unsigned char)*o)) return *o;
  std::string msg = std::string(name) + " ('" + arg + "') must be one of the following characters: ";
  for (const char *o = opts; *o; ++o) {
    if (o != opts) msg += ", ";
    msg += "'";
    msg += *o;
    msg += "'";
  }
  arg_error("%s.\n", msg.c_str());
}

// Case-insensitive selector (reference util/arg.h:51-79).
const char *arg2str(const char *name, const char *arg, const char *const *opts, int nopts) {
  if (arg) {
    const size_t la = strlen(arg);
    for (int i = 0; i < nopts; ++i) {
      if (strlen(opts[i]) != la) continue;
      bool eq = true;
      for (size_t c = 0; c < la && eq; ++c) eq = toupper((unsigned char)arg[c]) == toupper((unsigned char)opts[i][c]);
      if (eq) return opts[i];
    }
  }
  std::string msg = std::string(name) + " ('" + (arg ? arg : "(null)") + "') must be one of the following strings: ";
  for (int i = 0; i < nopts; ++i) {
    if (i) msg += ", ";
    msg += "\"";
    msg += opts[i];
    msg += "\"";
  }
  arg_error("%s.\n", msg.c_str());
}

#if !defined(ISVD_MPI_SHIM)
// Built against a real MPI (isvd_b200/build.py --mpi-include): the ranks of the communicator in
// isvd_Param join as row blocks without isvd_gpu_set_allreduce, each exchange an in-place
// MPI_Allreduce (MPI_SUM) on the library's pinned host staging buffer, as the reference's stages
// reduce on that communicator.  A reduction installed by the program takes precedence.
MPI_Comm g_param_comm;

void mpi_param_allreduce(void *buf, size_t count, int dtype, void *stream, void *user) {
  (void)stream; (void)user;
  const size_t esz = dtype == ISVD_GPU_DTYPE_F64 ? sizeof(double) : sizeof(float);
  const size_t chunk = (size_t)1 << 30;  // MPI counts are int
  for (size_t off = 0; off < count; off += chunk) {
    const int n = (int)std::min(chunk, count - off);
    if (MPI_Allreduce(MPI_IN_PLACE, static_cast<char *>(buf) + off * esz, n,
                      dtype == ISVD_GPU_DTYPE_F64 ? MPI_DOUBLE : MPI_FLOAT, MPI_SUM, g_param_comm) != MPI_SUCCESS)
      fail(kErrUnsupported, "MPI_Allreduce failed on the communicator of isvd_Param");
  }
}

void join_param_comm(const isvd_Param &p) {
  Collective &c = collective();
  if (c.fn && !c.from_comm) return;  // the program's own reduction
  if (p.mpi_size > 1) {
    g_param_comm = p.mpi_comm;
    c.fn = mpi_param_allreduce;
    c.user = nullptr;
    c.nranks = p.mpi_size;
    c.rank = p.mpi_rank;
    c.on_device = 0;
    c.from_comm = true;
  } else if (c.from_comm) {
    c = Collective();
  }
}
#endif

void require_single_rank(const isvd_Param &p) {
#if !defined(ISVD_MPI_SHIM)
  join_param_comm(p);
#endif
  // several ranks: only through the caller's AllReduce (isvd_gpu_set_allreduce), row blocks
  const Collective &cl = collective();
  if (p.mpi_size != 1 && !(cl.nranks == p.mpi_size && cl.rank == p.mpi_rank))
    fail(kErrUnsupported, "MPI size %d: this build joins several ranks only through isvd_gpu_set_allreduce",
         (int)p.mpi_size);
  // the ILP64 build takes 64-bit sizes at the boundary; one GPU's kernels index rows, columns and
  // sketch widths with 32-bit integers (element offsets are 64-bit)
  const long long lim = 2147483647LL;
  if ((long long)p.nrow > lim || (long long)p.ncol > lim || (long long)p.dim_sketch_total > lim)
    fail(kErrUnsupported, "sizes beyond 2^31 - 1 rows, columns or sketch columns are not supported on one GPU");
}

template <class T>
struct TypeName;
template <>
struct TypeName<float> { static constexpr const char *name = "Real Single"; };
template <>
struct TypeName<double> { static constexpr const char *name = "Real Double"; };

// ============================================================================ marshalling
// A caller matrix region: `outer` lines of `inner` contiguous elements, line stride `ld`.
template <class T>
struct View {
  T *d = nullptr;
  DBuf<T> own;
  T *host = nullptr;
  long long inner = 0, outer = 0, ld = 0;

  void bind(const T *p, long long inner_, long long outer_, long long ld_, bool copy_in, cudaStream_t st) {
    inner = inner_; outer = outer_; ld = ld_;
    if (p == nullptr || inner <= 0 || outer <= 0) { d = const_cast<T *>(p); return; }
    if (is_device_pointer(p)) { d = const_cast<T *>(p); return; }
    host = const_cast<T *>(p);
    own.alloc((size_t)((outer - 1) * ld + inner));
    d = own.p;
    if (copy_in)
      CK(cudaMemcpy2DAsync(d, ld * sizeof(T), p, ld * sizeof(T), inner * sizeof(T), outer, cudaMemcpyHostToDevice,
                           st));
  }
  // Copy `cols` leading elements of each line back to the host buffer.
  void back(cudaStream_t st, long long cols = -1) {
    if (!host) return;
    if (cols < 0) cols = inner;
    CK(cudaMemcpy2DAsync(host, ld * sizeof(T), d, ld * sizeof(T), cols * sizeof(T), outer, cudaMemcpyDeviceToHost,
                         st));
  }
};

// Out of core: rows per streamed panel of a host A (ml x n held by this rank), or 0 when A fits on
// the device beside the solve's other buffers (Y, Qbar, the Nl x Nl and n x l FP64 work) and is
// copied whole.  MIXED keeps A as bf16 planes instead of the FP32/FP64 copy.
template <class T>
long long plan_a_panels(const T *a, long long ml, long long n, long long Nl, long long l, bool mixed) {
  if (a == nullptr || ml <= 0 || n <= 0 || is_device_pointer(a)) return 0;
  const size_t s = sizeof(T), pld = (size_t)plane_ld(n);
  const size_t resident = mixed ? (size_t)plane_rows(ml) * pld * 2 * sketch_planes() : (size_t)ml * n * s;
  const size_t row_bytes = 2 * (size_t)n * s + (mixed ? pld * 2 * 3 : 0);  // two staging rows + planes
  const size_t work = (size_t)ml * Nl * s * 3 + (size_t)ml * l * s * 4 + (size_t)Nl * Nl * 8 * 4 +
                      (size_t)n * l * 8 * 4 + (size_t)n * Nl * s + ((size_t)64 << 20);
  return host_panel_rows(ml, n, resident, row_bytes, work, s);
}

struct Ctx {
  StageCtx sc;
  explicit Ctx(int precision) {
    Runtime &rt = Runtime::get();
    sc.st = rt.stream;
    sc.precision = precision < 0 ? default_precision() : precision;
    sc.status = reinterpret_cast<int *>(rt.ctl + 16);
    CK(cudaMemsetAsync(sc.status, 0, sizeof(int), sc.st));
  }
};

// ============================================================================ stages
// Sketching (reference core/stage/@x@_sketch_gaussian_projection.c:46-84, @x@_sketch.h).
template <class T>
void sketch_api(const isvd_Param &p, const T *argv, isvd_int_t argc, T *retv, isvd_int_t retc, char dista,
                char ordera, const T *a, isvd_int_t lda, const T *omega, isvd_int_t ldomega, T *yst,
                isvd_int_t ldyst, isvd_int_t seed, int precision) {
  if (argc > 0) REQUIRE(argv != nullptr);
  if (retc > 0) REQUIRE(retv != nullptr);
  if (argc < 0) return;
  const char dista_ = arg2char("DISTA", dista, "CR");
  const char ordera_ = arg2char("ORDERA", ordera, "CR");
  require_single_rank(p);
  // several ranks: row blocks hold rows [rowidxbegin, rowidxend) of A, column blocks (dista 'C') all
  // rows and columns [colidxbegin, colidxend); either way this rank's rows of Y are returned
  const bool colblk = p.mpi_size > 1 && dista_ == 'C';
  const int m = p.mpi_size > 1 ? (int)p.nrow_proc : (int)p.nrow, n = p.ncol, Nl = p.dim_sketch_total;
  const int arows = colblk ? (int)p.nrow : m, acols = colblk ? (int)p.ncol_proc : n;
  if (dista_ == 'C') {
    REQUIRE(ordera_ == 'C' ? lda >= p.nrow : lda >= p.ncol_proc);
    REQUIRE(ldyst == Nl);
  } else {
    REQUIRE(ordera_ == 'C' ? lda >= p.nrow_proc : lda >= n);
    REQUIRE(ldyst >= Nl);
  }
  if (omega) REQUIRE(ldomega >= Nl);
  Ctx c(precision);
  if (colblk) {
    c.sc.col_begin = p.colidxbegin;
    c.sc.a_cols = acols;
  }
  View<T> A, Om, Y;
  c.sc.a_panel_rows = plan_a_panels<T>(a, arows, acols, Nl, p.dim_sketch, c.sc.precision == kMixed);
  if (c.sc.a_panel_rows == 0) {  // otherwise a host A is streamed in row panels by the sketch
    if (ordera_ == 'R') A.bind(a, acols, arows, lda, true, c.sc.st);
    else A.bind(a, arows, acols, lda, true, c.sc.st);
  }
  if (omega) Om.bind(omega + (colblk ? (size_t)p.colidxbegin * ldomega : 0), Nl, acols, ldomega, true, c.sc.st);
  Y.bind(yst, Nl, m, ldyst, false, c.sc.st);
  const T *a_use = c.sc.a_panel_rows ? a : A.d;
  if (colblk) {  // Y = sum over the ranks of A_j Omega_j, then this rank's rows (@x@_sketch.h:82)
    DBuf<T> Yf((size_t)arows * Nl);
    sketch_dev<T>(c.sc, arows, acols, Nl, ordera_, a_use, lda, omega ? Om.d : nullptr, ldomega,
                  (uint64_t)(uint32_t)seed, Yf.p, Nl);
    allreduce_sum(Yf.p, (size_t)arows * Nl, c.sc.st);
    CK(cudaMemcpyAsync(Y.d, Yf.p + (size_t)p.rowidxbegin * Nl, (size_t)m * Nl * sizeof(T), cudaMemcpyDeviceToDevice,
                       c.sc.st));
    Y.back(c.sc.st);
    sync();
    return;
  }
  sketch_dev<T>(c.sc, m, n, Nl, ordera_, a_use, lda, omega ? Om.d : nullptr, ldomega, (uint64_t)(uint32_t)seed, Y.d,
                ldyst);
  Y.back(c.sc.st);
  sync();
}

template <class T>
void orth_api(const isvd_Param &p, const T *argv, isvd_int_t argc, T *retv, isvd_int_t retc, T *yst,
              isvd_int_t ldyst, bool tsqr) {
  if (argc > 0) REQUIRE(argv != nullptr);
  if (retc > 0) REQUIRE(retv != nullptr);
  if (argc < 0) return;
  require_single_rank(p);
  const int m = p.nrow_proc, l = p.dim_sketch, N = p.num_sketch, Nl = p.dim_sketch_total;
  REQUIRE(ldyst >= Nl);
  if (tsqr) REQUIRE(p.nrow >= l);
  Ctx c(-1);
  if (p.mpi_size > 1) c.sc.m_total = p.nrow;
  View<T> Y;
  Y.bind(yst, Nl, m, ldyst, true, c.sc.st);
  if (tsqr) orth_tsqr_dev<T>(c.sc, m, l, N, Y.d, ldyst);
  else orth_gramian_dev<T>(c.sc, m, l, N, Y.d, ldyst);
  Y.back(c.sc.st);
  sync();
}

template <class T>
void query_kn(T *retv, isvd_int_t retc) {
  int i = -1;
  if (retc > ++i) retv[i] = (T)256;
  if (retc > ++i) retv[i] = (T)1e-4;
}

template <class T>
void query_wy(T *retv, isvd_int_t retc) {
  const double d[9] = {256, 1e-3, 1.0, 1e14, 1e-14, 20, 0.5, 1e-4, 0.85};
  for (int i = 0; i < 9 && i < retc; ++i) retv[i] = (T)d[i];
}

template <class T>
void integrate_api(const isvd_Param &p, const T *argv, isvd_int_t argc, T *retv, isvd_int_t retc, T *yst,
                   isvd_int_t ldyst, T *qt, isvd_int_t ldqt, int alg) {
  if (argc > 0) REQUIRE(argv != nullptr);
  if (retc > 0) REQUIRE(retv != nullptr);
  if (argc < 0) {
    if (alg == 0) query_kn(retv, retc);
    if (alg == 1) query_wy(retv, retc);
    return;
  }
  require_single_rank(p);
  const int m = p.nrow_proc, l = p.dim_sketch, N = p.num_sketch, Nl = p.dim_sketch_total;
  REQUIRE(ldyst >= Nl);
  REQUIRE(ldqt >= l);
  Ctx c(-1);
  View<T> Y, Q;
  Y.bind(yst, Nl, m, ldyst, true, c.sc.st);
  Q.bind(qt, l, m, ldqt, false, c.sc.st);
  IterResult r;
  if (alg == 0) {
    int ai = -1;
    const int maxit = (argc > ++ai) ? (int)argv[ai] : 256;
    const double tol = (argc > ++ai) ? (double)argv[ai] : 1e-4;
    REQUIRE(maxit >= 0);
    REQUIRE(tol >= 0);
    r = integrate_kn_dev<T>(c.sc, m, l, N, Y.d, ldyst, Q.d, ldqt, maxit, tol);
  } else if (alg == 1) {
    WyArgs w;
    int ai = -1;
    if (argc > ++ai) w.maxit = (int)argv[ai];
    if (argc > ++ai) w.tol = argv[ai];
    if (argc > ++ai) w.tau0 = argv[ai];
    if (argc > ++ai) w.taumax = argv[ai];
    if (argc > ++ai) w.taumin = argv[ai];
    if (argc > ++ai) w.taumaxit = (int)argv[ai];
    if (argc > ++ai) w.beta = argv[ai];
    if (argc > ++ai) w.sigma = argv[ai];
    if (argc > ++ai) w.eta = argv[ai];
    REQUIRE(w.maxit >= 0 && w.tol >= 0 && w.tau0 >= 0 && w.taumax >= 0 && w.taumin >= 0 && w.taumaxit >= 0);
    REQUIRE(w.beta > 0 && w.beta < 1 && w.sigma > 0 && w.sigma < 1 && w.eta > 0 && w.eta < 1);
    r = integrate_wy_dev<T>(c.sc, m, l, N, Y.d, ldyst, Q.d, ldqt, w);
  } else {
    integrate_hr_dev<T>(c.sc, m, l, N, Y.d, ldyst, Q.d, ldqt);
    Y.back(c.sc.st);  // the reference overwrites yst
  }
  Q.back(c.sc.st);
  sync();
  if (alg != 2) {
    int ri = -1;
    if (retc > ++ri) retv[ri] = (T)r.iterations;
    if (retc > ++ri) retv[ri] = (T)r.error;
  }
}

// Postprocessing (reference @x@_postprocess_{gramian,tall_skinny_qr,symmetric}.c).  alg 0 GR, 1 TS, 2 SY.
template <class T>
void post_api(const isvd_Param &p, const T *argv, isvd_int_t argc, T *retv, isvd_int_t retc, char dista,
              char ordera, const T *a, isvd_int_t lda, const T *qt, isvd_int_t ldqt, T *s, T *ut, isvd_int_t ldut,
              T *vt, isvd_int_t ldvt, mpi_int_t ut_root, mpi_int_t vt_root, int alg, int precision) {
  if (argc > 0) REQUIRE(argv != nullptr);
  if (retc > 0) REQUIRE(retv != nullptr);
  if (argc < 0) return;
  const char dista_ = arg2char("DISTA", dista, "CR");
  const char ordera_ = arg2char("ORDERA", ordera, "CR");
  require_single_rank(p);
  if (p.mpi_size > 1) fail(kErrUnsupported, "several ranks: postprocessing runs inside isvd_?Isvd (the driver)");
  const int m = p.nrow, n = p.ncol, k = p.rank, l = p.dim_sketch;
  if (alg == 2) {
    // symmetric: U and V are the same matrix; the first requested one is computed (:101-104)
    REQUIRE(p.nrow_proc == p.ncol_proc);
    const mpi_int_t r = (ut_root >= -1) ? ut_root : vt_root;
    const isvd_int_t ld = (ut_root >= -1) ? ldut : ldvt;
    if (r >= 0) REQUIRE(ld == l);
    else if (r == -1) REQUIRE(ld >= l);
  } else {
    if (ut_root >= 0) REQUIRE(ldut == l);
    else if (ut_root == -1) REQUIRE(ldut >= l);
    if (vt_root >= 0) REQUIRE(ldvt == l);
    else if (vt_root == -1) REQUIRE(ldvt >= l);
  }
  if (dista_ == 'C') {
    REQUIRE(ordera_ == 'C' ? lda >= m : lda >= p.ncol_proc);
    REQUIRE(ldqt == l);
  } else {
    REQUIRE(ordera_ == 'C' ? lda >= p.nrow_proc : lda >= n);
    REQUIRE(ldqt >= l);
  }
  if (alg == 1) REQUIRE(n >= l);
  Ctx c(precision);
  View<T> A, Q, S, U, V;
  c.sc.a_panel_rows = plan_a_panels<T>(a, m, n, 0, l, c.sc.precision == kMixed);
  if (c.sc.a_panel_rows == 0) {  // otherwise a host A is streamed in row panels by the projection
    if (ordera_ == 'R') A.bind(a, n, m, lda, true, c.sc.st);
    else A.bind(a, m, n, lda, true, c.sc.st);
  }
  const T *a_use = c.sc.a_panel_rows ? a : A.d;
  Q.bind(qt, l, m, ldqt, true, c.sc.st);
  S.bind(s, l, 1, l, false, c.sc.st);
  if (alg == 2) {
    const bool wu = ut_root >= -1 || vt_root >= -1;
    T *u = (ut_root >= -1) ? ut : vt;
    const isvd_int_t ld = (ut_root >= -1) ? ldut : ldvt;
    U.bind(u, k, m, ld, false, c.sc.st);
    post_symmetric_dev<T>(c.sc, m, n, k, l, ordera_, a_use, lda, Q.d, ldqt, S.d, U.d, ld, wu);
    S.back(c.sc.st);
    if (wu) U.back(c.sc.st, k);
    if (ut_root >= -1 && vt_root >= -1) {
      // the reference copies U into V as well (:162-164)
      View<T> V2;
      V2.bind(vt, k, m, ldvt, false, c.sc.st);
      CK(cudaMemcpy2DAsync(V2.d, ldvt * sizeof(T), U.d, ld * sizeof(T), k * sizeof(T), m, cudaMemcpyDeviceToDevice,
                           c.sc.st));
      V2.back(c.sc.st, k);
      sync();
    }
    sync();
    return;
  }
  const bool wu = ut_root >= -1, wv = vt_root >= -1;
  const int vcols = (alg == 1) ? l : k;
  if (wu) U.bind(ut, k, m, ldut, false, c.sc.st);
  if (wv) V.bind(vt, vcols, n, ldvt, false, c.sc.st);
  if (alg == 0)
    post_gramian_dev<T>(c.sc, m, n, k, l, ordera_, a_use, lda, Q.d, ldqt, S.d, U.d, ldut, V.d, ldvt, wu, wv);
  else
    post_tsqr_dev<T>(c.sc, m, n, k, l, ordera_, a_use, lda, Q.d, ldqt, S.d, U.d, ldut, V.d, ldvt, wu, wv);
  S.back(c.sc.st);
  if (wu) U.back(c.sc.st, k);
  if (wv) V.back(c.sc.st, vcols);
  sync();
}

// ============================================================================ driver
const char *const kOptsS[] = {"GP", "GP_gpu"};
const char *const kOptsO[] = {"TS", "GR", "TS_gpu", "GR_gpu"};
const char *const kOptsI[] = {"KN", "WY", "HR", "KN_gpu", "WY_gpu", "HR_gpu"};
const char *const kOptsP[] = {"TS", "GR", "SY", "TS_gpu", "GR_gpu", "SY_gpu"};

std::string base(const char *sel) {
  std::string s(sel);
  const size_t u = s.find('_');
  return u == std::string::npos ? s : s.substr(0, u);
}

const char *alg_name(char stage, const std::string &b, bool gpu) {
  static thread_local std::string out;
  const char *what = "";
  if (stage == 'S') what = "Gaussian Projection Sketching";
  if (stage == 'O') what = (b == "TS") ? "Tall-Skinny QR Orthogonalization" : "Gramian Orthogonalization";
  if (stage == 'I')
    what = (b == "KN") ? "Kolmogorov-Nagumo Integration"
                       : (b == "WY") ? "Wen-Yin Integration" : "Hierarchical Reduction Integration";
  if (stage == 'P')
    what = (b == "TS") ? "Tall-Skinny QR Postprocessing"
                       : (b == "GR") ? "Gramian Postprocessing" : "Symmetric Postprocessing";
  out = std::string(gpu ? "GPU " : "") + what;
  return out.c_str();
}

struct StageTimer {
  cudaEvent_t ev[5];
  StageTimer() { for (auto &e : ev) CK(cudaEventCreate(&e)); }
  ~StageTimer() { for (auto &e : ev) cudaEventDestroy(e); }
  void mark(int i, cudaStream_t st) { CK(cudaEventRecord(ev[i], st)); }
  double sec(int i) {
    float ms = 0.f;
    CK(cudaEventElapsedTime(&ms, ev[i], ev[i + 1]));
    return ms * 1e-3;
  }
};

template <class T>
void driver(const isvd_Param &p, const char *alg_s, const char *alg_o, const char *alg_i, const char *alg_p,
            const T *argv[4], const isvd_int_t argc[4], T *retv[4], const isvd_int_t retc[4], double time[4],
            FILE *stream, char dista, char ordera, const T *a, isvd_int_t lda, T *s, T *ut, isvd_int_t ldut, T *vt,
            isvd_int_t ldvt, isvd_int_t seed, mpi_int_t ut_root, mpi_int_t vt_root, const T *omega,
            isvd_int_t ldomega, int precision) {
  // Selectors (reference core/driver/@x@_isvd.c:135-149)
  const std::string bs = base(arg2str("ALG_S", alg_s, kOptsS, 2));
  const std::string bo = base(arg2str("ALG_O", alg_o, kOptsO, 4));
  const std::string bi = base(arg2str("ALG_I", alg_i, kOptsI, 6));
  const std::string bp = base(arg2str("ALG_P", alg_p, kOptsP, 6));
  (void)bs;
  const T *av[4] = {nullptr, nullptr, nullptr, nullptr};
  isvd_int_t ac[4] = {0, 0, 0, 0};
  T *rv[4] = {nullptr, nullptr, nullptr, nullptr};
  isvd_int_t rc[4] = {0, 0, 0, 0};
  for (int i = 0; i < 4; ++i) {
    if (argv) { av[i] = argv[i]; ac[i] = argc[i]; }
    if (retv) { rv[i] = retv[i]; rc[i] = retc[i]; }
    if (ac[i] > 0) REQUIRE(av[i] != nullptr);
    if (rc[i] > 0) REQUIRE(rv[i] != nullptr);
  }
  // Default-argument query (:199-218): only the integration stages have defaults.
  bool query = false;
  for (int i = 0; i < 4; ++i) query |= ac[i] < 0;
  if (query) {
    if (ac[2] < 0) {
      if (bi == "KN") query_kn(rv[2], rc[2]);
      if (bi == "WY") query_wy(rv[2], rc[2]);
    }
    return;
  }
  const char dista_ = arg2char("DISTA", dista, "CR");
  const char ordera_ = arg2char("ORDERA", ordera, "CR");
  require_single_rank(p);
  const int m = p.nrow, n = p.ncol, k = p.rank, l = p.dim_sketch, N = p.num_sketch, Nl = p.dim_sketch_total;
  const bool root = p.mpi_rank == p.mpi_root;
  // several ranks (isvd_gpu_set_allreduce): this rank holds rows [rowidxbegin, rowidxend) of A
  const bool multi = p.mpi_size > 1;
  const int ml = multi ? (int)p.nrow_proc : m;  // rows of A held here
  if (stream && root) {
    const char *tn = TypeName<T>::name;
    fprintf(stream, "Using %s Precision %s.\n", tn, alg_name('S', "GP", true));
    fprintf(stream, "Using %s Precision %s.\n", tn, alg_name('O', bo, true));
    fprintf(stream, "Using %s Precision %s.\n", tn, alg_name('I', bi, true));
    fprintf(stream, "Using %s Precision %s.\n", tn, alg_name('P', bp, true));
    fprintf(stream, "\n");
  }
  // Argument checks of the stages (sketch / postprocess), done up front
  if (dista_ == 'C') REQUIRE(ordera_ == 'C' ? lda >= m : lda >= p.ncol_proc);
  else REQUIRE(ordera_ == 'C' ? lda >= p.nrow_proc : lda >= n);
  if (ut_root >= 0) REQUIRE(ldut == l); else if (ut_root == -1) REQUIRE(ldut >= l);
  if (vt_root >= 0) REQUIRE(ldvt == l); else if (vt_root == -1) REQUIRE(ldvt >= l);
  if (bo == "TS") REQUIRE(m >= l);
  if (bp == "TS") REQUIRE(n >= l);
  if (bp == "SY") REQUIRE(m == n);
  if (omega) REQUIRE(ldomega >= Nl);

  Ctx c(precision);
  cudaStream_t st = c.sc.st;
  MixedCache mcache;  // A's bf16 planes, shared by the sketch and the postprocess
  c.sc.cache = &mcache;
  // column blocks over several ranks (dista 'C'): A holds all m rows and this rank's columns; Y is
  // summed over the ranks and each keeps its row block, so that the orthogonalization and the
  // integration run on row blocks as with dista 'R'
  const bool colblk = multi && dista_ == 'C';
  const int arows = colblk ? m : ml, acols = colblk ? (int)p.ncol_proc : n;  // A held here
  if (multi) {
    c.sc.m_total = m;
    c.sc.row_begin = p.rowidxbegin;
  }
  if (colblk) {
    c.sc.col_begin = p.colidxbegin;
    c.sc.a_cols = acols;
  }
  StageTimer tm;
  auto progress = [&](const char *what) {
    if (stream && root) { fprintf(stream, "%s", what); fflush(stream); }
  };
  auto done = [&]() {
    if (stream && root) { fprintf(stream, "done.\n"); fflush(stream); }
  };

  // ---- sketch (includes moving A to the device when it is on the host)
  progress("Sketching ..................... ");
  tm.mark(0, st);
  // MIXED precision streams a host A through the device in panels inside the sketch and keeps
  // only its bf16 planes (reused by the postprocess); NATIVE precision copies A once.
  const bool mixed = c.sc.precision == kMixed;
  // out of core: a host A that does not fit beside the solve's buffers is streamed in row panels
  // by the sketch and again by the projection
  c.sc.a_panel_rows = plan_a_panels<T>(a, arows, acols, Nl, l, mixed);
  View<T> A, Om;
  if (!mixed && c.sc.a_panel_rows == 0) {
    if (ordera_ == 'R') A.bind(a, acols, arows, lda, true, st);
    else A.bind(a, arows, acols, lda, true, st);
  }
  const T *a_use = (mixed || c.sc.a_panel_rows > 0) ? a : A.d;
  // Omega passed in: all n rows; column blocks use the rows of their own columns
  if (omega) Om.bind(omega + (colblk ? (size_t)p.colidxbegin * ldomega : 0), Nl, acols, ldomega, true, st);
  DBuf<T> Y((size_t)ml * Nl), Q((size_t)ml * l);
  // MIXED GP / GR / (KN | WY) on one process: the sketch and the Gramian apply hand their outputs
  // to the next stage as bf16 planes (what that stage would split them into), so Y and Qs are never
  // written as values nor split again (ISVD_GPU_PLANE_HANDOFF=0 keeps the values)
  PlaneHandoff hand;
  struct HandoffScope {
    StageCtx &sc;
    ~HandoffScope() { sc.handoff = nullptr; }
  } hand_scope{c.sc};
  {
    const char *e = getenv("ISVD_GPU_PLANE_HANDOFF");
    if (mixed && !multi && bo == "GR" && (bi == "KN" || bi == "WY") && l % 64 == 0 && handoff_shape_ok(Nl) &&
        !(e && atoi(e) == 0))
      c.sc.handoff = &hand;
  }
  if (colblk) {  // Y = sum over the ranks of A_j Omega_j, then this rank's rows (reference
    DBuf<T> Yf((size_t)m * Nl);  // MPI_Reduce_scatter_block, @x@_sketch.h:82)
    sketch_dev<T>(c.sc, m, acols, Nl, ordera_, a_use, lda, omega ? Om.d : nullptr, ldomega, (uint64_t)(uint32_t)seed,
                  Yf.p, Nl);
    allreduce_sum(Yf.p, (size_t)m * Nl, st);
    CK(cudaMemcpyAsync(Y.p, Yf.p + (size_t)p.rowidxbegin * Nl, (size_t)ml * Nl * sizeof(T), cudaMemcpyDeviceToDevice,
                       st));
    sync();
  } else {
    sketch_dev<T>(c.sc, ml, n, Nl, ordera_, a_use, lda, omega ? Om.d : nullptr, ldomega, (uint64_t)(uint32_t)seed,
                  Y.p, Nl);
  }
  tm.mark(1, st);
  sync();
  done();
  // ---- orthogonalize
  progress("Orthogonalizing ............... ");
  if (bo == "TS") {
    orth_tsqr_dev<T>(c.sc, ml, l, N, Y.p, Nl);
    // MIXED: KN and WY re-orthonormalize the blocks in the coordinates of G (G_ii = I exactly),
    // removing what the tensor-core CholeskyQR leaves of non-orthogonality
    c.sc.deferred_orth = (bi == "KN" || bi == "WY");
  } else {
    // KN and WY form G = Qs' Qs anyway: they take over the second pass in the coordinates of G
    c.sc.deferred_orth = (bi == "KN" || bi == "WY");
    // KN, WY and HR are equivariant under Q_i -> Q_i R_i and GR / SY postprocessing is invariant,
    // so the blocks' bases are free: Cholesky factors instead of eigendecompositions.  (The TS
    // postprocessing of the reference depends on the basis of Qbar, so it keeps the eigenbasis.)
    c.sc.chol_basis = (bp != "TS");
    orth_gramian_dev<T>(c.sc, ml, l, N, Y.p, Nl);
    c.sc.chol_basis = false;
  }
  tm.mark(2, st);
  sync();
  done();
  // ---- integrate
  progress("Integrating ................... ");
  IterResult ir;
  if (bi == "KN") {
    int ai = -1;
    const int maxit = (ac[2] > ++ai) ? (int)av[2][ai] : 256;
    const double tol = (ac[2] > ++ai) ? (double)av[2][ai] : 1e-4;
    REQUIRE(maxit >= 0 && tol >= 0);
    ir = integrate_kn_dev<T>(c.sc, ml, l, N, Y.p, Nl, Q.p, l, maxit, tol);
  } else if (bi == "WY") {
    WyArgs w;
    int ai = -1;
    const T *x = av[2];
    if (ac[2] > ++ai) w.maxit = (int)x[ai];
    if (ac[2] > ++ai) w.tol = x[ai];
    if (ac[2] > ++ai) w.tau0 = x[ai];
    if (ac[2] > ++ai) w.taumax = x[ai];
    if (ac[2] > ++ai) w.taumin = x[ai];
    if (ac[2] > ++ai) w.taumaxit = (int)x[ai];
    if (ac[2] > ++ai) w.beta = x[ai];
    if (ac[2] > ++ai) w.sigma = x[ai];
    if (ac[2] > ++ai) w.eta = x[ai];
    ir = integrate_wy_dev<T>(c.sc, ml, l, N, Y.p, Nl, Q.p, l, w);
  } else {
    integrate_hr_dev<T>(c.sc, ml, l, N, Y.p, Nl, Q.p, l);
  }
  c.sc.handoff = nullptr;
  tm.mark(3, st);
  sync();
  done();
  if (bi != "HR") {
    int ri = -1;
    if (rc[2] > ++ri) rv[2][ri] = (T)ir.iterations;
    if (rc[2] > ++ri) rv[2][ri] = (T)ir.error;
  }
  // ---- postprocess
  progress("Postprocessing ................ ");
  View<T> S, U, V;
  S.bind(s, l, 1, l, false, st);
  if (bp == "SY" && !multi) {
    const bool wu = ut_root >= -1 || vt_root >= -1;
    T *u = (ut_root >= -1) ? ut : vt;
    const isvd_int_t ld = (ut_root >= -1) ? ldut : ldvt;
    U.bind(u, k, m, ld, false, st);
    post_symmetric_dev<T>(c.sc, m, n, k, l, ordera_, a_use, lda, Q.p, l, S.d, U.d, ld, wu);
    tm.mark(4, st);
    S.back(st);
    if (wu) U.back(st, k);
    if (ut_root >= -1 && vt_root >= -1) {
      View<T> V2;
      V2.bind(vt, k, m, ldvt, false, st);
      CK(cudaMemcpy2DAsync(V2.d, ldvt * sizeof(T), U.d, ld * sizeof(T), k * sizeof(T), m, cudaMemcpyDeviceToDevice,
                           st));
      V2.back(st, k);
      sync();
    }
  } else if (multi) {
    // row blocks: U rows of this rank; V (all n rows) is the same on every rank.  Symmetric: U and
    // V are the same matrix (reference @x@_postprocess_symmetric.c:101-104, 170-191)
    const bool sy = bp == "SY";
    const bool wu = ut_root >= -1 || (sy && vt_root >= -1), wv = !sy && vt_root >= -1;
    const int vcols = (bp == "TS") ? l : k;  // TS: all l columns of V (@x@_postprocess_tall_skinny_qr.c:286)
    DBuf<T> Ul((size_t)ml * l), Vf((size_t)n * l);
    if (bp == "GR")
      post_gramian_dev<T>(c.sc, ml, n, k, l, ordera_, a_use, lda, Q.p, l, S.d, Ul.p, l, Vf.p, l, wu, wv);
    else if (bp == "TS")
      post_tsqr_dev<T>(c.sc, ml, n, k, l, ordera_, a_use, lda, Q.p, l, S.d, Ul.p, l, Vf.p, l, wu, wv);
    else
      post_symmetric_dev<T>(c.sc, ml, n, k, l, ordera_, a_use, lda, Q.p, l, S.d, Ul.p, l, wu);
    tm.mark(4, st);
    S.back(st);
    // U: this rank's rows, and all rows at the root (reference MPI_Gather,
    // @x@_postprocess_gramian.c:162-165) through a sum of zero-padded copies of the ranks' rows
    auto emit_u = [&](T *out, isvd_int_t ld, mpi_int_t root) {
      View<T> Uo;
      if (root < 0 || root != p.mpi_rank) {  // this rank's rows only
        Uo.bind(out, k, ml, ld, false, st);
        CK(cudaMemcpy2DAsync(Uo.d, ld * sizeof(T), Ul.p, l * sizeof(T), k * sizeof(T), ml, cudaMemcpyDeviceToDevice,
                             st));
        Uo.back(st, k);
      }
      if (root >= 0) {
        DBuf<T> Ug((size_t)m * l);
        CK(cudaMemsetAsync(Ug.p, 0, (size_t)m * l * sizeof(T), st));
        CK(cudaMemcpyAsync(Ug.p + (size_t)p.rowidxbegin * l, Ul.p, (size_t)ml * l * sizeof(T),
                           cudaMemcpyDeviceToDevice, st));
        allreduce_sum(Ug.p, (size_t)m * l, st);
        if (root == p.mpi_rank) {
          View<T> Ua;
          Ua.bind(out, k, m, ld, false, st);
          CK(cudaMemcpy2DAsync(Ua.d, ld * sizeof(T), Ug.p, l * sizeof(T), k * sizeof(T), m, cudaMemcpyDeviceToDevice,
                               st));
          Ua.back(st, k);
        }
      }
      sync();
    };
    if (ut_root >= -1) emit_u(ut, ldut, ut_root);
    if (sy && vt_root >= -1) emit_u(vt, ldvt, vt_root);
    if (wv) {  // this rank's column block; all rows at the root (reference MPI_Gather, :176-183)
      const bool all = vt_root >= 0 && vt_root == p.mpi_rank;
      const long long v0 = all ? 0 : (long long)p.colidxbegin;
      const long long vn = all ? (long long)n : (long long)p.ncol_proc;
      V.bind(vt, vcols, vn, ldvt, false, st);
      CK(cudaMemcpy2DAsync(V.d, ldvt * sizeof(T), Vf.p + v0 * l, l * sizeof(T), vcols * sizeof(T), vn,
                           cudaMemcpyDeviceToDevice, st));
      V.back(st, vcols);
    }
  } else {
    const bool wu = ut_root >= -1, wv = vt_root >= -1;
    const int vcols = (bp == "TS") ? l : k;
    if (wu) U.bind(ut, k, m, ldut, false, st);
    if (wv) V.bind(vt, vcols, n, ldvt, false, st);
    if (bp == "GR")
      post_gramian_dev<T>(c.sc, m, n, k, l, ordera_, a_use, lda, Q.p, l, S.d, U.d, ldut, V.d, ldvt, wu, wv);
    else
      post_tsqr_dev<T>(c.sc, m, n, k, l, ordera_, a_use, lda, Q.p, l, S.d, U.d, ldut, V.d, ldvt, wu, wv);
    tm.mark(4, st);
    S.back(st);
    if (wu) U.back(st, k);
    if (wv) V.back(st, vcols);
  }
  sync();
  done();
  if (time) for (int i = 0; i < 4; ++i) time[i] = tm.sec(i);
}

}  // namespace

// ============================================================================ exported C ABI
namespace {

// Batched iSVD (isvd/b200.h).
template <class T>
isvd_gpu_batch *batch_create_api(isvd_int_t count, const isvd_int_t *m, const isvd_int_t *n, const isvd_int_t *k,
                                 const isvd_int_t *p, isvd_int_t N) {
  BatchPlan *plan = nullptr;
  api_call([&] {
    REQUIRE(count > 0 && m && n && k && p && N > 0);
    std::vector<int> mm(count), nn(count), kk(count), pp(count);
    for (isvd_int_t b = 0; b < count; ++b) {
      mm[b] = (int)m[b]; nn[b] = (int)n[b]; kk[b] = (int)k[b]; pp[b] = (int)p[b];
    }
    plan = batch_plan_create<T>((int)count, mm.data(), nn.data(), kk.data(), pp.data(), (int)N);
  });
  return reinterpret_cast<isvd_gpu_batch *>(plan);
}

template <class T>
int batch_isvd_api(isvd_gpu_batch *batch, const T *const *a, const isvd_int_t *lda, T *const *s, T *const *ut,
                   const isvd_int_t *ldut, T *const *vt, const isvd_int_t *ldvt, const isvd_int_t *seed, const T *argv,
                   isvd_int_t argc, isvd_int_t *iterations, T *errors) {
  return api_call([&] {
    REQUIRE(batch != nullptr && a && lda && s && ut && ldut && vt && ldvt && seed);
    if (argc > 0) REQUIRE(argv != nullptr);
    BatchPlan *plan = reinterpret_cast<BatchPlan *>(batch);
    if (plan->elem != (int)sizeof(T)) fail(kErrArgument, "batched iSVD: plan created for another element type");
    int ai = -1;
    const int maxit = (argc > ++ai) ? (int)argv[ai] : 256;
    const double tol = (argc > ++ai) ? (double)argv[ai] : 1e-4;
    REQUIRE(maxit >= 0 && tol >= 0);
    const int count = plan_count(plan);
    std::vector<long long> la(count), lu(count), lv(count);
    std::vector<unsigned long long> sd(count);
    for (int b = 0; b < count; ++b) {
      la[b] = lda[b]; lu[b] = ldut[b]; lv[b] = ldvt[b];
      sd[b] = (unsigned long long)(uint32_t)seed[b];  // as the single-solve driver
    }
    std::vector<int> it(count);
    std::vector<double> er(count);
    batch_solve<T>(plan, a, la.data(), s, ut, lu.data(), vt, lv.data(), sd.data(), maxit, tol, it.data(), er.data());
    for (int b = 0; b < count; ++b) {
      if (iterations) iterations[b] = it[b];
      if (errors) errors[b] = (T)er[b];
    }
  });
}

// Adjoint of the truncated SVD (isvd/b200.h).
template <class T>
int adjoint_api(isvd_int_t m, isvd_int_t n, isvd_int_t k, char ordera, const T *a, isvd_int_t lda, const T *s,
                const T *ut, isvd_int_t ldut, const T *vt, isvd_int_t ldvt, const T *ds, const T *dut,
                isvd_int_t lddut, const T *dvt, isvd_int_t lddvt, T *da, isvd_int_t ldda, int cg_iters, double tol,
                int *iterations) {
  int its = 0;
  const int st = api_call([&] {
    const char ordera_ = arg2char("ORDERA", ordera, "CR");
    REQUIRE(m > 0 && n > 0 && k > 0 && k <= m && k <= n);
    REQUIRE(a != nullptr && s != nullptr && ut != nullptr && vt != nullptr && da != nullptr);
    REQUIRE(ordera_ == 'R' ? (lda >= n && ldda >= n) : (lda >= m && ldda >= m));
    REQUIRE(ldut >= k && ldvt >= k);
    if (dut) REQUIRE(lddut >= k);
    if (dvt) REQUIRE(lddvt >= k);
    REQUIRE(cg_iters >= 0 && tol >= 0);
    Ctx c(-1);  // the library precision mode: MIXED puts the FP32 products by A on tensor cores
    cudaStream_t sst = c.sc.st;
    View<T> A, S, U, V, dS, dU, dV, dA;
    if (ordera_ == 'R') {
      A.bind(a, n, m, lda, true, sst);
      dA.bind(da, n, m, ldda, false, sst);
    } else {
      A.bind(a, m, n, lda, true, sst);
      dA.bind(da, m, n, ldda, false, sst);
    }
    S.bind(s, k, 1, k, true, sst);
    U.bind(ut, k, m, ldut, true, sst);
    V.bind(vt, k, n, ldvt, true, sst);
    if (ds) dS.bind(ds, k, 1, k, true, sst);
    if (dut) dU.bind(dut, k, m, lddut, true, sst);
    if (dvt) dV.bind(dvt, k, n, lddvt, true, sst);
    its = svd_adjoint_dev<T>(c.sc, m, n, k, ordera_, A.d, lda, U.d, ldut, S.d, V.d, ldvt, dut ? dU.d : nullptr, lddut,
                             ds ? dS.d : nullptr, dvt ? dV.d : nullptr, lddvt, dA.d, ldda, cg_iters, tol);
    dA.back(sst);
    sync();
  });
  if (iterations) *iterations = its;
  return st;
}

}  // namespace

#pragma GCC visibility push(default)
extern "C" {

size_t isvd_gpu_memory_limit = 0;

int isvd_gpu_get_last_error(void) { return t_last_error; }
const char *isvd_gpu_get_error_string(void) { return t_last_msg.c_str(); }
void isvd_gpu_clear_error(void) { t_last_error = 0; t_last_msg.clear(); }
void isvd_gpu_set_precision(int mode) { set_default_precision(mode == ISVD_GPU_PRECISION_MIXED ? kMixed : kNative); }
int isvd_gpu_get_precision(void) { return default_precision(); }
unsigned long long isvd_gpu_kernel_launch_count(void) { return g_launches.load(); }
void isvd_gpu_set_stream(void *stream) {
  api_call([&] {
    Runtime &rt = Runtime::get();
    rt.stream = stream ? (cudaStream_t)stream : rt.own_stream;
  });
}
void *isvd_gpu_get_stream(void) { return Runtime::initialised() ? (void *)Runtime::get().stream : nullptr; }
void isvd_gpu_profile_enable(int on) { set_profiling(on != 0); }
void isvd_gpu_profile_reset(void) { profile_reset(); }
int isvd_gpu_profile_get(const char *tag, double *ms, unsigned long long *launches, double *flops) {
  return (tag && profile_get(tag, ms, launches, flops)) ? 0 : -1;
}

// ---------------------------------------------------------------- utilities
mpi_int_t isvd_getMpiSize(const isvd_MpiComm comm) {
  // ranks joined by isvd_gpu_set_allreduce (a join from a communicator defers to that communicator)
  if (collective().nranks > 1 && !collective().from_comm) return collective().nranks;
  int s = 0;
  MPI_Comm_size(comm, &s);
  return s;
}
mpi_int_t isvd_getMpiRank(const isvd_MpiComm comm) {
  if (collective().nranks > 1 && !collective().from_comm) return collective().rank;
  int r = 0;
  MPI_Comm_rank(comm, &r);
  return r;
}
void isvd_gpu_set_allreduce(isvd_gpu_allreduce_fn fn, void *user, int nranks, int rank, int on_device) {
  api_call([&] {
    REQUIRE(nranks >= 1 && rank >= 0 && rank < nranks);
    Collective &c = collective();
    if (!fn || nranks == 1) {
      c = Collective();
      return;
    }
    c.fn = fn;
    c.user = user;
    c.nranks = nranks;
    c.rank = rank;
    c.on_device = on_device ? 1 : 0;
    c.from_comm = false;
  });
}

static void *aligned64(size_t bytes) {
  void *p = nullptr;
  if (bytes == 0) bytes = 64;
  if (posix_memalign(&p, 64, bytes) != 0) return nullptr;
  return p;
}
isvd_int_t *isvd_iMalloc(const size_t num) { return (isvd_int_t *)aligned64(num * sizeof(isvd_int_t)); }
isvd_s_val_t *isvd_sMalloc(const size_t num) { return (isvd_s_val_t *)aligned64(num * sizeof(isvd_s_val_t)); }
isvd_d_val_t *isvd_dMalloc(const size_t num) { return (isvd_d_val_t *)aligned64(num * sizeof(isvd_d_val_t)); }
void isvd_Free(void *ptr) { free(ptr); }
void isvd_iMemset0(isvd_int_t *ptr, const size_t num) { memset(ptr, 0, num * sizeof(*ptr)); }
void isvd_sMemset0(isvd_s_val_t *ptr, const size_t num) { memset(ptr, 0, num * sizeof(*ptr)); }
void isvd_dMemset0(isvd_d_val_t *ptr, const size_t num) { memset(ptr, 0, num * sizeof(*ptr)); }
void isvd_iMemcpy(isvd_int_t *d, const isvd_int_t *s, const size_t num) { memcpy(d, s, num * sizeof(*d)); }
void isvd_sMemcpy(isvd_s_val_t *d, const isvd_s_val_t *s, const size_t num) { memcpy(d, s, num * sizeof(*d)); }
void isvd_dMemcpy(isvd_d_val_t *d, const isvd_d_val_t *s, const size_t num) { memcpy(d, s, num * sizeof(*d)); }

// ---------------------------------------------------------------- environment
// ---------------------------------------------------------------- text I/O, OpenMP queries
void isvd_iFget(FILE *stream, isvd_int_t *varp) {
  long long v = 0;
  if (stream && varp && fscanf(stream, "%lld", &v) == 1) { *varp = (isvd_int_t)v; return; }
  record_error(kErrArgument, "isvd_iFget: no integer could be read");
}
void isvd_sFget(FILE *stream, isvd_s_val_t *varp) {
  if (!(stream && varp && fscanf(stream, "%f", varp) == 1)) record_error(kErrArgument, "isvd_sFget: no value could be read");
}
void isvd_dFget(FILE *stream, isvd_d_val_t *varp) {
  if (!(stream && varp && fscanf(stream, "%lf", varp) == 1)) record_error(kErrArgument, "isvd_dFget: no value could be read");
}
omp_int_t isvd_getOmpMaxSize(void) { return 1; }
omp_int_t isvd_getOmpSize(void) { return 1; }
omp_int_t isvd_getOmpRank(void) { return 0; }

#define ISVD_MTX(x, T)                                                                                          \
  int isvd_##x##MtxRead(const char *path, isvd_int_t *m, isvd_int_t *n, T *a, const isvd_int_t lda,             \
                        const char ordera) {                                                                    \
    return api_call([&] {                                                                                       \
      const MtxInfo h = mtx_read<T>(path, a, lda, ordera);                                                      \
      if (m) *m = (isvd_int_t)h.m;                                                                              \
      if (n) *n = (isvd_int_t)h.n;                                                                              \
    });                                                                                                         \
  }                                                                                                             \
  int isvd_##x##MtxWrite(const char *path, const isvd_int_t m, const isvd_int_t n, const T *a,                  \
                         const isvd_int_t lda, const char ordera) {                                             \
    return api_call([&] { mtx_write<T>(path, m, n, a, lda, ordera); });                                         \
  }
ISVD_MTX(s, float)
ISVD_MTX(d, double)
#undef ISVD_MTX

void isvd_Init_cpu(int *argcp, char ***argvp, const isvd_MpiComm mpi_comm) {
  (void)mpi_comm;
  MPI_Init(argcp, argvp);
}
void isvd_Finalize_cpu(void) { MPI_Finalize(); }
void isvd_PrintEnvironment_cpu(const isvd_MpiComm comm) {
  printf("iSVD %s (B200 implementation %s), %d MPI process(es)\n", ISVD_VERSION, ISVD_B200_VERSION,
         (int)isvd_getMpiSize(comm));
}
void isvd_Init_gpu(int *argcp, char ***argvp, const isvd_MpiComm mpi_comm) {
  (void)argcp; (void)argvp;
  api_call([&] {
    int count = 0;
    CK(cudaGetDeviceCount(&count));
    if (count == 0) fail(kErrCuda, "no CUDA device");
    CK(cudaSetDevice(isvd_getMpiRank(mpi_comm) % count));
    Runtime::get();
  });
}
void isvd_Finalize_gpu(void) {
  api_call([] { Runtime::reset(); });
}
void isvd_PrintEnvironment_gpu(const isvd_MpiComm comm) {
  (void)comm;
  api_call([] {
    Runtime &rt = Runtime::get();
    cudaDeviceProp prop;
    CK(cudaGetDeviceProperties(&prop, rt.device));
    printf("GPU %d: %s, sm_%d%d, %d SMs, %.1f GiB\n\n", rt.device, prop.name, prop.major, prop.minor,
           prop.multiProcessorCount, prop.totalGlobalMem / 1073741824.0);
  });
}

// ---------------------------------------------------------------- parameters
isvd_Param isvd_createParam(const isvd_int_t nrow, const isvd_int_t ncol, const isvd_int_t rank,
                            const isvd_int_t over_rank, const isvd_int_t num_sketch, const mpi_int_t mpi_root,
                            const isvd_MpiComm mpi_comm) {
  const mpi_int_t P = isvd_getMpiSize(mpi_comm), j = isvd_getMpiRank(mpi_comm);
  if (!(nrow > 0 && ncol > 0 && rank > 0 && over_rank >= 0 && num_sketch > 0))
    record_error(kErrArgument, "isvd_createParam: sizes must be positive (nrow, ncol, rank, num_sketch > 0, "
                               "over_rank >= 0)");
  const isvd_int_t mb = (nrow - 1) / P + 1, nb = (ncol - 1) / P + 1;
  isvd_int_t rb = j * mb, re = rb + mb, cb = j * nb, ce = cb + nb;
  if (rb > nrow) rb = nrow;
  if (re > nrow) re = nrow;
  if (cb > ncol) cb = ncol;
  if (ce > ncol) ce = ncol;
  isvd_Param p = {mpi_comm, P, mpi_root, j, nrow, ncol, re - rb, ce - cb, mb, nb, mb * P, nb * P, rb, re, cb, ce,
                  rank, over_rank, rank + over_rank, (rank + over_rank) * num_sketch, num_sketch};
  return p;
}

// ---------------------------------------------------------------- stages
#define ISVD_STAGES(x, T)                                                                                          \
  void isvd_##x##SketchGaussianProjection(const isvd_Param param, const T *argv, const isvd_int_t argc, T *retv,    \
                                          const isvd_int_t retc, const char dista, const char ordera, const T *a,    \
                                          const isvd_int_t lda, T *yst, const isvd_int_t ldyst,                      \
                                          const isvd_int_t seed, const mpi_int_t mpi_root) {                         \
    (void)mpi_root;                                                                                                \
    api_call([&] {                                                                                                 \
      sketch_api<T>(param, argv, argc, retv, retc, dista, ordera, a, lda, nullptr, 0, yst, ldyst, seed, -1);      \
    });                                                                                                            \
  }                                                                                                                \
  void isvd_##x##SketchGaussianProjection_gpu(const isvd_Param param, const T *argv, const isvd_int_t argc,         \
                                              T *retv, const isvd_int_t retc, const char dista, const char ordera, \
                                              const T *a, const isvd_int_t lda, T *yst, const isvd_int_t ldyst,    \
                                              const isvd_int_t seed, const mpi_int_t mpi_root) {                   \
    isvd_##x##SketchGaussianProjection(param, argv, argc, retv, retc, dista, ordera, a, lda, yst, ldyst, seed,     \
                                       mpi_root);                                                                  \
  }                                                                                                                \
  void isvd_##x##SketchGaussianProjectionOmega(const isvd_Param param, const T *argv, const isvd_int_t argc,        \
                                               T *retv, const isvd_int_t retc, const char dista,                   \
                                               const char ordera, const T *a, const isvd_int_t lda,                \
                                               const T *omega, const isvd_int_t ldomega, T *yst,                   \
                                               const isvd_int_t ldyst) {                                           \
    api_call([&] {                                                                                                 \
      if (!omega) fail(kErrArgument, "isvd_" #x "SketchGaussianProjectionOmega: omega is NULL");                   \
      sketch_api<T>(param, argv, argc, retv, retc, dista, ordera, a, lda, omega, ldomega, yst, ldyst, 0, -1);     \
    });                                                                                                            \
  }                                                                                                                \
  void isvd_##x##OrthogonalizeTallSkinnyQr(const isvd_Param param, const T *argv, const isvd_int_t argc, T *retv,   \
                                           const isvd_int_t retc, T *yst, const isvd_int_t ldyst) {                \
    api_call([&] { orth_api<T>(param, argv, argc, retv, retc, yst, ldyst, true); });                                \
  }                                                                                                                \
  void isvd_##x##OrthogonalizeGramian(const isvd_Param param, const T *argv, const isvd_int_t argc, T *retv,        \
                                      const isvd_int_t retc, T *yst, const isvd_int_t ldyst) {                     \
    api_call([&] { orth_api<T>(param, argv, argc, retv, retc, yst, ldyst, false); });                               \
  }                                                                                                                \
  void isvd_##x##IntegrateKolmogorovNagumo(const isvd_Param param, const T *argv, const isvd_int_t argc, T *retv,   \
                                           const isvd_int_t retc, const T *yst, const isvd_int_t ldyst, T *qt,     \
                                           const isvd_int_t ldqt) {                                                \
    api_call([&] { integrate_api<T>(param, argv, argc, retv, retc, const_cast<T *>(yst), ldyst, qt, ldqt, 0); });  \
  }                                                                                                                \
  void isvd_##x##IntegrateWenYin(const isvd_Param param, const T *argv, const isvd_int_t argc, T *retv,             \
                                 const isvd_int_t retc, const T *yst, const isvd_int_t ldyst, T *qt,               \
                                 const isvd_int_t ldqt) {                                                          \
    api_call([&] { integrate_api<T>(param, argv, argc, retv, retc, const_cast<T *>(yst), ldyst, qt, ldqt, 1); });  \
  }                                                                                                                \
  void isvd_##x##IntegrateHierarchicalReduction(const isvd_Param param, const T *argv, const isvd_int_t argc,       \
                                                T *retv, const isvd_int_t retc, T *yst, const isvd_int_t ldyst,    \
                                                T *qt, const isvd_int_t ldqt) {                                    \
    api_call([&] { integrate_api<T>(param, argv, argc, retv, retc, yst, ldyst, qt, ldqt, 2); });                    \
  }                                                                                                                \
  ISVD_POST(x, T, PostprocessGramian, 0)                                                                           \
  ISVD_POST(x, T, PostprocessTallSkinnyQr, 1)                                                                      \
  ISVD_POST(x, T, PostprocessSymmetric, 2)                                                                         \
  void isvd_##x##Isvd(const isvd_Param param, const char *alg_s, const char *alg_o, const char *alg_i,             \
                      const char *alg_p, const T *argv[4], const isvd_int_t argc[4], T *retv[4],                   \
                      const isvd_int_t retc[4], double time[4], FILE *stream, const char dista, const char ordera, \
                      const T *a, const isvd_int_t lda, T *s, T *ut, const isvd_int_t ldut, T *vt,                 \
                      const isvd_int_t ldvt, const isvd_int_t seed, const mpi_int_t ut_root,                       \
                      const mpi_int_t vt_root) {                                                                   \
    api_call([&] {                                                                                                 \
      driver<T>(param, alg_s, alg_o, alg_i, alg_p, argv, argc, retv, retc, time, stream, dista, ordera, a, lda, s, \
                ut, ldut, vt, ldvt, seed, ut_root, vt_root, nullptr, 0, -1);                                       \
    });                                                                                                            \
  }                                                                                                                \
  int isvd_##x##Isvd_ex(const isvd_Param param, const char *alg_s, const char *alg_o, const char *alg_i,           \
                        const char *alg_p, const T *argv[4], const isvd_int_t argc[4], T *retv[4],                 \
                        const isvd_int_t retc[4], double time[4], FILE *stream, const char dista,                  \
                        const char ordera, const T *a, const isvd_int_t lda, T *s, T *ut, const isvd_int_t ldut,   \
                        T *vt, const isvd_int_t ldvt, const isvd_int_t seed, const mpi_int_t ut_root,              \
                        const mpi_int_t vt_root, const T *omega, const isvd_int_t ldomega, const int precision) {  \
    return api_call([&] {                                                                                          \
      driver<T>(param, alg_s, alg_o, alg_i, alg_p, argv, argc, retv, retc, time, stream, dista, ordera, a, lda, s, \
                ut, ldut, vt, ldvt, seed, ut_root, vt_root, omega, ldomega,                                        \
                precision == ISVD_GPU_PRECISION_MIXED ? (int)kMixed                                               \
                : precision == ISVD_GPU_PRECISION_NATIVE ? (int)kNative : -1);                                     \
    });                                                                                                            \
  }

#define ISVD_POST(x, T, NAME, ALG)                                                                                 \
  void isvd_##x##NAME(const isvd_Param param, const T *argv, const isvd_int_t argc, T *retv, const isvd_int_t retc, \
                      const char dista, const char ordera, const T *a, const isvd_int_t lda, const T *qt,          \
                      const isvd_int_t ldqt, T *s, T *ut, const isvd_int_t ldut, T *vt, const isvd_int_t ldvt,     \
                      const mpi_int_t ut_root, const mpi_int_t vt_root) {                                          \
    api_call([&] {                                                                                                 \
      post_api<T>(param, argv, argc, retv, retc, dista, ordera, a, lda, qt, ldqt, s, ut, ldut, vt, ldvt, ut_root,  \
                  vt_root, ALG, -1);                                                                               \
    });                                                                                                            \
  }                                                                                                                \
  void isvd_##x##NAME##_gpu(const isvd_Param param, const T *argv, const isvd_int_t argc, T *retv,                 \
                            const isvd_int_t retc, const char dista, const char ordera, const T *a,                \
                            const isvd_int_t lda, const T *qt, const isvd_int_t ldqt, T *s, T *ut,                 \
                            const isvd_int_t ldut, T *vt, const isvd_int_t ldvt, const mpi_int_t ut_root,          \
                            const mpi_int_t vt_root) {                                                             \
    isvd_##x##NAME(param, argv, argc, retv, retc, dista, ordera, a, lda, qt, ldqt, s, ut, ldut, vt, ldvt, ut_root, \
                   vt_root);                                                                                       \
  }

ISVD_STAGES(s, float)
ISVD_STAGES(d, double)

// Kolmogorov-Nagumo integration without device allocation (isvd/b200.h).  Argument meaning and
// checks as isvd_dIntegrateKolmogorovNagumo; the stage itself is integrate_kn_static.
int isvd_dIntegrateKolmogorovNagumo_noalloc(const isvd_Param param, const isvd_d_val_t *argv, const isvd_int_t argc,
                                            isvd_d_val_t *retv, const isvd_int_t retc, const isvd_d_val_t *yst,
                                            const isvd_int_t ldyst, isvd_d_val_t *qt, const isvd_int_t ldqt,
                                            void *stream) {
  return api_call([&] {
    if (argc > 0) REQUIRE(argv != nullptr);
    if (retc > 0) REQUIRE(retv != nullptr);
    if (argc < 0) {
      query_kn(retv, retc);
      return;
    }
    // one rank only: this variant never sums G = Qs'Qs over the ranks joined by
    // isvd_gpu_set_allreduce, so each rank would iterate on its own partial Gram
    if (param.mpi_size != 1 || collective().nranks > 1)
      fail(kErrUnsupported, "Kolmogorov-Nagumo on static scratch: one rank only (MPI size %d, %d joined ranks)",
           (int)param.mpi_size, collective().nranks);
    require_single_rank(param);
    const int m = param.nrow_proc, l = param.dim_sketch, N = param.num_sketch, Nl = param.dim_sketch_total;
    REQUIRE(ldyst >= Nl);
    REQUIRE(ldqt >= l);
    int ai = -1;
    const int maxit = (argc > ++ai) ? (int)argv[ai] : 256;
    const double tol = (argc > ++ai) ? argv[ai] : 1e-4;
    REQUIRE(maxit >= 0);
    REQUIRE(tol >= 0);
    const IterResult r = integrate_kn_static(static_cast<cudaStream_t>(stream), m, l, N, yst, ldyst, qt, ldqt,
                                             maxit, tol);
    int ri = -1;
    if (retc > ++ri) retv[ri] = (double)r.iterations;
    if (retc > ++ri) retv[ri] = r.error;
  });
}

isvd_gpu_batch *isvd_sBatchCreate(const isvd_int_t count, const isvd_int_t *m, const isvd_int_t *n,
                                  const isvd_int_t *k, const isvd_int_t *p, const isvd_int_t N) {
  return batch_create_api<float>(count, m, n, k, p, N);
}

isvd_gpu_batch *isvd_dBatchCreate(const isvd_int_t count, const isvd_int_t *m, const isvd_int_t *n,
                                  const isvd_int_t *k, const isvd_int_t *p, const isvd_int_t N) {
  return batch_create_api<double>(count, m, n, k, p, N);
}

int isvd_sBatchIsvd(isvd_gpu_batch *batch, const isvd_s_val_t *const *a, const isvd_int_t *lda,
                    isvd_s_val_t *const *s, isvd_s_val_t *const *ut, const isvd_int_t *ldut, isvd_s_val_t *const *vt,
                    const isvd_int_t *ldvt, const isvd_int_t *seed, const isvd_s_val_t *argv, const isvd_int_t argc,
                    isvd_int_t *iterations, isvd_s_val_t *errors) {
  return batch_isvd_api<float>(batch, a, lda, s, ut, ldut, vt, ldvt, seed, argv, argc, iterations, errors);
}

int isvd_dBatchIsvd(isvd_gpu_batch *batch, const isvd_d_val_t *const *a, const isvd_int_t *lda,
                    isvd_d_val_t *const *s, isvd_d_val_t *const *ut, const isvd_int_t *ldut, isvd_d_val_t *const *vt,
                    const isvd_int_t *ldvt, const isvd_int_t *seed, const isvd_d_val_t *argv, const isvd_int_t argc,
                    isvd_int_t *iterations, isvd_d_val_t *errors) {
  return batch_isvd_api<double>(batch, a, lda, s, ut, ldut, vt, ldvt, seed, argv, argc, iterations, errors);
}

void isvd_gpu_batch_destroy(isvd_gpu_batch *batch) {
  api_call([&] {
    delete reinterpret_cast<BatchPlan *>(batch);
    sync();
  });
}

int isvd_sSvdAdjoint(const isvd_int_t m, const isvd_int_t n, const isvd_int_t k, const char ordera,
                     const isvd_s_val_t *a, const isvd_int_t lda, const isvd_s_val_t *s, const isvd_s_val_t *ut,
                     const isvd_int_t ldut, const isvd_s_val_t *vt, const isvd_int_t ldvt, const isvd_s_val_t *ds,
                     const isvd_s_val_t *dut, const isvd_int_t lddut, const isvd_s_val_t *dvt,
                     const isvd_int_t lddvt, isvd_s_val_t *da, const isvd_int_t ldda, const int cg_iters,
                     const double tol, int *iterations) {
  return adjoint_api<float>(m, n, k, ordera, a, lda, s, ut, ldut, vt, ldvt, ds, dut, lddut, dvt, lddvt, da, ldda,
                            cg_iters, tol, iterations);
}

int isvd_dSvdAdjoint(const isvd_int_t m, const isvd_int_t n, const isvd_int_t k, const char ordera,
                     const isvd_d_val_t *a, const isvd_int_t lda, const isvd_d_val_t *s, const isvd_d_val_t *ut,
                     const isvd_int_t ldut, const isvd_d_val_t *vt, const isvd_int_t ldvt, const isvd_d_val_t *ds,
                     const isvd_d_val_t *dut, const isvd_int_t lddut, const isvd_d_val_t *dvt,
                     const isvd_int_t lddvt, isvd_d_val_t *da, const isvd_int_t ldda, const int cg_iters,
                     const double tol, int *iterations) {
  return adjoint_api<double>(m, n, k, ordera, a, lda, s, ut, ldut, vt, ldvt, ds, dut, lddut, dvt, lddvt, da, ldda,
                             cg_iters, tol, iterations);
}

}  // extern "C"
#pragma GCC visibility pop
