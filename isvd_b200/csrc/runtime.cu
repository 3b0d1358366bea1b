// Device context, errors and stream-ordered allocation for libisvd_gpu_b200.
#include "runtime.h"

#include <algorithm>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <vector>

extern "C" size_t isvd_gpu_memory_limit;  // include/isvd/gpu/env.h

namespace isvdb {

std::atomic<unsigned long long> g_launches{0};

static Runtime g_rt;
static bool g_init = false;
static std::mutex g_init_mu;
static int g_precision = -1;

void fail(int code, const char *fmt, ...) {
  char buf[1024];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  throw Error(code, buf);
}

void check_cuda(cudaError_t e, const char *what, const char *file, int line) {
  if (e == cudaSuccess) return;
  int code = (e == cudaErrorMemoryAllocation) ? kErrMemory : kErrCuda;
  fail(code, "CUDA error %s (%s) in %s at %s:%d", cudaGetErrorName(e), cudaGetErrorString(e), what, file, line);
}

bool Runtime::initialised() { return g_init; }

Runtime &Runtime::get() {
  if (g_init) return g_rt;
  std::lock_guard<std::mutex> lk(g_init_mu);
  if (g_init) return g_rt;
  int dev = 0;
  CK(cudaGetDevice(&dev));
  cudaDeviceProp prop;
  CK(cudaGetDeviceProperties(&prop, dev));
  g_rt.device = dev;
  g_rt.num_sms = prop.multiProcessorCount;
  g_rt.cc_major = prop.major;
  g_rt.cc_minor = prop.minor;
  g_rt.smem_optin = prop.sharedMemPerBlockOptin;
  CK(cudaStreamCreateWithFlags(&g_rt.own_stream, cudaStreamNonBlocking));
  g_rt.stream = g_rt.own_stream;
  CK(cudaStreamCreateWithFlags(&g_rt.copy_stream, cudaStreamNonBlocking));
  // Keep freed pool memory cached: repeated solves reuse it without new cudaMalloc calls.
  cudaMemPool_t pool;
  CK(cudaDeviceGetDefaultMemPool(&pool, dev));
  uint64_t thr = UINT64_MAX;
  CK(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr));
  CK(cudaMalloc(&g_rt.ctl, 4096));
  CK(cudaMemset(g_rt.ctl, 0, 4096));
  CK(cudaMallocHost(&g_rt.host_pin, 64 * sizeof(double)));
  g_init = true;
  return g_rt;
}

void Runtime::reset() {
  std::lock_guard<std::mutex> lk(g_init_mu);
  if (!g_init) return;
  cudaStreamSynchronize(g_rt.stream);
  cudaFree(g_rt.ctl);
  cudaFreeHost(g_rt.host_pin);
  cudaStreamDestroy(g_rt.own_stream);
  cudaStreamDestroy(g_rt.copy_stream);
  g_rt = Runtime();
  g_init = false;
}

int default_precision() {
  if (g_precision < 0) {
    const char *e = getenv("ISVD_GPU_PRECISION");
    g_precision = (e && (!strcmp(e, "mixed") || !strcmp(e, "1"))) ? kMixed : kNative;
  }
  return g_precision;
}

void set_default_precision(int p) { g_precision = p; }

void *dev_alloc(size_t bytes) {
  Runtime &rt = Runtime::get();
  void *p = nullptr;
  cudaError_t e = cudaMallocAsync(&p, bytes, rt.stream);
  if (e != cudaSuccess) {
    cudaGetLastError();
    fail(kErrMemory, "device allocation of %zu bytes failed (%s)", bytes, cudaGetErrorString(e));
  }
  return p;
}

size_t device_budget() {
  Runtime &rt = Runtime::get();
  size_t free_b = 0, total_b = 0;
  CK(cudaMemGetInfo(&free_b, &total_b));
  // memory the library's pool holds but does not use counts as free (it is reused first)
  cudaMemPool_t pool;
  CK(cudaDeviceGetDefaultMemPool(&pool, rt.device));
  unsigned long long reserved = 0, used = 0;
  CK(cudaMemPoolGetAttribute(pool, cudaMemPoolAttrReservedMemCurrent, &reserved));
  CK(cudaMemPoolGetAttribute(pool, cudaMemPoolAttrUsedMemCurrent, &used));
  if (reserved > used) free_b += (size_t)(reserved - used);
  const size_t lim = isvd_gpu_memory_limit;
  return lim > 0 ? std::min(free_b, lim) : free_b;
}

long long host_panel_rows(long long m, long long n, size_t resident_bytes, size_t row_bytes, size_t work_bytes,
                          size_t elem) {
  const size_t budget = device_budget();
  if (resident_bytes + work_bytes <= budget) return 0;
  const size_t avail = budget > work_bytes ? budget - work_bytes : 0;
  long long P = (long long)(avail / std::max<size_t>(row_bytes, 1));
  const long long cap = std::max<long long>(128, (long long)((1ll << 30) / ((long long)n * (long long)elem)));
  P = std::min(P, cap);
  if (P >= m) return m;
  P = P / 128 * 128;
  if (P < 128)
    fail(kErrMemory, "not enough GPU memory for a host A streamed in panels of 128 rows (%zu bytes usable, "
                     "%zu needed)", budget, work_bytes + 128 * row_bytes);
  return P;
}

void dev_free(void *p) {
  if (!p || !g_init) return;
  cudaFreeAsync(p, g_rt.stream);
}

bool is_device_pointer(const void *p) {
  if (!p) return false;
  cudaPointerAttributes attr;
  cudaError_t e = cudaPointerGetAttributes(&attr, p);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return attr.type == cudaMemoryTypeDevice || attr.type == cudaMemoryTypeManaged;
}

void sync() { CK(cudaStreamSynchronize(Runtime::get().stream)); }

struct ProfEntry {
  double ms = 0.0, flops = 0.0;
  unsigned long long count = 0;
};
static std::map<std::string, ProfEntry> g_prof;
static std::mutex g_prof_mu;
static bool g_profiling = false;

bool profiling() { return g_profiling; }
void set_profiling(bool on) { g_profiling = on; }

unsigned long long count_kernel_nodes(cudaGraph_t g) {
  size_t n = 0;
  CK(cudaGraphGetNodes(g, nullptr, &n));
  std::vector<cudaGraphNode_t> nodes(n);
  if (n) CK(cudaGraphGetNodes(g, nodes.data(), &n));
  unsigned long long k = 0;
  for (size_t i = 0; i < n; ++i) {
    cudaGraphNodeType t;
    CK(cudaGraphNodeGetType(nodes[i], &t));
    if (t == cudaGraphNodeTypeKernel) ++k;
  }
  return k;
}

GraphPair::GraphPair(cudaStream_t s) : st(s) {
  const char *env = getenv("ISVD_GPU_GRAPHS");
  const bool off = env && env[0] == '0';
  // stream-ordered allocations inside the body go to the library stream: only that one is captured
  usable = !off && s != nullptr && s != cudaStreamLegacy && s != cudaStreamPerThread && !profiling() &&
           s == Runtime::get().stream;
}

GraphPair::~GraphPair() {
  for (int i = 0; i < 2; ++i)
    if (exec[i]) cudaGraphExecDestroy(exec[i]);
}
Collective &collective() {
  static Collective c;
  return c;
}

namespace {
template <class T>
void allreduce_impl(T *p, size_t count, int dtype, cudaStream_t st) {
  Collective &c = collective();
  if (c.nranks <= 1 || !c.fn || count == 0) return;
  if (c.on_device) {
    c.fn(p, count, dtype, st, c.user);
    CK(cudaGetLastError());
    return;
  }
  static void *pin = nullptr;
  static size_t pin_bytes = 0;
  const size_t bytes = count * sizeof(T);
  if (bytes > pin_bytes) {
    if (pin) cudaFreeHost(pin);
    pin = nullptr;
    pin_bytes = 0;
    if (cudaMallocHost(&pin, bytes) != cudaSuccess) fail(kErrMemory, "pinned staging for the AllReduce");
    pin_bytes = bytes;
  }
  CK(cudaMemcpyAsync(pin, p, bytes, cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  c.fn(pin, count, dtype, st, c.user);
  CK(cudaMemcpyAsync(p, pin, bytes, cudaMemcpyHostToDevice, st));
  CK(cudaStreamSynchronize(st));  // the staging buffer is reused by the next call
}
}  // namespace

void allreduce_sum(double *p, size_t count, cudaStream_t st) { allreduce_impl(p, count, 1, st); }
void allreduce_sum(float *p, size_t count, cudaStream_t st) { allreduce_impl(p, count, 0, st); }

void profile_add(const char *tag, double ms, double flops) {
  std::lock_guard<std::mutex> lk(g_prof_mu);
  ProfEntry &e = g_prof[tag];
  e.ms += ms;
  e.flops += flops;
  e.count += 1;
}
bool profile_get(const char *tag, double *ms, unsigned long long *count, double *flops) {
  std::lock_guard<std::mutex> lk(g_prof_mu);
  auto it = g_prof.find(tag);
  if (it == g_prof.end()) return false;
  if (ms) *ms = it->second.ms;
  if (count) *count = it->second.count;
  if (flops) *flops = it->second.flops;
  return true;
}
void profile_reset() {
  std::lock_guard<std::mutex> lk(g_prof_mu);
  g_prof.clear();
}

}  // namespace isvdb
