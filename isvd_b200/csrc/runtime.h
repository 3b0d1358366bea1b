// Host-side runtime of libisvd_gpu_b200: device context, stream, errors, device buffers.
#pragma once

#include <cuda_runtime.h>

#include <atomic>
#include <cstddef>
#include <cstdint>
#include <stdexcept>
#include <string>

namespace isvdb {

// Status codes (mirror include/isvd/b200.h).
enum Status : int {
  kSuccess = 0,
  kErrArgument = 1,
  kErrCuda = 2,
  kErrMemory = 3,
  kErrTimeout = 4,
  kErrNumerical = 5,
  kErrUnsupported = 6,
};

struct Error : std::runtime_error {
  int code;
  Error(int c, const std::string &m) : std::runtime_error(m), code(c) {}
};

[[noreturn]] void fail(int code, const char *fmt, ...);
void check_cuda(cudaError_t e, const char *what, const char *file, int line);

#define CK(x) ::isvdb::check_cuda((x), #x, __FILE__, __LINE__)

extern std::atomic<unsigned long long> g_launches;
// Every kernel launch of the library goes through KLAUNCHED() right after the <<<>>>.
#define KLAUNCHED()                                    \
  do {                                                 \
    ::isvdb::g_launches.fetch_add(1);                  \
    ::isvdb::check_cuda(cudaGetLastError(), "kernel launch", __FILE__, __LINE__); \
  } while (0)

enum Precision : int { kNative = 0, kMixed = 1 };

struct Runtime {
  int device = -1;
  cudaStream_t stream = nullptr;      // stream in use
  cudaStream_t own_stream = nullptr;  // the library's own stream
  cudaStream_t copy_stream = nullptr; // host-to-device panel transfers overlapped with compute
  int num_sms = 0;
  int cc_major = 0, cc_minor = 0;
  size_t smem_optin = 0;
  // Device-resident control block (barrier counters, status words), zeroed at init.
  unsigned int *ctl = nullptr;
  // Pinned host block (64 doubles) for small asynchronous read-backs (iteration errors).
  double *host_pin = nullptr;
  static Runtime &get();  // initialises on first use (device = current device)
  static bool initialised();
  static void reset();    // releases stream and control block (isvd_Finalize_gpu)
};

int default_precision();
void set_default_precision(int p);

// Stream-ordered device buffer (cudaMallocAsync on the library stream; pool memory is retained).
template <class T>
struct DBuf {
  T *p = nullptr;
  size_t n = 0;
  DBuf() = default;
  explicit DBuf(size_t count) { alloc(count); }
  DBuf(const DBuf &) = delete;
  DBuf &operator=(const DBuf &) = delete;
  DBuf(DBuf &&o) noexcept : p(o.p), n(o.n) { o.p = nullptr; o.n = 0; }
  DBuf &operator=(DBuf &&o) noexcept {
    if (this != &o) { release(); p = o.p; n = o.n; o.p = nullptr; o.n = 0; }
    return *this;
  }
  ~DBuf() { release(); }
  void alloc(size_t count);
  void ensure(size_t count) {  // keep the buffer when it already holds count elements
    if (!p || n != count) alloc(count);
  }
  void release();
  T *get() const { return p; }
  operator T *() const { return p; }
};

void *dev_alloc(size_t bytes);
void dev_free(void *p);

template <class T>
void DBuf<T>::alloc(size_t count) {
  release();
  n = count;
  p = count ? static_cast<T *>(dev_alloc(count * sizeof(T))) : nullptr;
}
template <class T>
void DBuf<T>::release() {
  if (p) dev_free(p);
  p = nullptr;
  n = 0;
}

// Pointer classification: true when the GPU can dereference `p` directly.
bool is_device_pointer(const void *p);

void sync();  // synchronise the library stream, converting errors into Error

// Multi-rank execution through a caller-provided sum-AllReduce (isvd_gpu_set_allreduce).
struct Collective {
  void (*fn)(void *, size_t, int, void *, void *) = nullptr;
  void *user = nullptr;
  int nranks = 1, rank = 0, on_device = 0;
  // installed by the library itself from the communicator of an isvd_Param (real-MPI builds), not
  // by isvd_gpu_set_allreduce
  bool from_comm = false;
};
Collective &collective();
// In-place sum over the ranks of `count` values at the device pointer p, ordered on st (no-op on
// one rank).  A host-memory reduction goes through pinned memory after a stream synchronisation.
void allreduce_sum(double *p, size_t count, cudaStream_t st);
void allreduce_sum(float *p, size_t count, cudaStream_t st);

// Optional per-kernel timing (CUDA events on the launching stream), off by default.
bool profiling();
void set_profiling(bool on);

unsigned long long count_kernel_nodes(cudaGraph_t g);

// Two CUDA graphs for the two parities of a ping-pong loop body: captured from the body's
// enqueues on first use and replayed afterwards.  Not used (the caller runs the body eagerly) on
// the legacy default stream, while kernel timing is on, or with ISVD_GPU_GRAPHS=0.
struct GraphPair {
  cudaStream_t st;
  bool usable;
  cudaGraphExec_t exec[2] = {nullptr, nullptr};
  unsigned long long kernels[2] = {0, 0};  // kernel nodes per graph (added to the launch counter)
  explicit GraphPair(cudaStream_t s);
  ~GraphPair();
  GraphPair(const GraphPair &) = delete;
  GraphPair &operator=(const GraphPair &) = delete;
  template <class F>
  void run(int par, F &&body) {
    if (!exec[par]) {
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
      kernels[par] = count_kernel_nodes(g);
      const cudaError_t e = cudaGraphInstantiate(&exec[par], g, 0);
      cudaGraphDestroy(g);
      CK(e);
    }
    CK(cudaGraphLaunch(exec[par], st));
    g_launches.fetch_add(kernels[par]);
  }
};
void profile_add(const char *tag, double ms, double flops);
bool profile_get(const char *tag, double *ms, unsigned long long *count, double *flops);
void profile_reset();

}  // namespace isvdb
