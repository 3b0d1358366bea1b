// Out-of-core A: a matrix in host memory streamed through the device in row panels, for matrices
// that do not fit in device memory beside the solve's own buffers (reference
// gpu/stage/@x@_sketch_gpu.h:65-135 and @x@_postprocess_gpu.h, which stream A in column panels
// sized by isvd_gpu_memory_limit).  Row panels keep Y's rows independent (the sketch of a panel
// is final) and make the projection Z = sum over panels of A_p' Qbar_p.
#pragma once

#include <algorithm>
#include <cstddef>

#include "runtime.h"
#include "stages.h"

namespace isvdb {

// Device memory the library may use now: the free memory, capped by isvd_gpu_memory_limit when
// that is non-zero (reference gpu/stage/@x@_sketch_gpu.h:66-68).
size_t device_budget();

// Rows per panel for a host A (m x n): 0 when `resident_bytes` of A-derived device data fit
// beside `work_bytes` of the solve's other buffers; otherwise the largest multiple of 128 rows
// (at most about 1 GiB of A) whose `row_bytes` per row of staging fit.  Fails with kErrMemory
// when not even 128 rows fit (the reference: "No enough GPU memory").
long long host_panel_rows(long long m, long long n, size_t resident_bytes, size_t row_bytes, size_t work_bytes,
                          size_t elem);

// Calls fn(r0, rows, panel, ldp) for consecutive row panels [r0, r0 + rows) of the host matrix a
// (m x n; ordera 'R': row-major with row stride lda, 'C': column-major with column stride lda).
// The panel lies on the device in the same order: 'R' rows x n with ldp = n, 'C' n columns of
// `rows` elements with ldp = rows.  Panel p + 1 is copied on the runtime's copy stream while fn
// enqueues panel p's work on c.st; the copy into a staging buffer waits for the work that read
// it two panels before.
template <class T, class F>
void for_each_host_panel(const StageCtx &c, const T *a, long long lda, char ordera, long long m, long long n,
                         long long P, F &&fn) {
  Runtime &rt = Runtime::get();
  P = std::max<long long>(1, std::min(P, m));
  DBuf<T> stage[2];
  cudaEvent_t copied[2] = {nullptr, nullptr}, consumed[2] = {nullptr, nullptr}, ready = nullptr;
  auto destroy = [&] {
    for (int b = 0; b < 2; ++b) {
      if (copied[b]) cudaEventDestroy(copied[b]);
      if (consumed[b]) cudaEventDestroy(consumed[b]);
    }
    if (ready) cudaEventDestroy(ready);
  };
  try {
    for (int b = 0; b < 2; ++b) {
      stage[b].alloc((size_t)P * n);
      CK(cudaEventCreateWithFlags(&copied[b], cudaEventDisableTiming));
      CK(cudaEventCreateWithFlags(&consumed[b], cudaEventDisableTiming));
    }
    CK(cudaEventCreateWithFlags(&ready, cudaEventDisableTiming));
    CK(cudaEventRecord(ready, c.st));  // staging buffers and earlier work ordered before the copies
    CK(cudaStreamWaitEvent(rt.copy_stream, ready, 0));
    int p = 0;
    for (long long r0 = 0; r0 < m; r0 += P, ++p) {
      const long long rows = std::min<long long>(P, m - r0);
      const int b = p & 1;
      if (p >= 2) CK(cudaStreamWaitEvent(rt.copy_stream, consumed[b], 0));
      if (ordera == 'R') {
        CK(cudaMemcpy2DAsync(stage[b].p, n * sizeof(T), a + r0 * lda, lda * sizeof(T), n * sizeof(T), rows,
                             cudaMemcpyHostToDevice, rt.copy_stream));
      } else {
        CK(cudaMemcpy2DAsync(stage[b].p, rows * sizeof(T), a + r0, lda * sizeof(T), rows * sizeof(T), n,
                             cudaMemcpyHostToDevice, rt.copy_stream));
      }
      CK(cudaEventRecord(copied[b], rt.copy_stream));
      CK(cudaStreamWaitEvent(c.st, copied[b], 0));
      fn(r0, rows, (const T *)stage[b].p, ordera == 'R' ? n : rows);
      CK(cudaEventRecord(consumed[b], c.st));
    }
    CK(cudaStreamSynchronize(c.st));  // the staging buffers are released below
  } catch (...) {
    cudaStreamSynchronize(rt.copy_stream);
    cudaStreamSynchronize(c.st);
    destroy();
    throw;
  }
  destroy();
}

}  // namespace isvdb
