// MIXED precision engine (placeholder until the tcgen05 kernels land).
#include "mixed.h"
#include "runtime.h"

namespace isvdb {

#define ISVD_MIXED_TODO(name) fail(kErrUnsupported, "mixed precision: %s not available in this build", name)

template <class T>
void mixed_sketch(const StageCtx &, int, int, int, char, const T *, long long, const T *, long long, uint64_t, T *,
                  long long) { ISVD_MIXED_TODO("sketch"); }
template <class T>
void mixed_block_gram(const StageCtx &, int, int, int, const T *, long long, double *) { ISVD_MIXED_TODO("gram"); }
template <class T>
void mixed_block_apply(const StageCtx &, int, int, int, const T *, long long, const T *, T *, long long) {
  ISVD_MIXED_TODO("apply");
}
template <class T>
void mixed_gram_full(const StageCtx &, int, int, const T *, long long, double *) { ISVD_MIXED_TODO("gram"); }
template <class T>
void mixed_apply_coeff(const StageCtx &, int, int, int, const T *, long long, const double *, T *, long long) {
  ISVD_MIXED_TODO("apply");
}
template <class T>
void mixed_project(const StageCtx &, int, int, int, char, const T *, long long, const T *, long long, T *) {
  ISVD_MIXED_TODO("project");
}

#define ISVD_INST(T)                                                                                        \
  template void mixed_sketch<T>(const StageCtx &, int, int, int, char, const T *, long long, const T *,      \
                                long long, uint64_t, T *, long long);                                      \
  template void mixed_block_gram<T>(const StageCtx &, int, int, int, const T *, long long, double *);         \
  template void mixed_block_apply<T>(const StageCtx &, int, int, int, const T *, long long, const T *, T *,  \
                                     long long);                                                           \
  template void mixed_gram_full<T>(const StageCtx &, int, int, const T *, long long, double *);              \
  template void mixed_apply_coeff<T>(const StageCtx &, int, int, int, const T *, long long, const double *,  \
                                     T *, long long);                                                      \
  template void mixed_project<T>(const StageCtx &, int, int, int, char, const T *, long long, const T *,     \
                                 long long, T *);
ISVD_INST(float)
ISVD_INST(double)

}  // namespace isvdb
