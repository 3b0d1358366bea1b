// Householder-QR based stages (TSQR orthogonalization, TSQR postprocessing) and Wen-Yin integration.
#include "kernels.h"
#include "runtime.h"
#include "stages.h"

namespace isvdb {

template <class T>
void orth_tsqr_dev(const StageCtx &, int, int, int, T *, long long) {
  fail(kErrUnsupported, "tall-skinny QR orthogonalization is not available in this build");
}
template <class T>
IterResult integrate_wy_dev(const StageCtx &, int, int, int, const T *, long long, T *, long long, const WyArgs &) {
  fail(kErrUnsupported, "Wen-Yin integration is not available in this build");
}
template <class T>
void post_tsqr_dev(const StageCtx &, int, int, int, int, char, const T *, long long, const T *, long long, T *, T *,
                   long long, T *, long long, bool, bool) {
  fail(kErrUnsupported, "tall-skinny QR postprocessing is not available in this build");
}

#define ISVD_INST(T)                                                                                         \
  template void orth_tsqr_dev<T>(const StageCtx &, int, int, int, T *, long long);                           \
  template IterResult integrate_wy_dev<T>(const StageCtx &, int, int, int, const T *, long long, T *, long long, \
                                          const WyArgs &);                                                   \
  template void post_tsqr_dev<T>(const StageCtx &, int, int, int, int, char, const T *, long long, const T *,  \
                                 long long, T *, T *, long long, T *, long long, bool, bool);
ISVD_INST(float)
ISVD_INST(double)

}  // namespace isvdb
