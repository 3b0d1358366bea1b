// Device helpers shared by the Kolmogorov-Nagumo step kernels.
#pragma once

namespace isvdb {

// Number of coupled Newton-Schulz steps so that rho^(2^k) <= target (rho: bound of ||I - X||_2).
__device__ __forceinline__ int kn_ns_steps(double rho, double target) {
  if (!(rho < 0.999)) return 40;
  if (rho < 1e-300) return 1;
  const double need = -log(target) / -log(rho);
  int k = 0;
  double p = 1.0;
  while (p < need && k < 40) {
    p *= 2.0;
    ++k;
  }
  return k + 1;
}

}  // namespace isvdb
