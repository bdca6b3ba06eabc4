// Elementwise math shared by the Sinkhorn kernels.
#pragma once

#include <cuda_runtime.h>
#include <math.h>

namespace wdl {

// log(x) of a positive FP32 value returned in FP64 with an absolute error of a
// few 1e-8 instead of logf's one ulp of |log x| (~1e-6 at |log x| ~ 10): x is
// split as m * 2^e with m in [sqrt(1/2), sqrt(2)), e*ln2 is formed in FP64 and
// only log(m), which is small, comes from logf.  Used where FP32 logarithms are
// summed in FP64 over a whole grid (weight-gradient dot products, the weighted
// geometric mean), so that the sums keep FP32-level relative accuracy.
__device__ __forceinline__ double log_f32_precise(float x) {
  int e;
  float m = frexpf(x, &e);  // x = m * 2^e, m in [0.5, 1)
  if (m < 0.70710678f) {
    m *= 2.0f;
    e -= 1;
  }
  return (double)e * 0.6931471805599453 + (double)logf(m);
}

// exp(s) for an FP64 exponent returned in FP32: s = n*ln2 + r with |r| <= ln2/2,
// exp(s) = 2^n * expf(r); relative error ~1e-7 for the whole FP32 range.
__device__ __forceinline__ float exp_to_f32(double s) {
  if (s < -110.0) return 0.0f;
  if (s > 89.0) return INFINITY;
  const double n = rint(s * 1.4426950408889634);
  const float r = (float)(s - n * 0.6931471805599453);
  return ldexpf(expf(r), (int)n);
}

}  // namespace wdl
