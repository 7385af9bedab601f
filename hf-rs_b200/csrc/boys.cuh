// Boys function F_m(T) = int_0^1 t^{2m} exp(-T t^2) dt on the device.
//
// Same scheme as hf-rs (src/integrals.rs:20-101): for T <= 50 a Taylor
// expansion of order 7 about the nearest point of a 0.05-step grid,
// d^k F_m / dT^k = (-1)^k F_{m+k}; for T > 50 the closed form
// F_0 = sqrt(pi)/(2 sqrt(T)) (erf(sqrt(T)) is 1 to double precision there)
// and the upward recursion F_m = ((2m-1) F_{m-1} - e^{-T}) / (2T).
// The grid values are produced on the host by the convergent series at the
// highest order followed by downward recursion (boys_table_host()).
//
// The FP32 flavour uses a float copy of the same grid with a Taylor order of
// 4 (truncation below 1e-9 relative for |dT| <= 0.025) and fast-math
// exponentials; it is only used for quartets whose Schwarz bound is small.
#pragma once
#include <cuda_runtime.h>

namespace hfg {

constexpr int kBoysCols = 16;   // F_0 .. F_15 stored per grid point (L <= 8)
constexpr int kBoysRows = 1002; // T in [0, 50.05]
constexpr double kBoysStep = 0.05;
constexpr double kBoysTSwitch = 50.0;
constexpr double kHalfSqrtPi = 0.88622692545275801365;

template <typename T> struct BoysTable;

// F[0..L] for T; table is row-major [row][kBoysCols].
template <int L>
__device__ __forceinline__ void boys_eval(double t, const double* __restrict__ table, double* F) {
  if (t > kBoysTSwitch) {
    const double r = rsqrt(t);
    F[0] = kHalfSqrtPi * r;
    if (L > 0) {
      const double e = exp(-t);
      const double inv2t = 0.5 * r * r;
#pragma unroll
      for (int m = 1; m <= L; ++m) F[m] = ((2 * m - 1) * F[m - 1] - e) * inv2t;
    }
    return;
  }
  const int idx = min(max(__double2int_rn(t * 20.0), 0), kBoysRows - 1);
  const double dt = t - idx * kBoysStep;
  const double* row = table + idx * kBoysCols;
  const double x = -dt;
  // Horner in x with coefficients F_{m+k}/k!
#pragma unroll
  for (int m = 0; m <= L; ++m) {
    double acc = __ldg(row + m + 7) * (1.0 / 5040.0);
    acc = fma(acc, x, __ldg(row + m + 6) * (1.0 / 720.0));
    acc = fma(acc, x, __ldg(row + m + 5) * (1.0 / 120.0));
    acc = fma(acc, x, __ldg(row + m + 4) * (1.0 / 24.0));
    acc = fma(acc, x, __ldg(row + m + 3) * (1.0 / 6.0));
    acc = fma(acc, x, __ldg(row + m + 2) * 0.5);
    acc = fma(acc, x, __ldg(row + m + 1));
    acc = fma(acc, x, __ldg(row + m));
    F[m] = acc;
  }
}

template <int L>
__device__ __forceinline__ void boys_eval(float t, const float* __restrict__ table, float* F) {
  if (t > 50.0f) {
    const float r = rsqrtf(t);
    F[0] = 0.88622692545f * r;
    if (L > 0) {
      const float e = __expf(-t);
      const float inv2t = 0.5f * r * r;
#pragma unroll
      for (int m = 1; m <= L; ++m) F[m] = ((2 * m - 1) * F[m - 1] - e) * inv2t;
    }
    return;
  }
  const int idx = min(max(__float2int_rn(t * 20.0f), 0), kBoysRows - 1);
  const float x = -(t - idx * 0.05f);
  const float* row = table + idx * kBoysCols;
#pragma unroll
  for (int m = 0; m <= L; ++m) {
    float acc = __ldg(row + m + 4) * (1.0f / 24.0f);
    acc = fmaf(acc, x, __ldg(row + m + 3) * (1.0f / 6.0f));
    acc = fmaf(acc, x, __ldg(row + m + 2) * 0.5f);
    acc = fmaf(acc, x, __ldg(row + m + 1));
    acc = fmaf(acc, x, __ldg(row + m));
    F[m] = acc;
  }
}

}  // namespace hfg
