// Boys function F_m(T) = int_0^1 t^{2m} exp(-T t^2) dt on the device.
//
// Grid values are those of hf-rs's table (src/integrals.rs:20-57): T on a
// 0.05 step, produced on the host by the convergent series at order 47 and
// downward recursion (boys_table_host()).  On the device, for a class of
// total angular momentum L:
//
//  * T <= 36: F_L by the order-7 Taylor expansion about the nearest grid
//    point T0, d^k F_L/dT^k = (-1)^k F_{L+k} (hf-rs's scheme,
//    src/integrals.rs:83-100); e^{-T} = e^{-T0} e^{-dT} with an order-7
//    Taylor of e^{-dT} (|dT| <= 0.025, truncation < 1e-17); then the
//    downward recursion F_m = (2T F_{m+1} + e^{-T}) / (2m+1), stable for all
//    T.  The row F_L/0!, ..., F_{L+7}/7!, e^{-T0} of every grid point with
//    T <= 36 is staged once per block in shared memory (9 doubles per row;
//    the odd stride spreads the rows over the banks).
//  * T > 36: F_0 = sqrt(pi)/(2 sqrt T) (erf(sqrt T) is 1 to double precision
//    there) and the upward recursion F_m = ((2m-1) F_{m-1} - e^{-T})/(2T),
//    stable for T > m (hf-rs's branch beyond its switch,
//    src/integrals.rs:73-80).  For L <= 2 the e^{-T} < 2.4e-16 F_0 term
//    changes F_m by less than 1e-13 relative and is dropped.
//
// The FP32 flavour (only for quartets with small Schwarz bounds) uses an
// order-4 Taylor row F_L/k!, k = 0..4 plus e^{-T0}, and an order-4 Taylor of
// e^{-dT}, for T <= 36 (truncation below 1e-9 relative); for T > 36 it
// evaluates the FP64 branch above and rounds each F_m to FP32.
#pragma once
#include <cuda_runtime.h>

namespace hfg {

constexpr int kBoysCols = 24;   // F_0 .. F_23 per grid point in the global table (L <= 16 with order 7)
constexpr int kBoysRows = 1002; // T in [0, 50.05]
constexpr double kBoysStep = 0.05;
constexpr int kBoysSmemRows = 721;  // T <= 36
constexpr double kBoysTMax = 36.0;
constexpr double kHalfSqrtPi = 0.88622692545275801365;

template <typename T> struct BoysSmem;
template <> struct BoysSmem<double> {
  static constexpr int kTerms = 8;
  static constexpr int kStride = 9;
};
template <> struct BoysSmem<float> {
  static constexpr int kTerms = 5;
  static constexpr int kStride = 7;
};

template <typename T>
__host__ __device__ constexpr size_t boys_smem_bytes() {
  return (size_t)kBoysSmemRows * BoysSmem<T>::kStride * sizeof(T);
}

// Stage F_{L+k}/k! (k < terms) and e^{-T0} for T0 <= 36 in shared memory.
// `table` holds F_0..F_15 per grid row; `expt` holds e^{-T0} per row.
template <typename T, int L>
__device__ __forceinline__ void boys_stage(T* __restrict__ sm, const T* __restrict__ table,
                                           const T* __restrict__ expt) {
  constexpr int terms = BoysSmem<T>::kTerms, stride = BoysSmem<T>::kStride;
  const T inv_fact[8] = {(T)1.0, (T)1.0, (T)0.5, (T)(1.0 / 6.0), (T)(1.0 / 24.0), (T)(1.0 / 120.0),
                         (T)(1.0 / 720.0), (T)(1.0 / 5040.0)};
  for (int i = threadIdx.x; i < kBoysSmemRows * (terms + 1); i += blockDim.x) {
    const int r = i / (terms + 1), c = i - r * (terms + 1);
    sm[r * stride + c] = c < terms ? table[r * kBoysCols + L + c] * inv_fact[c] : expt[r];
  }
}

template <int L>
__device__ __forceinline__ void boys_eval(double t, const double* __restrict__ sm, double* F) {
  if (t > kBoysTMax) {
    const double r = rsqrt(t);
    F[0] = kHalfSqrtPi * r;
    if (L > 0) {
      const double inv2t = 0.5 * r * r;
      if (L <= 2) {
#pragma unroll
        for (int m = 1; m <= L; ++m) F[m] = (2 * m - 1) * F[m - 1] * inv2t;
      } else {
        const double e = exp(-t);
#pragma unroll
        for (int m = 1; m <= L; ++m) F[m] = ((2 * m - 1) * F[m - 1] - e) * inv2t;
      }
    }
    return;
  }
  const int idx = min(max(__double2int_rn(t * 20.0), 0), kBoysSmemRows - 1);
  const double x = idx * kBoysStep - t;  // -(T - T0)
  const double* row = sm + idx * 9;
  double acc = fma(row[7], x, row[6]);
  acc = fma(acc, x, row[5]);
  acc = fma(acc, x, row[4]);
  acc = fma(acc, x, row[3]);
  acc = fma(acc, x, row[2]);
  acc = fma(acc, x, row[1]);
  F[L] = fma(acc, x, row[0]);
  if (L > 0) {
    // e^{-T} = e^{-T0} * e^{x}
    double ex = fma(x, 1.0 / 5040.0, 1.0 / 720.0);
    ex = fma(ex, x, 1.0 / 120.0);
    ex = fma(ex, x, 1.0 / 24.0);
    ex = fma(ex, x, 1.0 / 6.0);
    ex = fma(ex, x, 0.5);
    ex = fma(ex, x, 1.0);
    ex = fma(ex, x, 1.0);
    const double e = row[8] * ex;
    const double t2 = 2.0 * t;
#pragma unroll
    for (int m = L - 1; m >= 0; --m) F[m] = (t2 * F[m + 1] + e) * (1.0 / (2 * m + 1));
  }
}

template <int L>
__device__ __forceinline__ void boys_eval(float t, const float* __restrict__ sm, float* F) {
  if (t > 36.0f) {
    // large T in FP64: the asymptotic F_0 and the upward recursion of the
    // FP64 flavour, rounded to FP32 once per order
    const double td = t;
    const double r = rsqrt(td);
    double f = kHalfSqrtPi * r;
    F[0] = (float)f;
    if (L > 0) {
      const double inv2t = 0.5 * r * r;
      const double e = L <= 2 ? 0.0 : exp(-td);
#pragma unroll
      for (int m = 1; m <= L; ++m) {
        f = ((2 * m - 1) * f - e) * inv2t;
        F[m] = (float)f;
      }
    }
    return;
  }
  // nearest grid point by adding and subtracting 1.5 * 2^23, which rounds
  // 20 t (0 <= 20 t <= 720 here) to an integer in the FP32 adder and leaves
  // it in the low mantissa bits; no float<->int conversions (the clamp also
  // catches a NaN t)
  const float y = t * 20.0f + 12582912.0f;
  const int idx = min(max(__float_as_int(y) - 0x4B400000, 0), kBoysSmemRows - 1);
  const float x = (y - 12582912.0f) * 0.05f - t;
  const float* row = sm + idx * 7;
  float acc = fmaf(row[4], x, row[3]);
  acc = fmaf(acc, x, row[2]);
  acc = fmaf(acc, x, row[1]);
  F[L] = fmaf(acc, x, row[0]);
  if (L > 0) {
    // e^{x}, |x| <= 0.025: order-4 Taylor (truncation below 1e-10 relative)
    float ex = fmaf(x, 1.0f / 24.0f, 1.0f / 6.0f);
    ex = fmaf(ex, x, 0.5f);
    ex = fmaf(ex, x, 1.0f);
    ex = fmaf(ex, x, 1.0f);
    const float e = row[5] * ex;
    const float t2 = 2.0f * t;
#pragma unroll
    for (int m = L - 1; m >= 0; --m) F[m] = (t2 * F[m + 1] + e) * (1.0f / (2 * m + 1));
  }
}

}  // namespace hfg
