// Dispatch of the per-class J/K launches (one translation unit per class).
#pragma once
#include <cuda_runtime.h>

#include "hfg_internal.h"

namespace hfg {

// Lane-group sizes G built per class: classes with many contracted
// accumulators keep one quartet per lane (the accumulators would not fit a
// shuffle reduction in registers).
constexpr int kMaxAccG32 = 36;
constexpr int kMaxAccG8 = 100;

#define HFG_DECL(a, b, c, d) cudaError_t launch_jk_##a##b##c##d(const JKLaunchArgs&, int, bool, cudaStream_t);
HFG_DECL(0, 0, 0, 0)
HFG_DECL(1, 0, 0, 0)
HFG_DECL(1, 0, 1, 0)
HFG_DECL(1, 1, 0, 0)
HFG_DECL(1, 1, 1, 0)
HFG_DECL(1, 1, 1, 1)
HFG_DECL(2, 0, 0, 0)
HFG_DECL(2, 0, 1, 0)
HFG_DECL(2, 0, 1, 1)
HFG_DECL(2, 0, 2, 0)
HFG_DECL(2, 1, 0, 0)
HFG_DECL(2, 1, 1, 0)
HFG_DECL(2, 1, 1, 1)
HFG_DECL(2, 1, 2, 0)
HFG_DECL(2, 1, 2, 1)
HFG_DECL(2, 2, 0, 0)
HFG_DECL(2, 2, 1, 0)
HFG_DECL(2, 2, 1, 1)
HFG_DECL(2, 2, 2, 0)
HFG_DECL(2, 2, 2, 1)
HFG_DECL(2, 2, 2, 2)
#undef HFG_DECL

// Contracted accumulator count of class (la lb|lc ld): the Cartesian
// components of |e| in [la, la+lb] times those of |f| in [lc, lc+ld].
inline int class_nacc(int la, int lb, int lc, int ld) {
  auto nc = [](int l) { return (l + 1) * (l + 2) / 2; };
  int e = 0, f = 0;
  for (int l = la; l <= la + lb; ++l) e += nc(l);
  for (int l = lc; l <= lc + ld; ++l) f += nc(l);
  return e * f;
}

// Lane-group size for a class with nominal primitive-quartet count kk.
inline int choose_group(int la, int lb, int lc, int ld, long kk) {
  const int nacc = class_nacc(la, lb, lc, ld);
  if (kk >= 256 && nacc <= kMaxAccG32) return 32;
  if (kk >= 16 && nacc <= kMaxAccG8) return 8;
  return 1;
}

cudaError_t launch_jk(int la, int lb, int lc, int ld, int G, bool fp32, const JKLaunchArgs& a, cudaStream_t st);
cudaError_t launch_schwarz(int la, int lb, const PairInfo* pairs, const PrimPair* prims, int first, int count,
                           const double* boys, double* out, int prim_mode, cudaStream_t st);
cudaError_t launch_quartet(int la, int lb, int lc, int ld, const PairInfo* pairs, const PrimPair* prims,
                           const double* boys, double* out, cudaStream_t st);

}  // namespace hfg
