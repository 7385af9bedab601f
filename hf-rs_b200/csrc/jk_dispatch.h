// Dispatch of the per-class J/K launches (one translation unit per class).
#pragma once
#include <cuda_runtime.h>

#include "hfg_internal.h"

namespace hfg {

// Classes with at most this many contracted accumulators would also be built
// with the cooperative kernels (G = 8 or 32 lanes per shell quartet).  On the
// cc-pVDZ water clusters one quartet per lane was faster at every
// contraction length (most quartets keep few primitive quartets after
// screening, and G > 1 multiplies the per-task work), so none are built.
constexpr int kMaxAccCoop = 0;

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

cudaError_t launch_jk(int la, int lb, int lc, int ld, int G, bool fp32, const JKLaunchArgs& a, cudaStream_t st);

// Contracted accumulator count of class (la lb|lc ld): Cartesian components
// of |e| in [la, la+lb] times those of |f| in [lc, lc+ld].
inline int class_nacc(int la, int lb, int lc, int ld) {
  auto nc = [](int l) { return (l + 1) * (l + 2) / 2; };
  int e = 0, f = 0;
  for (int l = la; l <= la + lb; ++l) e += nc(l);
  for (int l = lc; l <= lc + ld; ++l) f += nc(l);
  return e * f;
}

// Lanes per shell quartet from the nominal primitive-quartet count kk.
inline int choose_group(int la, int lb, int lc, int ld, long kk) {
  if (kMaxAccCoop == 0 || class_nacc(la, lb, lc, ld) > kMaxAccCoop) return 1;
  if (kk >= 1024) return 32;
  if (kk >= 128) return 8;
  return 1;
}
cudaError_t launch_schwarz(int la, int lb, const PairInfo* pairs, const PrimPair* prims, int first, int count,
                           const double* boys, const double* expt, double* out, int prim_mode, cudaStream_t st);
// out[0] += evaluated primitive quartets, out[1] += evaluated shell quartets
cudaError_t launch_count(const JKEntry* entries, const long long* prefix, int nentries, long long nwarps, int G,
                         const PairInfo* pairs, const double* pairQ, double thr, const float* pbound, double eps,
                         unsigned long long* out, cudaStream_t st);
cudaError_t fma_peak(int fp32, double* tflops);
cudaError_t launch_eri_packed(int la, int lb, int lc, int ld, const JKEntry* entries, const long long* prefix,
                              int nentries, long long nwarps, const PairInfo* pairs, const double* pairQ,
                              double thr, const PrimRec64* rec,
                              const double* boys, const double* expt, double* out, cudaStream_t st);
cudaError_t launch_quartet(int la, int lb, int lc, int ld, const PairInfo* pairs, const PrimPair* prims,
                           const double* boys, const double* expt, double* out, cudaStream_t st);

}  // namespace hfg
