// Dispatch of the per-class J/K launches (one translation unit per class).
#pragma once
#include <cuda_runtime.h>

#include "hfg_internal.h"

namespace hfg {

#define HFG_DECL(a, b, c, d)                                                            \
  cudaError_t launch_jk_##a##b##c##d(const JKLaunchArgs&, bool fp32, cudaStream_t); \
  cudaError_t launch_jkb_##a##b##c##d(const JKLaunchArgs&, bool fp32, cudaStream_t);
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

cudaError_t launch_jk(int la, int lb, int lc, int ld, bool fp32, const JKLaunchArgs& a, cudaStream_t st);
// The same over several molecules (a.jobs, a.job_steps, a.njobs; RHF).
cudaError_t launch_jk_batch(int la, int lb, int lc, int ld, bool fp32, const JKLaunchArgs& a, cudaStream_t st);
cudaError_t launch_schwarz(int la, int lb, const PairInfo* pairs, const PrimPair* prims, int first, int count,
                           const double* boys, const double* expt, double* out, int prim_mode, cudaStream_t st);
// out[0] += evaluated primitive quartets, out[1] += evaluated shell quartets
cudaError_t launch_count(const JKEntry* entries, const long long* prefix, int nentries, long long nwarps,
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
