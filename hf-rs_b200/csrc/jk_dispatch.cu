// Dispatch tables for the J/K, Schwarz and single-quartet kernels: the
// generated kernels for s, p and d, the generic engine (eri_md.cu) for
// classes with an f shell.
#include "jk_dispatch.h"
#include "eri_md.h"
#include "eri_prim.cuh"

namespace hfg {

cudaError_t launch_jk(int la, int lb, int lc, int ld, bool fp32, const JKLaunchArgs& a, cudaStream_t st) {
  // classes with an f shell: the generic engine, FP64 only
  if (la > kLMax || lb > kLMax || lc > kLMax || ld > kLMax)
    return fp32 ? cudaErrorInvalidValue : launch_jk_md(la, lb, lc, ld, a, st);
#define HFG_CASE(A, B, C, D) \
  if (la == A && lb == B && lc == C && ld == D) return launch_jk_##A##B##C##D(a, fp32, st);
  HFG_CASE(0, 0, 0, 0)
  HFG_CASE(1, 0, 0, 0)
  HFG_CASE(1, 0, 1, 0)
  HFG_CASE(1, 1, 0, 0)
  HFG_CASE(1, 1, 1, 0)
  HFG_CASE(1, 1, 1, 1)
  HFG_CASE(2, 0, 0, 0)
  HFG_CASE(2, 0, 1, 0)
  HFG_CASE(2, 0, 1, 1)
  HFG_CASE(2, 0, 2, 0)
  HFG_CASE(2, 1, 0, 0)
  HFG_CASE(2, 1, 1, 0)
  HFG_CASE(2, 1, 1, 1)
  HFG_CASE(2, 1, 2, 0)
  HFG_CASE(2, 1, 2, 1)
  HFG_CASE(2, 2, 0, 0)
  HFG_CASE(2, 2, 1, 0)
  HFG_CASE(2, 2, 1, 1)
  HFG_CASE(2, 2, 2, 0)
  HFG_CASE(2, 2, 2, 1)
  HFG_CASE(2, 2, 2, 2)
#undef HFG_CASE
  return cudaErrorInvalidValue;
}

cudaError_t launch_jk_batch(int la, int lb, int lc, int ld, bool fp32, const JKLaunchArgs& a, cudaStream_t st) {
  if (la > kLMax || lb > kLMax || lc > kLMax || ld > kLMax) return cudaErrorInvalidValue;
#define HFG_CASE(A, B, C, D) \
  if (la == A && lb == B && lc == C && ld == D) return launch_jkb_##A##B##C##D(a, fp32, st);
  HFG_CASE(0, 0, 0, 0)
  HFG_CASE(1, 0, 0, 0)
  HFG_CASE(1, 0, 1, 0)
  HFG_CASE(1, 1, 0, 0)
  HFG_CASE(1, 1, 1, 0)
  HFG_CASE(1, 1, 1, 1)
  HFG_CASE(2, 0, 0, 0)
  HFG_CASE(2, 0, 1, 0)
  HFG_CASE(2, 0, 1, 1)
  HFG_CASE(2, 0, 2, 0)
  HFG_CASE(2, 1, 0, 0)
  HFG_CASE(2, 1, 1, 0)
  HFG_CASE(2, 1, 1, 1)
  HFG_CASE(2, 1, 2, 0)
  HFG_CASE(2, 1, 2, 1)
  HFG_CASE(2, 2, 0, 0)
  HFG_CASE(2, 2, 1, 0)
  HFG_CASE(2, 2, 1, 1)
  HFG_CASE(2, 2, 2, 0)
  HFG_CASE(2, 2, 2, 1)
  HFG_CASE(2, 2, 2, 2)
#undef HFG_CASE
  return cudaErrorInvalidValue;
}

cudaError_t launch_schwarz(int la, int lb, const PairInfo* pairs, const PrimPair* prims, int first, int count,
                           const double* boys, const double* expt, double* out, int prim_mode, cudaStream_t st) {
  if (count <= 0) return cudaSuccess;
  if (la > kLMax || lb > kLMax) return launch_schwarz_md(la, lb, pairs, prims, first, count, boys, expt, out, prim_mode, st);
  const int smem = (int)boys_smem_bytes<double>();
  const int block = 64, grid = (count + block - 1) / block;
#define HFG_CASE(A, B)                                                                             \
  if (la == A && lb == B) {                                                                        \
    cudaFuncSetAttribute(schwarz_kernel<A, B>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);             \
    schwarz_kernel<A, B><<<grid, block, smem, st>>>(pairs, prims, first, count, boys, expt, out, prim_mode);   \
    return cudaGetLastError();                                                                     \
  }
  HFG_CASE(0, 0)
  HFG_CASE(1, 0)
  HFG_CASE(1, 1)
  HFG_CASE(2, 0)
  HFG_CASE(2, 1)
  HFG_CASE(2, 2)
#undef HFG_CASE
  return cudaErrorInvalidValue;
}

cudaError_t launch_quartet(int la, int lb, int lc, int ld, const PairInfo* pairs, const PrimPair* prims,
                           const double* boys, const double* expt, double* out, cudaStream_t st) {
  if (la > kLMax || lb > kLMax || lc > kLMax || ld > kLMax)
    return launch_quartet_md(la, lb, lc, ld, pairs, prims, boys, expt, out, st);
  const int smem = (int)boys_smem_bytes<double>();
#define HFG_CASE(A, B, C, D)                                                    \
  if (la == A && lb == B && lc == C && ld == D) {                               \
    cudaFuncSetAttribute(quartet_kernel<A, B, C, D>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem); \
    quartet_kernel<A, B, C, D><<<1, 32, smem, st>>>(pairs, prims, boys, expt, out);                  \
    return cudaGetLastError();                                                  \
  }
#define HFG_KET(A, B) \
  HFG_CASE(A, B, 0, 0) HFG_CASE(A, B, 1, 0) HFG_CASE(A, B, 1, 1) HFG_CASE(A, B, 2, 0) HFG_CASE(A, B, 2, 1) HFG_CASE(A, B, 2, 2)
  HFG_KET(0, 0)
  HFG_KET(1, 0)
  HFG_KET(1, 1)
  HFG_KET(2, 0)
  HFG_KET(2, 1)
  HFG_KET(2, 2)
#undef HFG_KET
#undef HFG_CASE
  return cudaErrorInvalidValue;
}

}  // namespace hfg
