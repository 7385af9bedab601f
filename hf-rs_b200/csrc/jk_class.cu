// One angular class of the J/K kernels, compiled once per class with
// -DHFG_LA=.. -DHFG_LB=.. -DHFG_LC=.. -DHFG_LD=.. so the 21 classes build in
// parallel.  Exports launch_jk_<LA><LB><LC><LD>().
#include "jk_kernels.cuh"
#include "jk_dispatch.h"

#ifndef HFG_LA
#error "compile with -DHFG_LA -DHFG_LB -DHFG_LC -DHFG_LD"
#endif

namespace hfg {

template <int G>
static cudaError_t launch_g(const JKLaunchArgs& a, bool fp32, cudaStream_t st) {
  const long long threads = a.nwarps * 32;
  const int block = 128;
  const long long grid = (threads + block - 1) / block;
  if (grid == 0) return cudaSuccess;
  if (fp32) jk_kernel<HFG_LA, HFG_LB, HFG_LC, HFG_LD, G, float><<<(unsigned)grid, block, 0, st>>>(a);
  else jk_kernel<HFG_LA, HFG_LB, HFG_LC, HFG_LD, G, double><<<(unsigned)grid, block, 0, st>>>(a);
  return cudaGetLastError();
}

#define HFG_CAT2(a, b, c, d) launch_jk_##a##b##c##d
#define HFG_CAT(a, b, c, d) HFG_CAT2(a, b, c, d)
cudaError_t HFG_CAT(HFG_LA, HFG_LB, HFG_LC, HFG_LD)(const JKLaunchArgs& a, int G, bool fp32, cudaStream_t st) {
  constexpr int nacc = EriClass<HFG_LA, HFG_LB, HFG_LC, HFG_LD>::NACC;
  if (G == 1) return launch_g<1>(a, fp32, st);
  if constexpr (nacc <= kMaxAccG8) {
    if (G == 8) return launch_g<8>(a, fp32, st);
  }
  if constexpr (nacc <= kMaxAccG32) {
    if (G == 32) return launch_g<32>(a, fp32, st);
  }
  return cudaErrorInvalidValue;
}

}  // namespace hfg
