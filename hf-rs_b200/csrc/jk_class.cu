// One angular class of the J/K kernels, compiled once per class with
// -DHFG_LA=.. -DHFG_LB=.. -DHFG_LC=.. -DHFG_LD=.. so the 21 classes build in
// parallel.  Exports launch_jk_<LA><LB><LC><LD>().
#include <atomic>

#include "jk_dispatch.h"
#include "jk_kernels.cuh"

#ifndef HFG_LA
#error "compile with -DHFG_LA -DHFG_LB -DHFG_LC -DHFG_LD"
#endif

namespace hfg {

// Persistent grid: as many resident blocks as the kernel's occupancy allows
// on every SM, capped by the work.
template <typename T, int NS, bool BATCH = false>
static cudaError_t launch_t(const JKLaunchArgs& a, cudaStream_t st) {
  constexpr int block = 256;
  const size_t smem = boys_smem_bytes<T>();
  auto kern = BATCH ? jk_batch_kernel<HFG_LA, HFG_LB, HFG_LC, HFG_LD, T> : jk_kernel<HFG_LA, HFG_LB, HFG_LC, HFG_LD, T, NS>;
  // resident blocks per device (a process may drive different device
  // models), looked up once per device
  constexpr int kMaxDev = 64;
  static std::atomic<int> resident_by_dev[kMaxDev];
  int dev = 0;
  cudaGetDevice(&dev);
  int resident = (dev >= 0 && dev < kMaxDev) ? resident_by_dev[dev].load(std::memory_order_relaxed) : 0;
  if (resident <= 0) {
    int sms = 0, per_sm = 0;
    cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
#ifdef HFG_JK_CARVEOUT
    cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout, HFG_JK_CARVEOUT);
#endif
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, block, smem);
    resident = sms * (per_sm > 0 ? per_sm : 1);
    if (dev >= 0 && dev < kMaxDev) resident_by_dev[dev].store(resident, std::memory_order_relaxed);
  }
  // FP32 launches read the FP32 density copies (a batched launch carries
  // them in its molecule table)
  if (sizeof(T) == 4 && !BATCH && (!a.Dtot32 || (NS == 2 && !a.Dspin32))) return cudaErrorInvalidValue;
  if (a.serial) {
    if (a.nchunks > 0) kern<<<1, 32, smem, st>>>(a);
    return cudaGetLastError();
  }
  const long long want = (a.nchunks + (block / 32) - 1) / (block / 32);
  const long long grid = want < resident ? want : resident;
  if (grid <= 0) return cudaSuccess;
  kern<<<(unsigned)grid, block, smem, st>>>(a);
  return cudaGetLastError();
}

#define HFG_CAT2(a, b, c, d) launch_jk_##a##b##c##d
#define HFG_CAT(a, b, c, d) HFG_CAT2(a, b, c, d)
#define HFG_CATB2(a, b, c, d) launch_jkb_##a##b##c##d
#define HFG_CATB(a, b, c, d) HFG_CATB2(a, b, c, d)

// a batched launch over several molecules (RHF); a.nchunks is the total of
// their steps
cudaError_t HFG_CATB(HFG_LA, HFG_LB, HFG_LC, HFG_LD)(const JKLaunchArgs& a, bool fp32, cudaStream_t st) {
  return fp32 ? launch_t<float, 1, true>(a, st) : launch_t<double, 1, true>(a, st);
}

cudaError_t HFG_CAT(HFG_LA, HFG_LB, HFG_LC, HFG_LD)(const JKLaunchArgs& a, bool fp32, cudaStream_t st) {
  if (a.nspin == 2) return fp32 ? launch_t<float, 2>(a, st) : launch_t<double, 2>(a, st);
  return fp32 ? launch_t<float, 1>(a, st) : launch_t<double, 1>(a, st);
}

}  // namespace hfg
