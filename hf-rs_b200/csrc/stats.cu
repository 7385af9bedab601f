// Work accounting and pipe-peak measurement.
//
// count_kernel walks the same work entries as the J/K kernels and counts the
// primitive quartets that survive primitive screening, so that the
// McMurchie-Davidson work unit of the roofline counts only evaluated work.
// fma_peak_kernel measures the FP64 / FP32 FMA pipe peak of this device with
// independent FMA chains in registers.
#include <cuda_runtime.h>

#include "hfg_internal.h"

namespace hfg {

__global__ void count_kernel(const JKEntry* __restrict__ entries, const long long* __restrict__ prefix, int nentries,
                             long long nwarps, const PairInfo* __restrict__ pairs,
                             const double* __restrict__ pairQ, double thr, const float* __restrict__ pbound,
                             double eps, unsigned long long* __restrict__ out) {
  const long long warp = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (warp >= nwarps) return;
  const int lane = threadIdx.x & 31;
  int lo = 0, hi = nentries;
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (prefix[mid] <= warp) lo = mid; else hi = mid;
  }
  const JKEntry e = entries[lo];
  const int k = e.k_lo + (int)(warp - prefix[lo]) * 32 + lane;
  unsigned long long c = 0, quartets = 0;
  if (k < e.k_hi && pairQ[k] * pairQ[e.bra] > thr) {
    quartets = 1;
    const PairInfo b = pairs[e.bra], q = pairs[k];
    // the kernels' loop: ket primitive pairs surviving against the largest bra
    // one, then bra primitive pairs while the product stays above eps
    // (FP32 products, as in the kernels)
    const float feps = (float)eps;
    const float bmax = pbound[b.rec_off];
    for (int ik = 0; ik < q.npp; ++ik) {
      const float qb = pbound[q.rec_off + (size_t)ik * q.rec_stride];
      if (qb * bmax < feps) break;
      int l = 0, h = b.npp;  // bounds sorted descending
      while (l < h) {
        const int m = (l + h) >> 1;
        if (pbound[b.rec_off + (size_t)m * b.rec_stride] * qb >= feps) l = m + 1; else h = m;
      }
      c += (unsigned long long)l;
    }
  }
  for (int off = 16; off > 0; off >>= 1) {
    c += __shfl_xor_sync(0xffffffffu, c, off);
    quartets += __shfl_xor_sync(0xffffffffu, quartets, off);
  }
  if (lane == 0 && c) atomicAdd(out, c);
  if (lane == 0 && quartets) atomicAdd(out + 1, quartets);
}

cudaError_t launch_count(const JKEntry* entries, const long long* prefix, int nentries, long long nwarps,
                         const PairInfo* pairs, const double* pairQ, double thr, const float* pbound, double eps,
                         unsigned long long* out, cudaStream_t st) {
  const long long threads = nwarps * 32;
  if (threads == 0) return cudaSuccess;
  count_kernel<<<(unsigned)((threads + 127) / 128), 128, 0, st>>>(entries, prefix, nentries, nwarps, pairs, pairQ,
                                                                   thr, pbound, eps, out);
  return cudaGetLastError();
}

template <typename T>
__global__ void fma_peak_kernel(T* out, int iters, T seed) {
  T a0 = seed + threadIdx.x, a1 = a0 + 1, a2 = a0 + 2, a3 = a0 + 3, a4 = a0 + 4, a5 = a0 + 5, a6 = a0 + 6,
    a7 = a0 + 7;
  const T m = (T)0.999999, c = (T)1e-7;
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int k = 0; k < 16; ++k) {
      a0 = a0 * m + c; a1 = a1 * m + c; a2 = a2 * m + c; a3 = a3 * m + c;
      a4 = a4 * m + c; a5 = a5 * m + c; a6 = a6 * m + c; a7 = a7 * m + c;
    }
  }
  const T s = a0 + a1 + a2 + a3 + a4 + a5 + a6 + a7;
  if (s == (T)-1) out[0] = s;  // keeps the chains live; never true
}

cudaError_t fma_peak(int fp32, double* tflops) {
  int dev = 0, sms = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  void* out = nullptr;
  cudaError_t e = cudaMalloc(&out, 16);
  if (e != cudaSuccess) return e;
  const int block = 256, grid = sms * 8, iters = 4096;
  cudaEvent_t a, b;
  cudaEventCreate(&a);
  cudaEventCreate(&b);
  float best = 1e30f;
  for (int rep = 0; rep < 4; ++rep) {
    cudaEventRecord(a);
    if (fp32) fma_peak_kernel<float><<<grid, block>>>((float*)out, iters, 1.0f);
    else fma_peak_kernel<double><<<grid, block>>>((double*)out, iters, 1.0);
    cudaEventRecord(b);
    cudaEventSynchronize(b);
    float ms = 0;
    cudaEventElapsedTime(&ms, a, b);
    if (rep > 0) best = ms < best ? ms : best;
  }
  e = cudaGetLastError();
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  cudaFree(out);
  const double flops = 2.0 * 8 * 16 * (double)iters * grid * block;
  *tflops = flops / (best * 1e-3) / 1e12;
  return e;
}

}  // namespace hfg
