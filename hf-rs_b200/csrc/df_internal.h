// Density-fitting data shared by df.cu (host) and df_kernels.cu (device).
#pragma once
#include <cuda_runtime.h>

#include "hfg_internal.h"

namespace hfg {

struct Df3cArgs {
  const PairInfo* bra_pairs;
  const PrimPair* bra_prims;
  const int* bra_idx;        // bra pairs of this launch (indices into bra_pairs)
  const long long* bra_col;  // first output column of each of them
  int nbra;
  const PairInfo* ket_pairs;  // unit-paired auxiliary shells
  const PrimPair* ket_prims;
  const int* ket_idx;
  int nket;
  const double* boys;
  const double* expt;
  double* out;  // out[aux function][column], leading dimension ld
  long long ld;
};

cudaError_t launch_df3c(int la, int lb, int lc, const Df3cArgs& args, cudaStream_t st);
cudaError_t launch_df_unpack(int mode, const void* B, long long ldb, const int2* colmn, long long ncol, int q0, int qc,
                             int n, void* out, cudaStream_t st);
cudaError_t launch_convert(int mode, const double* in, void* out, long long len, cudaStream_t st);
cudaError_t launch_convert_cols(int mode, const double* in, int w, long long rows, void* out, long long ldo,
                                long long c0, cudaStream_t st);
cudaError_t launch_df_j(int mode, const void* B, long long ncol, int rank, const double* p, double* gam, double* j,
                        cudaStream_t st);
cudaError_t launch_pack_density(const double* P, const int2* colmn, long long ncol, int n, double* p, cudaStream_t st);
cudaError_t launch_unpack_j(const double* j, const int2* colmn, long long ncol, int n, double* J, cudaStream_t st);
cudaError_t launch_convert_f32(int mode, const float* in, void* out, long long len, cudaStream_t st);
cudaError_t launch_accumulate_f32(double* acc, const float* src, double scale, long long len, cudaStream_t st);

}  // namespace hfg
