// Pivoted Cholesky decomposition of the AO ERI supermatrix on the device.
//
// Stands in for hf-rs's pivoted_cholesky_eri (src/cholesky.rs:42-190):
// (pq|rs) ~ sum_K L_K(pq) L_K(rs), the pivot at each step being the largest
// residual diagonal (diagonals within 1e-12 relative of it are ties, taken
// by the smallest packed pair index), until the largest residual is at or
// below the threshold.  The vectors are returned as an hfg_df factor over
// every packed AO pair (compound_index order), so hfg_df_jk and hfg_scf_df
// run Cholesky-factorised RHF (run_cd_hf, src/hf_variants/cholesky_df.rs).
//
// Layout of the work: the ERI supermatrix V[pq][rs] is held on the device
// (packed 8-fold, from the J/K engine's integrals for quartets with
// Q_ab Q_cd > 1e-15, the column filter hf-rs uses), which bounds the
// system size to n_p (n_p + 1) / 2 doubles of device memory; hf-rs instead
// evaluates the pivots' columns on the fly.  Each step: the residual
// diagonal comes back to the host (the pivot rule must match exactly), the
// pivot column is gathered from V, the previous vectors' projection is
// removed with one DGEMV, and the diagonal is updated and checked on the
// device.
#include <cublas_v2.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <vector>

#include "df_handle.h"

using namespace hfg;

namespace {

__device__ __forceinline__ unsigned long long packed(unsigned long long i, unsigned long long j) {
  return i >= j ? i * (i + 1) / 2 + j : j * (j + 1) / 2 + i;
}

__global__ void chol_diag_kernel(const double* __restrict__ V, long long np, double* __restrict__ d) {
  for (long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x; k < np; k += (long long)gridDim.x * blockDim.x)
    d[k] = V[packed(k, k)];
}

__global__ void chol_column_kernel(const double* __restrict__ V, long long np, long long pivot, double* __restrict__ c) {
  for (long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x; k < np; k += (long long)gridDim.x * blockDim.x)
    c[k] = V[packed(k, pivot)];
}

// row = column / root with row[pivot] = root; diag -= row^2, with the check
// and clamp of src/cholesky.rs:172-178 (bad[0] set on a residual below
// -1e-10 scale)
__global__ void chol_update_kernel(double* __restrict__ row, long long np, long long pivot, double root, double scale,
                                   double* __restrict__ diag, int* __restrict__ bad) {
  for (long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x; k < np; k += (long long)gridDim.x * blockDim.x) {
    const double r = k == pivot ? root : row[k] / root;
    row[k] = r;
    const double d = diag[k] - r * r;
    if (d < -1e-10 * scale) *bad = 1;
    diag[k] = fmax(d, 0.0);
  }
}

}  // namespace

extern "C" int hfg_cholesky_eri(hfg_ctx* ctx, double threshold, size_t budget, hfg_df** out, double* max_residual,
                                long long* pivots, int max_pivots, int* n_pivots) {
  if (!ctx) return HFG_ERR_INVALID_INPUT;
  if (!out) return set_error(ctx, HFG_ERR_INVALID_INPUT, "null pointer");
  *out = nullptr;
  if (!(threshold >= 0.0) || !std::isfinite(threshold))
    return set_error(ctx, HFG_ERR_INVALID_INPUT, "Cholesky requires a basis and a finite, nonnegative threshold");
  std::lock_guard<std::mutex> lk(ctx->mu);
  cudaSetDevice(ctx->device);
  AllocScope alloc_scope(ctx->stream);
  cudaStream_t st = ctx->stream;
  const long long n = ctx->n, np = n * (n + 1) / 2;
  const size_t vlen = (size_t)np * (np + 1) / 2;
  int rc = HFG_OK;
#define CK(call)                         \
  do {                                   \
    rc = cuda_check(ctx, (call), #call); \
    if (rc != HFG_OK) return rc;         \
  } while (0)
  DevBuf<double> V, diag, col;
  DevBuf<int> bad;
  if (V.alloc(vlen) != cudaSuccess) {
    cudaGetLastError();
    return set_error(ctx, HFG_ERR_OOM, "pivoted Cholesky ERI decomposition: the ERI supermatrix does not fit");
  }
  CK(diag.alloc(np));
  CK(col.alloc(np));
  CK(bad.alloc(1));
  rc = eri_packed_locked(ctx, 1e-15, V.p, vlen);
  if (rc != HFG_OK) return rc;
  const unsigned g = (unsigned)std::min<long long>((np + 255) / 256, 4096);
  chol_diag_kernel<<<g, 256, 0, st>>>(V.p, np, diag.p);
  CK(cudaGetLastError());
  CK(cudaMemsetAsync(bad.p, 0, 4, st));
  std::vector<double> d(np);
  CK(cudaMemcpyAsync(d.data(), diag.p, np * 8, cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  double scale = 1.0;
  for (double x : d) scale = std::max(scale, x);
  for (double x : d)
    if (x < -1e-12 * scale)
      return set_error(ctx, HFG_ERR_INTEGRAL,
                       "pivoted Cholesky ERI decomposition: negative ERI diagonal; the Coulomb metric is not positive "
                       "semidefinite");
  // the vectors, row-major [rank][np]; capacity bounded by the budget
  const long long cap = std::max<long long>(1, std::min<long long>(np, (long long)(budget / (8 * (size_t)np))));
  auto df = std::make_unique<hfg_df>();
  df->ctx = ctx;
  df->n = (int)n;
  df->storage = HFG_DF_FP64;
  CK(df->B64.alloc((size_t)cap * np));
  if (cublasCreate(&df->blas) != CUBLAS_STATUS_SUCCESS) return set_error(ctx, HFG_ERR_CUDA, "cublasCreate");
  cublasSetStream(df->blas, st);
  std::vector<long long> piv;
  long long rank = 0;
  double maxres = 0.0;
  for (;;) {
    double largest = -INFINITY;
    for (double x : d) largest = std::max(largest, x);
    long long pivot = 0;
    while (!(d[pivot] >= largest - 1e-12 * std::fabs(largest))) ++pivot;
    const double maximum = d[pivot];
    if (maximum <= threshold || rank == np) {
      maxres = std::max(maximum, 0.0);
      break;
    }
    if (8.0 * (double)np * (double)(rank + 2) > (double)budget || rank >= cap)
      return set_error(ctx, HFG_ERR_INTEGRAL, "pivoted Cholesky ERI decomposition: factor storage exceeds the memory budget");
    const double root = std::sqrt(maximum);
    double* row = df->B64.p + (size_t)rank * np;
    chol_column_kernel<<<g, 256, 0, st>>>(V.p, np, pivot, row);
    CK(cudaGetLastError());
    if (rank > 0) {
      // row -= sum_K L_K L_K[pivot]: L column-major (np x rank, ld np), x = L[:, pivot] (stride np)
      const double m1 = -1.0, one = 1.0;
      if (cublasDgemv(df->blas, CUBLAS_OP_N, (int)np, (int)rank, &m1, df->B64.p, (int)np, df->B64.p + pivot, (int)np,
                      &one, row, 1) != CUBLAS_STATUS_SUCCESS)
        return set_error(ctx, HFG_ERR_CUDA, "Cholesky projection GEMV");
    }
    chol_update_kernel<<<g, 256, 0, st>>>(row, np, pivot, root, scale, diag.p, bad.p);
    CK(cudaGetLastError());
    int hbad = 0;
    CK(cudaMemcpyAsync(d.data(), diag.p, np * 8, cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(&hbad, bad.p, 4, cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    if (hbad) return set_error(ctx, HFG_ERR_INTEGRAL, "pivoted Cholesky ERI decomposition: nonpositive residual Coulomb diagonal");
    piv.push_back(pivot);
    ++rank;
  }
  if (rank == 0)
    return set_error(ctx, HFG_ERR_INTEGRAL,
                     "pivoted Cholesky ERI decomposition: threshold exceeds every ERI diagonal; no Cholesky vectors were "
                     "generated");
  // the factor over every packed AO pair, compound_index order
  std::vector<int2> colmn((size_t)np);
  for (long long p = 0; p < n; ++p)
    for (long long q = 0; q <= p; ++q) colmn[(size_t)(p * (p + 1) / 2 + q)] = make_int2((int)p, (int)q);
  CK(df->colmn.alloc(np));
  CK(cudaMemcpyAsync(df->colmn.p, colmn.data(), np * sizeof(int2), cudaMemcpyHostToDevice, st));
  CK(cudaStreamSynchronize(st));
  df->naux = df->rank = df->rank_total = (int)rank;
  df->ncol = np;
  if (max_residual) *max_residual = maxres;
  if (n_pivots) *n_pivots = (int)rank;
  if (pivots)
    for (long long k = 0; k < rank && k < max_pivots; ++k) pivots[k] = piv[k];
  *out = df.release();
#undef CK
  return HFG_OK;
}
