// DF factor in a molecular-orbital basis and the RI-MP2 energy on the device.
//
// Stand in for hf-rs's DfTensor::transform and DfTensor::mp2_energy
// (src/df.rs:182-236):
//   transform: B^MO_Q = C^T B_Q C for every retained auxiliary function Q,
//              packed over p >= q (compound_index, src/scf.rs:222-235);
//   mp2_energy: E = sum_{ij in active occ, ab in virt} v_iajb (2 v_iajb - v_ibja)
//              / (e_i + e_j - e_a - e_b), v_iajb = sum_Q B_Q,ia B_Q,jb.
// FP64 throughout, on the stored factor (FP32 / BF16 storage converted while
// unpacking).  Per chunk of Q: unpack B_Q dense, T_Q = C^T B_Q and
// M_Q = T_Q C by batched cuBLAS DGEMMs (plain library GEMMs), then either
// pack M_Q or keep its occupied-virtual block L[Q][i][a].  The MP2 energy is
// one DGEMM per active occupied i, V_i[a][(j, b)] = sum_Q L[Q][i][a] L[Q][j][b],
// and a reduction kernel that applies the denominators (this library's own,
// one partial sum per block, summed on the host in a fixed order).
#include <cublas_v2.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <vector>

#include "df_handle.h"
#include "df_internal.h"

using namespace hfg;

namespace {

// pack the lower triangle of every m x m matrix of the chunk:
// out[q][p (p + 1) / 2 + r] = M[q][p][r], p >= r
__global__ void pack_mo_kernel(const double* __restrict__ M, int m, int qn, double* __restrict__ out) {
  const long long np = (long long)m * (m + 1) / 2;
  const long long tot = np * qn;
  for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < tot; t += (long long)gridDim.x * blockDim.x) {
    const int q = (int)(t / np);
    const long long k = t % np;
    int p = (int)((sqrt(8.0 * (double)k + 1.0) - 1.0) * 0.5);
    while ((long long)p * (p + 1) / 2 > k) --p;
    while ((long long)(p + 1) * (p + 2) / 2 <= k) ++p;
    const int r = (int)(k - (long long)p * (p + 1) / 2);
    out[t] = M[(size_t)q * m * m + (size_t)p * m + r];
  }
}

// L[q][i][a] = M[q][o0 + i][v0 + a] for the occupied-virtual block
__global__ void ov_block_kernel(const double* __restrict__ M, int m, int qn, int o0, int no, int v0, int nv,
                                double* __restrict__ L) {
  const long long tot = (long long)qn * no * nv;
  for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < tot; t += (long long)gridDim.x * blockDim.x) {
    const int q = (int)(t / ((long long)no * nv));
    const int r = (int)(t % ((long long)no * nv));
    const int i = r / nv, a = r % nv;
    L[t] = M[(size_t)q * m * m + (size_t)(o0 + i) * m + v0 + a];
  }
}

// Energy of one occupied i: V is (j, b, a) with V[(j * nv + b) * nv + a] =
// v_iajb.  Each block writes one partial sum.
__global__ void mp2_pair_kernel(const double* __restrict__ V, const double* __restrict__ eps, int i, int o0, int no,
                                int v0, int nv, double* __restrict__ part) {
  double s = 0.0;
  const long long tot = (long long)no * nv * nv;
  const double ei = eps[o0 + i];
  for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < tot; t += (long long)gridDim.x * blockDim.x) {
    const int j = (int)(t / ((long long)nv * nv));
    const int r = (int)(t % ((long long)nv * nv));
    const int b = r / nv, a = r % nv;
    const double v = V[t];                                   // v_iajb
    const double w = V[((size_t)j * nv + a) * nv + b];        // v_ibja
    const double gap = ei + eps[o0 + j] - eps[v0 + a] - eps[v0 + b];
    s += v * (2.0 * v - w) / gap;
  }
  for (int off = 16; off > 0; off >>= 1) s += __shfl_xor_sync(0xffffffffu, s, off);
  __shared__ double w32[32];
  if ((threadIdx.x & 31) == 0) w32[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int k = 0; k < (int)(blockDim.x >> 5); ++k) t += w32[k];
    part[blockIdx.x] = t;
  }
}

// M_Q = C^T B_Q C for the chunk [q0, q0 + qn): C row-major n x m on the device.
int mo_chunk(hfg_df* df, const double* dC, int m, int q0, int qn, double* dense, double* T, double* M) {
  hfg_ctx* ctx = df->ctx;
  cudaStream_t st = ctx->stream;
  const int n = df->n;
  const long long nn = (long long)n * n;
  int rc = cuda_check(ctx, cudaMemsetAsync(dense, 0, (size_t)qn * nn * 8, st), "clear");
  if (rc != HFG_OK) return rc;
  const int um = df->storage == HFG_DF_FP64 ? 0 : (df->storage == HFG_DF_FP32 ? 3 : 4);
  const void* Bs = df->storage == HFG_DF_FP64 ? (const void*)df->B64.p
                   : df->storage == HFG_DF_FP32 ? (const void*)df->B32.p : (const void*)df->B16.p;
  rc = cuda_check(ctx, launch_df_unpack(um, Bs, df->ncol, df->colmn.p, df->ncol, q0, qn, n, dense, st), "unpack");
  if (rc != HFG_OK) return rc;
  const double one = 1.0, zero = 0.0;
  // column-major views: C row-major (n x m) is Cc = C^T (m x n, ld m); the
  // unpack interleaves the chunk as [row][q][col], so B_Q (symmetric) starts
  // at dense + q n with leading dimension qn n.  T^T := Cc B_Q (m x n), then
  // M = T^T C (m x m): Cc with OP_T.
  if (cublasDgemmStridedBatched(df->blas, CUBLAS_OP_N, CUBLAS_OP_N, m, n, n, &one, dC, m, 0, dense, (long long)qn * n,
                                n, &zero, T, m, (long long)m * n, qn) != CUBLAS_STATUS_SUCCESS)
    return set_error(ctx, HFG_ERR_CUDA, "MO transform GEMM");
  if (cublasDgemmStridedBatched(df->blas, CUBLAS_OP_N, CUBLAS_OP_T, m, m, n, &one, T, m, (long long)m * n, dC, m, 0,
                                &zero, M, m, (long long)m * m, qn) != CUBLAS_STATUS_SUCCESS)
    return set_error(ctx, HFG_ERR_CUDA, "MO transform GEMM");
  return HFG_OK;
}

int chunk_size(const hfg_df* df, int m) {
  size_t free_b = 0, total_b = 0;
  cudaMemGetInfo(&free_b, &total_b);
  const size_t budget = std::max<size_t>((size_t)64 << 20, std::min<size_t>((size_t)4 << 30, free_b / 4));
  const size_t per_q = ((size_t)df->n * df->n + (size_t)m * df->n + (size_t)m * m) * 8;
  return (int)std::max<size_t>(1, std::min<size_t>((size_t)df->rank, budget / per_q));
}

}  // namespace

extern "C" int hfg_df_transform(hfg_df* df, const double* C, int m, double* out, size_t len) {
  if (!df) return HFG_ERR_INVALID_INPUT;
  hfg_ctx* ctx = df->ctx;
  if (!C || !out || m <= 0) return set_error(ctx, HFG_ERR_INVALID_INPUT, "DF MO coefficient dimension mismatch");
  const size_t np = (size_t)m * (m + 1) / 2;
  if (len != (size_t)df->rank * np) return set_error(ctx, HFG_ERR_INVALID_INPUT, "MO factor length must be rank * m (m + 1) / 2");
  for (size_t k = 0; k < (size_t)df->n * m; ++k)
    if (!std::isfinite(C[k])) return set_error(ctx, HFG_ERR_INVALID_INPUT, "non-finite MO coefficients");
  std::lock_guard<std::mutex> lk(ctx->mu);
  cudaSetDevice(ctx->device);
  AllocScope alloc_scope(ctx->stream);
  cudaStream_t st = ctx->stream;
  const int n = df->n, qc = chunk_size(df, m);
  DevBuf<double> dC, dense, T, M, P;
  int rc = cuda_check(ctx, dC.alloc((size_t)n * m), "alloc");
  if (rc == HFG_OK) rc = cuda_check(ctx, dense.alloc((size_t)qc * n * n), "alloc");
  if (rc == HFG_OK) rc = cuda_check(ctx, T.alloc((size_t)qc * m * n), "alloc");
  if (rc == HFG_OK) rc = cuda_check(ctx, M.alloc((size_t)qc * m * m), "alloc");
  if (rc == HFG_OK) rc = cuda_check(ctx, P.alloc((size_t)qc * np), "alloc");
  if (rc == HFG_OK) rc = cuda_check(ctx, cudaMemcpyAsync(dC.p, C, (size_t)n * m * 8, cudaMemcpyHostToDevice, st), "copy C");
  if (rc != HFG_OK) return rc;
  for (int q0 = 0; q0 < df->rank; q0 += qc) {
    const int qn = std::min(qc, df->rank - q0);
    rc = mo_chunk(df, dC.p, m, q0, qn, dense.p, T.p, M.p);
    if (rc != HFG_OK) return rc;
    pack_mo_kernel<<<1184, 256, 0, st>>>(M.p, m, qn, P.p);
    rc = cuda_check(ctx, cudaGetLastError(), "pack");
    if (rc == HFG_OK)
      rc = cuda_check(ctx, cudaMemcpyAsync(out + (size_t)q0 * np, P.p, (size_t)qn * np * 8, cudaMemcpyDeviceToHost, st),
                      "copy back");
    if (rc == HFG_OK) rc = cuda_check(ctx, cudaStreamSynchronize(st), "transform");
    if (rc != HFG_OK) return rc;
  }
  return HFG_OK;
}

extern "C" int hfg_df_mp2(hfg_df* df, const double* C, const double* eps, int m, int n_occ, int n_frozen,
                          double* energy) {
  if (!df) return HFG_ERR_INVALID_INPUT;
  hfg_ctx* ctx = df->ctx;
  if (!C || !eps || !energy || m <= 0) return set_error(ctx, HFG_ERR_INVALID_INPUT, "null pointer");
  if (n_frozen < 0 || n_frozen > n_occ || n_occ > m)
    return set_error(ctx, HFG_ERR_INVALID_INPUT, "invalid RI-MP2 orbital partition");
  // (ia|jb) sums over every auxiliary function before the energy expression
  if (df->shard()) return set_error(ctx, HFG_ERR_INVALID_INPUT, "RI-MP2 needs the whole factor, not a shard of it");
  const int no = n_occ - n_frozen, nv = m - n_occ;
  *energy = 0.0;
  if (no == 0 || nv == 0) return HFG_OK;
  // hf-rs rejects any denominator within 1e-12 of zero
  {
    std::vector<double> so, sv;
    for (int i = n_frozen; i < n_occ; ++i)
      for (int j = n_frozen; j < n_occ; ++j) so.push_back(eps[i] + eps[j]);
    for (int a = n_occ; a < m; ++a)
      for (int b = n_occ; b < m; ++b) sv.push_back(eps[a] + eps[b]);
    std::sort(sv.begin(), sv.end());
    for (double x : so) {
      auto it = std::lower_bound(sv.begin(), sv.end(), x);
      if ((it != sv.end() && std::fabs(*it - x) < 1e-12) || (it != sv.begin() && std::fabs(*(it - 1) - x) < 1e-12))
        return set_error(ctx, HFG_ERR_SCF, "singular RI-MP2 denominator");
    }
  }
  std::lock_guard<std::mutex> lk(ctx->mu);
  cudaSetDevice(ctx->device);
  AllocScope alloc_scope(ctx->stream);
  cudaStream_t st = ctx->stream;
  const int n = df->n, qc = chunk_size(df, m), rank = df->rank;
  DevBuf<double> dC, dE, dense, T, M, L, V, part;
  constexpr int kBlocks = 296;
  int rc = cuda_check(ctx, dC.alloc((size_t)n * m), "alloc");
  if (rc == HFG_OK) rc = cuda_check(ctx, dE.alloc(m), "alloc");
  if (rc == HFG_OK) rc = cuda_check(ctx, dense.alloc((size_t)qc * n * n), "alloc");
  if (rc == HFG_OK) rc = cuda_check(ctx, T.alloc((size_t)qc * m * n), "alloc");
  if (rc == HFG_OK) rc = cuda_check(ctx, M.alloc((size_t)qc * m * m), "alloc");
  if (rc == HFG_OK) rc = cuda_check(ctx, L.alloc((size_t)rank * no * nv), "alloc (ia|Q) factor");
  if (rc == HFG_OK) rc = cuda_check(ctx, V.alloc((size_t)nv * no * nv), "alloc");
  if (rc == HFG_OK) rc = cuda_check(ctx, part.alloc(kBlocks), "alloc");
  if (rc == HFG_OK) rc = cuda_check(ctx, cudaMemcpyAsync(dC.p, C, (size_t)n * m * 8, cudaMemcpyHostToDevice, st), "copy C");
  if (rc == HFG_OK) rc = cuda_check(ctx, cudaMemcpyAsync(dE.p, eps, (size_t)m * 8, cudaMemcpyHostToDevice, st), "copy eps");
  if (rc != HFG_OK) return rc;
  for (int q0 = 0; q0 < rank; q0 += qc) {
    const int qn = std::min(qc, rank - q0);
    rc = mo_chunk(df, dC.p, m, q0, qn, dense.p, T.p, M.p);
    if (rc != HFG_OK) return rc;
    ov_block_kernel<<<1184, 256, 0, st>>>(M.p, m, qn, n_frozen, no, n_occ, nv, L.p + (size_t)q0 * no * nv);
    rc = cuda_check(ctx, cudaGetLastError(), "occupied-virtual block");
    if (rc != HFG_OK) return rc;
  }
  const double one = 1.0, zero = 0.0;
  const int ld = no * nv;
  std::vector<double> h(kBlocks);
  double e = 0.0;
  for (int i = 0; i < no; ++i) {
    // V[a][(j, b)] = sum_Q L[Q][i][a] L[Q][j][b]
    if (cublasDgemm(df->blas, CUBLAS_OP_N, CUBLAS_OP_T, nv, no * nv, rank, &one, L.p + (size_t)i * nv, ld, L.p, ld,
                    &zero, V.p, nv) != CUBLAS_STATUS_SUCCESS)
      return set_error(ctx, HFG_ERR_CUDA, "RI-MP2 GEMM");
    mp2_pair_kernel<<<kBlocks, 256, 0, st>>>(V.p, dE.p, i, n_frozen, no, n_occ, nv, part.p);
    rc = cuda_check(ctx, cudaGetLastError(), "RI-MP2 energy");
    if (rc == HFG_OK) rc = cuda_check(ctx, cudaMemcpyAsync(h.data(), part.p, kBlocks * 8, cudaMemcpyDeviceToHost, st), "copy");
    if (rc == HFG_OK) rc = cuda_check(ctx, cudaStreamSynchronize(st), "RI-MP2");
    if (rc != HFG_OK) return rc;
    for (double x : h) e += x;
  }
  *energy = e;
  return HFG_OK;
}
