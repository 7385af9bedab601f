// Density fitting: DfTensor::build and coulomb_exchange_rhf on the device.
//
// Stands in for hf-rs's DfTensor::build / build_in_space (src/df.rs:89-127)
// in the Cartesian auxiliary space and coulomb_exchange_rhf
// (src/df.rs:133-174):
//   M = (P|Q), X = canonical_orthogonalizer(M, cutoff) (src/df.rs:16-28),
//   B = X^T (P|mn) over unique AO pairs m >= n,
//   J = sum_Q (B_Q . P) B_Q,  K = 2 sum_Q (B_Q C_occ)(B_Q C_occ)^T.
// Differences of layout, not of arithmetic: B is kept only for the AO pairs
// of shell pairs whose Schwarz bound exceeds `pair_threshold` (0 keeps all,
// as hf-rs does), and may be stored in FP32 or BF16.  J uses two GEMVs on
// the packed B; K runs chunks of auxiliary functions through two GEMMs on
// dense unpacked blocks (FP64, TF32 or BF16 tensor-core GEMMs with FP32
// accumulation, summed into FP64).
#include <cublas_v2.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cstdlib>
#include <cusolverDn.h>

#include <algorithm>
#include <cmath>
#include <map>
#include <vector>

#include "df_handle.h"
#include "df_internal.h"
#include "df_umma.h"
#include "hfg_ctx.h"

using namespace hfg;


namespace {

// The auxiliary basis as unit-paired "pairs" on the device, grouped by
// angular momentum (hf-rs's constant() partner, src/df.rs:30-41).
struct AuxSet {
  hfg_ctx shells;
  DevBuf<PairInfo> dup;
  DevBuf<PrimPair> dupr;
  std::map<int, std::vector<int>> by_l;
  std::map<int, DevBuf<int>> idx;
};

int make_aux_set(hfg_ctx* ctx, const hfg_basis* aux, AuxSet& ax) {
  cudaStream_t st = ctx->stream;
  // the three-centre kernels cover orbital pairs of s, p and d shells
  if (ctx->lmax > kLMax)
    return set_error(ctx, HFG_ERR_UNSUPPORTED, "density fitting covers orbital s, p and d shells");
  int rc = build_shell_list(&ax.shells, aux, 4);
  if (rc != HFG_OK) return set_error(ctx, rc, "auxiliary basis: " + ax.shells.err);
  std::vector<PairInfo> upairs(ax.shells.shells.size());
  std::vector<PrimPair> uprims;
  for (size_t s = 0; s < ax.shells.shells.size(); ++s) {
    const Shell& sh = ax.shells.shells[s];
    PairInfo& pi = upairs[s];
    pi = PairInfo{};
    pi.Ax = sh.c[0];
    pi.Ay = sh.c[1];
    pi.Az = sh.c[2];
    pi.ao_a = sh.ao;
    pi.pp_off = (int)uprims.size();
    pi.npp = sh.K;
    for (int q = 0; q < sh.K; ++q) {
      PrimPair p{};
      p.p = ax.shells.exps[sh.prim_off + q];
      p.inv_p = 1.0 / p.p;
      p.kp = ax.shells.coefs[sh.prim_off + q] * p.inv_p;  // unit partner: coefficient 1, exp(0) = 1
      uprims.push_back(p);
    }
  }
  rc = cuda_check(ctx, ax.dup.alloc(upairs.size()), "alloc");
  if (rc == HFG_OK) rc = cuda_check(ctx, ax.dupr.alloc(uprims.size()), "alloc");
  if (rc == HFG_OK)
    rc = cuda_check(ctx, cudaMemcpyAsync(ax.dup.p, upairs.data(), upairs.size() * sizeof(PairInfo),
                                         cudaMemcpyHostToDevice, st), "copy");
  if (rc == HFG_OK)
    rc = cuda_check(ctx, cudaMemcpyAsync(ax.dupr.p, uprims.data(), uprims.size() * sizeof(PrimPair),
                                         cudaMemcpyHostToDevice, st), "copy");
  if (rc != HFG_OK) return rc;
  for (size_t s = 0; s < ax.shells.shells.size(); ++s) ax.by_l[ax.shells.shells[s].l].push_back((int)s);
  for (auto& kv : ax.by_l) {
    rc = cuda_check(ctx, ax.idx[kv.first].alloc(kv.second.size()), "alloc");
    if (rc == HFG_OK)
      rc = cuda_check(ctx, cudaMemcpyAsync(ax.idx[kv.first].p, kv.second.data(), kv.second.size() * 4,
                                           cudaMemcpyHostToDevice, st), "copy");
    if (rc != HFG_OK) return rc;
  }
  // the host copies above are pageable: complete them before they go away
  return cuda_check(ctx, cudaStreamSynchronize(st), "aux set");
}

int gemm_ex(hfg_ctx* ctx, cublasHandle_t h, cublasOperation_t ta, cublasOperation_t tb, int m, int n, int k,
            const void* A, cudaDataType ta_t, int lda, const void* B, cudaDataType tb_t, int ldb, float beta,
            float* C, int ldc, cublasComputeType_t ct) {
  const float alpha = 1.0f;
  const cublasStatus_t s =
      cublasGemmEx(h, ta, tb, m, n, k, &alpha, A, ta_t, lda, B, tb_t, ldb, &beta, C, CUDA_R_32F, ldc, ct,
                   CUBLAS_GEMM_DEFAULT);
  return s == CUBLAS_STATUS_SUCCESS ? HFG_OK : set_error(ctx, HFG_ERR_CUDA, "cublasGemmEx failed");
}

int ensure_tiles(hfg_df* df, int kind) {
  if (df->tiles_ready[kind]) return HFG_OK;
  hfg_ctx* ctx = df->ctx;
  std::vector<int2> colmn((size_t)df->ncol);
  int rc = cuda_check(ctx, cudaMemcpy(colmn.data(), df->colmn.p, colmn.size() * sizeof(int2), cudaMemcpyDeviceToHost),
                      "copy pair map");
  if (rc != HFG_OK) return rc;
  TileStructure& t = df->tiles[kind];
  t.build(colmn, df->n, kind);
  auto up = [&](DevBuf<int>& d, const std::vector<int>& h) -> int {
    int r = cuda_check(ctx, d.alloc(std::max<size_t>(1, h.size())), "alloc tile structure");
    if (r == HFG_OK && !h.empty())
      r = cuda_check(ctx, cudaMemcpyAsync(d.p, h.data(), h.size() * 4, cudaMemcpyHostToDevice, ctx->stream),
                     "copy tile structure");
    return r;
  };
  if ((rc = up(df->tile_off[kind], t.tile_off)) != HFG_OK) return rc;
  if ((rc = up(df->tile_kt[kind], t.tile_kt)) != HFG_OK) return rc;
  if ((rc = up(df->tile_map[kind], t.tile_map)) != HFG_OK) return rc;
  rc = cuda_check(ctx, cudaStreamSynchronize(ctx->stream), "tile structure");
  if (rc != HFG_OK) return rc;
  t.tile_map.clear();
  t.tile_map.shrink_to_fit();
  df->tiles_ready[kind] = true;
  return HFG_OK;
}

}  // namespace

extern "C" {

int hfg_df_build(hfg_ctx* ctx, const hfg_basis* aux, double metric_cutoff, double pair_threshold, int storage,
                 hfg_df** out) {
  return hfg_df_build_shard(ctx, aux, metric_cutoff, pair_threshold, storage, 0, 1, out);
}

int hfg_df_build_shard(hfg_ctx* ctx, const hfg_basis* aux, double metric_cutoff, double pair_threshold, int storage,
                       int shard, int nshards, hfg_df** out) {
  if (!ctx || !aux || !out) return HFG_ERR_INVALID_INPUT;
  *out = nullptr;
  if (nshards < 1 || shard < 0 || shard >= nshards) return set_error(ctx, HFG_ERR_INVALID_INPUT, "invalid shard");
  if (!(metric_cutoff > 0) || !std::isfinite(metric_cutoff))
    return set_error(ctx, HFG_ERR_INVALID_INPUT, "DF metric cutoff must be finite and positive");
  if (storage < HFG_DF_FP64 || storage > HFG_DF_BF16) return set_error(ctx, HFG_ERR_INVALID_INPUT, "storage");
  std::lock_guard<std::mutex> lk(ctx->mu);
  cudaSetDevice(ctx->device);
  AllocScope alloc_scope(ctx->stream);
  auto df = std::make_unique<hfg_df>();
  df->ctx = ctx;
  df->n = ctx->n;
  df->storage = storage;
  cudaStream_t st = ctx->stream;
  int rc = HFG_OK;
#define CK(call)                         \
  do {                                   \
    rc = cuda_check(ctx, (call), #call); \
    if (rc != HFG_OK) return rc;         \
  } while (0)
  // auxiliary shells and their unit-partner "pairs"
  AuxSet ax;
  rc = make_aux_set(ctx, aux, ax);
  if (rc != HFG_OK) return rc;
  hfg_ctx& auxc = ax.shells;
  const int naux = auxc.n;
  df->naux = naux;
  DevBuf<PairInfo>& dup = ax.dup;
  DevBuf<PrimPair>& dupr = ax.dupr;
  std::map<int, std::vector<int>>& aux_by_l = ax.by_l;
  std::map<int, DevBuf<int>>& aux_idx = ax.idx;
  // metric (P|Q): bra and ket both unit-paired auxiliary shells
  CK(df->metric.alloc((size_t)naux * naux));
  for (auto& bk : aux_by_l) {
    std::vector<long long> cols;
    for (int s : bk.second) cols.push_back(auxc.shells[s].ao);
    DevBuf<long long> dcols;
    CK(dcols.alloc(cols.size()));
    CK(cudaMemcpyAsync(dcols.p, cols.data(), cols.size() * 8, cudaMemcpyHostToDevice, st));
    for (auto& kk : aux_by_l) {
      Df3cArgs a{dup.p, dupr.p, aux_idx[bk.first].p, dcols.p, (int)bk.second.size(), dup.p, dupr.p,
                 aux_idx[kk.first].p, (int)kk.second.size(), ctx->d_boys64.p, ctx->d_expt64.p, df->metric.p, naux};
      CK(launch_df3c(bk.first, 0, kk.first, a, st));
    }
    CK(cudaStreamSynchronize(st));
  }
  // canonical orthogonaliser of the metric (cutoff on its eigenvalues)
  cusolverDnHandle_t solver = nullptr;
  if (cusolverDnCreate(&solver) != CUSOLVER_STATUS_SUCCESS) return set_error(ctx, HFG_ERR_CUDA, "cusolver");
  cusolverDnSetStream(solver, st);
  DevBuf<double> V, w, work;
  DevBuf<int> info;
  CK(V.alloc((size_t)naux * naux));
  CK(w.alloc(naux));
  CK(info.alloc(1));
  CK(cudaMemcpyAsync(V.p, df->metric.p, (size_t)naux * naux * 8, cudaMemcpyDeviceToDevice, st));
  int lwork = 0;
  cusolverDnDsyevd_bufferSize(solver, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_LOWER, naux, V.p, naux, w.p, &lwork);
  CK(work.alloc(lwork));
  if (cusolverDnDsyevd(solver, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_LOWER, naux, V.p, naux, w.p, work.p, lwork,
                       info.p) != CUSOLVER_STATUS_SUCCESS) {
    cusolverDnDestroy(solver);
    return set_error(ctx, HFG_ERR_CUDA, "metric eigendecomposition failed");
  }
  std::vector<double> wh(naux);
  CK(cudaMemcpyAsync(wh.data(), w.p, naux * 8, cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  cusolverDnDestroy(solver);
  if (wh[0] < -metric_cutoff) return set_error(ctx, HFG_ERR_INTEGRAL, "DF metric has a negative eigenvalue");
  int first = 0;
  while (first < naux && wh[first] < metric_cutoff) ++first;
  const int rank_total = naux - first;
  if (rank_total <= 0) return set_error(ctx, HFG_ERR_INTEGRAL, "DF metric has zero retained rank");
  // this shard's rows of B: whitened functions [row0, row0 + rank)
  const int row0 = (int)((long long)rank_total * shard / nshards);
  const int rank = (int)((long long)rank_total * (shard + 1) / nshards) - row0;
  if (rank <= 0) return set_error(ctx, HFG_ERR_INVALID_INPUT, "more DF shards than retained auxiliary functions");
  df->rank = rank;
  df->rank_total = rank_total;
  df->row0 = row0;
  // Xm = V[:, first + row0 : first + row0 + rank] diag(w^-1/2), column-major
  // naux x rank (columns move left only, so none is overwritten before use)
  {
    std::vector<double> Vh((size_t)naux * naux);
    CK(cudaMemcpyAsync(Vh.data(), V.p, Vh.size() * 8, cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    for (int c = 0; c < rank; ++c) {
      const double sc = 1.0 / std::sqrt(wh[first + row0 + c]);
      for (int r = 0; r < naux; ++r) Vh[(size_t)c * naux + r] = Vh[(size_t)(first + row0 + c) * naux + r] * sc;
    }
    CK(cudaMemcpyAsync(V.p, Vh.data(), (size_t)naux * rank * 8, cudaMemcpyHostToDevice, st));
  }

  // significant orbital shell pairs (in pair order) and their unique AO-pair columns
  struct SigPair {
    int pair, la, lb;
    long long col;
  };
  std::vector<SigPair> sig;
  std::vector<int2> colmn;
  long long ncol = 0;
  for (size_t i = 0; i < ctx->h_pairs.size(); ++i) {
    if (!(ctx->sorted_Q[i] > pair_threshold)) continue;
    const PairInfo& pi = ctx->h_pairs[i];
    const PairClass& c = ctx->classes[pi.cls];
    const int na = (c.la + 1) * (c.la + 2) / 2, nb = (c.lb + 1) * (c.lb + 2) / 2;
    sig.push_back({(int)i, c.la, c.lb, ncol});
    for (int a = 0; a < na; ++a)
      for (int b = 0; b < nb; ++b) {
        if (pi.same && b > a) continue;
        colmn.push_back(make_int2(pi.ao_a + a, pi.ao_b + b));
      }
    ncol += pi.same ? na * (na + 1) / 2 : na * nb;
  }
  df->ncol = ncol;
  CK(df->colmn.alloc(ncol));
  CK(cudaMemcpyAsync(df->colmn.p, colmn.data(), ncol * sizeof(int2), cudaMemcpyHostToDevice, st));
  if (cublasCreate(&df->blas) != CUBLAS_STATUS_SUCCESS) return set_error(ctx, HFG_ERR_CUDA, "cublasCreate");
  cublasSetStream(df->blas, st);
  // the stored factor B (row-major [rank][ncol]) in its storage precision
  if (storage == HFG_DF_FP64) CK(df->B64.alloc((size_t)rank * ncol));
  else if (storage == HFG_DF_FP32) CK(df->B32.alloc((size_t)rank * ncol));
  else CK(df->B16.alloc((size_t)rank * ncol));
  // (P|mn) and B = Xm^T (P|mn) over chunks of consecutive columns, so that
  // only one chunk of the FP64 three-centre integrals (naux x width) and of
  // the FP64 product (rank x width) is held at a time: about 8 GiB, or a
  // quarter of the free device memory if that is less
  size_t free_b = 0, total_b = 0;
  cudaMemGetInfo(&free_b, &total_b);
  const double budget = std::min(8.0 * (1ull << 30), 0.25 * (double)free_b);
  const long long per_col = 8LL * (naux + (storage == HFG_DF_FP64 ? 0 : rank));
  long long width_max = std::max(256LL, std::min(ncol, (long long)(budget / (double)per_col)));
  // HFG_DF_CHUNK_COLS caps the chunk width (tests use it to exercise chunking
  // on small systems)
  if (const char* ev = getenv("HFG_DF_CHUNK_COLS")) {
    const long long v = atoll(ev);
    if (v > 0) width_max = std::min(width_max, std::max(64LL, v));
  }
  DevBuf<double> T3, Bt;
  CK(T3.alloc((size_t)naux * std::min(width_max + 64, ncol)));
  if (storage != HFG_DF_FP64) CK(Bt.alloc((size_t)rank * std::min(width_max + 64, ncol)));
  size_t p0 = 0;
  while (p0 < sig.size()) {
    // pairs [p0, p1) whose columns fit in the chunk (one pair has at most 36)
    const long long c0 = sig[p0].col;
    size_t p1 = p0;
    while (p1 < sig.size() && sig[p1].col - c0 < width_max) ++p1;
    const long long c1 = p1 < sig.size() ? sig[p1].col : ncol;
    const int w = (int)(c1 - c0);
    std::map<std::pair<int, int>, std::pair<std::vector<int>, std::vector<long long>>> by_class;
    for (size_t k = p0; k < p1; ++k) {
      auto& e = by_class[{sig[k].la, sig[k].lb}];
      e.first.push_back(sig[k].pair);
      e.second.push_back(sig[k].col - c0);
    }
    for (auto& bc : by_class) {
      DevBuf<int> bidx;
      DevBuf<long long> bcol;
      CK(bidx.alloc(bc.second.first.size()));
      CK(bcol.alloc(bc.second.second.size()));
      CK(cudaMemcpyAsync(bidx.p, bc.second.first.data(), bc.second.first.size() * 4, cudaMemcpyHostToDevice, st));
      CK(cudaMemcpyAsync(bcol.p, bc.second.second.data(), bc.second.second.size() * 8, cudaMemcpyHostToDevice, st));
      for (auto& kk : aux_by_l) {
        Df3cArgs a{ctx->d_pairs.p, ctx->d_prims.p, bidx.p, bcol.p, (int)bc.second.first.size(), dup.p, dupr.p,
                   aux_idx[kk.first].p, (int)kk.second.size(), ctx->d_boys64.p, ctx->d_expt64.p, T3.p, w};
        CK(launch_df3c(bc.first.first, bc.first.second, kk.first, a, st));
      }
      CK(cudaStreamSynchronize(st));  // the index buffers are released at the end of this scope
    }
    // column-major view: T3c (w x naux, ld w) times Xm (naux x rank) gives the
    // chunk's columns of B (row-major [rank][ncol] = column-major ncol x rank)
    const double one = 1.0, zero = 0.0;
    double* dst = storage == HFG_DF_FP64 ? df->B64.p + c0 : Bt.p;
    const int ldc = storage == HFG_DF_FP64 ? (int)ncol : w;
    if (cublasDgemm(df->blas, CUBLAS_OP_N, CUBLAS_OP_N, w, rank, naux, &one, T3.p, w, V.p, naux, &zero, dst, ldc) !=
        CUBLAS_STATUS_SUCCESS)
      return set_error(ctx, HFG_ERR_CUDA, "B = X^T (P|mn) GEMM failed");
    if (storage != HFG_DF_FP64)
      CK(launch_convert_cols(storage == HFG_DF_FP32 ? 1 : 2, Bt.p, w, rank,
                             storage == HFG_DF_FP32 ? (void*)df->B32.p : (void*)df->B16.p, ncol, c0, st));
    p0 = p1;
  }
  CK(cudaStreamSynchronize(st));
  T3.release();
  Bt.release();
  *out = df.release();
#undef CK
  return HFG_OK;
}

int hfg_df_destroy(hfg_df* df) {
  if (!df) return HFG_OK;
  cudaSetDevice(df->ctx->device);
  AllocScope alloc_scope(df->ctx->stream);
  cudaStreamSynchronize(df->ctx->stream);
  delete df;
  return HFG_OK;
}

int hfg_df_sizes(const hfg_df* df, int* naux, int* rank, long long* ncol) {
  if (!df) return HFG_ERR_INVALID_INPUT;
  if (naux) *naux = df->naux;
  if (rank) *rank = df->rank;
  if (ncol) *ncol = df->ncol;
  return HFG_OK;
}

int hfg_df_metric(hfg_df* df, double* M) {
  if (!df || !M) return HFG_ERR_INVALID_INPUT;
  if (!df->metric.p) return set_error(df->ctx, HFG_ERR_INVALID_INPUT, "this factor has no fitting metric (Cholesky vectors)");
  cudaSetDevice(df->ctx->device);
  const size_t len = (size_t)df->naux * df->naux;
  if (cudaMemcpy(M, df->metric.p, len * 8, cudaMemcpyDeviceToHost) != cudaSuccess)
    return set_error(df->ctx, HFG_ERR_CUDA, "copy metric");
  return HFG_OK;
}

int hfg_df_last_stats(hfg_df* df, double* k_ms, double* k_flops, double* tiles_fraction) {
  if (!df) return HFG_ERR_INVALID_INPUT;
  if (!df->k_timed) return set_error(df->ctx, HFG_ERR_INVALID_INPUT, "no tensor-core exchange has run on this factor");
  cudaSetDevice(df->ctx->device);
  float ms = 0.f;
  int rc = cuda_check(df->ctx, cudaEventSynchronize(df->kev[1]), "exchange event");
  if (rc == HFG_OK) rc = cuda_check(df->ctx, cudaEventElapsedTime(&ms, df->kev[0], df->kev[1]), "exchange time");
  if (rc != HFG_OK) return rc;
  if (k_ms) *k_ms = ms;
  if (k_flops) *k_flops = df->k_flops;
  if (tiles_fraction) *tiles_fraction = df->tiles_fraction;
  return HFG_OK;
}

// three_center_integrals (src/df.rs:60-78): (P|mu nu) for every auxiliary
// function P (rows) and every AO pair mu >= nu (packed columns
// compound_index(mu, nu) = mu (mu + 1) / 2 + nu), row-major, unscreened.
int hfg_df_three_center(hfg_ctx* ctx, const hfg_basis* aux, double* out, size_t len) {
  if (!ctx) return HFG_ERR_INVALID_INPUT;
  if (!aux || !out) return set_error(ctx, HFG_ERR_INVALID_INPUT, "null pointer");
  std::lock_guard<std::mutex> lk(ctx->mu);
  cudaSetDevice(ctx->device);
  AllocScope alloc_scope(ctx->stream);
  cudaStream_t st = ctx->stream;
  AuxSet ax;
  int rc = make_aux_set(ctx, aux, ax);
  if (rc != HFG_OK) return rc;
  const int naux = ax.shells.n;
  const long long n = ctx->n, np = n * (n + 1) / 2;
  if (len != (size_t)naux * (size_t)np)
    return set_error(ctx, HFG_ERR_INVALID_INPUT, "three-centre length must be n_aux * n (n + 1) / 2");
  // every shell pair's block in its own columns (as the factor build lays
  // them out), then scattered to the packed AO-pair order on the host
  std::vector<int2> colmn;
  std::map<std::pair<int, int>, std::pair<std::vector<int>, std::vector<long long>>> by_class;
  long long ncol = 0;
  for (size_t i = 0; i < ctx->h_pairs.size(); ++i) {
    const PairInfo& pi = ctx->h_pairs[i];
    const PairClass& c = ctx->classes[pi.cls];
    const int na = (c.la + 1) * (c.la + 2) / 2, nb = (c.lb + 1) * (c.lb + 2) / 2;
    auto& e = by_class[{c.la, c.lb}];
    e.first.push_back((int)i);
    e.second.push_back(ncol);
    for (int a = 0; a < na; ++a)
      for (int b = 0; b < nb; ++b) {
        if (pi.same && b > a) continue;
        colmn.push_back(make_int2(pi.ao_a + a, pi.ao_b + b));
      }
    ncol += pi.same ? na * (na + 1) / 2 : na * nb;
  }
  if (ncol != np) return set_error(ctx, HFG_ERR_INTEGRAL, "AO pair count mismatch");
  DevBuf<double> T3;
  rc = cuda_check(ctx, T3.alloc((size_t)naux * ncol), "alloc three-centre");
  if (rc != HFG_OK) return rc;
  for (auto& bc : by_class) {
    DevBuf<int> bidx;
    DevBuf<long long> bcol;
    rc = cuda_check(ctx, bidx.alloc(bc.second.first.size()), "alloc");
    if (rc == HFG_OK) rc = cuda_check(ctx, bcol.alloc(bc.second.second.size()), "alloc");
    if (rc == HFG_OK)
      rc = cuda_check(ctx, cudaMemcpyAsync(bidx.p, bc.second.first.data(), bc.second.first.size() * 4,
                                           cudaMemcpyHostToDevice, st), "copy");
    if (rc == HFG_OK)
      rc = cuda_check(ctx, cudaMemcpyAsync(bcol.p, bc.second.second.data(), bc.second.second.size() * 8,
                                           cudaMemcpyHostToDevice, st), "copy");
    for (auto& kk : ax.by_l) {
      if (rc != HFG_OK) break;
      Df3cArgs a{ctx->d_pairs.p, ctx->d_prims.p, bidx.p, bcol.p, (int)bc.second.first.size(), ax.dup.p, ax.dupr.p,
                 ax.idx[kk.first].p, (int)kk.second.size(), ctx->d_boys64.p, ctx->d_expt64.p, T3.p, ncol};
      rc = cuda_check(ctx, launch_df3c(bc.first.first, bc.first.second, kk.first, a, st), "three-centre kernel");
    }
    if (rc == HFG_OK) rc = cuda_check(ctx, cudaStreamSynchronize(st), "three-centre");
    if (rc != HFG_OK) return rc;
  }
  std::vector<double> h((size_t)naux * ncol);
  rc = cuda_check(ctx, cudaMemcpyAsync(h.data(), T3.p, h.size() * 8, cudaMemcpyDeviceToHost, st), "copy back");
  if (rc == HFG_OK) rc = cuda_check(ctx, cudaStreamSynchronize(st), "three-centre");
  if (rc != HFG_OK) return rc;
  for (long long c = 0; c < ncol; ++c) {
    const long long mu = std::max(colmn[c].x, colmn[c].y), nu = std::min(colmn[c].x, colmn[c].y);
    const long long k = mu * (mu + 1) / 2 + nu;
    for (int p = 0; p < naux; ++p) out[(size_t)p * np + k] = h[(size_t)p * ncol + c];
  }
  return HFG_OK;
}

}  // extern "C"

namespace hfg {

bool df_is_shard(const hfg_df* df) { return df->shard(); }

// J and K from occupied coefficients on the device: dC column-major n x nocc
// (leading dimension n), i.e. the first nocc columns of an SCF C matrix.
int df_jk_device(hfg_df* df, const double* dC, int nocc, double* dJ, double* dK, int mma, int q_lo, int q_hi) {
  hfg_ctx* ctx = df->ctx;
  cudaStream_t st = ctx->stream;
  const int n = df->n;
  // auxiliary functions [q_lo, q_hi) of the factor (a shard of the sum over Q)
  if (q_hi < 0) q_hi = df->rank;
  if (q_lo < 0 || q_lo > q_hi || q_hi > df->rank) return set_error(ctx, HFG_ERR_INVALID_INPUT, "auxiliary range");
  const int rank = q_hi - q_lo;
  const long long ncol = df->ncol, nn = (long long)n * n;
  int rc = HFG_OK;
#define CK(call)                         \
  do {                                   \
    rc = cuda_check(ctx, (call), #call); \
    if (rc != HFG_OK) return rc;         \
  } while (0)
  // arithmetic of the K GEMMs: FP64 storage always FP64; FP32 storage TF32
  // or BF16 tensor cores (the factor rounded to BF16 while unpacking) or FP64
  // on the converted factor; BF16 storage BF16 tensor cores or FP64 on the
  // converted factor
  if (df->storage == HFG_DF_FP64) mma = HFG_DF_FP64;
  if (df->storage == HFG_DF_BF16 && mma == HFG_DF_FP32) mma = HFG_DF_BF16;
  const double one = 1.0, zero = 0.0, two = 2.0;
  // P = 2 C C^T
  CK(df->P.alloc(nn));
  if (cublasDgemm(df->blas, CUBLAS_OP_N, CUBLAS_OP_T, n, n, nocc, &two, dC, n, dC, n, &zero, df->P.p, n) !=
      CUBLAS_STATUS_SUCCESS)
    return set_error(ctx, HFG_ERR_CUDA, "P GEMM");
  // J: gamma = B p, j = B^T gamma (B row-major [rank][ncol] = column-major ncol x rank)
  CK(df->pvec.alloc(ncol));
  CK(df->gam.alloc(std::max(rank, 1)));
  CK(df->jcol.alloc(ncol));
  CK(launch_pack_density(df->P.p, df->colmn.p, ncol, n, df->pvec.p, st));
  if (df->storage == HFG_DF_FP64) {
    const double* Bq = df->B64.p + (size_t)q_lo * ncol;
    if (rank > 0) {
      cublasDgemv(df->blas, CUBLAS_OP_T, (int)ncol, rank, &one, Bq, (int)ncol, df->pvec.p, 1, &zero, df->gam.p, 1);
      cublasDgemv(df->blas, CUBLAS_OP_N, (int)ncol, rank, &one, Bq, (int)ncol, df->gam.p, 1, &zero, df->jcol.p, 1);
    } else {
      CK(cudaMemsetAsync(df->jcol.p, 0, ncol * 8, st));
    }
  } else {
    // the stored FP32 / BF16 factor with FP64 accumulation (J is
    // memory-bound; the density is not rounded)
    const bool bf = df->storage == HFG_DF_BF16;
    if (rank == 0) CK(cudaMemsetAsync(df->jcol.p, 0, ncol * 8, st));
    CK(launch_df_j(bf ? 2 : 1, bf ? (const void*)(df->B16.p + (size_t)q_lo * ncol) : (const void*)(df->B32.p + (size_t)q_lo * ncol), ncol, rank, df->pvec.p,
                   df->gam.p, df->jcol.p, st));
  }
  CK(cudaMemsetAsync(dJ, 0, nn * 8, st));
  CK(launch_unpack_j(df->jcol.p, df->colmn.p, ncol, n, dJ, st));

  // K on the tensor cores: this library's tcgen05 kernels (df_umma.cu).
  // HFG_DF_K_CUBLAS=1 selects the cuBLAS GEMMs below instead, kept only to
  // time the two side by side.
  const char* kc = getenv("HFG_DF_K_CUBLAS");
  const bool k_cublas = kc && kc[0] == '1';
  if (mma != HFG_DF_FP64 && !k_cublas) {
    const int kind = mma == HFG_DF_BF16 ? kBF16 : kTF32;
    rc = ensure_tiles(df, kind);
    if (rc != HFG_OK) return rc;
    UmmaDfArgs ua;
    ua.device = ctx->device;
    ua.n = n;
    ua.nocc = nocc;
    ua.rank = rank;
    ua.rank_offset = q_lo;
    ua.kind = kind;
    ua.storage = df->storage == HFG_DF_BF16 ? 2 : 1;
    ua.ncol = ncol;
    ua.B = df->storage == HFG_DF_BF16 ? (const void*)df->B16.p : (const void*)df->B32.p;
    ua.C = dC;
    ua.K = dK;
    ua.tiles = &df->tiles[kind];
    ua.tile_off_dev = df->tile_off[kind].p;
    ua.tile_kt_dev = df->tile_kt[kind].p;
    ua.tile_map_dev = df->tile_map[kind].p;
    size_t free_b = 0, total_b = 0;
    cudaMemGetInfo(&free_b, &total_b);
    ua.chunk_bytes = std::max<size_t>((size_t)64 << 20, std::min<size_t>((size_t)4 << 30, free_b / 4));
    if (const char* ev = getenv("HFG_DF_K_CHUNK")) ua.max_chunk = atoi(ev);  // tests: many chunks
    int status = 0;
    if (!df->kev[0]) {
      CK(cudaEventCreate(&df->kev[0]));
      CK(cudaEventCreate(&df->kev[1]));
    }
    CK(cudaEventRecord(df->kev[0], st));
    CK(df_k_tensor_cores(ua, df->uws, &status, st));
    CK(cudaEventRecord(df->kev[1], st));
    df->k_flops = df->uws.flops_executed;
    df->tiles_fraction = df->uws.tiles_fraction;
    df->k_timed = true;
    if (status != 0)
      return set_error(ctx, HFG_ERR_TIMEOUT, "DF exchange kernel: a bounded wait ran out (code " +
                                                 std::to_string(status) + ")");
    return HFG_OK;
  }

  // K: chunks of qc auxiliary functions
  df->k_timed = false;
  const size_t esz = mma == HFG_DF_FP64 ? 8 : (mma == HFG_DF_FP32 ? 4 : 2);
  size_t free_b = 0, total_b = 0;
  cudaMemGetInfo(&free_b, &total_b);
  const size_t budget = std::max<size_t>((size_t)64 << 20, std::min<size_t>((size_t)4 << 30, free_b / 4));
  int qc = (int)std::max<size_t>(1, std::min<size_t>((size_t)std::max(rank, 1), budget / ((size_t)nn * esz)));
  CK(df->dense.alloc((size_t)qc * nn * esz));
  CK(cudaMemsetAsync(dK, 0, nn * 8, st));
  if (mma == HFG_DF_FP64) {
    CK(df->T64.alloc((size_t)qc * n * nocc));
    for (int q0 = q_lo; q0 < q_hi; q0 += qc) {
      const int qn = std::min(qc, q_hi - q0);
      CK(cudaMemsetAsync(df->dense.p, 0, (size_t)qn * nn * 8, st));
      // FP64 arithmetic on the stored factor, converted while unpacking
      const int um = df->storage == HFG_DF_FP64 ? 0 : (df->storage == HFG_DF_FP32 ? 3 : 4);
      const void* Bs = df->storage == HFG_DF_FP64 ? (const void*)df->B64.p
                       : df->storage == HFG_DF_FP32 ? (const void*)df->B32.p : (const void*)df->B16.p;
      CK(launch_df_unpack(um, Bs, ncol, df->colmn.p, ncol, q0, qn, n, df->dense.p, st));
      const double* Bd = (const double*)df->dense.p;
      // T^T (nocc x n*qn) = C^T (nocc x n) * Bd2^T (n x n*qn)
      cublasDgemm(df->blas, CUBLAS_OP_T, CUBLAS_OP_N, nocc, n * qn, n, &one, dC, n, Bd, n, &zero, df->T64.p, nocc);
      // K += 2 U U^T, U (row-major n x qn*nocc) = column-major (qn*nocc x n)
      cublasDgemm(df->blas, CUBLAS_OP_T, CUBLAS_OP_N, n, n, qn * nocc, &two, df->T64.p, qn * nocc, df->T64.p,
                  qn * nocc, &one, dK, n);
    }
  } else {
    const bool bf = mma == HFG_DF_BF16;
    const cudaDataType it = bf ? CUDA_R_16BF : CUDA_R_32F;
    const cublasComputeType_t ct = bf ? CUBLAS_COMPUTE_32F : CUBLAS_COMPUTE_32F_FAST_TF32;
    CK(df->Tf.alloc((size_t)qc * n * nocc));
    CK(df->Kf.alloc(nn));
    const void* Cin;
    if (bf) {
      CK(df->Cb.alloc((size_t)n * nocc));
      CK(launch_convert(2, dC, df->Cb.p, (long long)n * nocc, st));
      Cin = df->Cb.p;
      CK(df->Tb.alloc((size_t)qc * n * nocc));
    } else {
      CK(df->Cf.alloc((size_t)n * nocc));
      CK(launch_convert(1, dC, df->Cf.p, (long long)n * nocc, st));
      Cin = df->Cf.p;
    }
    const void* Bsrc = df->storage == HFG_DF_BF16 ? (const void*)df->B16.p : (const void*)df->B32.p;
    const int umode = df->storage == HFG_DF_BF16 ? 2 : (bf ? 5 : 1);
    for (int q0 = q_lo; q0 < q_hi; q0 += qc) {
      const int qn = std::min(qc, q_hi - q0);
      CK(cudaMemsetAsync(df->dense.p, 0, (size_t)qn * nn * esz, st));
      CK(launch_df_unpack(umode, Bsrc, ncol, df->colmn.p, ncol, q0, qn, n, df->dense.p, st));
      rc = gemm_ex(ctx, df->blas, CUBLAS_OP_T, CUBLAS_OP_N, nocc, n * qn, n, Cin, it, n, df->dense.p, it, n, 0.0f,
                   df->Tf.p, nocc, ct);
      if (rc != HFG_OK) return rc;
      const void* U = df->Tf.p;
      if (bf) {
        // T (FP32 accumulated) back to BF16 for the second product
        CK(launch_convert_f32(2, df->Tf.p, df->Tb.p, (long long)qn * n * nocc, st));
        U = df->Tb.p;
      }
      rc = gemm_ex(ctx, df->blas, CUBLAS_OP_T, CUBLAS_OP_N, n, n, qn * nocc, U, it, qn * nocc, U, it, qn * nocc, 0.0f,
                   df->Kf.p, n, ct);
      if (rc != HFG_OK) return rc;
      CK(launch_accumulate_f32(dK, df->Kf.p, 2.0, nn, st));
    }
  }
#undef CK
  return HFG_OK;
}

}  // namespace hfg

namespace {

// the shard's auxiliary functions: [shard * rank / nshards, (shard + 1) * rank / nshards)
void shard_range(const hfg_df* df, int shard, int nshards, int& q_lo, int& q_hi) {
  q_lo = (int)((long long)df->rank * shard / nshards);
  q_hi = (int)((long long)df->rank * (shard + 1) / nshards);
}

int df_jk_host(hfg_df* df, const double* C_occ, int nocc, double* J, double* K, int mma, int shard, int nshards) {
  if (!df || !C_occ || !J || !K || nocc <= 0) return HFG_ERR_INVALID_INPUT;
  hfg_ctx* ctx = df->ctx;
  if (nshards < 1 || shard < 0 || shard >= nshards) return set_error(ctx, HFG_ERR_INVALID_INPUT, "invalid shard");
  std::lock_guard<std::mutex> lk(ctx->mu);
  cudaSetDevice(ctx->device);
  AllocScope alloc_scope(ctx->stream);
  const long long nn = (long long)df->n * df->n;
  int rc = cuda_check(ctx, df->Cd.alloc((size_t)df->n * nocc), "alloc");
  if (rc == HFG_OK) rc = cuda_check(ctx, df->J.alloc(nn), "alloc");
  if (rc == HFG_OK) rc = cuda_check(ctx, df->K.alloc(nn), "alloc");
  if (rc != HFG_OK) return rc;
  // row-major n x nocc -> column-major (leading dimension n)
  std::vector<double> ct((size_t)df->n * nocc);
  for (int i = 0; i < df->n; ++i)
    for (int k = 0; k < nocc; ++k) ct[(size_t)k * df->n + i] = C_occ[(size_t)i * nocc + k];
  cudaMemcpyAsync(df->Cd.p, ct.data(), ct.size() * 8, cudaMemcpyHostToDevice, ctx->stream);
  int q_lo, q_hi;
  shard_range(df, shard, nshards, q_lo, q_hi);
  rc = df_jk_device(df, df->Cd.p, nocc, df->J.p, df->K.p, mma, q_lo, q_hi);
  if (rc != HFG_OK) return rc;
  cudaMemcpyAsync(J, df->J.p, nn * 8, cudaMemcpyDeviceToHost, ctx->stream);
  cudaMemcpyAsync(K, df->K.p, nn * 8, cudaMemcpyDeviceToHost, ctx->stream);
  return cuda_check(ctx, cudaStreamSynchronize(ctx->stream), "df_jk sync");
}

}  // namespace

extern "C" int hfg_df_jk(hfg_df* df, const double* C_occ, int nocc, double* J, double* K, int mma) {
  return df_jk_host(df, C_occ, nocc, J, K, mma, 0, 1);
}

extern "C" int hfg_df_jk_shard(hfg_df* df, const double* C_occ, int nocc, double* J, double* K, int mma, int shard,
                               int nshards) {
  return df_jk_host(df, C_occ, nocc, J, K, mma, shard, nshards);
}

extern "C" int hfg_df_jk_device_shard(hfg_df* df, const double* d_C, int nocc, double* d_J, double* d_K, int mma,
                                      int shard, int nshards) {
  if (!df || !d_C || !d_J || !d_K || nocc <= 0) return HFG_ERR_INVALID_INPUT;
  hfg_ctx* ctx = df->ctx;
  if (nshards < 1 || shard < 0 || shard >= nshards) return set_error(ctx, HFG_ERR_INVALID_INPUT, "invalid shard");
  std::lock_guard<std::mutex> lk(ctx->mu);
  cudaSetDevice(ctx->device);
  AllocScope alloc_scope(ctx->stream);
  int q_lo, q_hi;
  shard_range(df, shard, nshards, q_lo, q_hi);
  return df_jk_device(df, d_C, nocc, d_J, d_K, mma, q_lo, q_hi);
}
