// The DF factor handle (hfg_df) shared by the DF translation units.
#pragma once
#include <cublas_v2.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include "df_umma.h"
#include "hfg_ctx.h"

// B = X^T (P|mn) over the stored AO pairs, row-major [rank][ncol], in its
// storage precision, and the scratch of the J/K builds.
struct hfg_df {
  hfg_ctx* ctx = nullptr;
  int n = 0, naux = 0, rank = 0;
  // a shard factor holds rows [row0, row0 + rank) of the full rank_total rows
  int rank_total = 0, row0 = 0;
  bool shard() const { return rank != rank_total; }
  long long ncol = 0;
  int storage = HFG_DF_FP64;
  hfg::DevBuf<double> B64;
  hfg::DevBuf<float> B32;
  hfg::DevBuf<__nv_bfloat16> B16;
  hfg::DevBuf<int2> colmn;
  hfg::DevBuf<double> metric;  // kept for inspection (naux x naux)
  cublasHandle_t blas = nullptr;
  hfg::DevBuf<double> P, pvec, gam, jcol, Cd, J, K, T64;
  hfg::DevBuf<float> gam32, jcol32, pvec32, Kf, Tf, Cf;
  hfg::DevBuf<__nv_bfloat16> Cb, Tb;
  hfg::DevBuf<unsigned char> dense;
  // tensor-core exchange: tile structure of the unpacked factor per operand
  // type (built on first use) and its scratch
  hfg::TileStructure tiles[2];
  bool tiles_ready[2] = {false, false};
  hfg::DevBuf<int> tile_off[2], tile_kt[2], tile_map[2];
  hfg::UmmaWorkspace uws;
  // device time of the last exchange (K) and its executed tensor-core flops
  cudaEvent_t kev[2] = {nullptr, nullptr};
  double k_flops = 0.0, tiles_fraction = 0.0;
  bool k_timed = false;
  ~hfg_df() {
    for (auto& e : kev)
      if (e) cudaEventDestroy(e);
    if (blas) cublasDestroy(blas);
  }
};
