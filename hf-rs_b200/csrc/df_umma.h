// Tensor-core DF exchange (df_umma.cu): tile structure of the unpacked
// factor, scratch buffers and the host entry.
#pragma once
#include <cuda_runtime.h>

#include <vector>

#include "hfg_ctx.h"

namespace hfg {

constexpr int kBF16 = 0, kTF32 = 1;  // operand type of both exchange GEMMs

// Non-zero 128 x TK tiles of B_Q (the same for every Q): the AO pairs stored
// in the factor decide which tiles of the symmetric n x n unpack hold
// anything.  tile_off[mt] .. tile_off[mt + 1] are the tiles of row block mt
// (column blocks tile_kt[]); tile_map holds, per tile, the packed factor
// column of each of its 128 x TK elements (-1: zero).
struct TileStructure {
  int n = 0, tk = 0, ntiles = 0, total_tiles = 0;
  std::vector<int> tile_off, tile_kt, tile_map;
  int build(const std::vector<int2>& colmn, int n, int kind);
};

struct UmmaWorkspace {
  DevBuf<unsigned char> dense, T, Ct, Kf, err, lower;
  double flops_executed = 0.0;  // tensor-core flops of the last exchange (both GEMMs)
  double tiles_fraction = 0.0;  // non-zero share of the 128 x TK tiles of B_Q
  static cudaError_t grow(DevBuf<unsigned char>& b, size_t bytes) { return b.alloc(bytes); }
};

struct UmmaDfArgs {
  int device = 0, n = 0, nocc = 0;
  int rank = 0;         // auxiliary functions processed: factor rows [rank_offset, rank_offset + rank)
  int rank_offset = 0;
  int kind = kBF16;     // operand type
  int storage = 1;      // stored factor: 1 FP32, 2 BF16
  long long ncol = 0;   // packed columns of the factor
  const void* B = nullptr;
  const double* C = nullptr;  // column-major n x nocc (ld n)
  double* K = nullptr;        // n x n, overwritten with 2 sum_Q A_Q A_Q^T
  const TileStructure* tiles = nullptr;
  const int* tile_off_dev = nullptr;
  const int* tile_kt_dev = nullptr;
  const int* tile_map_dev = nullptr;
  size_t chunk_bytes = (size_t)4 << 30;  // scratch for one chunk of Q
  int max_chunk = 0;                      // > 0: at most this many Q per chunk
};

// K on the tensor cores; *status (host) receives the kernels' error code
// (0 ok, > 0: a bounded wait ran out).
cudaError_t df_k_tensor_cores(const UmmaDfArgs& p, UmmaWorkspace& ws, int* status, cudaStream_t st);

}  // namespace hfg
