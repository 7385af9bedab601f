// DF exchange on the 5th-generation tensor cores (tcgen05 + TMEM + TMA).
//
// Stands in for the K half of hf-rs's DfTensor::coulomb_exchange_rhf
// (src/df.rs:133-174): per auxiliary function Q, B_Q is the symmetric n x n
// unpack of row Q of the factor, A = B_Q C_occ, K += 2 A A^T.  Here, for a
// chunk of consecutive Q:
//
//   1. unpack  : row Q of the packed factor (FP32 or BF16 storage) into the
//                non-zero 128 x TK tiles of B_Q only ("tile-compact" dense
//                chunk [Q][tile][128][TK]), through a per-tile index map;
//                tiles of B_Q that hold no significant AO pair are never
//                written or read.
//   2. GEMM 1  : T_Q = B_Q C (n x nocc, FP32 accumulation in TMEM) for every
//                Q of the chunk, summing only over the non-zero tiles of the
//                row block; T is stored in the operand type (BF16 or FP32)
//                as [Q][m][i].
//   3. GEMM 2  : K_lower += U U^T with U[m, (Q, i)] = T_Q[m, i]: only the
//                output tiles on or below the diagonal (K is symmetric, half
//                the flops of a GEMM), split over Q ranges, FP32 atomics into
//                an n x n FP32 accumulator.
//
// Both GEMMs are one warp-specialised kernel: warp 0 issues TMA tile loads
// (cp.async.bulk.tensor, 128-byte swizzle) into a 4-stage shared-memory
// ring, warp 1 allocates TMEM and issues tcgen05.mma (one elected thread;
// M = 128, N = up to 256, K = 16 (BF16) or 8 (TF32) per instruction) and
// releases ring slots with tcgen05.commit, warps 2-5 read the accumulator
// back with tcgen05.ld and store it.  All tensor maps cover this GPU's own
// memory, with no cluster multicast.  Every mbarrier wait is bounded: on
// timeout the kernel records an error code, drains its own copies and MMAs,
// frees TMEM and returns, and the host reports HFG_ERR_TIMEOUT.
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <mutex>
#include <vector>

#include "df_umma.h"

namespace hfg {
namespace umma {

constexpr int kStages = 4;
constexpr int kBM = 128;
constexpr int kBN = 256;
constexpr int kRowBytes = 128;  // one swizzle span: BK elements of the operand type
constexpr int kThreads = 192;   // warp 0 TMA, warp 1 MMA, warps 2-5 epilogue
constexpr int kTmemCols = 256;

constexpr int kStageA = kBM * kRowBytes;  // 16 KB
constexpr int kStageB = kBN * kRowBytes;  // 32 KB
constexpr size_t kSmemBytes = (size_t)kStages * (kStageA + kStageB) + 1024 /*align*/ + 256 /*barriers*/;

// ------------------------------------------------------------ PTX helpers --
__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}\n"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
__device__ __forceinline__ uint64_t global_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}
// Wait for the phase of `parity` to complete; false after kWaitNs of wall
// time or when another role of the block has given up (*abort set).  A wait
// in a working kernel lasts at most one output tile's main loop (well under
// a millisecond).
constexpr uint64_t kWaitNs = 2000000000ull;
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, volatile int* abort) {
  const uint64_t t0 = global_ns();
  for (uint32_t i = 0;; ++i) {
    if (mbar_try_wait(bar, parity)) return true;
    if ((i & 255u) == 255u && (*abort || global_ns() - t0 > kWaitNs)) return false;
  }
}
// Drain-only wait (no abort check): lets this block's own in-flight copies
// or MMAs finish before it frees TMEM and exits; bounded the same way.
__device__ __forceinline__ bool mbar_wait_drain(uint64_t* bar, uint32_t parity) {
  const uint64_t t0 = global_ns();
  for (uint32_t i = 0;; ++i) {
    if (mbar_try_wait(bar, parity)) return true;
    if ((i & 255u) == 255u && global_ns() - t0 > kWaitNs) return false;
  }
}

__device__ __forceinline__ void tma_load_3d(void* dst, const CUtensorMap* map, uint64_t* bar, int x, int y, int z) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4, %5}], [%2];" ::
          "r"(smem_u32(dst)),
      "l"(map), "r"(smem_u32(bar)), "r"(x), "r"(y), "r"(z)
      : "memory");
}

__device__ __forceinline__ void tmem_alloc(uint32_t* dst, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(dst)), "r"(ncols)
               : "memory");
}
__device__ __forceinline__ void tmem_relinquish() {
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

template <int KIND>
__device__ __forceinline__ void umma(uint32_t d, uint64_t a, uint64_t b, uint32_t idesc, uint32_t accumulate) {
  if constexpr (KIND == kBF16) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(d),
        "l"(a), "l"(b), "r"(idesc), "r"(accumulate)
        : "memory");
  } else {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(d),
        "l"(a), "l"(b), "r"(idesc), "r"(accumulate)
        : "memory");
  }
}
__device__ __forceinline__ void umma_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
               : "memory");
}

// 16 consecutive FP32 accumulator columns of this thread's TMEM lane.
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float* v) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
      "%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int k = 0; k < 16; ++k) v[k] = __uint_as_float(r[k]);
}

// Operand conversion.  The tensor cores read the top 19 bits of an FP32
// operand (TF32) and drop the rest, a truncation toward zero whose error is
// biased and adds up coherently in K = T T^T; FP32 operands are therefore
// rounded to the nearest TF32 value where they are written.
template <typename TD> __device__ __forceinline__ TD to_operand(float x);
template <> __device__ __forceinline__ __nv_bfloat16 to_operand<__nv_bfloat16>(float x) { return __float2bfloat16_rn(x); }
template <> __device__ __forceinline__ float to_operand<float>(float x) {
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
  return __uint_as_float(r);
}

// Shared-memory matrix descriptor of a K-major tile written by TMA with
// 128-byte swizzling: rows of 128 bytes, 8-row (1024-byte) swizzle atoms.
__device__ __forceinline__ uint64_t sw128_desc(uint32_t saddr) {
  uint64_t d = 0;
  d |= (uint64_t)((saddr >> 4) & 0x3FFFu);  // start address
  d |= (uint64_t)1u << 16;                  // leading-dimension offset (unused for swizzled K-major)
  d |= (uint64_t)(1024u >> 4) << 32;        // stride between 8-row groups
  d |= (uint64_t)1u << 46;                  // descriptor version (sm_100)
  d |= (uint64_t)2u << 61;                  // 128-byte swizzle
  return d;
}

// Instruction descriptor: FP32 accumulator, A and B of format `fmt`
// (1 = BF16, 2 = TF32), both K-major, M x N.
__device__ __forceinline__ uint32_t make_idesc(uint32_t fmt, uint32_t M, uint32_t N) {
  return (1u << 4) | (fmt << 7) | (fmt << 10) | ((N >> 3) << 17) | ((M >> 4) << 24);
}

__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

// ----------------------------------------------------------------- kernel --
// Persistent: one block per SM walks the launch's work units (output tiles,
// or output tile x Q range for the symmetric update) with a grid stride.
// The shared-memory ring runs continuously across units, and the TMEM
// accumulator is double-buffered (2 x 256 columns), so the epilogue of one
// unit overlaps the main loop of the next.
struct GemmArgs {
  int mode;    // 0: T_Q = B_Q C over non-zero tiles; 1: K_lower += T T^T
  int m_rows;  // valid rows of the output (n)
  int n_cols;  // valid columns of the output (mode 0: nocc_pad; mode 1: n)
  int bn;      // output tile width (<= 256, multiple of 16)
  long long units;  // work units of the launch
  // mode 0: unit = (nt, mt, Q), nt fastest
  const int* tile_off;  // per row block: its non-zero tiles [tile_off[mt], tile_off[mt + 1])
  const int* tile_kt;   // column block of each non-zero tile (tiles numbered in row-block order)
  int n_ntiles, n_mtiles;
  // mode 1: unit = (lower tile, Q range), lower tile fastest
  const int2* out_tiles;  // (mt, nt) of every lower output tile
  int n_lower;
  int q_count;  // Q of the chunk
  int q_per_split;
  int i_tiles;  // K tiles per Q (ceil(nocc_pad / BK))
  // output
  void* out;
  long long ldo;           // row stride (elements)
  long long batch_stride;  // mode 0: per Q (elements)
  int* err;
};

struct Unit {
  int mt, nt, q, q0, nk;
};

template <int MODE>
__device__ __forceinline__ Unit unit_of(const GemmArgs& a, long long u) {
  Unit w;
  if (MODE == 0) {
    w.nt = (int)(u % a.n_ntiles);
    const long long r = u / a.n_ntiles;
    w.mt = (int)(r % a.n_mtiles);
    w.q = (int)(r / a.n_mtiles);
    w.q0 = 0;
    w.nk = __ldg(a.tile_off + w.mt + 1) - __ldg(a.tile_off + w.mt);
  } else {
    const int t = (int)(u % a.n_lower), sp = (int)(u / a.n_lower);
    const int2 tt = a.out_tiles[t];
    w.mt = tt.x;
    w.nt = tt.y;
    w.q = 0;
    w.q0 = sp * a.q_per_split;
    const int q1 = min(a.q_count, w.q0 + a.q_per_split);
    w.nk = q1 > w.q0 ? (q1 - w.q0) * a.i_tiles : 0;
  }
  return w;
}

// MMA N of a unit: its output columns rounded up to 16 (columns past
// n_cols read zero-filled rows of B and are not stored)
__device__ __forceinline__ int unit_cols(const GemmArgs& a, const Unit& w) {
  return (min(a.bn, a.n_cols - w.nt * a.bn) + 15) & ~15;
}

template <int KIND, int MODE>
__global__ void __launch_bounds__(kThreads, 1)
    umma_gemm_kernel(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB, const GemmArgs a) {
  constexpr uint32_t kFmt = KIND == kBF16 ? 1u : 2u;
  constexpr int kEl = KIND == kBF16 ? 2 : 4;  // operand bytes; 32 bytes of K per instruction
  extern __shared__ unsigned char smem_raw[];
  unsigned char* base = (unsigned char*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  unsigned char* sA = base;
  unsigned char* sB = base + kStages * kStageA;
  uint64_t* full = (uint64_t*)(sB + kStages * kStageB);
  uint64_t* empty = full + kStages;
  uint64_t* tfull = empty + kStages;  // accumulator buffer b holds a finished unit
  uint64_t* tempty = tfull + 2;       // accumulator buffer b has been read out
  uint64_t* done = tempty + 2;
  uint32_t* tmem_slot = (uint32_t*)(done + 1);
  volatile int* abort_flag = (volatile int*)(tmem_slot + 1);

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (threadIdx.x == 0) {
    for (int s = 0; s < kStages; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
    }
    for (int b = 0; b < 2; ++b) {
      mbar_init(&tfull[b], 1);
      mbar_init(&tempty[b], 4);  // one arrival per epilogue warp
    }
    mbar_init(done, 1);
    *abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 1) {
    tmem_alloc(tmem_slot, 2 * kTmemCols);
    tmem_relinquish();
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;

  if (warp == 0 && lane == 0) {
    // ---------------------------------------------------------- producer
    int last_round[kStages];
#pragma unroll
    for (int s = 0; s < kStages; ++s) last_round[s] = -1;
    const uint32_t bytes = (uint32_t)(kStageA + kStageB);
    long long it = 0;
    for (long long u = blockIdx.x; u < a.units && !*abort_flag; u += gridDim.x) {
      const Unit w = unit_of<MODE>(a, u);
      for (int k = 0; k < w.nk; ++k, ++it) {
        const int s = (int)(it % kStages);
        const uint32_t round = (uint32_t)(it / kStages);
        if (!mbar_wait(&empty[s], (round & 1u) ^ 1u, abort_flag)) {
          if (!*abort_flag) atomicExch(a.err, 1);
          *abort_flag = 1;
          break;
        }
        mbar_expect_tx(&full[s], bytes);
        int ax, ay, az, bx, by, bz;
        if (MODE == 0) {
          const int t = __ldg(a.tile_off + w.mt) + k;
          ax = 0;
          ay = t * kBM;
          az = w.q;
          bx = __ldg(a.tile_kt + t) * (kRowBytes / kEl);
          by = w.nt * a.bn;
          bz = 0;
        } else {
          const int q = w.q0 + k / a.i_tiles, ib = k % a.i_tiles;
          ax = bx = ib * (kRowBytes / kEl);
          ay = w.mt * kBM;
          by = w.nt * a.bn;
          az = bz = q;
        }
        tma_load_3d(sA + s * kStageA, &tmA, &full[s], ax, ay, az);
        tma_load_3d(sB + s * kStageB, &tmB, &full[s], bx, by, bz);
        last_round[s] = (int)round;
      }
    }
    // let every copy this thread issued land before the block may exit
    for (int s = 0; s < kStages; ++s)
      if (last_round[s] >= 0 && !mbar_wait_drain(&full[s], (uint32_t)(last_round[s] & 1))) atomicExch(a.err, 2);
  } else if (warp == 1 && lane == 0) {
    // ------------------------------------------------------- MMA issuer
    long long it = 0;
    int lt = 0;
    for (long long u = blockIdx.x; u < a.units && !*abort_flag; u += gridDim.x, ++lt) {
      const Unit w = unit_of<MODE>(a, u);
      const int b = lt & 1;
      const uint32_t use = (uint32_t)(lt >> 1);
      if (!mbar_wait(&tempty[b], (use & 1u) ^ 1u, abort_flag)) {
        if (!*abort_flag) atomicExch(a.err, 3);
        *abort_flag = 1;
        break;
      }
      tc_fence_after();
      const uint32_t d = tmem + (uint32_t)(b * kTmemCols);
      const uint32_t idesc = make_idesc(kFmt, kBM, (uint32_t)unit_cols(a, w));
      bool ok = true;
      for (int k = 0; k < w.nk; ++k, ++it) {
        const int s = (int)(it % kStages);
        const uint32_t round = (uint32_t)(it / kStages);
        if (!mbar_wait(&full[s], round & 1u, abort_flag)) {
          if (!*abort_flag) atomicExch(a.err, 4);
          *abort_flag = 1;
          ok = false;
          break;
        }
        tc_fence_after();
        const uint32_t a0 = smem_u32(sA + s * kStageA), b0 = smem_u32(sB + s * kStageB);
#pragma unroll
        for (int kk = 0; kk < 4; ++kk)  // 4 x 32 bytes of K per 128-byte row
          umma<KIND>(d, sw128_desc(a0 + 32 * kk), sw128_desc(b0 + 32 * kk), idesc, (k > 0 || kk > 0) ? 1u : 0u);
        umma_commit(&empty[s]);  // the slot is free once these MMAs have read it
      }
      if (!ok) break;
      umma_commit(&tfull[b]);  // with no MMAs (nk = 0) it arrives at once
    }
    // every MMA issued above completes before TMEM is freed
    umma_commit(done);
    if (!mbar_wait_drain(done, 0u)) atomicExch(a.err, 5);
  } else if (warp >= 2) {
    // --------------------------------------------------------- epilogue
    const int quarter = warp & 3;  // TMEM lanes 32*quarter .. +31 belong to this warp
    int lt = 0;
    for (long long u = blockIdx.x; u < a.units; u += gridDim.x, ++lt) {
      const Unit w = unit_of<MODE>(a, u);
      const int b = lt & 1;
      const uint32_t use = (uint32_t)(lt >> 1);
      bool ok = mbar_wait(&tfull[b], use & 1u, abort_flag);
      // tcgen05.ld is warp-collective: the whole warp reads or none of it
      ok = __all_sync(0xffffffffu, ok);
      if (!ok) {
        if (lane == 0) {
          if (!*abort_flag) atomicExch(a.err, 6);
          *abort_flag = 1;
        }
        break;
      }
      tc_fence_after();
      const int row = w.mt * kBM + quarter * 32 + lane;
      const int n0 = w.nt * a.bn, ncols = unit_cols(a, w);
      const uint32_t lane_addr = tmem + ((uint32_t)(quarter * 32) << 16) + (uint32_t)(b * kTmemCols);
      for (int c = 0; c < ncols; c += 16) {
        float v[16];
        if (w.nk > 0) {
          tmem_ld16(lane_addr + (uint32_t)c, v);
        } else {
#pragma unroll
          for (int k = 0; k < 16; ++k) v[k] = 0.f;
        }
        if (row >= a.m_rows) continue;
        if (MODE == 0) {
          // n_cols (nocc_pad) and every unit's width are multiples of 16
          const long long off = (long long)w.q * a.batch_stride + (long long)row * a.ldo + n0 + c;
          if (KIND == kBF16) {
            __nv_bfloat16* o = (__nv_bfloat16*)a.out + off;
            uint4 q4[2];
            __nv_bfloat162* h = (__nv_bfloat162*)q4;
#pragma unroll
            for (int k = 0; k < 8; ++k) h[k] = __floats2bfloat162_rn(v[2 * k], v[2 * k + 1]);
            ((uint4*)o)[0] = q4[0];
            ((uint4*)o)[1] = q4[1];
          } else {
            float4* o = (float4*)((float*)a.out + off);
#pragma unroll
            for (int k = 0; k < 4; ++k)
              o[k] = make_float4(to_operand<float>(v[4 * k]), to_operand<float>(v[4 * k + 1]),
                                 to_operand<float>(v[4 * k + 2]), to_operand<float>(v[4 * k + 3]));
          }
        } else {
          float* o = (float*)a.out + (long long)row * a.ldo + n0 + c;
#pragma unroll
          for (int k = 0; k < 16; ++k)
            if (n0 + c + k < a.n_cols) atomicAdd(o + k, v[k]);
        }
      }
      // hand the buffer back to the MMA issuer once this warp's reads are done
      tc_fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive(&tempty[b]);
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 1) {
    tc_fence_after();
    tmem_dealloc(tmem, 2 * kTmemCols);
  }
}

// ----------------------------------------------------------------- unpack --
// Tile-compact unpack: block = one non-zero 128 x TK tile of the row-block
// structure; each thread keeps its elements' packed-column indices and walks
// the Q of the chunk.  dst[Q][tile][r][c] (row stride TK).
template <typename TS, typename TD, int TK>
__global__ void __launch_bounds__(256) unpack_tiles_kernel(const TS* __restrict__ B, long long ncol,
                                                           const int* __restrict__ tile_map, int ntiles, int q0,
                                                           int qn, TD* __restrict__ dst) {
  constexpr int kPer = kBM * TK / 256;
  const int t = blockIdx.x;
  if (t >= ntiles) return;
  const int* m = tile_map + (size_t)t * kBM * TK;
  int idx[kPer];
#pragma unroll
  for (int k = 0; k < kPer; ++k) idx[k] = __ldg(m + threadIdx.x + k * 256);
  for (int q = blockIdx.y; q < qn; q += gridDim.y) {
    const TS* row = B + (size_t)(q0 + q) * ncol;
    TD* o = dst + ((size_t)q * ntiles + t) * kBM * TK;
#pragma unroll
    for (int k = 0; k < kPer; ++k) {
      const int e = idx[k];
      float v = 0.f;
      if (e >= 0) v = (float)row[e];
      o[threadIdx.x + k * 256] = to_operand<TD>(v);
    }
  }
}

// C^T in the operand type: ct[i][k] = C[k + i * n] (column-major C, ld n),
// zero outside nocc x n (rows up to nocc_pad, columns up to ldk).
template <typename TD>
__global__ void ct_kernel(const double* __restrict__ C, int n, int nocc, int nocc_pad, int ldk, TD* __restrict__ ct) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)nocc_pad * ldk) return;
  const int i = (int)(t / ldk), k = (int)(t % ldk);
  ct[t] = to_operand<TD>((i < nocc && k < n) ? (float)C[(size_t)i * n + k] : 0.f);
}

// K (FP64, n x n) = scale * symmetric completion of the lower triangle of Kf.
__global__ void k_finalize_kernel(const float* __restrict__ Kf, int n, double scale, double* __restrict__ K) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)n * n) return;
  const int i = (int)(t / n), j = (int)(t % n);
  const int r = max(i, j), c = min(i, j);
  K[t] = scale * (double)Kf[(size_t)r * n + c];
}

// ------------------------------------------------------------------- host --
PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = (PFN_cuTensorMapEncodeTiled_v12000)p;
  });
  return fn;
}

// 3-D tensor map (x fastest) with 128-byte swizzle and a box of
// (128 bytes, rows, 1).
static bool make_map(CUtensorMap* m, int kind, const void* base, long long d0, long long d1, long long d2,
                     long long stride1_bytes, long long stride2_bytes, int box_rows) {
  auto fn = encode_fn();
  if (!fn) return false;
  const int el = kind == kBF16 ? 2 : 4;
  cuuint64_t dims[3] = {(cuuint64_t)d0, (cuuint64_t)d1, (cuuint64_t)d2};
  cuuint64_t strides[2] = {(cuuint64_t)stride1_bytes, (cuuint64_t)stride2_bytes};
  cuuint32_t box[3] = {(cuuint32_t)(kRowBytes / el), (cuuint32_t)box_rows, 1};
  cuuint32_t estr[3] = {1, 1, 1};
  const CUresult r =
      fn(m, kind == kBF16 ? CU_TENSOR_MAP_DATA_TYPE_BFLOAT16 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3,
         const_cast<void*>(base), dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
         CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS;
}

template <int KIND, int MODE>
static cudaError_t launch_gemm(const CUtensorMap& A, const CUtensorMap& B, const GemmArgs& a, dim3 grid,
                               cudaStream_t st) {
  auto k = umma_gemm_kernel<KIND, MODE>;
  static std::once_flag once[64];
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev >= 0 && dev < 64)
    std::call_once(once[dev], [&] { cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSmemBytes); });
  k<<<grid, kThreads, kSmemBytes, st>>>(A, B, a);
  return cudaGetLastError();
}

}  // namespace umma

using namespace umma;

int TileStructure::build(const std::vector<int2>& colmn, int n, int kind) {
  this->n = n;
  tk = kind == kBF16 ? 64 : 32;
  const int nmt = (n + kBM - 1) / kBM, nkt = (n + tk - 1) / tk;
  // packed column of every (row, col) of B_Q, -1 where no significant pair
  std::vector<int> full((size_t)n * n, -1);
  for (size_t c = 0; c < colmn.size(); ++c) {
    const int i = colmn[c].x, j = colmn[c].y;
    full[(size_t)i * n + j] = (int)c;
    full[(size_t)j * n + i] = (int)c;
  }
  std::vector<char> nz((size_t)nmt * nkt, 0);
  for (int i = 0; i < n; ++i)
    for (int j = 0; j < n; ++j)
      if (full[(size_t)i * n + j] >= 0) nz[(size_t)(i / kBM) * nkt + j / tk] = 1;
  tile_off.assign(nmt + 1, 0);
  tile_kt.clear();
  for (int mt = 0; mt < nmt; ++mt) {
    for (int kt = 0; kt < nkt; ++kt)
      if (nz[(size_t)mt * nkt + kt]) tile_kt.push_back(kt);
    tile_off[mt + 1] = (int)tile_kt.size();
  }
  ntiles = (int)tile_kt.size();
  tile_map.assign((size_t)ntiles * kBM * tk, -1);
  for (int mt = 0; mt < nmt; ++mt)
    for (int t = tile_off[mt]; t < tile_off[mt + 1]; ++t) {
      const int kt = tile_kt[t];
      for (int r = 0; r < kBM; ++r) {
        const int i = mt * kBM + r;
        if (i >= n) break;
        for (int c = 0; c < tk; ++c) {
          const int j = kt * tk + c;
          if (j >= n) break;
          tile_map[((size_t)t * kBM + r) * tk + c] = full[(size_t)i * n + j];
        }
      }
    }
  total_tiles = nmt * nkt;
  return 0;
}

// K = 2 sum_Q (B_Q C)(B_Q C)^T on the tensor cores; see the file comment.
// Bsrc: packed factor [rank][ncol] (storage 1 = FP32, 2 = BF16); kind: the
// operand type of both GEMMs.  Scratch comes from `ws` (grown as needed).
cudaError_t df_k_tensor_cores(const UmmaDfArgs& p, UmmaWorkspace& ws, int* status, cudaStream_t st) {
  const int n = p.n, nocc = p.nocc, kind = p.kind;
  const int el = kind == kBF16 ? 2 : 4;
  const TileStructure& ts = *p.tiles;
  const int tk = ts.tk;
  const int nocc_pad = (nocc + 15) / 16 * 16;
  const int ldk = (n + 7) / 8 * 8;  // row stride of C^T: 16-byte multiple for TMA
  const int nmt = (n + kBM - 1) / kBM;
  const int i_tiles = (nocc_pad * el + kRowBytes - 1) / kRowBytes;
  cudaError_t e;
  // per-Q bytes: the tile-compact chunk and T
  const size_t per_q = (size_t)ts.ntiles * kBM * tk * el + (size_t)n * nocc_pad * el;
  int qc = (int)std::max<size_t>(1, std::min<size_t>((size_t)p.rank, p.chunk_bytes / std::max<size_t>(per_q, 1)));
  if (p.max_chunk > 0) qc = std::min(qc, p.max_chunk);
  if ((e = ws.grow(ws.dense, (size_t)qc * ts.ntiles * kBM * tk * el)) != cudaSuccess) return e;
  if ((e = ws.grow(ws.T, (size_t)qc * n * nocc_pad * el)) != cudaSuccess) return e;
  if ((e = ws.grow(ws.Ct, (size_t)nocc_pad * ldk * el)) != cudaSuccess) return e;
  if ((e = ws.grow(ws.Kf, (size_t)n * n * 4)) != cudaSuccess) return e;
  if ((e = ws.grow(ws.err, 4)) != cudaSuccess) return e;
  if ((e = cudaMemsetAsync(ws.Kf.p, 0, (size_t)n * n * 4, st)) != cudaSuccess) return e;
  if ((e = cudaMemsetAsync(ws.err.p, 0, 4, st)) != cudaSuccess) return e;
  {
    const long long tot = (long long)nocc_pad * ldk;
    const unsigned g = (unsigned)((tot + 255) / 256);
    if (kind == kBF16) ct_kernel<__nv_bfloat16><<<g, 256, 0, st>>>(p.C, n, nocc, nocc_pad, ldk, (__nv_bfloat16*)ws.Ct.p);
    else ct_kernel<float><<<g, 256, 0, st>>>(p.C, n, nocc, nocc_pad, ldk, (float*)ws.Ct.p);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
  }
  // lower output tiles of the symmetric update
  std::vector<int2> lower;
  for (int mt = 0; mt < nmt; ++mt)
    for (int nt = 0; nt * kBN < n; ++nt)
      if (nt * kBN <= mt * kBM + kBM - 1) lower.push_back(make_int2(mt, nt));
  if ((e = ws.grow(ws.lower, lower.size() * sizeof(int2))) != cudaSuccess) return e;
  if ((e = cudaMemcpyAsync(ws.lower.p, lower.data(), lower.size() * sizeof(int2), cudaMemcpyHostToDevice, st)) !=
      cudaSuccess)
    return e;
  CUtensorMap mCt, mA1, mT_A, mT_B;
  if (!make_map(&mCt, kind, ws.Ct.p, ldk, nocc_pad, 1, (long long)ldk * el, (long long)nocc_pad * ldk * el, kBN))
    return cudaErrorInvalidValue;
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, p.device);
  // executed MMA work: GEMM 1 over the non-zero tiles of every row block,
  // GEMM 2 over the lower output tiles (N of the edge tiles as issued)
  {
    // (the column tiles' widths sum to nocc_pad)
    double f1 = 2.0 * kBM * tk * (double)ts.ntiles * nocc_pad;
    double f2 = 0.0;
    for (const int2& t : lower) f2 += 2.0 * kBM * (double)((std::min(kBN, n - t.y * kBN) + 15) / 16 * 16);
    f2 *= (double)i_tiles * (kRowBytes / el);
    ws.flops_executed = (f1 + f2) * p.rank;
    ws.tiles_fraction = ts.total_tiles > 0 ? (double)ts.ntiles / ts.total_tiles : 0.0;
  }
  // HFG_PROFILE=1: device time of each phase, summed over the chunks, on stderr
  static const bool profile = getenv("HFG_PROFILE") && getenv("HFG_PROFILE")[0] == '1';
  cudaEvent_t pev[4] = {nullptr, nullptr, nullptr, nullptr};
  float pms[3] = {0.f, 0.f, 0.f};
  if (profile)
    for (auto& x : pev) cudaEventCreate(&x);
  for (int q0 = 0; q0 < p.rank; q0 += qc) {
    const int qn = std::min(qc, p.rank - q0);
    if (profile) cudaEventRecord(pev[0], st);
    // 1. unpack the chunk's non-zero tiles
    {
      dim3 g((unsigned)ts.ntiles, (unsigned)std::min(qn, 64));
      if (ts.ntiles > 0) {
        if (kind == kBF16) {
          if (p.storage == 1)
            unpack_tiles_kernel<float, __nv_bfloat16, 64><<<g, 256, 0, st>>>(
                (const float*)p.B, p.ncol, p.tile_map_dev, ts.ntiles, p.rank_offset + q0, qn, (__nv_bfloat16*)ws.dense.p);
          else
            unpack_tiles_kernel<__nv_bfloat16, __nv_bfloat16, 64><<<g, 256, 0, st>>>(
                (const __nv_bfloat16*)p.B, p.ncol, p.tile_map_dev, ts.ntiles, p.rank_offset + q0, qn,
                (__nv_bfloat16*)ws.dense.p);
        } else {
          unpack_tiles_kernel<float, float, 32><<<g, 256, 0, st>>>((const float*)p.B, p.ncol, p.tile_map_dev,
                                                                   ts.ntiles, p.rank_offset + q0, qn, (float*)ws.dense.p);
        }
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
      }
    }
    if (profile) cudaEventRecord(pev[1], st);
    // 2. T_Q = B_Q C: A = tile-compact chunk (x: tk, y: tile rows, z: Q)
    if (!make_map(&mA1, kind, ws.dense.p, tk, (long long)ts.ntiles * kBM, qn, (long long)tk * el,
                  (long long)ts.ntiles * kBM * tk * el, kBM))
      return cudaErrorInvalidValue;
    GemmArgs g1{};
    g1.mode = 0;
    g1.m_rows = n;
    g1.n_cols = nocc_pad;
    g1.tile_off = p.tile_off_dev;
    g1.tile_kt = p.tile_kt_dev;
    g1.out = ws.T.p;
    g1.ldo = nocc_pad;
    g1.batch_stride = (long long)n * nocc_pad;
    g1.err = (int*)ws.err.p;
    // equal column tiles of at most 256 (a narrow remainder tile would run
    // the tensor cores below their rate)
    g1.n_ntiles = (nocc_pad + kBN - 1) / kBN;
    g1.bn = ((nocc_pad + g1.n_ntiles - 1) / g1.n_ntiles + 15) / 16 * 16;
    g1.n_mtiles = nmt;
    g1.units = (long long)g1.n_ntiles * nmt * qn;
    dim3 grid1((unsigned)std::min<long long>(g1.units, sms));
    e = kind == kBF16 ? launch_gemm<kBF16, 0>(mA1, mCt, g1, grid1, st) : launch_gemm<kTF32, 0>(mA1, mCt, g1, grid1, st);
    if (e != cudaSuccess) return e;
    if (profile) cudaEventRecord(pev[2], st);
    // 3. K_lower += T T^T over this chunk's Q, split so that the grid covers
    //    the SMs a few times
    if (!make_map(&mT_A, kind, ws.T.p, nocc_pad, n, qn, (long long)nocc_pad * el, (long long)n * nocc_pad * el, kBM) ||
        !make_map(&mT_B, kind, ws.T.p, nocc_pad, n, qn, (long long)nocc_pad * el, (long long)n * nocc_pad * el, kBN))
      return cudaErrorInvalidValue;
    // work units: (lower tile, Q range), about eight per SM for balance
    int splits = std::max(1, std::min(qn, (8 * sms + (int)lower.size() - 1) / (int)lower.size()));
    const int qps = (qn + splits - 1) / splits;
    splits = (qn + qps - 1) / qps;
    GemmArgs g2{};
    g2.mode = 1;
    g2.m_rows = n;
    g2.n_cols = n;
    g2.bn = kBN;
    g2.out_tiles = (const int2*)ws.lower.p;
    g2.n_lower = (int)lower.size();
    g2.q_count = qn;
    g2.q_per_split = qps;
    g2.i_tiles = i_tiles;
    g2.units = (long long)lower.size() * splits;
    g2.out = ws.Kf.p;
    g2.ldo = n;
    g2.err = (int*)ws.err.p;
    dim3 grid2((unsigned)std::min<long long>(g2.units, sms));
    e = kind == kBF16 ? launch_gemm<kBF16, 1>(mT_A, mT_B, g2, grid2, st)
                      : launch_gemm<kTF32, 1>(mT_A, mT_B, g2, grid2, st);
    if (e != cudaSuccess) return e;
    if (profile) {
      cudaEventRecord(pev[3], st);
      cudaEventSynchronize(pev[3]);
      for (int k = 0; k < 3; ++k) {
        float ms = 0.f;
        cudaEventElapsedTime(&ms, pev[k], pev[k + 1]);
        pms[k] += ms;
      }
    }
  }
  if (profile) {
    fprintf(stderr, "hfg-profile df-exchange %s n %d nocc %d rank %d chunk %d tiles %d/%d: unpack %.3f ms, "
                    "T = B C %.3f ms, K += T T^T %.3f ms\n",
            kind == kBF16 ? "bf16" : "tf32", n, nocc, p.rank, qc, ts.ntiles, ts.total_tiles, pms[0], pms[1], pms[2]);
    for (auto& x : pev) cudaEventDestroy(x);
  }
  {
    const long long tot = (long long)n * n;
    k_finalize_kernel<<<(unsigned)((tot + 255) / 256), 256, 0, st>>>((const float*)ws.Kf.p, n, 2.0, p.K);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
  }
  if (status) {
    if ((e = cudaMemcpyAsync(status, ws.err.p, 4, cudaMemcpyDeviceToHost, st)) != cudaSuccess) return e;
    if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return e;
  }
  return cudaSuccess;
}

}  // namespace hfg
