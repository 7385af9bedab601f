// Direct J/K build: one kernel per angular class (la lb|lc ld), Obara-Saika
// VRR per primitive quartet, contraction in registers, HRR, and the J/K
// digestion fused in the same kernel.
//
// Replaces hf-rs's chain compute_shell_eri_tensor -> packed 8-fold tensor ->
// contract_jk (src/shell_integrals.rs:92-240, src/scf.rs:337-364): the same
// Schwarz-screened shell quartets (Q_ab Q_cd > threshold), digested into
// the same J and K, without storing integrals.
//
// Digestion of one unique shell quartet (ab|cd) with degeneracy weight
// deg = (a==b ? 1/2 : 1)(c==d ? 1/2 : 1)(ab==cd ? 1/2 : 1) applied to the full
// Cartesian block accumulates into unsymmetrised J', K' and the host-side
// epilogue forms J = (J' + J'^T)/2, K = (K' + K'^T)/2:
//   J'[a,b] += 4 w Σ (ab|cd) D[c,d]      J'[c,d] += 4 w Σ (ab|cd) D[a,b]
//   K'[a,c] += 2 w Σ (ab|cd) D[b,d]      K'[b,c] += 2 w Σ (ab|cd) D[a,d]
//   K'[a,d] += 2 w Σ (ab|cd) D[b,c]      K'[b,d] += 2 w Σ (ab|cd) D[a,c]
// which equals contract_jk's 8-permutation loop for symmetric densities.
//
// Work split: a warp takes one bra shell pair and up to 32 ket pairs of one
// pair class, one shell quartet per lane.  Each lane keeps its ket
// primitive pair in registers (outer loop) while the warp walks the bra
// primitive pairs together (inner loop: every lane reads the same address,
// one broadcast transaction).  Primitive pairs are sorted by their own
// Cauchy-Schwarz bound, so primitive screening ends both loops early.
// Blocks are persistent: each stages the Boys Taylor rows it needs in shared
// memory once and then strides over the launch's warp tasks.  The J'[a,b]
// contribution, common to the warp's bra pair, is reduced across the warp
// before its atomics.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

#include "eri_prim.cuh"

namespace hfg {

// Density blocks needed by the digestion of one quartet.
// The blocks are held in the kernel's arithmetic type: FP32 quartets have
// |(ab|cd)| below the FP32 threshold (<= 1e-7), so rounding D to FP32 adds
// at most ~1e-14 relative to the largest contribution to J/K.
template <int LA, int LB, int LC, int LD, int NS, typename DT>
struct DBlocks {
  static constexpr int NA = ncart(LA), NB = ncart(LB), NC = ncart(LC), ND = ncart(LD);
  DT cd[NC * ND], ab[NA * NB];
  DT bd[NS][NB * ND], ad[NS][NA * ND], bc[NS][NB * NC], ac[NS][NA * NC];
  __device__ __forceinline__ void load(const PairInfo& bra, const PairInfo& ket, const JKLaunchArgs& a) {
    // FP32 launches read the build's FP32 copies (half the bytes, no
    // conversions); their launcher refuses to start without them
    if constexpr (sizeof(DT) == 4) fill(bra, ket, a.n, a.Dtot32, a.Dspin32);
    else fill(bra, ket, a.n, a.Dtot, a.Dspin);
  }
  template <typename ST>
  __device__ __forceinline__ void fill(const PairInfo& bra, const PairInfo& ket, int n, const ST* __restrict__ Dt,
                                       const ST* __restrict__ Ds) {
    const int i0 = bra.ao_a, j0 = bra.ao_b, k0 = ket.ao_a, l0 = ket.ao_b;
#pragma unroll
    for (int k = 0; k < NC; ++k)
#pragma unroll
      for (int l = 0; l < ND; ++l) cd[k * ND + l] = (DT)__ldg(Dt + (size_t)(k0 + k) * n + l0 + l);
#pragma unroll
    for (int i = 0; i < NA; ++i)
#pragma unroll
      for (int j = 0; j < NB; ++j) ab[i * NB + j] = (DT)__ldg(Dt + (size_t)(i0 + i) * n + j0 + j);
#pragma unroll
    for (int sp = 0; sp < NS; ++sp) {
      const ST* D = Ds + (size_t)sp * n * n;
#pragma unroll
      for (int j = 0; j < NB; ++j)
#pragma unroll
        for (int l = 0; l < ND; ++l) bd[sp][j * ND + l] = (DT)__ldg(D + (size_t)(j0 + j) * n + l0 + l);
#pragma unroll
      for (int i = 0; i < NA; ++i)
#pragma unroll
        for (int l = 0; l < ND; ++l) ad[sp][i * ND + l] = (DT)__ldg(D + (size_t)(i0 + i) * n + l0 + l);
#pragma unroll
      for (int j = 0; j < NB; ++j)
#pragma unroll
        for (int k = 0; k < NC; ++k) bc[sp][j * NC + k] = (DT)__ldg(D + (size_t)(j0 + j) * n + k0 + k);
#pragma unroll
      for (int i = 0; i < NA; ++i)
#pragma unroll
        for (int k = 0; k < NC; ++k) ac[sp][i * NC + k] = (DT)__ldg(D + (size_t)(i0 + i) * n + k0 + k);
    }
  }
};

// Fused digestion of one scaled Cartesian block (w already includes deg and
// the component scales), except J'[a,b] which the caller reduces across the
// warp (jab receives this lane's sum over c,d).  With SEG, K'[a,c] and
// K'[b,c] are returned in kac / kbc for the caller's segmented reduction
// over lanes that share shell c, instead of being added here.
template <int LA, int LB, int LC, int LD, int NS, typename DT, bool SEG>
__device__ __forceinline__ void digest(const DT* __restrict__ w, const PairInfo& bra, const PairInfo& ket,
                                       const JKLaunchArgs& a, const DBlocks<LA, LB, LC, LD, NS, DT>& d,
                                       DT* __restrict__ jab, DT (*__restrict__ kac)[ncart(LA) * ncart(LC)],
                                       DT (*__restrict__ kbc)[ncart(LB) * ncart(LC)]) {
  constexpr int NA = ncart(LA), NB = ncart(LB), NC = ncart(LC), ND = ncart(LD);
  const int n = a.n;
  const int i0 = bra.ao_a, j0 = bra.ao_b, k0 = ket.ao_a, l0 = ket.ao_b;
#pragma unroll
  for (int ij = 0; ij < NA * NB; ++ij) {
    DT s = (DT)0;
#pragma unroll
    for (int kl = 0; kl < NC * ND; ++kl) s += w[ij * NC * ND + kl] * d.cd[kl];
    jab[ij] = (DT)4 * s;
  }
#pragma unroll
  for (int k = 0; k < NC; ++k)
#pragma unroll
    for (int l = 0; l < ND; ++l) {
      DT s = (DT)0;
#pragma unroll
      for (int ij = 0; ij < NA * NB; ++ij) s += w[ij * NC * ND + k * ND + l] * d.ab[ij];
      atomicAdd(a.Jacc + (size_t)(k0 + k) * n + l0 + l, 4.0 * (double)s);
    }
#pragma unroll
  for (int sp = 0; sp < NS; ++sp) {
    double* K = a.Kacc + (size_t)sp * n * n;
#pragma unroll
    for (int i = 0; i < NA; ++i)
#pragma unroll
      for (int k = 0; k < NC; ++k) {
        DT s = (DT)0;
#pragma unroll
        for (int j = 0; j < NB; ++j)
#pragma unroll
          for (int l = 0; l < ND; ++l) s += w[((i * NB + j) * NC + k) * ND + l] * d.bd[sp][j * ND + l];
        if (SEG) kac[sp][i * NC + k] = s;
        else atomicAdd(K + (size_t)(i0 + i) * n + k0 + k, 2.0 * (double)s);
      }
#pragma unroll
    for (int j = 0; j < NB; ++j)
#pragma unroll
      for (int k = 0; k < NC; ++k) {
        DT s = (DT)0;
#pragma unroll
        for (int i = 0; i < NA; ++i)
#pragma unroll
          for (int l = 0; l < ND; ++l) s += w[((i * NB + j) * NC + k) * ND + l] * d.ad[sp][i * ND + l];
        if (SEG) kbc[sp][j * NC + k] = s;
        else atomicAdd(K + (size_t)(j0 + j) * n + k0 + k, 2.0 * (double)s);
      }
#pragma unroll
    for (int i = 0; i < NA; ++i)
#pragma unroll
      for (int l = 0; l < ND; ++l) {
        DT s = (DT)0;
#pragma unroll
        for (int j = 0; j < NB; ++j)
#pragma unroll
          for (int k = 0; k < NC; ++k) s += w[((i * NB + j) * NC + k) * ND + l] * d.bc[sp][j * NC + k];
        atomicAdd(K + (size_t)(i0 + i) * n + l0 + l, 2.0 * (double)s);
      }
#pragma unroll
    for (int j = 0; j < NB; ++j)
#pragma unroll
      for (int l = 0; l < ND; ++l) {
        DT s = (DT)0;
#pragma unroll
        for (int i = 0; i < NA; ++i)
#pragma unroll
          for (int k = 0; k < NC; ++k) s += w[((i * NB + j) * NC + k) * ND + l] * d.ac[sp][i * NC + k];
        atomicAdd(K + (size_t)(j0 + j) * n + l0 + l, 2.0 * (double)s);
      }
  }
}

// Resident blocks per SM that the register allocation of class
// (LA LB|LC LD) is tuned for (measured on (H2O)64 cc-pVDZ): the light FP32
// classes gain from 3-4 blocks; classes whose contracted accumulators do not
// fit in 128 registers (FP64 with L >= 4, FP32 with L >= 5 and (pp|pp)) run
// one block with up to 255 registers, since their spills cost more than the
// lost occupancy.  The HFG_JK_MIN_BLOCKS_F64 / _F32 macros override the
// table for tuning builds.
template <int LA, int LB, int LC, int LD, typename T> struct MinBlocks {
  static constexpr int code = LA * 1000 + LB * 100 + LC * 10 + LD;
  static constexpr int L = LA + LB + LC + LD;
#ifndef HFG_JK_F64_LIGHT_BLOCKS
#define HFG_JK_F64_LIGHT_BLOCKS 2
#endif
#ifdef HFG_JK_MIN_BLOCKS_F64
  static constexpr int f64 = HFG_JK_MIN_BLOCKS_F64;
#else
  static constexpr int f64 = L >= 4 ? 1 : (L <= 2 ? HFG_JK_F64_LIGHT_BLOCKS : 2);
#endif
#ifdef HFG_JK_MIN_BLOCKS_F32
  static constexpr int f32 = HFG_JK_MIN_BLOCKS_F32;
#else
  static constexpr int f32 = (code == 0 || code == 1000 || code == 1010 || code == 1100 || code == 2000) ? 4
                             : (code == 2100 || code == 1110 || code == 2010)                           ? 3
                             : (L >= 5 || code == 1111)                                                 ? 1
                                                                                                        : 2;
#endif
  static constexpr int value = sizeof(T) == 4 ? f32 : f64;
};

// 1: start fetching the next task's ket primitive records while this task
// computes.  It pays in the FP64 launches; the FP32 ones ran 1% faster
// without it on (H2O)64 cc-pVDZ.
#ifndef HFG_JK_PREFETCH_F64
#define HFG_JK_PREFETCH_F64 1
#endif
#ifndef HFG_JK_PREFETCH_F32
#define HFG_JK_PREFETCH_F32 0
#endif
// Bring the 128-byte line holding p into L1 without waiting for it.
__device__ __forceinline__ void prefetch_l1(const void* p) { asm volatile("prefetch.global.L1 [%0];" ::"l"(p)); }


// K'[a,c], K'[b,c] are summed over the lanes that share the ket's first
// shell c before their atomics (kets are ordered by AO index within each
// Schwarz bucket, so such lanes are neighbours) in the launches where that
// measured faster on (H2O)64 cc-pVDZ: FP32 launches except (21|11), (21|20)
// and (22|10), and the FP64 launches of (10|10), (11|10), (20|10) (4-12%
// each).  The others add per lane.  HFG_JK_SEG_F64 / HFG_JK_SEG_F32 = 0 or 1
// override this in tuning builds.
#ifndef HFG_JK_SEG_F64
#define HFG_JK_SEG_F64 -1
#endif
#ifndef HFG_JK_SEG_F32
#define HFG_JK_SEG_F32 -1
#endif
template <int LA, int LB, int LC, int LD, typename T> struct SegReduce {
  static constexpr int code = LA * 1000 + LB * 100 + LC * 10 + LD;
  static constexpr bool f64_table = code == 1010 || code == 1110 || code == 2010;
  static constexpr bool f32_table = !(code == 2111 || code == 2120 || code == 2210);
  static constexpr bool value = sizeof(T) == 4 ? (HFG_JK_SEG_F32 < 0 ? f32_table : HFG_JK_SEG_F32 != 0)
                                               : (HFG_JK_SEG_F64 < 0 ? f64_table : HFG_JK_SEG_F64 != 0);
};

// Sum of v over this lane's run of lanes [lane, end), left in the run's
// first lane (segmented tree over contiguous runs of at most 32 lanes).
template <typename T>
__device__ __forceinline__ T run_sum(T v, int lane, int end) {
#pragma unroll
  for (int off = 1; off < 32; off <<= 1) {
    const T o = __shfl_down_sync(0xffffffffu, v, off);
    if (lane + off < end) v += o;
  }
  return v;
}

// One work-queue step of a launch: a warp takes one bra shell pair and up
// to 32 ket pairs of one pair class per task, one shell quartet per lane.
// Step c holds tasks [chunk_start[c], chunk_start[c + 1]) and chunk_entry[c]
// is the entry of its first task; later tasks of the step walk the prefix
// forward.
template <int LA, int LB, int LC, int LD, typename T, int NS>
__device__ __forceinline__ void jk_step(const JKLaunchArgs& a, long long c, int lane, const T* __restrict__ sm) {
  using C = EriClass<LA, LB, LC, LD>;
  constexpr bool SEG = SegReduce<LA, LB, LC, LD, T>::value;
  constexpr int NA = ncart(LA), NB = ncart(LB), NC = ncart(LC), ND = ncart(LD), NAB = NA * NB;
  {
    const long long t0 = __ldg(a.chunk_start + c), t1 = __ldg(a.chunk_start + c + 1);
    int e = __ldg(a.chunk_entry + c);
    long long next = __ldg(a.prefix + e + 1);
    const int turns = a.serial ? 32 : 1;
    for (long long warp = t0; warp < t1; ++warp) {
      while (warp >= next) {
        ++e;
        next = a.prefix[e + 1];
      }
      for (int turn = 0; turn < turns; ++turn) {
        const JKEntry ent = a.entries[e];
        const int kidx = ent.k_lo + (int)(warp - a.prefix[e]) * 32 + lane;
        // kets are bucketed by bound: the exact Schwarz test per quartet (in
        // deterministic mode, only lane `turn`'s quartet on this turn)
        const bool active = kidx < ent.k_hi && __ldg(a.pairQ + kidx) * __ldg(a.pairQ + ent.bra) > a.thr &&
                            (turns == 1 || lane == turn);
        const PairInfo bra = a.pairs[ent.bra];
        PairInfo ket;
        {
          const int kx = active ? kidx : ent.k_lo;
          const double2 v0 = __ldg(a.kets.a0 + kx), v1 = __ldg(a.kets.a1 + kx), v2 = __ldg(a.kets.a2 + kx);
          const int4 ii = __ldg(a.kets.ii + kx);
          const int2 nn = __ldg(a.kets.nn + kx);
          ket.Ax = v0.x;
          ket.Ay = v0.y;
          ket.Az = v1.x;
          ket.ABx = v1.y;
          ket.ABy = v2.x;
          ket.ABz = v2.y;
          ket.ao_a = ii.x;
          ket.ao_b = ii.y;
          ket.rec_off = ii.z;
          ket.rec_stride = ii.w;
          ket.npp = nn.x;
          ket.same = nn.y;
        }
        // the next task usually continues this entry: start fetching its
        // first primitive records (kets of one class have equal primitive
        // counts and consecutive records, so they start 32 on)
        constexpr bool kPrefetch = sizeof(T) == 4 ? HFG_JK_PREFETCH_F32 != 0 : HFG_JK_PREFETCH_F64 != 0;
        if (kPrefetch && warp + 1 < t1 && kidx + 32 < ent.k_hi) {
          prefetch_l1(RecOf<T>::get(a) + ket.rec_off + 32);
          prefetch_l1(a.pbound + ket.rec_off + 32);
        }
        T acc[C::NACC];
#pragma unroll
        for (int x = 0; x < C::NACC; ++x) acc[x] = (T)0;
        if (active) {
          using Rec = typename RecOf<T>::type;
          const T ACx = (T)(bra.Ax - ket.Ax), ACy = (T)(bra.Ay - ket.Ay), ACz = (T)(bra.Az - ket.Az);
          const T bABx = (T)bra.ABx, bABy = (T)bra.ABy, bABz = (T)bra.ABz;
          const T kABx = (T)ket.ABx, kABy = (T)ket.ABy, kABz = (T)ket.ABz;
          const Rec* __restrict__ br = RecOf<T>::get(a) + bra.rec_off;
          const Rec* __restrict__ kr = RecOf<T>::get(a) + ket.rec_off;
          const float* __restrict__ bb = a.pbound + bra.rec_off;
          const float* __restrict__ kb = a.pbound + ket.rec_off;
          const int nb = bra.npp, nk = ket.npp, bs = bra.rec_stride, ks = ket.rec_stride;
          // screening products in FP32 (bounds are stored as floats; count_kernel
          // evaluates the same products)
          const float eps = (float)a.prim_eps;
          const float bmax = bb[0];
          // ket primitive pairs while they survive against the largest bra one
          // (bounds sorted descending); the next record and bound are fetched
          // one iteration ahead
          Rec Qn = kr[0];
          float qbn = kb[0];
          for (int ik = 0; ik < nk; ++ik) {
            const Rec Q = Qn;
            const float qb = qbn;
            if (qb * bmax < eps) break;
            if (ik + 1 < nk) {
              Qn = kr[(ik + 1) * ks];
              qbn = kb[(ik + 1) * ks];
            }
            const T QCx = -Q.bp * kABx, QCy = -Q.bp * kABy, QCz = -Q.bp * kABz;
            const T ACQx = ACx - QCx, ACQy = ACy - QCy, ACQz = ACz - QCz;
            const T ckq = (T)kTwoPiPow25 * Q.kp;
            int ib = 0;
            if constexpr (C::NACC <= 9) {
              // two independent primitive quartets per step (bra primitive pairs
              // are sorted by bound: if the second survives, so does the first)
              for (; ib + 1 < nb; ib += 2) {
                if (bb[(ib + 1) * bs] * qb < eps) break;
                const Rec P0 = br[ib * bs], P1 = br[(ib + 1) * bs];
                prim_quartet_k<LA, LB, LC, LD, T>(acc, P0.p, P0.inv_p, P0.kp, -P0.bp * bABx, -P0.bp * bABy,
                                                  -P0.bp * bABz, Q.p, Q.inv_p, ckq, QCx, QCy, QCz, ACQx, ACQy, ACQz,
                                                  sm);
                prim_quartet_k<LA, LB, LC, LD, T>(acc, P1.p, P1.inv_p, P1.kp, -P1.bp * bABx, -P1.bp * bABy,
                                                  -P1.bp * bABz, Q.p, Q.inv_p, ckq, QCx, QCy, QCz, ACQx, ACQy, ACQz,
                                                  sm);
              }
            }
            Rec P = br[(ib < nb ? ib : 0) * bs];
            for (; ib < nb; ++ib) {
              const Rec Pn = br[(ib + 1 < nb ? ib + 1 : ib) * bs];
              if (bb[ib * bs] * qb < eps) break;
              prim_quartet_k<LA, LB, LC, LD, T>(acc, P.p, P.inv_p, P.kp, -P.bp * bABx, -P.bp * bABy, -P.bp * bABz,
                                                Q.p, Q.inv_p, ckq, QCx, QCy, QCz, ACQx, ACQy, ACQz, sm);
              P = Pn;
            }
          }
        }
        T jab[NAB];
        T kac[NS][NA * NC], kbc[NS][NB * NC];
        if (active) {
          DBlocks<LA, LB, LC, LD, NS, T> dblk;
          dblk.load(bra, ket, a);
          T out[C::NOUT];
          C::hrr(acc, out, (T)bra.ABx, (T)bra.ABy, (T)bra.ABz, (T)ket.ABx, (T)ket.ABy, (T)ket.ABz);
          T deg = (T)1;
          if (bra.same) deg *= (T)0.5;
          if (ket.same) deg *= (T)0.5;
          if (kidx == ent.bra) deg *= (T)0.5;
          // scaled in place (a second block-sized array would double the
          // per-thread footprint of the large classes)
#pragma unroll
          for (int i = 0; i < NA; ++i)
#pragma unroll
            for (int j = 0; j < NB; ++j)
#pragma unroll
              for (int k = 0; k < NC; ++k)
#pragma unroll
                for (int l = 0; l < ND; ++l) {
                  const int x = ((i * NB + j) * NC + k) * ND + l;
                  out[x] *= deg * (T)(comp_scale(LA, i) * comp_scale(LB, j) * comp_scale(LC, k) * comp_scale(LD, l));
                }
          digest<LA, LB, LC, LD, NS, T, SEG>(out, bra, ket, a, dblk, jab, kac, kbc);
        } else {
#pragma unroll
          for (int x = 0; x < NAB; ++x) jab[x] = (T)0;
          if (SEG) {
#pragma unroll
            for (int sp = 0; sp < NS; ++sp) {
#pragma unroll
              for (int x = 0; x < NA * NC; ++x) kac[sp][x] = (T)0;
#pragma unroll
              for (int x = 0; x < NB * NC; ++x) kbc[sp][x] = (T)0;
            }
          }
        }
        if (SEG) {
          // runs of consecutive lanes whose kets share shell c (first AO
          // ket.ao_a); inactive lanes form runs of their own
          const int key = active ? ket.ao_a : -1 - lane;
          const int prev = __shfl_up_sync(0xffffffffu, key, 1);
          const unsigned heads = __ballot_sync(0xffffffffu, lane == 0 || key != prev);
          const unsigned later = heads & (0xfffffffeu << lane);
          const int end = later ? __ffs(later) - 1 : 32;
          const bool head = (heads >> lane) & 1u;
          const int n = a.n, i0 = bra.ao_a, j0 = bra.ao_b, k0 = ket.ao_a;
#pragma unroll
          for (int sp = 0; sp < NS; ++sp) {
            double* K = a.Kacc + (size_t)sp * n * n;
#pragma unroll
            for (int i = 0; i < NA; ++i)
#pragma unroll
              for (int k = 0; k < NC; ++k) {
                const T v = run_sum(kac[sp][i * NC + k], lane, end);
                if (head && active) atomicAdd(K + (size_t)(i0 + i) * n + k0 + k, 2.0 * (double)v);
              }
#pragma unroll
            for (int j = 0; j < NB; ++j)
#pragma unroll
              for (int k = 0; k < NC; ++k) {
                const T v = run_sum(kbc[sp][j * NC + k], lane, end);
                if (head && active) atomicAdd(K + (size_t)(j0 + j) * n + k0 + k, 2.0 * (double)v);
              }
          }
        }
        // J'[a,b]: the whole warp shares the bra pair
#pragma unroll
        for (int x = 0; x < NAB; ++x) {
          T v = jab[x];
#pragma unroll
          for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
          if (lane == 0) atomicAdd(a.Jacc + (size_t)(bra.ao_a + x / NB) * a.n + bra.ao_b + x % NB, (double)v);
        }
      }
    }
  }
}

// Persistent blocks: each stages the Boys Taylor rows of its class in shared
// memory once, then takes work-queue steps from the launch's atomic counter
// until the launch is done.
template <int LA, int LB, int LC, int LD, typename T, int NS>
__global__ void __launch_bounds__(256, (MinBlocks<LA, LB, LC, LD, T>::value)) jk_kernel(const JKLaunchArgs a) {
  using C = EriClass<LA, LB, LC, LD>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* sm = reinterpret_cast<T*>(smem_raw);
  boys_stage<T, C::L>(sm, Prec<T>::table(a), Prec<T>::expt(a));
  __syncthreads();
  const int lane = threadIdx.x & 31;
  for (;;) {
    unsigned long long c = 0;
    if (lane == 0) c = atomicAdd(a.counter, 1ull);
    c = __shfl_sync(0xffffffffu, c, 0);
    if ((long long)c >= a.nchunks) break;
    jk_step<LA, LB, LC, LD, T, NS>(a, (long long)c, lane, sm);
  }
}

// One launch of class (LA LB|LC LD) over the work queues of several
// molecules (RHF): the launch's steps are the molecules' steps one after
// another (job_steps[j] is the first step of molecule j), and each step runs
// with its molecule's pair tables, records, thresholds, density and
// accumulators.
template <int LA, int LB, int LC, int LD, typename T>
__global__ void __launch_bounds__(256, (MinBlocks<LA, LB, LC, LD, T>::value)) jk_batch_kernel(const JKLaunchArgs a) {
  using C = EriClass<LA, LB, LC, LD>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* sm = reinterpret_cast<T*>(smem_raw);
  boys_stage<T, C::L>(sm, Prec<T>::table(a), Prec<T>::expt(a));
  __syncthreads();
  const int lane = threadIdx.x & 31;
  for (;;) {
    unsigned long long c = 0;
    if (lane == 0) c = atomicAdd(a.counter, 1ull);
    c = __shfl_sync(0xffffffffu, c, 0);
    if ((long long)c >= a.nchunks) break;
    int lo = 0, hi = a.njobs;  // last job whose first step is <= c
    while (hi - lo > 1) {
      const int mid = (lo + hi) >> 1;
      if (__ldg(a.job_steps + mid) <= (long long)c) lo = mid; else hi = mid;
    }
    const JKJob& jb = a.jobs[lo];
    JKLaunchArgs la = a;
    la.entries = jb.entries;
    la.prefix = jb.prefix;
    la.chunk_start = jb.chunk_start;
    la.chunk_entry = jb.chunk_entry;
    la.pairs = jb.pairs;
    la.kets = jb.kets;
    la.pairQ = jb.pairQ;
    la.rec64 = jb.rec64;
    la.rec32 = jb.rec32;
    la.pbound = jb.pbound;
    la.Dtot = jb.Dtot;
    la.Dspin = jb.Dtot;
    la.Dtot32 = jb.Dtot32;
    la.Dspin32 = jb.Dtot32;
    la.Jacc = jb.Jacc;
    la.Kacc = jb.Kacc;
    la.n = jb.n;
    la.thr = jb.thr;
    la.prim_eps = jb.prim_eps;
    jk_step<LA, LB, LC, LD, T, 1>(la, (long long)c - __ldg(a.job_steps + lo), lane, sm);
  }
}

}  // namespace hfg
