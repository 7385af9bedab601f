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

#include "boys.cuh"
#include "eri_gen.cuh"
#include "hfg_internal.h"

namespace hfg {

constexpr double kTwoPiPow25 = 34.986836655249726164477;

__host__ __device__ constexpr int ncart(int l) { return (l + 1) * (l + 2) / 2; }

// Per-component scale 1/sqrt(prod (2l_i-1)!!) in hf-rs component order
// (src/basis.rs:123-132 with the contraction normalisation factored out).
__device__ __forceinline__ double comp_scale(int l, int i) {
  if (l < 2) return 1.0;
  return i < 3 ? 0.57735026918962576451 : 1.0;
}

template <typename T> struct Prec;
template <> struct Prec<double> {
  __device__ static const double* table(const JKLaunchArgs& a) { return a.boys64; }
  __device__ static const double* expt(const JKLaunchArgs& a) { return a.expt64; }
};
template <> struct Prec<float> {
  __device__ static const float* table(const JKLaunchArgs& a) { return a.boys32; }
  __device__ static const float* expt(const JKLaunchArgs& a) { return a.expt32; }
};

template <typename T> __device__ __forceinline__ T rsqrt_t(T x);
template <> __device__ __forceinline__ double rsqrt_t<double>(double x) { return rsqrt(x); }
template <> __device__ __forceinline__ float rsqrt_t<float>(float x) { return rsqrtf(x); }

// One primitive quartet added into acc: bra primitive pair (p, 1/p, kp,
// P - A) and ket primitive pair (q, 1/q, kq, Q - C); AC = A - C.
template <int LA, int LB, int LC, int LD, typename T>
__device__ __forceinline__ void prim_quartet(T* __restrict__ acc, T p, T inv_p, T kpp, T PAx, T PAy, T PAz, T q,
                                             T inv_q, T kpq, T QCx, T QCy, T QCz, T ACx, T ACy, T ACz,
                                             const T* __restrict__ sm) {
  using C = EriClass<LA, LB, LC, LD>;
  constexpr int L = C::L;
  const T PQx = ACx + PAx - QCx, PQy = ACy + PAy - QCy, PQz = ACz + PAz - QCz;
  const T s = p + q;
  const T r = rsqrt_t<T>(s);
  const T inv_s = r * r;
  const T pq_s = p * q * inv_s;
  const T tt = pq_s * (PQx * PQx + PQy * PQy + PQz * PQz);
  T F[L + 1];
  boys_eval<L>(tt, sm, F);
  const T pref = (T)kTwoPiPow25 * kpp * kpq * r;
#pragma unroll
  for (int m = 0; m <= L; ++m) F[m] *= pref;
  const T qs = q * inv_s, ps = p * inv_s;
  C::prim(acc, F, PAx, PAy, PAz, -qs * PQx, -qs * PQy, -qs * PQz, QCx, QCy, QCz, ps * PQx, ps * PQy, ps * PQz,
          (T)0.5 * inv_p, (T)0.5 * inv_q, (T)0.5 * inv_s, qs, ps);
}

template <int LA, int LB, int LC, int LD>
__device__ __forceinline__ void prim_quartet_pp(double* __restrict__ acc, const PrimPair& P, const PrimPair& Q,
                                                double ACx, double ACy, double ACz, const double* __restrict__ sm) {
  prim_quartet<LA, LB, LC, LD, double>(acc, P.p, P.inv_p, P.kp, P.PAx, P.PAy, P.PAz, Q.p, Q.inv_p, Q.kp, Q.PAx,
                                       Q.PAy, Q.PAz, ACx, ACy, ACz, sm);
}

template <typename T> struct RecOf;
template <> struct RecOf<double> {
  using type = PrimRec64;
  __device__ static const PrimRec64* get(const JKLaunchArgs& a) { return a.rec64; }
};
template <> struct RecOf<float> {
  using type = PrimRec32;
  __device__ static const PrimRec32* get(const JKLaunchArgs& a) { return a.rec32; }
};

// Fused digestion of one scaled Cartesian block (w already includes deg and
// the component scales).
// Density blocks needed by the digestion of one quartet (loaded before the
// primitive loop so their latency overlaps the integral work).
template <int LA, int LB, int LC, int LD, int NS>
struct DBlocks {
  static constexpr int NA = ncart(LA), NB = ncart(LB), NC = ncart(LC), ND = ncart(LD);
  double cd[NC * ND], ab[NA * NB];
  double bd[NS][NB * ND], ad[NS][NA * ND], bc[NS][NB * NC], ac[NS][NA * NC];
  __device__ __forceinline__ void load(const PairInfo& bra, const PairInfo& ket, const JKLaunchArgs& a) {
    const int n = a.n;
    const int i0 = bra.ao_a, j0 = bra.ao_b, k0 = ket.ao_a, l0 = ket.ao_b;
#pragma unroll
    for (int k = 0; k < NC; ++k)
#pragma unroll
      for (int l = 0; l < ND; ++l) cd[k * ND + l] = __ldg(a.Dtot + (size_t)(k0 + k) * n + l0 + l);
#pragma unroll
    for (int i = 0; i < NA; ++i)
#pragma unroll
      for (int j = 0; j < NB; ++j) ab[i * NB + j] = __ldg(a.Dtot + (size_t)(i0 + i) * n + j0 + j);
#pragma unroll
    for (int sp = 0; sp < NS; ++sp) {
      const double* D = a.Dspin + (size_t)sp * n * n;
#pragma unroll
      for (int j = 0; j < NB; ++j)
#pragma unroll
        for (int l = 0; l < ND; ++l) bd[sp][j * ND + l] = __ldg(D + (size_t)(j0 + j) * n + l0 + l);
#pragma unroll
      for (int i = 0; i < NA; ++i)
#pragma unroll
        for (int l = 0; l < ND; ++l) ad[sp][i * ND + l] = __ldg(D + (size_t)(i0 + i) * n + l0 + l);
#pragma unroll
      for (int j = 0; j < NB; ++j)
#pragma unroll
        for (int k = 0; k < NC; ++k) bc[sp][j * NC + k] = __ldg(D + (size_t)(j0 + j) * n + k0 + k);
#pragma unroll
      for (int i = 0; i < NA; ++i)
#pragma unroll
        for (int k = 0; k < NC; ++k) ac[sp][i * NC + k] = __ldg(D + (size_t)(i0 + i) * n + k0 + k);
    }
  }
};

// Fused digestion of one scaled Cartesian block (w already includes deg and
// the component scales), except J'[a,b] which the caller reduces across the
// warp (jab receives this lane's sum over c,d).
template <int LA, int LB, int LC, int LD, int NS>
__device__ __forceinline__ void digest(const double* __restrict__ w, const PairInfo& bra, const PairInfo& ket,
                                       const JKLaunchArgs& a, const DBlocks<LA, LB, LC, LD, NS>& d,
                                       double* __restrict__ jab) {
  constexpr int NA = ncart(LA), NB = ncart(LB), NC = ncart(LC), ND = ncart(LD);
  const int n = a.n;
  const int i0 = bra.ao_a, j0 = bra.ao_b, k0 = ket.ao_a, l0 = ket.ao_b;
#pragma unroll
  for (int ij = 0; ij < NA * NB; ++ij) {
    double s = 0.0;
#pragma unroll
    for (int kl = 0; kl < NC * ND; ++kl) s += w[ij * NC * ND + kl] * d.cd[kl];
    jab[ij] = 4.0 * s;
  }
#pragma unroll
  for (int k = 0; k < NC; ++k)
#pragma unroll
    for (int l = 0; l < ND; ++l) {
      double s = 0.0;
#pragma unroll
      for (int ij = 0; ij < NA * NB; ++ij) s += w[ij * NC * ND + k * ND + l] * d.ab[ij];
      atomicAdd(a.Jacc + (size_t)(k0 + k) * n + l0 + l, 4.0 * s);
    }
#pragma unroll
  for (int sp = 0; sp < NS; ++sp) {
    double* K = a.Kacc + (size_t)sp * n * n;
#pragma unroll
    for (int i = 0; i < NA; ++i)
#pragma unroll
      for (int k = 0; k < NC; ++k) {
        double s = 0.0;
#pragma unroll
        for (int j = 0; j < NB; ++j)
#pragma unroll
          for (int l = 0; l < ND; ++l) s += w[((i * NB + j) * NC + k) * ND + l] * d.bd[sp][j * ND + l];
        atomicAdd(K + (size_t)(i0 + i) * n + k0 + k, 2.0 * s);
      }
#pragma unroll
    for (int j = 0; j < NB; ++j)
#pragma unroll
      for (int k = 0; k < NC; ++k) {
        double s = 0.0;
#pragma unroll
        for (int i = 0; i < NA; ++i)
#pragma unroll
          for (int l = 0; l < ND; ++l) s += w[((i * NB + j) * NC + k) * ND + l] * d.ad[sp][i * ND + l];
        atomicAdd(K + (size_t)(j0 + j) * n + k0 + k, 2.0 * s);
      }
#pragma unroll
    for (int i = 0; i < NA; ++i)
#pragma unroll
      for (int l = 0; l < ND; ++l) {
        double s = 0.0;
#pragma unroll
        for (int j = 0; j < NB; ++j)
#pragma unroll
          for (int k = 0; k < NC; ++k) s += w[((i * NB + j) * NC + k) * ND + l] * d.bc[sp][j * NC + k];
        atomicAdd(K + (size_t)(i0 + i) * n + l0 + l, 2.0 * s);
      }
#pragma unroll
    for (int j = 0; j < NB; ++j)
#pragma unroll
      for (int l = 0; l < ND; ++l) {
        double s = 0.0;
#pragma unroll
        for (int i = 0; i < NA; ++i)
#pragma unroll
          for (int k = 0; k < NC; ++k) s += w[((i * NB + j) * NC + k) * ND + l] * d.ac[sp][i * NC + k];
        atomicAdd(K + (size_t)(j0 + j) * n + l0 + l, 2.0 * s);
      }
  }
}

__device__ __forceinline__ int find_entry(const long long* __restrict__ prefix, int n, long long w) {
  int lo = 0, hi = n;  // largest e with prefix[e] <= w
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (__ldg(prefix + mid) <= w) lo = mid; else hi = mid;
  }
  return lo;
}

// Warp tasks are handed out in chunks of kChunk consecutive tasks through
// a per-launch atomic counter; consecutive tasks usually share a work entry,
// so the entry lookup is a binary search once per chunk.
constexpr int kChunk = 8;

// Resident blocks per SM the register allocation is tuned for.
#ifndef HFG_JK_MIN_BLOCKS
#define HFG_JK_MIN_BLOCKS 2
#endif

// G lanes per shell quartet (G = 1: one quartet per lane).  With G > 1 the
// lanes of a group take the quartet's ket primitive pairs round-robin (they
// are sorted by bound, so neighbouring lanes see similar screening), all
// walk the shared bra primitive pairs, and the group reduces its
// accumulators with shuffles before one lane digests the block.
template <int LA, int LB, int LC, int LD, typename T, int NS, int G>
__global__ void __launch_bounds__(256, HFG_JK_MIN_BLOCKS) jk_kernel(const JKLaunchArgs a) {
  constexpr int QPW = 32 / G;
  using C = EriClass<LA, LB, LC, LD>;
  constexpr int NA = ncart(LA), NB = ncart(LB), NC = ncart(LC), ND = ncart(LD), NAB = NA * NB;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* sm = reinterpret_cast<T*>(smem_raw);
  boys_stage<T, C::L>(sm, Prec<T>::table(a), Prec<T>::expt(a));
  __syncthreads();
  const int lane = threadIdx.x & 31;
  for (;;) {
    long long t0 = 0;
    if (lane == 0) t0 = (long long)atomicAdd(a.counter, (unsigned long long)kChunk);
    t0 = __shfl_sync(0xffffffffu, t0, 0);
    if (t0 >= a.nwarps) break;
    const long long t1 = t0 + kChunk < a.nwarps ? t0 + kChunk : a.nwarps;
    int e = find_entry(a.prefix, a.nentries, t0);
    long long next = a.prefix[e + 1];
    for (long long warp = t0; warp < t1; ++warp) {
      while (warp >= next) {
        ++e;
        next = a.prefix[e + 1];
      }
      const JKEntry ent = a.entries[e];
      const int grp = lane / G, gl = lane - grp * G;
      const int kidx = ent.k_lo + (int)(warp - a.prefix[e]) * QPW + grp;
      const bool active = kidx < ent.k_hi;
      const PairInfo bra = a.pairs[ent.bra];
      const PairInfo ket = a.pairs[active ? kidx : ent.k_lo];
      // the next task usually continues this entry: touch its ket pair now
      if (warp + 1 < t1 && kidx + QPW < ent.k_hi) (void)__ldg(&a.pairs[kidx + QPW].pp_off);
      DBlocks<LA, LB, LC, LD, NS> dblk;
      if (active && gl == 0) dblk.load(bra, ket, a);

      T acc[C::NACC];
#pragma unroll
      for (int x = 0; x < C::NACC; ++x) acc[x] = (T)0;

      if (active) {
        using Rec = typename RecOf<T>::type;
        const T ACx = (T)(bra.Ax - ket.Ax), ACy = (T)(bra.Ay - ket.Ay), ACz = (T)(bra.Az - ket.Az);
        const T bABx = (T)bra.ABx, bABy = (T)bra.ABy, bABz = (T)bra.ABz;
        const T kABx = (T)ket.ABx, kABy = (T)ket.ABy, kABz = (T)ket.ABz;
        const Rec* __restrict__ br = RecOf<T>::get(a) + bra.pp_off;
        const Rec* __restrict__ kr = RecOf<T>::get(a) + ket.pp_off;
        const float* __restrict__ bb = a.pbound + bra.pp_off;
        const float* __restrict__ kb = a.pbound + ket.pp_off;
        const int nb = bra.npp, nk = ket.npp;
        const double eps = a.prim_eps;
        const double bmax = bb[0];
        // ket primitive pairs that survive against the largest bra one
        // (bounds sorted descending: binary search)
        int nke = 0;
        {
          int hi = nk;
          while (nke < hi) {
            const int mid = (nke + hi) >> 1;
            if ((double)kb[mid] * bmax >= eps) nke = mid + 1; else hi = mid;
          }
        }
        Rec Qn = kr[gl < nk ? gl : 0];
        for (int ik = gl; ik < nke; ik += G) {
          const Rec Q = Qn;
          if (ik + G < nke) Qn = kr[ik + G];
          const double qb = kb[ik];
          const T QCx = -Q.bp * kABx, QCy = -Q.bp * kABy, QCz = -Q.bp * kABz;
          int ib = 0;
          if constexpr (C::NACC <= 9) {
            // two independent primitive quartets per step (bra primitive pairs
            // are sorted by bound: if the second survives, so does the first)
            for (; ib + 1 < nb; ib += 2) {
              if ((double)bb[ib + 1] * qb < eps) break;
              const Rec P0 = br[ib], P1 = br[ib + 1];
              prim_quartet<LA, LB, LC, LD, T>(acc, P0.p, P0.inv_p, P0.kp, -P0.bp * bABx, -P0.bp * bABy,
                                              -P0.bp * bABz, Q.p, Q.inv_p, Q.kp, QCx, QCy, QCz, ACx, ACy, ACz, sm);
              prim_quartet<LA, LB, LC, LD, T>(acc, P1.p, P1.inv_p, P1.kp, -P1.bp * bABx, -P1.bp * bABy,
                                              -P1.bp * bABz, Q.p, Q.inv_p, Q.kp, QCx, QCy, QCz, ACx, ACy, ACz, sm);
            }
          }
          Rec P = br[ib < nb ? ib : 0];
          for (; ib < nb; ++ib) {
            const Rec Pn = br[ib + 1 < nb ? ib + 1 : ib];
            if ((double)bb[ib] * qb < eps) break;
            prim_quartet<LA, LB, LC, LD, T>(acc, P.p, P.inv_p, P.kp, -P.bp * bABx, -P.bp * bABy, -P.bp * bABz, Q.p,
                                            Q.inv_p, Q.kp, QCx, QCy, QCz, ACx, ACy, ACz, sm);
            P = Pn;
          }
        }
      }
      if (G > 1) {
#pragma unroll
        for (int x = 0; x < C::NACC; ++x) {
#pragma unroll
          for (int off = G / 2; off > 0; off >>= 1) acc[x] += __shfl_xor_sync(0xffffffffu, acc[x], off);
        }
      }
      double jab[NAB];
      if (active && gl == 0) {
        T out[C::NOUT];
        C::hrr(acc, out, (T)bra.ABx, (T)bra.ABy, (T)bra.ABz, (T)ket.ABx, (T)ket.ABy, (T)ket.ABz);
        double deg = 1.0;
        if (bra.same) deg *= 0.5;
        if (ket.same) deg *= 0.5;
        if (kidx == ent.bra) deg *= 0.5;
        double w[C::NOUT];
#pragma unroll
        for (int i = 0; i < NA; ++i)
#pragma unroll
          for (int j = 0; j < NB; ++j)
#pragma unroll
            for (int k = 0; k < NC; ++k)
#pragma unroll
              for (int l = 0; l < ND; ++l) {
                const int x = ((i * NB + j) * NC + k) * ND + l;
                w[x] = (double)out[x] *
                       (deg * comp_scale(LA, i) * comp_scale(LB, j) * comp_scale(LC, k) * comp_scale(LD, l));
              }
        digest<LA, LB, LC, LD, NS>(w, bra, ket, a, dblk, jab);
      } else {
#pragma unroll
        for (int x = 0; x < NAB; ++x) jab[x] = 0.0;
      }
      // J'[a,b]: the whole warp shares the bra pair
#pragma unroll
      for (int x = 0; x < NAB; ++x) {
        double v = jab[x];
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
        if (lane == 0) atomicAdd(a.Jacc + (size_t)(bra.ao_a + x / NB) * a.n + bra.ao_b + x % NB, v);
      }
    }
  }
}

// ---------------------------------------------------------------------------
// Schwarz bounds.  One thread per shell pair (contracted, all primitives) or
// per primitive pair (prim_mode): max over the diagonal (ij|ij) of the scaled
// block, square-rooted.
template <int LA, int LB>
__global__ void schwarz_kernel(const PairInfo* __restrict__ pairs, const PrimPair* __restrict__ prims, int first,
                               int count, const double* __restrict__ boys, const double* __restrict__ expt,
                               double* __restrict__ out, int prim_mode) {
  using C = EriClass<LA, LB, LA, LB>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  double* sm = reinterpret_cast<double*>(smem_raw);
  boys_stage<double, C::L>(sm, boys, expt);
  __syncthreads();
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= count) return;
  // pair mode: t indexes shell pairs first + t; prim_mode: t indexes
  // primitive pairs first + t, whose owning shell pair index is stored in
  // PrimPair::pad.
  const int p0 = prim_mode ? first + t : pairs[first + t].pp_off;
  const int np = prim_mode ? 1 : pairs[first + t].npp;
  const PairInfo owner = prim_mode ? pairs[(int)prims[p0].pad] : pairs[first + t];
  double acc[C::NACC];
#pragma unroll
  for (int x = 0; x < C::NACC; ++x) acc[x] = 0.0;
  for (int ib = 0; ib < np; ++ib)
    for (int ik = 0; ik < np; ++ik)
      prim_quartet_pp<LA, LB, LA, LB>(acc, prims[p0 + ib], prims[p0 + ik], 0.0, 0.0, 0.0, sm);
  double blk[C::NOUT];
  C::hrr(acc, blk, owner.ABx, owner.ABy, owner.ABz, owner.ABx, owner.ABy, owner.ABz);
  constexpr int NA = ncart(LA), NB = ncart(LB), NAB = NA * NB;
  double m = 0.0;
#pragma unroll
  for (int i = 0; i < NA; ++i)
#pragma unroll
    for (int j = 0; j < NB; ++j) {
      const double s = comp_scale(LA, i) * comp_scale(LB, j);
      const int ij = i * NB + j;
      m = fmax(m, blk[ij * NAB + ij] * s * s);
    }
  out[t] = sqrt(m);
}

// One full Cartesian block (ab|cd) for the single-quartet entry point.
template <int LA, int LB, int LC, int LD>
__global__ void quartet_kernel(const PairInfo* __restrict__ pairs, const PrimPair* __restrict__ prims,
                               const double* __restrict__ boys, const double* __restrict__ expt,
                               double* __restrict__ out) {
  using C = EriClass<LA, LB, LC, LD>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  double* sm = reinterpret_cast<double*>(smem_raw);
  boys_stage<double, C::L>(sm, boys, expt);
  __syncthreads();
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  const PairInfo bra = pairs[0], ket = pairs[1];
  double acc[C::NACC];
  for (int x = 0; x < C::NACC; ++x) acc[x] = 0.0;
  for (int ib = 0; ib < bra.npp; ++ib)
    for (int ik = 0; ik < ket.npp; ++ik)
      prim_quartet_pp<LA, LB, LC, LD>(acc, prims[bra.pp_off + ib], prims[ket.pp_off + ik], bra.Ax - ket.Ax,
                                      bra.Ay - ket.Ay, bra.Az - ket.Az, sm);
  double blk[C::NOUT];
  C::hrr(acc, blk, bra.ABx, bra.ABy, bra.ABz, ket.ABx, ket.ABy, ket.ABz);
  constexpr int NA = ncart(LA), NB = ncart(LB), NC = ncart(LC), ND = ncart(LD);
  for (int i = 0; i < NA; ++i)
    for (int j = 0; j < NB; ++j)
      for (int k = 0; k < NC; ++k)
        for (int l = 0; l < ND; ++l) {
          const int x = ((i * NB + j) * NC + k) * ND + l;
          out[x] = blk[x] * comp_scale(LA, i) * comp_scale(LB, j) * comp_scale(LC, k) * comp_scale(LD, l);
        }
}

}  // namespace hfg
