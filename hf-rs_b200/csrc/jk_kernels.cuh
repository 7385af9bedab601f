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
// Work split: a warp takes one bra shell pair and up to 32/G ket pairs of
// one pair class; a group of G lanes evaluates one shell quartet, its lanes
// striding over the primitive quartets, then reduces its accumulators with
// warp shuffles.  G is chosen per launch from the contraction lengths so that
// heavily contracted quartets (cc-pVDZ oxygen 1s/2s: 81 primitive pairs)
// spread over a whole warp while uncontracted ones take one lane each.
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
};
template <> struct Prec<float> {
  __device__ static const float* table(const JKLaunchArgs& a) { return a.boys32; }
};

// One primitive quartet added into acc.  AC = A - C of the two pairs.
template <int LA, int LB, int LC, int LD, typename T>
__device__ __forceinline__ void prim_quartet(T* __restrict__ acc, const PrimPair& P, const PrimPair& Q, T ACx, T ACy,
                                             T ACz, const T* __restrict__ table) {
  using C = EriClass<LA, LB, LC, LD>;
  constexpr int L = C::L;
  const T p = (T)P.p, q = (T)Q.p;
  const T PAx = (T)P.PAx, PAy = (T)P.PAy, PAz = (T)P.PAz;
  const T QCx = (T)Q.PAx, QCy = (T)Q.PAy, QCz = (T)Q.PAz;
  const T PQx = ACx + PAx - QCx, PQy = ACy + PAy - QCy, PQz = ACz + PAz - QCz;
  const T s = p + q;
  T r;
  if constexpr (sizeof(T) == 8) r = rsqrt(s); else r = rsqrtf(s);
  const T inv_s = r * r;
  const T pq_s = p * q * inv_s;
  const T tt = pq_s * (PQx * PQx + PQy * PQy + PQz * PQz);
  T F[L + 1];
  boys_eval<L>(tt, table, F);
  const T pref = (T)kTwoPiPow25 * (T)P.kp * (T)Q.kp * r;
#pragma unroll
  for (int m = 0; m <= L; ++m) F[m] *= pref;
  const T qs = q * inv_s, ps = p * inv_s;
  C::prim(acc, F, PAx, PAy, PAz, -qs * PQx, -qs * PQy, -qs * PQz, QCx, QCy, QCz, ps * PQx, ps * PQy, ps * PQz,
          (T)0.5 * (T)P.inv_p, (T)0.5 * (T)Q.inv_p, (T)0.5 * inv_s, qs, ps);
}

// Fused digestion of one scaled Cartesian block (w already includes deg and
// the component scales).
template <int LA, int LB, int LC, int LD>
__device__ __forceinline__ void digest(const double* __restrict__ w, const PairInfo& bra, const PairInfo& ket,
                                       const JKLaunchArgs& a) {
  constexpr int NA = ncart(LA), NB = ncart(LB), NC = ncart(LC), ND = ncart(LD);
  const int n = a.n;
  const int i0 = bra.ao_a, j0 = bra.ao_b, k0 = ket.ao_a, l0 = ket.ao_b;
  {
    double dcd[NC * ND], dab[NA * NB];
#pragma unroll
    for (int k = 0; k < NC; ++k)
#pragma unroll
      for (int l = 0; l < ND; ++l) dcd[k * ND + l] = __ldg(a.Dtot + (size_t)(k0 + k) * n + l0 + l);
#pragma unroll
    for (int i = 0; i < NA; ++i)
#pragma unroll
      for (int j = 0; j < NB; ++j) dab[i * NB + j] = __ldg(a.Dtot + (size_t)(i0 + i) * n + j0 + j);
#pragma unroll
    for (int i = 0; i < NA; ++i)
#pragma unroll
      for (int j = 0; j < NB; ++j) {
        double s = 0.0;
#pragma unroll
        for (int kl = 0; kl < NC * ND; ++kl) s += w[(i * NB + j) * NC * ND + kl] * dcd[kl];
        atomicAdd(a.Jacc + (size_t)(i0 + i) * n + j0 + j, 4.0 * s);
      }
#pragma unroll
    for (int k = 0; k < NC; ++k)
#pragma unroll
      for (int l = 0; l < ND; ++l) {
        double s = 0.0;
#pragma unroll
        for (int ij = 0; ij < NA * NB; ++ij) s += w[ij * NC * ND + k * ND + l] * dab[ij];
        atomicAdd(a.Jacc + (size_t)(k0 + k) * n + l0 + l, 4.0 * s);
      }
  }
  for (int sp = 0; sp < a.nspin; ++sp) {
    const double* D = a.Dspin + (size_t)sp * n * n;
    double* K = a.Kacc + (size_t)sp * n * n;
    double dbd[NB * ND], dad[NA * ND], dbc[NB * NC], dac[NA * NC];
#pragma unroll
    for (int j = 0; j < NB; ++j)
#pragma unroll
      for (int l = 0; l < ND; ++l) dbd[j * ND + l] = __ldg(D + (size_t)(j0 + j) * n + l0 + l);
#pragma unroll
    for (int i = 0; i < NA; ++i)
#pragma unroll
      for (int l = 0; l < ND; ++l) dad[i * ND + l] = __ldg(D + (size_t)(i0 + i) * n + l0 + l);
#pragma unroll
    for (int j = 0; j < NB; ++j)
#pragma unroll
      for (int k = 0; k < NC; ++k) dbc[j * NC + k] = __ldg(D + (size_t)(j0 + j) * n + k0 + k);
#pragma unroll
    for (int i = 0; i < NA; ++i)
#pragma unroll
      for (int k = 0; k < NC; ++k) dac[i * NC + k] = __ldg(D + (size_t)(i0 + i) * n + k0 + k);
    // K'[a,c] += 2 Σ_{b,d} w D[b,d]
#pragma unroll
    for (int i = 0; i < NA; ++i)
#pragma unroll
      for (int k = 0; k < NC; ++k) {
        double s = 0.0;
#pragma unroll
        for (int j = 0; j < NB; ++j)
#pragma unroll
          for (int l = 0; l < ND; ++l) s += w[((i * NB + j) * NC + k) * ND + l] * dbd[j * ND + l];
        atomicAdd(K + (size_t)(i0 + i) * n + k0 + k, 2.0 * s);
      }
    // K'[b,c] += 2 Σ_{a,d} w D[a,d]
#pragma unroll
    for (int j = 0; j < NB; ++j)
#pragma unroll
      for (int k = 0; k < NC; ++k) {
        double s = 0.0;
#pragma unroll
        for (int i = 0; i < NA; ++i)
#pragma unroll
          for (int l = 0; l < ND; ++l) s += w[((i * NB + j) * NC + k) * ND + l] * dad[i * ND + l];
        atomicAdd(K + (size_t)(j0 + j) * n + k0 + k, 2.0 * s);
      }
    // K'[a,d] += 2 Σ_{b,c} w D[b,c]
#pragma unroll
    for (int i = 0; i < NA; ++i)
#pragma unroll
      for (int l = 0; l < ND; ++l) {
        double s = 0.0;
#pragma unroll
        for (int j = 0; j < NB; ++j)
#pragma unroll
          for (int k = 0; k < NC; ++k) s += w[((i * NB + j) * NC + k) * ND + l] * dbc[j * NC + k];
        atomicAdd(K + (size_t)(i0 + i) * n + l0 + l, 2.0 * s);
      }
    // K'[b,d] += 2 Σ_{a,c} w D[a,c]
#pragma unroll
    for (int j = 0; j < NB; ++j)
#pragma unroll
      for (int l = 0; l < ND; ++l) {
        double s = 0.0;
#pragma unroll
        for (int i = 0; i < NA; ++i)
#pragma unroll
          for (int k = 0; k < NC; ++k) s += w[((i * NB + j) * NC + k) * ND + l] * dac[i * NC + k];
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

template <int LA, int LB, int LC, int LD, int G, typename T>
__global__ void __launch_bounds__(128) jk_kernel(const JKLaunchArgs a) {
  using C = EriClass<LA, LB, LC, LD>;
  constexpr int QPW = 32 / G;  // quartets per warp
  const long long warp = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (warp >= a.nwarps) return;
  const int lane = threadIdx.x & 31;
  const int e = find_entry(a.prefix, a.nentries, warp);
  const JKEntry ent = a.entries[e];
  const long long chunk = warp - a.prefix[e];
  const int grp = lane / G, gl = lane % G;
  const int kidx = ent.k_lo + (int)chunk * QPW + grp;
  const bool active = kidx < ent.k_hi;
  const PairInfo bra = a.pairs[ent.bra];
  const PairInfo ket = a.pairs[active ? kidx : ent.k_lo];

  T acc[C::NACC];
#pragma unroll
  for (int x = 0; x < C::NACC; ++x) acc[x] = (T)0;

  if (active) {
    const T ACx = (T)(bra.Ax - ket.Ax), ACy = (T)(bra.Ay - ket.Ay), ACz = (T)(bra.Az - ket.Az);
    const PrimPair* __restrict__ bp = a.prims + bra.pp_off;
    const PrimPair* __restrict__ kp = a.prims + ket.pp_off;
    const int nb = bra.npp, nk = ket.npp;
    const double eps = a.prim_eps;
    if (G == 1) {
      for (int ib = 0; ib < nb; ++ib) {
        const PrimPair P = bp[ib];
        if (P.bound * kp[0].bound < eps) break;
        for (int ik = 0; ik < nk; ++ik) {
          const PrimPair Q = kp[ik];
          if (P.bound * Q.bound < eps) break;
          prim_quartet<LA, LB, LC, LD, T>(acc, P, Q, ACx, ACy, ACz, Prec<T>::table(a));
        }
      }
    } else {
      const int total = nb * nk;
      int ib = gl / nk, ik = gl - (gl / nk) * nk;
      for (int t = gl; t < total; t += G) {
        const PrimPair P = bp[ib];
        const PrimPair Q = kp[ik];
        if (P.bound * Q.bound >= eps) prim_quartet<LA, LB, LC, LD, T>(acc, P, Q, ACx, ACy, ACz, Prec<T>::table(a));
        ik += G;
        while (ik >= nk) {
          ik -= nk;
          ++ib;
        }
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
  if (!active || gl != 0) return;

  T out[C::NOUT];
  C::hrr(acc, out, (T)bra.ABx, (T)bra.ABy, (T)bra.ABz, (T)ket.ABx, (T)ket.ABy, (T)ket.ABz);
  double deg = 1.0;
  if (bra.same) deg *= 0.5;
  if (ket.same) deg *= 0.5;
  if (kidx == ent.bra) deg *= 0.5;
  constexpr int NA = ncart(LA), NB = ncart(LB), NC = ncart(LC), ND = ncart(LD);
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
          w[x] = (double)out[x] * (deg * comp_scale(LA, i) * comp_scale(LB, j) * comp_scale(LC, k) * comp_scale(LD, l));
        }
  digest<LA, LB, LC, LD>(w, bra, ket, a);
}

// ---------------------------------------------------------------------------
// Schwarz bounds.  One thread per shell pair (contracted, all primitives) or
// per primitive pair (prim_mode): max over the diagonal (ij|ij) of the scaled
// block, square-rooted.
template <int LA, int LB>
__global__ void schwarz_kernel(const PairInfo* __restrict__ pairs, const PrimPair* __restrict__ prims, int first,
                               int count, const double* __restrict__ boys, double* __restrict__ out, int prim_mode) {
  using C = EriClass<LA, LB, LA, LB>;
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
      prim_quartet<LA, LB, LA, LB, double>(acc, prims[p0 + ib], prims[p0 + ik], 0.0, 0.0, 0.0, boys);
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
                               const double* __restrict__ boys, double* __restrict__ out) {
  using C = EriClass<LA, LB, LC, LD>;
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  const PairInfo bra = pairs[0], ket = pairs[1];
  double acc[C::NACC];
  for (int x = 0; x < C::NACC; ++x) acc[x] = 0.0;
  for (int ib = 0; ib < bra.npp; ++ib)
    for (int ik = 0; ik < ket.npp; ++ik)
      prim_quartet<LA, LB, LC, LD, double>(acc, prims[bra.pp_off + ib], prims[ket.pp_off + ik], bra.Ax - ket.Ax,
                                           bra.Ay - ket.Ay, bra.Az - ket.Az, boys);
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
