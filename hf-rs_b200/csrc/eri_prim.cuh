// Primitive-quartet code shared by every ERI kernel: the Obara-Saika
// driver of one primitive quartet (scaled Boys values, then the generated
// vertical recursion of eri_gen.cuh), the per-component scales, the compact
// primitive-pair records, the work-entry lookup, and the Schwarz-bound and
// single-quartet kernels.
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
// P - A) and ket primitive pair (q, 1/q, ckq = 2 pi^{5/2} kq, Q - C), with
// ACQ = (A - C) - (Q - C), so that P - Q = (P - A) + ACQ.  The ket-side
// terms are formed once per ket primitive pair by the callers' outer loops.
template <int LA, int LB, int LC, int LD, typename T>
__device__ __forceinline__ void prim_quartet_k(T* __restrict__ acc, T p, T inv_p, T kpp, T PAx, T PAy, T PAz, T q,
                                               T inv_q, T ckq, T QCx, T QCy, T QCz, T ACQx, T ACQy, T ACQz,
                                               const T* __restrict__ sm) {
  using C = EriClass<LA, LB, LC, LD>;
  constexpr int L = C::L;
  const T PQx = PAx + ACQx, PQy = PAy + ACQy, PQz = PAz + ACQz;
  const T s = p + q;
  const T r = rsqrt_t<T>(s);
  const T inv_s = r * r;
  const T pq_s = p * q * inv_s;
  const T tt = pq_s * (PQx * PQx + PQy * PQy + PQz * PQz);
  T F[L + 1];
  boys_eval<L>(tt, sm, F);
  const T pref = kpp * ckq * r;
#pragma unroll
  for (int m = 0; m <= L; ++m) F[m] *= pref;
  const T qs = q * inv_s, ps = p * inv_s;
  C::prim(acc, F, PAx, PAy, PAz, -qs * PQx, -qs * PQy, -qs * PQz, QCx, QCy, QCz, ps * PQx, ps * PQy, ps * PQz,
          (T)0.5 * inv_p, (T)0.5 * inv_q, (T)0.5 * inv_s, qs, ps);
}

// The same from A - C and the ket's kq, for callers without an outer ket loop.
template <int LA, int LB, int LC, int LD, typename T>
__device__ __forceinline__ void prim_quartet(T* __restrict__ acc, T p, T inv_p, T kpp, T PAx, T PAy, T PAz, T q,
                                             T inv_q, T kpq, T QCx, T QCy, T QCz, T ACx, T ACy, T ACz,
                                             const T* __restrict__ sm) {
  prim_quartet_k<LA, LB, LC, LD, T>(acc, p, inv_p, kpp, PAx, PAy, PAz, q, inv_q, (T)kTwoPiPow25 * kpq, QCx, QCy, QCz,
                                    ACx - QCx, ACy - QCy, ACz - QCz, sm);
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

__device__ __forceinline__ int find_entry(const long long* __restrict__ prefix, int n, long long w) {
  int lo = 0, hi = n;  // largest e with prefix[e] <= w
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (__ldg(prefix + mid) <= w) lo = mid; else hi = mid;
  }
  return lo;
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
