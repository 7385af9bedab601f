// Packed 8-fold ERI tensor on the device: the counterpart of hf-rs's
// compute_eri_tensor (src/scf.rs:275-333 -> compute_shell_eri_tensor,
// src/shell_integrals.rs:156-240) for small systems and for consumers that
// want stored integrals (post-HF transforms).
//
// Layout (src/scf.rs:222-235): slot eri_index(mu,nu,lam,sig) =
// c(c(mu,nu), c(lam,sig)) with c(i,j) = max(i,j)(max(i,j)+1)/2 + min(i,j),
// holding the Cartesian (mu nu|lam sig) with the per-component scale of
// src/basis.rs:123-132.  Shell quartets with Q_ab Q_cd <= threshold stay
// zero, as in the reference.  The quartets are those of the FP64 J/K plan
// (every unique Schwarz-significant shell quartet once), one per thread, all
// primitive quartets evaluated (no primitive screening).  Every slot has one
// writer: within a same-shell pair only the i >= j components are written,
// and a quartet of a pair with itself writes only IJ >= KL.
#include "jk_dispatch.h"
#include "eri_prim.cuh"

namespace hfg {

__device__ __forceinline__ unsigned long long compound(unsigned long long i, unsigned long long j) {
  return i >= j ? i * (i + 1) / 2 + j : j * (j + 1) / 2 + i;
}

template <int LA, int LB, int LC, int LD>
__global__ void __launch_bounds__(128) eri_packed_kernel(const JKEntry* __restrict__ entries,
                                                         const long long* __restrict__ prefix, int nentries,
                                                         long long nwarps, const PairInfo* __restrict__ pairs,
                                                         const double* __restrict__ pairQ, double thr,
                                                         const PrimRec64* __restrict__ rec,
                                                         const double* __restrict__ boys,
                                                         const double* __restrict__ expt, double* __restrict__ out) {
  using C = EriClass<LA, LB, LC, LD>;
  constexpr int NA = ncart(LA), NB = ncart(LB), NC = ncart(LC), ND = ncart(LD);
  extern __shared__ __align__(16) unsigned char smem_raw[];
  double* sm = reinterpret_cast<double*>(smem_raw);
  boys_stage<double, C::L>(sm, boys, expt);
  __syncthreads();
  const long long warp = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (warp >= nwarps) return;
  const int lane = threadIdx.x & 31;
  const int e = find_entry(prefix, nentries, warp);
  const JKEntry ent = entries[e];
  const int kidx = ent.k_lo + (int)(warp - prefix[e]) * 32 + lane;
  if (kidx >= ent.k_hi || !(pairQ[kidx] * pairQ[ent.bra] > thr)) return;
  const PairInfo bra = pairs[ent.bra], ket = pairs[kidx];
  const double ACx = bra.Ax - ket.Ax, ACy = bra.Ay - ket.Ay, ACz = bra.Az - ket.Az;
  double acc[C::NACC];
#pragma unroll
  for (int x = 0; x < C::NACC; ++x) acc[x] = 0.0;
  for (int ik = 0; ik < ket.npp; ++ik) {
    const PrimRec64 Q = rec[ket.rec_off + (size_t)ik * ket.rec_stride];
    for (int ib = 0; ib < bra.npp; ++ib) {
      const PrimRec64 P = rec[bra.rec_off + (size_t)ib * bra.rec_stride];
      prim_quartet<LA, LB, LC, LD, double>(acc, P.p, P.inv_p, P.kp, -P.bp * bra.ABx, -P.bp * bra.ABy,
                                           -P.bp * bra.ABz, Q.p, Q.inv_p, Q.kp, -Q.bp * ket.ABx, -Q.bp * ket.ABy,
                                           -Q.bp * ket.ABz, ACx, ACy, ACz, sm);
    }
  }
  double blk[C::NOUT];
  C::hrr(acc, blk, bra.ABx, bra.ABy, bra.ABz, ket.ABx, ket.ABy, ket.ABz);
  const bool self = kidx == ent.bra;
#pragma unroll
  for (int i = 0; i < NA; ++i)
#pragma unroll
    for (int j = 0; j < NB; ++j) {
      const int mu = bra.ao_a + i, nu = bra.ao_b + j;
      if (bra.same && mu < nu) continue;
      const unsigned long long IJ = compound(mu, nu);
#pragma unroll
      for (int k = 0; k < NC; ++k)
#pragma unroll
        for (int l = 0; l < ND; ++l) {
          const int lam = ket.ao_a + k, sig = ket.ao_b + l;
          if (ket.same && lam < sig) continue;
          const unsigned long long KL = compound(lam, sig);
          if (self && IJ < KL) continue;
          const int x = ((i * NB + j) * NC + k) * ND + l;
          out[compound(IJ, KL)] =
              blk[x] * (comp_scale(LA, i) * comp_scale(LB, j) * comp_scale(LC, k) * comp_scale(LD, l));
        }
    }
}

cudaError_t launch_eri_packed(int la, int lb, int lc, int ld, const JKEntry* entries, const long long* prefix,
                              int nentries, long long nwarps, const PairInfo* pairs, const double* pairQ,
                              double thr, const PrimRec64* rec,
                              const double* boys, const double* expt, double* out, cudaStream_t st) {
  if (nwarps <= 0) return cudaSuccess;
  const int smem = (int)boys_smem_bytes<double>();
  const int block = 128;
  const long long grid = (nwarps * 32 + block - 1) / block;
#define HFG_CASE(A, B, C, D)                                                                                  \
  if (la == A && lb == B && lc == C && ld == D) {                                                             \
    cudaFuncSetAttribute(eri_packed_kernel<A, B, C, D>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);   \
    eri_packed_kernel<A, B, C, D><<<(unsigned)grid, block, smem, st>>>(entries, prefix, nentries, nwarps, pairs, \
                                                                      pairQ, thr, rec, boys, expt, out);      \
    return cudaGetLastError();                                                                                \
  }
  HFG_CASE(0, 0, 0, 0)
  HFG_CASE(1, 0, 0, 0)
  HFG_CASE(1, 0, 1, 0)
  HFG_CASE(1, 1, 0, 0)
  HFG_CASE(1, 1, 1, 0)
  HFG_CASE(1, 1, 1, 1)
  HFG_CASE(2, 0, 0, 0)
  HFG_CASE(2, 0, 1, 0)
  HFG_CASE(2, 0, 1, 1)
  HFG_CASE(2, 0, 2, 0)
  HFG_CASE(2, 1, 0, 0)
  HFG_CASE(2, 1, 1, 0)
  HFG_CASE(2, 1, 1, 1)
  HFG_CASE(2, 1, 2, 0)
  HFG_CASE(2, 1, 2, 1)
  HFG_CASE(2, 2, 0, 0)
  HFG_CASE(2, 2, 1, 0)
  HFG_CASE(2, 2, 1, 1)
  HFG_CASE(2, 2, 2, 0)
  HFG_CASE(2, 2, 2, 1)
  HFG_CASE(2, 2, 2, 2)
#undef HFG_CASE
  return cudaErrorInvalidValue;
}

}  // namespace hfg
