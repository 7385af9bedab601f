// Shell quartets with an f shell (l = 3): a generic McMurchie-Davidson
// engine, one thread block per shell quartet.
//
// The generated Obara-Saika kernels (eri_gen.cuh) cover s, p and d; their
// straight-line recursions grow too large to compile beyond that.  Classes
// with an f shell take this path instead, for every entry point: Schwarz
// bounds, the single-quartet block, the packed tensor and the direct J/K
// build (same work queues as the fast kernels, FP64 only).  It restates the
// scheme of hf-rs's shell engine (src/shell_integrals.rs:92-135 with
// src/integrals.rs:107-191 and :253-346):
//
//   (ab|cd) = 2 pi^{5/2} / (p q sqrt(p+q)) sum_{tuv} E^{ab}_{tuv}
//             sum_{tau nu phi} (-1)^{tau+nu+phi} E^{cd}_{tau nu phi}
//             R_{t+tau, u+nu, v+phi}(alpha, P - Q),  alpha = pq/(p+q),
//
// with Hermite coefficients E per axis from
//   E^{i+1,j}_t = E^{ij}_{t-1}/(2p) + X_PA E^{ij}_t + (t+1) E^{ij}_{t+1}
//   E^{i,j+1}_t = E^{ij}_{t-1}/(2p) + X_PB E^{ij}_t + (t+1) E^{ij}_{t+1}
// (E^{00}_0 = 1; the Gaussian product factor sits in the pair's K_p), and
//   R^{n}_{t+1,u,v} = t R^{n+1}_{t-1,u,v} + X_PQ R^{n+1}_{t,u,v},
//   R^{n}_{000} = (-2 alpha)^n F_n(alpha |PQ|^2).
// Per primitive quartet the block builds the R table level by level, then
// G[ab][tau nu phi] = sum_{tuv} E^{ab}_{tuv} R_{t+tau,u+nu,v+phi} and finally
// adds sum_{tau nu phi} (-1)^{...} E^{cd} G into the contracted block, all in
// shared memory (about 190 KB for (ff|ff)).
#include <cuda_runtime.h>

#include "eri_md.h"
#include "jk_dispatch.h"
#include "eri_prim.cuh"

namespace hfg {

namespace {

constexpr int kMDThreads = 256;
constexpr int kMDR = kMDLMax * 4 + 1;     // R cube edge: t, u, v <= 12
constexpr int kMDRCube = kMDR * kMDR * kMDR;
constexpr int kMDE = 2 * kMDLMax + 1;     // Hermite index range of one pair per axis
constexpr int kMDHCube = kMDE * kMDE * kMDE;
constexpr int kMDEAxis = (kMDLMax + 1) * (kMDLMax + 1) * kMDE;  // E[i][j][t] of one axis

__device__ __forceinline__ int ridx(int t, int u, int v) { return (t * kMDR + u) * kMDR + v; }
__device__ __forceinline__ int eidx(int ax, int i, int j, int t) {
  return ((ax * (kMDLMax + 1) + i) * (kMDLMax + 1) + j) * kMDE + t;
}

// Cartesian component c of angular momentum l in hf-rs order
// (src/basis.rs:418-445: d is xx, yy, zz, xy, xz, yz; the others are
// lexicographic with x descending, then y).
__device__ __forceinline__ void md_component(int l, int c, int* e) {
  if (l == 2) {
    const int d[6][3] = {{2, 0, 0}, {0, 2, 0}, {0, 0, 2}, {1, 1, 0}, {1, 0, 1}, {0, 1, 1}};
    e[0] = d[c][0];
    e[1] = d[c][1];
    e[2] = d[c][2];
    return;
  }
  int k = 0;
  for (int lx = l; lx >= 0; --lx)
    for (int ly = l - lx; ly >= 0; --ly) {
      if (k == c) {
        e[0] = lx;
        e[1] = ly;
        e[2] = l - lx - ly;
        return;
      }
      ++k;
    }
}

// 1/sqrt(prod (2 l_i - 1)!!): the per-component scale of src/basis.rs:123-132
__device__ __forceinline__ double md_comp_scale(const int* e) {
  double d = 1.0;
  for (int k = 0; k < 3; ++k)
    for (int m = 2 * e[k] - 1; m > 1; m -= 2) d *= m;
  return rsqrt(d);
}

// F_0..F_L at T for a run-time L <= 16: the device's Boys scheme (boys.cuh)
// read from the global grid table (kBoysCols columns per row).
__device__ void md_boys(double t, int L, const double* __restrict__ table, const double* __restrict__ expt,
                        double* F) {
  if (t > kBoysTMax) {
    const double r = rsqrt(t);
    F[0] = kHalfSqrtPi * r;
    const double inv2t = 0.5 * r * r, e = exp(-t);
    for (int m = 1; m <= L; ++m) F[m] = ((2 * m - 1) * F[m - 1] - e) * inv2t;
    return;
  }
  const int idx = min(max(__double2int_rn(t * 20.0), 0), kBoysSmemRows - 1);
  const double x = idx * kBoysStep - t;
  const double* row = table + (size_t)idx * kBoysCols + L;
  double acc = row[7] * (1.0 / 5040.0);
  acc = fma(acc, x, row[6] * (1.0 / 720.0));
  acc = fma(acc, x, row[5] * (1.0 / 120.0));
  acc = fma(acc, x, row[4] * (1.0 / 24.0));
  acc = fma(acc, x, row[3] * (1.0 / 6.0));
  acc = fma(acc, x, row[2] * 0.5);
  acc = fma(acc, x, row[1]);
  F[L] = fma(acc, x, row[0]);
  double ex = fma(x, 1.0 / 5040.0, 1.0 / 720.0);
  ex = fma(ex, x, 1.0 / 120.0);
  ex = fma(ex, x, 1.0 / 24.0);
  ex = fma(ex, x, 1.0 / 6.0);
  ex = fma(ex, x, 0.5);
  ex = fma(ex, x, 1.0);
  ex = fma(ex, x, 1.0);
  const double e = expt[idx] * ex, t2 = 2.0 * t;
  for (int m = L - 1; m >= 0; --m) F[m] = (t2 * F[m + 1] + e) / (2 * m + 1);
}

// Shared-memory layout of one block (offsets in doubles, then ints).
struct MDLayout {
  int nab, ncd, nherm;
  int out, G, R0, R1, Eb, Ek, F, S, dbl_end;
  __host__ __device__ MDLayout(const MDClass& c) {
    nab = c.na * c.nb;
    ncd = c.nc * c.nd;
    nherm = (c.lcd + 1) * (c.lcd + 2) * (c.lcd + 3) / 6;
    out = 0;
    G = out + nab * ncd;
    R0 = G + nab * nherm;
    R1 = R0 + kMDRCube;
    Eb = R1 + kMDRCube;
    Ek = Eb + 3 * kMDEAxis;
    F = Ek + 3 * kMDEAxis;
    S = F + 4 * kMDLMax + 8;
    dbl_end = S + 16;
  }
  // ints: Hermite index cube, Hermite list, components of the four shells
  __host__ __device__ size_t bytes() const {
    return (size_t)dbl_end * 8 + (size_t)(kMDHCube + 3 * kMDHCube + 4 * 10 * 3) * 4;
  }
};

struct MDShared {
  double *out, *G, *R0, *R1, *Eb, *Ek, *F, *S;
  int *hidx, *hlist, *comp;  // comp[(shell * 10 + c) * 3 + axis]
};

__device__ MDShared md_shared(const MDLayout& L, unsigned char* raw) {
  MDShared s;
  double* d = reinterpret_cast<double*>(raw);
  s.out = d + L.out;
  s.G = d + L.G;
  s.R0 = d + L.R0;
  s.R1 = d + L.R1;
  s.Eb = d + L.Eb;
  s.Ek = d + L.Ek;
  s.F = d + L.F;
  s.S = d + L.S;
  int* ip = reinterpret_cast<int*>(d + L.dbl_end);
  s.hidx = ip;
  s.hlist = ip + kMDHCube;
  s.comp = ip + 4 * kMDHCube;
  return s;
}

// Component and Hermite tables of the class (once per block).
__device__ void md_setup(const MDClass& c, const MDLayout& L, const MDShared& s) {
  const int ls[4] = {c.la, c.lb, c.lc, c.ld};
  for (int x = threadIdx.x; x < 4 * 10; x += blockDim.x) {
    const int sh = x / 10, k = x % 10;
    if (k < ncart(ls[sh])) md_component(ls[sh], k, s.comp + x * 3);
  }
  if (threadIdx.x == 0) {
    int h = 0;
    for (int t = 0; t < kMDE; ++t)
      for (int u = 0; u < kMDE; ++u)
        for (int v = 0; v < kMDE; ++v) {
          const int cell = (t * kMDE + u) * kMDE + v;
          if (t + u + v <= c.lcd) {
            s.hidx[cell] = h;
            s.hlist[3 * h] = t;
            s.hlist[3 * h + 1] = u;
            s.hlist[3 * h + 2] = v;
            ++h;
          } else {
            s.hidx[cell] = -1;
          }
        }
  }
  (void)L;
}

// E[axis][i][j][t] of one primitive pair for i <= li, j <= lj.
__device__ void md_hermite_axis(double* E, int ax, int li, int lj, double xpa, double xpb, double inv2p) {
  for (int i = 0; i <= li; ++i)
    for (int j = 0; j <= lj; ++j)
      for (int t = 0; t < kMDE; ++t) E[eidx(ax, i, j, t)] = 0.0;
  E[eidx(ax, 0, 0, 0)] = 1.0;
  for (int i = 0; i <= li; ++i)
    for (int j = 0; j <= lj; ++j) {
      if (i == 0 && j == 0) continue;
      const int pi = i > 0 ? i - 1 : 0, pj = i > 0 ? j : j - 1;
      const double x = i > 0 ? xpa : xpb;
      const int tmax = i + j;
      for (int t = 0; t <= tmax; ++t) {
        double v = x * E[eidx(ax, pi, pj, t)];
        if (t > 0) v += inv2p * E[eidx(ax, pi, pj, t - 1)];
        if (t + 1 <= tmax - 1) v += (t + 1) * E[eidx(ax, pi, pj, t + 1)];
        E[eidx(ax, i, j, t)] = v;
      }
    }
}

// One primitive pair: exponent sum, 1/p, K_p (contraction coefficients,
// Gaussian product factor and 1/p) and P - A.
struct MDPrim {
  double p, inv_p, kp, PA[3];
};

// R_{tuv} = R^{0}_{tuv} for t+u+v <= L into R0, from S[0..2] = P - Q,
// S[3] = -2 alpha and F[n] = F_n: level n from level n + 1 for n = L .. 0
// (level n in R0 for even n, R1 for odd n), the block synchronised after
// each level.
__device__ void md_build_R(int L, double* R0, double* R1, const double* S, const double* F) {
  const int tid = threadIdx.x, nt = blockDim.x;
  for (int n = L; n >= 0; --n) {
    double* cur = (n & 1) ? R1 : R0;
    const double* prev = (n & 1) ? R0 : R1;
    const int m = L - n, e1 = m + 1, cube = e1 * e1 * e1;
    for (int x = tid; x < cube; x += nt) {
      const int t = x / (e1 * e1), u = (x / e1) % e1, v = x % e1;
      if (t + u + v > m) continue;
      double r;
      if (t > 0) {
        r = S[0] * prev[ridx(t - 1, u, v)];
        if (t > 1) r += (t - 1) * prev[ridx(t - 2, u, v)];
      } else if (u > 0) {
        r = S[1] * prev[ridx(t, u - 1, v)];
        if (u > 1) r += (u - 1) * prev[ridx(t, u - 2, v)];
      } else if (v > 0) {
        r = S[2] * prev[ridx(t, u, v - 1)];
        if (v > 1) r += (v - 1) * prev[ridx(t, u, v - 2)];
      } else {
        double w = 1.0;
        for (int k = 0; k < n; ++k) w *= S[3];
        r = w * F[n];
      }
      cur[ridx(t, u, v)] = r;
    }
    __syncthreads();
  }
}

// Adds one primitive quartet into s.out (every thread of the block takes
// part; the caller synchronises before reusing the tables).
__device__ void md_prim_quartet(const MDClass& c, const MDLayout& L, const MDShared& s, const MDPrim& P,
                                const MDPrim& Q, const double* AB, const double* CD, const double* AC,
                                const double* __restrict__ boys, const double* __restrict__ expt) {
  const int tid = threadIdx.x, nt = blockDim.x;
  if (tid == 0) {
    double PQ[3];
    for (int k = 0; k < 3; ++k) PQ[k] = AC[k] + P.PA[k] - Q.PA[k];
    const double sum = P.p + Q.p, alpha = P.p * Q.p / sum;
    const double T = alpha * (PQ[0] * PQ[0] + PQ[1] * PQ[1] + PQ[2] * PQ[2]);
    md_boys(T, c.L, boys, expt, s.F);
    s.S[0] = PQ[0];
    s.S[1] = PQ[1];
    s.S[2] = PQ[2];
    s.S[3] = -2.0 * alpha;
    s.S[4] = kTwoPiPow25 * P.kp * Q.kp * rsqrt(sum);
  } else if (tid >= 32 && tid < 35) {
    const int ax = tid - 32;
    md_hermite_axis(s.Eb, ax, c.la, c.lb, P.PA[ax], P.PA[ax] + AB[ax], 0.5 * P.inv_p);
  } else if (tid >= 64 && tid < 67) {
    const int ax = tid - 64;
    md_hermite_axis(s.Ek, ax, c.lc, c.ld, Q.PA[ax], Q.PA[ax] + CD[ax], 0.5 * Q.inv_p);
  }
  __syncthreads();
  md_build_R(c.L, s.R0, s.R1, s.S, s.F);
  // G[ab][h] = sum_tuv E^{ab}_{tuv} R_{t+tau, u+nu, v+phi}
  for (int x = tid; x < L.nab * L.nherm; x += nt) {
    const int ab = x / L.nherm, h = x % L.nherm;
    const int* ea = s.comp + (0 * 10 + ab / c.nb) * 3;
    const int* eb = s.comp + (1 * 10 + ab % c.nb) * 3;
    const int ht = s.hlist[3 * h], hu = s.hlist[3 * h + 1], hv = s.hlist[3 * h + 2];
    double g = 0.0;
    for (int t = 0; t <= ea[0] + eb[0]; ++t) {
      const double ex = s.Eb[eidx(0, ea[0], eb[0], t)];
      for (int u = 0; u <= ea[1] + eb[1]; ++u) {
        const double exy = ex * s.Eb[eidx(1, ea[1], eb[1], u)];
        for (int v = 0; v <= ea[2] + eb[2]; ++v)
          g += exy * s.Eb[eidx(2, ea[2], eb[2], v)] * s.R0[ridx(t + ht, u + hu, v + hv)];
      }
    }
    s.G[x] = g;
  }
  __syncthreads();
  // out[ab][cd] += pref sum (-1)^{tau+nu+phi} E^{cd} G[ab]
  const double pref = s.S[4];
  for (int x = tid; x < L.nab * L.ncd; x += nt) {
    const int ab = x / L.ncd, cd = x % L.ncd;
    const int* ec = s.comp + (2 * 10 + cd / c.nd) * 3;
    const int* ed = s.comp + (3 * 10 + cd % c.nd) * 3;
    const double* g = s.G + (size_t)ab * L.nherm;
    double acc = 0.0;
    for (int t = 0; t <= ec[0] + ed[0]; ++t) {
      const double ex = (t & 1 ? -1.0 : 1.0) * s.Ek[eidx(0, ec[0], ed[0], t)];
      for (int u = 0; u <= ec[1] + ed[1]; ++u) {
        const double exy = (u & 1 ? -ex : ex) * s.Ek[eidx(1, ec[1], ed[1], u)];
        for (int v = 0; v <= ec[2] + ed[2]; ++v) {
          const double w = (v & 1 ? -exy : exy) * s.Ek[eidx(2, ec[2], ed[2], v)];
          acc += w * g[s.hidx[(t * kMDE + u) * kMDE + v]];
        }
      }
    }
    s.out[x] += pref * acc;
  }
  __syncthreads();
}

// A primitive pair from the 64-byte table (PrimPair, P - A stored).
__device__ __forceinline__ MDPrim md_from_pp(const PrimPair& q) {
  MDPrim m;
  m.p = q.p;
  m.inv_p = q.inv_p;
  m.kp = q.kp;
  m.PA[0] = q.PAx;
  m.PA[1] = q.PAy;
  m.PA[2] = q.PAz;
  return m;
}

// A primitive pair from the compact records (P - A = -(beta/p) AB).
__device__ __forceinline__ MDPrim md_from_rec(const PrimRec64& r, const PairInfo& pi) {
  MDPrim m;
  m.p = r.p;
  m.inv_p = r.inv_p;
  m.kp = r.kp;
  m.PA[0] = -r.bp * pi.ABx;
  m.PA[1] = -r.bp * pi.ABy;
  m.PA[2] = -r.bp * pi.ABz;
  return m;
}

__device__ __forceinline__ void md_zero_out(const MDLayout& L, const MDShared& s) {
  for (int x = threadIdx.x; x < L.nab * L.ncd; x += blockDim.x) s.out[x] = 0.0;
  __syncthreads();
}

// Contracted block of (bra|ket) from the compact records, primitive
// quartets with bound products below eps skipped (eps = 0: all).
__device__ void md_quartet_rec(const MDClass& c, const MDLayout& L, const MDShared& s, const PairInfo& bra,
                               const PairInfo& ket, const PrimRec64* __restrict__ rec,
                               const float* __restrict__ pbound, double eps, const double* __restrict__ boys,
                               const double* __restrict__ expt) {
  md_zero_out(L, s);
  const double AB[3] = {bra.ABx, bra.ABy, bra.ABz}, CD[3] = {ket.ABx, ket.ABy, ket.ABz};
  const double AC[3] = {bra.Ax - ket.Ax, bra.Ay - ket.Ay, bra.Az - ket.Az};
  const float feps = (float)eps;
  for (int ib = 0; ib < bra.npp; ++ib) {
    const float bb = pbound[bra.rec_off + (size_t)ib * bra.rec_stride];
    const MDPrim P = md_from_rec(rec[bra.rec_off + (size_t)ib * bra.rec_stride], bra);
    for (int ik = 0; ik < ket.npp; ++ik) {
      if (eps > 0.0 && bb * pbound[ket.rec_off + (size_t)ik * ket.rec_stride] < feps) continue;
      const MDPrim Q = md_from_rec(rec[ket.rec_off + (size_t)ik * ket.rec_stride], ket);
      md_prim_quartet(c, L, s, P, Q, AB, CD, AC, boys, expt);
    }
  }
}

// Scale factor of block element (ab, cd): the four component scales.
__device__ __forceinline__ double md_scale(const MDClass& c, const MDShared& s, int ab, int cd) {
  return md_comp_scale(s.comp + (0 * 10 + ab / c.nb) * 3) * md_comp_scale(s.comp + (1 * 10 + ab % c.nb) * 3) *
         md_comp_scale(s.comp + (2 * 10 + cd / c.nd) * 3) * md_comp_scale(s.comp + (3 * 10 + cd % c.nd) * 3);
}

// ---------------------------------------------------------------------------
// Schwarz bounds: one block per shell pair (prim_mode 0) or per primitive
// pair (prim_mode 1), sqrt of the largest scaled diagonal element.
__global__ void __launch_bounds__(kMDThreads) schwarz_md_kernel(MDClass c, const PairInfo* __restrict__ pairs,
                                                                const PrimPair* __restrict__ prims, int first,
                                                                const double* __restrict__ boys,
                                                                const double* __restrict__ expt,
                                                                double* __restrict__ out, int prim_mode) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const MDLayout L(c);
  const MDShared s = md_shared(L, smem_raw);
  __shared__ double red[kMDThreads];
  md_setup(c, L, s);
  md_zero_out(L, s);
  const int t = blockIdx.x;
  const int p0 = prim_mode ? first + t : pairs[first + t].pp_off;
  const int np = prim_mode ? 1 : pairs[first + t].npp;
  const PairInfo owner = prim_mode ? pairs[(int)prims[p0].pad] : pairs[first + t];
  const double AB[3] = {owner.ABx, owner.ABy, owner.ABz}, AC[3] = {0.0, 0.0, 0.0};
  for (int ib = 0; ib < np; ++ib)
    for (int ik = 0; ik < np; ++ik)
      md_prim_quartet(c, L, s, md_from_pp(prims[p0 + ib]), md_from_pp(prims[p0 + ik]), AB, AB, AC, boys, expt);
  double m = 0.0;
  for (int ij = threadIdx.x; ij < L.nab; ij += blockDim.x) {
    const double sc = md_scale(c, s, ij, ij);
    m = fmax(m, s.out[(size_t)ij * L.ncd + ij] * sc);
  }
  red[threadIdx.x] = m;
  __syncthreads();
  if (threadIdx.x == 0) {
    double r = 0.0;
    for (int k = 0; k < (int)blockDim.x; ++k) r = fmax(r, red[k]);
    out[t] = sqrt(r);
  }
}

// One full scaled block (ab|cd) of bra pairs[0], ket pairs[1].
__global__ void __launch_bounds__(kMDThreads) quartet_md_kernel(MDClass c, const PairInfo* __restrict__ pairs,
                                                                const PrimPair* __restrict__ prims,
                                                                const double* __restrict__ boys,
                                                                const double* __restrict__ expt,
                                                                double* __restrict__ out) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const MDLayout L(c);
  const MDShared s = md_shared(L, smem_raw);
  md_setup(c, L, s);
  md_zero_out(L, s);
  const PairInfo bra = pairs[0], ket = pairs[1];
  const double AB[3] = {bra.ABx, bra.ABy, bra.ABz}, CD[3] = {ket.ABx, ket.ABy, ket.ABz};
  const double AC[3] = {bra.Ax - ket.Ax, bra.Ay - ket.Ay, bra.Az - ket.Az};
  for (int ib = 0; ib < bra.npp; ++ib)
    for (int ik = 0; ik < ket.npp; ++ik)
      md_prim_quartet(c, L, s, md_from_pp(prims[bra.pp_off + ib]), md_from_pp(prims[ket.pp_off + ik]), AB, CD, AC,
                      boys, expt);
  for (int x = threadIdx.x; x < L.nab * L.ncd; x += blockDim.x)
    out[x] = s.out[x] * md_scale(c, s, x / L.ncd, x % L.ncd);
}

__device__ __forceinline__ unsigned long long md_compound(unsigned long long i, unsigned long long j) {
  return i >= j ? i * (i + 1) / 2 + j : j * (j + 1) / 2 + i;
}

// Packed 8-fold tensor slots of the plan's quartets (the writer rules of
// eri_packed_kernel: i >= j within a same-shell pair, IJ >= KL for a pair
// with itself).  One block per warp task of the plan, its kets in turn.
__global__ void __launch_bounds__(kMDThreads) eri_packed_md_kernel(
    MDClass c, const JKEntry* __restrict__ entries, const long long* __restrict__ prefix, int nentries,
    const PairInfo* __restrict__ pairs, const double* __restrict__ pairQ, double thr,
    const PrimRec64* __restrict__ rec, const float* __restrict__ pbound, const double* __restrict__ boys,
    const double* __restrict__ expt, double* __restrict__ out) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const MDLayout L(c);
  const MDShared s = md_shared(L, smem_raw);
  md_setup(c, L, s);
  __syncthreads();
  const long long warp = blockIdx.x;
  const int e = find_entry(prefix, nentries, warp);
  const JKEntry ent = entries[e];
  const int k0 = ent.k_lo + (int)(warp - prefix[e]) * 32, k1 = min(k0 + 32, ent.k_hi);
  const PairInfo bra = pairs[ent.bra];
  for (int kidx = k0; kidx < k1; ++kidx) {
    if (!(pairQ[kidx] * pairQ[ent.bra] > thr)) continue;
    const PairInfo ket = pairs[kidx];
    md_quartet_rec(c, L, s, bra, ket, rec, pbound, 0.0, boys, expt);
    const bool self = kidx == ent.bra;
    for (int x = threadIdx.x; x < L.nab * L.ncd; x += blockDim.x) {
      const int ab = x / L.ncd, cd = x % L.ncd;
      const int mu = bra.ao_a + ab / c.nb, nu = bra.ao_b + ab % c.nb;
      const int lam = ket.ao_a + cd / c.nd, sig = ket.ao_b + cd % c.nd;
      if (bra.same && mu < nu) continue;
      if (ket.same && lam < sig) continue;
      const unsigned long long IJ = md_compound(mu, nu), KL = md_compound(lam, sig);
      if (self && IJ < KL) continue;
      out[md_compound(IJ, KL)] = s.out[x] * md_scale(c, s, ab, cd);
    }
    __syncthreads();
  }
}

// Direct J/K (FP64) over a launch's work queue: persistent blocks take
// work-queue steps; each warp task's kets are evaluated one quartet at a
// time by the whole block and digested as the fast kernels do
// (jk_kernels.cuh): J'[a,b] += 4w sum D[c,d], J'[c,d] += 4w sum D[a,b],
// K'[a,c] += 2w sum D[b,d] and the three other exchange blocks, w the
// quartet's degeneracy weight.  In deterministic mode one block runs the
// queue and one thread issues every atomic of a quartet, quartet after
// quartet.
__global__ void __launch_bounds__(kMDThreads) jk_md_kernel(MDClass c, const JKLaunchArgs a) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const MDLayout L(c);
  const MDShared s = md_shared(L, smem_raw);
  __shared__ long long s_step;
  md_setup(c, L, s);
  const int n = a.n, NS = a.nspin;
  const int na = c.na, nb = c.nb, nc = c.nc, nd = c.nd;
  for (;;) {
    __syncthreads();
    if (threadIdx.x == 0) s_step = (long long)atomicAdd(a.counter, 1ull);
    __syncthreads();
    const long long step = s_step;
    if (step >= a.nchunks) break;
    const long long t0 = a.chunk_start[step], t1 = a.chunk_start[step + 1];
    int e = a.chunk_entry[step];
    for (long long w = t0; w < t1; ++w) {
      while (a.prefix[e + 1] <= w) ++e;
      const JKEntry ent = a.entries[e];
      const int k0 = ent.k_lo + (int)(w - a.prefix[e]) * 32, k1 = min(k0 + 32, ent.k_hi);
      const PairInfo bra = a.pairs[ent.bra];
      for (int kidx = k0; kidx < k1; ++kidx) {
        if (!(a.pairQ[kidx] * a.pairQ[ent.bra] > a.thr)) continue;
        const PairInfo ket = a.pairs[kidx];
        md_quartet_rec(c, L, s, bra, ket, a.rec64, a.pbound, a.prim_eps, a.boys64, a.expt64);
        double deg = 1.0;
        if (bra.same) deg *= 0.5;
        if (ket.same) deg *= 0.5;
        if (kidx == ent.bra) deg *= 0.5;
        for (int x = threadIdx.x; x < L.nab * L.ncd; x += blockDim.x)
          s.out[x] *= deg * md_scale(c, s, x / L.ncd, x % L.ncd);
        __syncthreads();
        const int i0 = bra.ao_a, j0 = bra.ao_b, kk0 = ket.ao_a, l0 = ket.ao_b;
        // items: J'[ab], J'[cd], then per spin K'[ac], K'[bc], K'[ad], K'[bd]
        const int nK = na * nc + nb * nc + na * nd + nb * nd;
        const int items = L.nab + L.ncd + NS * nK;
        // items can add into the same element (J'[ab] and J'[cd] of a pair
        // with itself, K' blocks of a same-shell pair): in deterministic mode
        // one thread takes every item in order
        const int x0 = a.serial ? (threadIdx.x == 0 ? 0 : items) : threadIdx.x;
        const int dx = a.serial ? 1 : blockDim.x;
        for (int x = x0; x < items; x += dx) {
          if (x < L.nab) {
            double v = 0.0;
            for (int cd = 0; cd < L.ncd; ++cd)
              v += s.out[(size_t)x * L.ncd + cd] * a.Dtot[(size_t)(kk0 + cd / nd) * n + l0 + cd % nd];
            atomicAdd(a.Jacc + (size_t)(i0 + x / nb) * n + j0 + x % nb, 4.0 * v);
            continue;
          }
          int y = x - L.nab;
          if (y < L.ncd) {
            double v = 0.0;
            for (int ab = 0; ab < L.nab; ++ab)
              v += s.out[(size_t)ab * L.ncd + y] * a.Dtot[(size_t)(i0 + ab / nb) * n + j0 + ab % nb];
            atomicAdd(a.Jacc + (size_t)(kk0 + y / nd) * n + l0 + y % nd, 4.0 * v);
            continue;
          }
          y -= L.ncd;
          const int sp = y / nK;
          int r = y % nK;
          const double* D = a.Dspin + (size_t)sp * n * n;
          double* K = a.Kacc + (size_t)sp * n * n;
          double v = 0.0;
          if (r < na * nc) {  // K'[a,c] from D[b,d]
            const int i = r / nc, k = r % nc;
            for (int j = 0; j < nb; ++j)
              for (int l = 0; l < nd; ++l)
                v += s.out[(size_t)(i * nb + j) * L.ncd + k * nd + l] * D[(size_t)(j0 + j) * n + l0 + l];
            atomicAdd(K + (size_t)(i0 + i) * n + kk0 + k, 2.0 * v);
            continue;
          }
          r -= na * nc;
          if (r < nb * nc) {  // K'[b,c] from D[a,d]
            const int j = r / nc, k = r % nc;
            for (int i = 0; i < na; ++i)
              for (int l = 0; l < nd; ++l)
                v += s.out[(size_t)(i * nb + j) * L.ncd + k * nd + l] * D[(size_t)(i0 + i) * n + l0 + l];
            atomicAdd(K + (size_t)(j0 + j) * n + kk0 + k, 2.0 * v);
            continue;
          }
          r -= nb * nc;
          if (r < na * nd) {  // K'[a,d] from D[b,c]
            const int i = r / nd, l = r % nd;
            for (int j = 0; j < nb; ++j)
              for (int k = 0; k < nc; ++k)
                v += s.out[(size_t)(i * nb + j) * L.ncd + k * nd + l] * D[(size_t)(j0 + j) * n + kk0 + k];
            atomicAdd(K + (size_t)(i0 + i) * n + l0 + l, 2.0 * v);
            continue;
          }
          r -= na * nd;
          {  // K'[b,d] from D[a,c]
            const int j = r / nd, l = r % nd;
            for (int i = 0; i < na; ++i)
              for (int k = 0; k < nc; ++k)
                v += s.out[(size_t)(i * nb + j) * L.ncd + k * nd + l] * D[(size_t)(i0 + i) * n + kk0 + k];
            atomicAdd(K + (size_t)(j0 + j) * n + l0 + l, 2.0 * v);
          }
        }
        if (a.serial) __threadfence();
        __syncthreads();
      }
    }
  }
}


// ---------------------------------------------------------------------------
// Nuclear derivatives of the two-electron energy (the ERI part of the HF
// gradient, hf-rs's contract_eri_derivatives, src/gradient.rs:33-69 with the
// densities of :287-301).  With G = P_ab P_cd - x (P_ac P_bd + P_ad P_bc)
// (x = 1/4 for a closed shell; per spin, x = 1/2 on the spin densities)
// the energy is E2 = 1/2 sum_abcd (ab|cd) G_abcd, so over unique quartets
//   dE2/dX = 4 sum w (d(ab|cd)/dX) G_abcd,
// w the degeneracy weight of the J/K kernels.  A centre derivative of a
// Gaussian raises and lowers its power, d/dA_x phi_a = 2 alpha phi_{a+1x}
// - a_x phi_{a-1x}, so the derivative integrals use the same R table (one
// order higher) with Hermite coefficients 2 alpha E^{i+1,j} - i E^{i-1,j};
// the fourth centre follows from translational invariance.  Per primitive
// quartet, G is first contracted with one side's Hermite coefficients and
// R (W, V for the bra; X, U for the ket), then with the derivative
// coefficients of the other side.
struct GradArgs {
  const JKEntry* entries;
  const long long* prefix;
  const long long* chunk_start;
  const int* chunk_entry;
  long long nchunks;
  unsigned long long* counter;
  const PairInfo* pairs;
  const double* pairQ;
  double thr;
  const PrimRec64* rec;
  const double* boys;
  const double* expt;
  const double* P;   // total density, n x n
  const double* Ps;  // nspin spin densities
  int nspin, n;
  const int* ao_atom;
  double* grad;  // natom x 3
};

struct GradLayout {
  int nab, ncd, hab, hcd, hab1, hcd1;
  int G, W, X, V, U, R0, R1, Eb, Ek, F, S, red, dbl_end;
  __host__ __device__ GradLayout(const MDClass& c) {
    nab = c.na * c.nb;
    ncd = c.nc * c.nd;
    hab = (c.lab + 1) * (c.lab + 2) * (c.lab + 3) / 6;
    hcd = (c.lcd + 1) * (c.lcd + 2) * (c.lcd + 3) / 6;
    hab1 = (c.lab + 2) * (c.lab + 3) * (c.lab + 4) / 6;
    hcd1 = (c.lcd + 2) * (c.lcd + 3) * (c.lcd + 4) / 6;
    G = 0;
    W = G + nab * ncd;
    X = W + nab * hcd;
    V = X + ncd * hab;
    U = V + nab * hab1;
    R0 = U + ncd * hcd1;
    R1 = R0 + kMDRCube;
    Eb = R1 + kMDRCube;
    Ek = Eb + 3 * kMDEAxis;
    F = Ek + 3 * kMDEAxis;
    S = F + 4 * kMDLMax + 8;
    red = S + 16;
    dbl_end = red + 9 * (kMDThreads / 32);
  }
  __host__ __device__ size_t bytes() const {
    return (size_t)dbl_end * 8 + (size_t)(kMDHCube + 3 * kMDHCube + 4 * 10 * 3) * 4;
  }
};

__global__ void __launch_bounds__(kMDThreads) grad_md_kernel(MDClass c, const GradArgs a) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const GradLayout L(c);
  double* d = reinterpret_cast<double*>(smem_raw);
  double *Gm = d + L.G, *W = d + L.W, *X = d + L.X, *V = d + L.V, *U = d + L.U;
  double *R0 = d + L.R0, *R1 = d + L.R1, *Eb = d + L.Eb, *Ek = d + L.Ek, *F = d + L.F, *S = d + L.S;
  double* red = d + L.red;
  int* ip = reinterpret_cast<int*>(d + L.dbl_end);
  int *hidx = ip, *hlist = ip + kMDHCube, *comp = ip + 4 * kMDHCube;
  __shared__ long long s_step;
  const int tid = threadIdx.x, nt = blockDim.x;
  // components of the four shells, and the Hermite triples in order of
  // total degree (those of degree <= k are the first nherm(k))
  {
    const int ls[4] = {c.la, c.lb, c.lc, c.ld};
    for (int x = tid; x < 4 * 10; x += nt) {
      const int sh = x / 10, k = x % 10;
      if (k < ncart(ls[sh])) md_component(ls[sh], k, comp + x * 3);
    }
    if (tid == 0) {
      for (int x = 0; x < kMDHCube; ++x) hidx[x] = -1;
      int h = 0;
      for (int deg = 0; deg < kMDE; ++deg)
        for (int t = deg; t >= 0; --t)
          for (int u = deg - t; u >= 0; --u) {
            const int v = deg - t - u;
            hidx[(t * kMDE + u) * kMDE + v] = h;
            hlist[3 * h] = t;
            hlist[3 * h + 1] = u;
            hlist[3 * h + 2] = v;
            ++h;
          }
    }
  }
  const int n = a.n, NS = a.nspin;
  const double xk = NS == 1 ? 0.25 : 0.5;
  const int Lg = c.L + 1;
  const int* ca = comp;
  const int* cb = comp + 30;
  const int* cc = comp + 60;
  const int* cdd = comp + 90;
  auto hm = [&](int t, int u, int v) { return hidx[(t * kMDE + u) * kMDE + v]; };
  for (;;) {
    __syncthreads();
    if (tid == 0) s_step = (long long)atomicAdd(a.counter, 1ull);
    __syncthreads();
    const long long step = s_step;
    if (step >= a.nchunks) break;
    const long long t0 = a.chunk_start[step], t1 = a.chunk_start[step + 1];
    int e = a.chunk_entry[step];
    for (long long w = t0; w < t1; ++w) {
      while (a.prefix[e + 1] <= w) ++e;
      const JKEntry ent = a.entries[e];
      const int k0 = ent.k_lo + (int)(w - a.prefix[e]) * 32, k1 = min(k0 + 32, ent.k_hi);
      const PairInfo bra = a.pairs[ent.bra];
      for (int kidx = k0; kidx < k1; ++kidx) {
        if (!(a.pairQ[kidx] * a.pairQ[ent.bra] > a.thr)) continue;
        const PairInfo ket = a.pairs[kidx];
        const int i0 = bra.ao_a, j0 = bra.ao_b, kk0 = ket.ao_a, l0 = ket.ao_b;
        // G with the component scales of the four functions
        for (int x = tid; x < L.nab * L.ncd; x += nt) {
          const int ab = x / L.ncd, cd = x % L.ncd;
          const int I = i0 + ab / c.nb, J = j0 + ab % c.nb, K = kk0 + cd / c.nd, M = l0 + cd % c.nd;
          double g = a.P[(size_t)I * n + J] * a.P[(size_t)K * n + M];
          for (int sp = 0; sp < NS; ++sp) {
            const double* D = a.Ps + (size_t)sp * n * n;
            g -= xk * (D[(size_t)I * n + K] * D[(size_t)J * n + M] + D[(size_t)I * n + M] * D[(size_t)J * n + K]);
          }
          Gm[x] = g * md_comp_scale(ca + (ab / c.nb) * 3) * md_comp_scale(cb + (ab % c.nb) * 3) *
                  md_comp_scale(cc + (cd / c.nd) * 3) * md_comp_scale(cdd + (cd % c.nd) * 3);
        }
        double acc[9];
        for (int k = 0; k < 9; ++k) acc[k] = 0.0;
        const double AB[3] = {bra.ABx, bra.ABy, bra.ABz}, CD[3] = {ket.ABx, ket.ABy, ket.ABz};
        const double AC[3] = {bra.Ax - ket.Ax, bra.Ay - ket.Ay, bra.Az - ket.Az};
        for (int ib = 0; ib < bra.npp; ++ib) {
          const PrimRec64 rb = a.rec[bra.rec_off + (size_t)ib * bra.rec_stride];
          for (int ik = 0; ik < ket.npp; ++ik) {
            const PrimRec64 rk = a.rec[ket.rec_off + (size_t)ik * ket.rec_stride];
            __syncthreads();  // G written; tables of the previous primitive quartet read
            const MDPrim Pp = md_from_rec(rb, bra), Qp = md_from_rec(rk, ket);
            if (tid == 0) {
              double PQ[3];
              for (int k = 0; k < 3; ++k) PQ[k] = AC[k] + Pp.PA[k] - Qp.PA[k];
              const double sum = Pp.p + Qp.p, alpha = Pp.p * Qp.p / sum;
              md_boys(alpha * (PQ[0] * PQ[0] + PQ[1] * PQ[1] + PQ[2] * PQ[2]), Lg, a.boys, a.expt, F);
              S[0] = PQ[0];
              S[1] = PQ[1];
              S[2] = PQ[2];
              S[3] = -2.0 * alpha;
              S[4] = kTwoPiPow25 * Pp.kp * Qp.kp * rsqrt(sum);
            } else if (tid >= 32 && tid < 35) {
              const int ax = tid - 32;
              md_hermite_axis(Eb, ax, c.la + 1, c.lb + 1, Pp.PA[ax], Pp.PA[ax] + AB[ax], 0.5 * Pp.inv_p);
            } else if (tid >= 64 && tid < 67) {
              const int ax = tid - 64;
              md_hermite_axis(Ek, ax, c.lc + 1, c.ld + 1, Qp.PA[ax], Qp.PA[ax] + CD[ax], 0.5 * Qp.inv_p);
            }
            __syncthreads();
            md_build_R(Lg, R0, R1, S, F);
            // W[ab][h] = sum_cd G s(h) E^{cd}_h;  X[cd][h] = sum_ab G E^{ab}_h
            for (int x = tid; x < L.nab * L.hcd + L.ncd * L.hab; x += nt) {
              if (x < L.nab * L.hcd) {
                const int ab = x / L.hcd, h = x % L.hcd;
                const int ht = hlist[3 * h], hu = hlist[3 * h + 1], hv = hlist[3 * h + 2];
                double v = 0.0;
                for (int cd = 0; cd < L.ncd; ++cd) {
                  const int* ec = cc + (cd / c.nd) * 3;
                  const int* ed = cdd + (cd % c.nd) * 3;
                  v += Gm[(size_t)ab * L.ncd + cd] * Ek[eidx(0, ec[0], ed[0], ht)] * Ek[eidx(1, ec[1], ed[1], hu)] *
                       Ek[eidx(2, ec[2], ed[2], hv)];
                }
                W[x] = ((ht + hu + hv) & 1) ? -v : v;
              } else {
                const int y = x - L.nab * L.hcd, cd = y / L.hab, h = y % L.hab;
                const int ht = hlist[3 * h], hu = hlist[3 * h + 1], hv = hlist[3 * h + 2];
                double v = 0.0;
                for (int ab = 0; ab < L.nab; ++ab) {
                  const int* ea = ca + (ab / c.nb) * 3;
                  const int* eb = cb + (ab % c.nb) * 3;
                  v += Gm[(size_t)ab * L.ncd + cd] * Eb[eidx(0, ea[0], eb[0], ht)] * Eb[eidx(1, ea[1], eb[1], hu)] *
                       Eb[eidx(2, ea[2], eb[2], hv)];
                }
                X[y] = v;
              }
            }
            __syncthreads();
            // V[ab][h'] = sum_h W[ab][h] R_{h'+h} (h' of degree <= lab + 1);
            // U[cd][h'] = sum_h X[cd][h] R_{h+h'} (h' of degree <= lcd + 1)
            for (int x = tid; x < L.nab * L.hab1 + L.ncd * L.hcd1; x += nt) {
              if (x < L.nab * L.hab1) {
                const int ab = x / L.hab1, h1 = x % L.hab1;
                const int t = hlist[3 * h1], u = hlist[3 * h1 + 1], v = hlist[3 * h1 + 2];
                double r = 0.0;
                for (int h = 0; h < L.hcd; ++h)
                  r += W[(size_t)ab * L.hcd + h] * R0[ridx(t + hlist[3 * h], u + hlist[3 * h + 1], v + hlist[3 * h + 2])];
                V[x] = r;
              } else {
                const int y = x - L.nab * L.hab1, cd = y / L.hcd1, h1 = y % L.hcd1;
                const int t = hlist[3 * h1], u = hlist[3 * h1 + 1], v = hlist[3 * h1 + 2];
                double r = 0.0;
                for (int h = 0; h < L.hab; ++h)
                  r += X[(size_t)cd * L.hab + h] * R0[ridx(hlist[3 * h] + t, hlist[3 * h + 1] + u, hlist[3 * h + 2] + v)];
                U[y] = ((t + u + v) & 1) ? -r : r;
              }
            }
            __syncthreads();
            // derivative coefficients against V (centres A, B) and U (C)
            const double pref = S[4];
            const double beta = rb.bp * rb.p, alpha_a = rb.p - beta;
            const double delta = rk.bp * rk.p, gamma_c = rk.p - delta;
            for (int x = tid; x < L.nab + L.ncd; x += nt) {
              const bool braside = x < L.nab;
              const int id = braside ? x : x - L.nab;
              const int* e1 = braside ? ca + (id / c.nb) * 3 : cc + (id / c.nd) * 3;
              const int* e2 = braside ? cb + (id % c.nb) * 3 : cdd + (id % c.nd) * 3;
              const double* E = braside ? Eb : Ek;
              const double* T = braside ? V + (size_t)id * L.hab1 : U + (size_t)id * L.hcd1;
              // first centre (A or C), then second (B), each x, y, z
              for (int centre = 0; centre < (braside ? 2 : 1); ++centre) {
                const double ex = centre == 0 ? (braside ? alpha_a : gamma_c) : beta;
                for (int ax = 0; ax < 3; ++ax) {
                  int p0[3] = {e1[0], e1[1], e1[2]}, q0[3] = {e2[0], e2[1], e2[2]};
                  int* dv = centre == 0 ? p0 : q0;  // the differentiated function's powers
                  const int lo = dv[ax];
                  double sacc = 0.0;
                  // 2 ex (raised) - lo (lowered), each a product of three axes
                  for (int term = 0; term < 2; ++term) {
                    if (term == 1 && lo == 0) break;
                    const double f = term == 0 ? 2.0 * ex : -(double)lo;
                    dv[ax] = term == 0 ? lo + 1 : lo - 1;
                    double s3 = 0.0;
                    for (int t = 0; t <= p0[0] + q0[0]; ++t) {
                      const double e0 = E[eidx(0, p0[0], q0[0], t)];
                      for (int u = 0; u <= p0[1] + q0[1]; ++u) {
                        const double e01 = e0 * E[eidx(1, p0[1], q0[1], u)];
                        for (int v = 0; v <= p0[2] + q0[2]; ++v)
                          s3 += e01 * E[eidx(2, p0[2], q0[2], v)] * T[hm(t, u, v)];
                      }
                    }
                    sacc += f * s3;
                    dv[ax] = lo;
                  }
                  acc[(braside ? 3 * centre : 6) + ax] += pref * sacc;
                }
              }
            }
          }
        }
        // block sums of the nine components, then the four centres
        for (int k = 0; k < 9; ++k) {
          double v = acc[k];
          for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
          if ((tid & 31) == 0) red[k * (kMDThreads / 32) + (tid >> 5)] = v;
        }
        __syncthreads();
        if (tid == 0) {
          double g[9];
          for (int k = 0; k < 9; ++k) {
            g[k] = 0.0;
            for (int wv = 0; wv < nt / 32; ++wv) g[k] += red[k * (kMDThreads / 32) + wv];
          }
          double deg = 1.0;
          if (bra.same) deg *= 0.5;
          if (ket.same) deg *= 0.5;
          if (kidx == ent.bra) deg *= 0.5;
          const double f = 4.0 * deg;
          const int atA = a.ao_atom[i0], atB = a.ao_atom[j0], atC = a.ao_atom[kk0], atD = a.ao_atom[l0];
          for (int ax = 0; ax < 3; ++ax) {
            atomicAdd(a.grad + 3 * atA + ax, f * g[ax]);
            atomicAdd(a.grad + 3 * atB + ax, f * g[3 + ax]);
            atomicAdd(a.grad + 3 * atC + ax, f * g[6 + ax]);
            atomicAdd(a.grad + 3 * atD + ax, -f * (g[ax] + g[3 + ax] + g[6 + ax]));
          }
        }
      }
    }
  }
}

int md_resident_blocks(const void* kern, size_t smem) {
  int dev = 0, sms = 0, per_sm = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kMDThreads, smem);
  return sms * (per_sm > 0 ? per_sm : 1);
}

}  // namespace

MDClass md_class(int la, int lb, int lc, int ld) {
  MDClass c;
  c.la = la;
  c.lb = lb;
  c.lc = lc;
  c.ld = ld;
  c.na = ncart(la);
  c.nb = ncart(lb);
  c.nc = ncart(lc);
  c.nd = ncart(ld);
  c.lab = la + lb;
  c.lcd = lc + ld;
  c.L = c.lab + c.lcd;
  return c;
}

size_t md_smem_bytes(const MDClass& c) { return MDLayout(c).bytes(); }

bool md_class_ok(int la, int lb, int lc, int ld) {
  return la >= 0 && lb >= 0 && lc >= 0 && ld >= 0 && la <= kMDLMax && lb <= kMDLMax && lc <= kMDLMax &&
         ld <= kMDLMax;
}

cudaError_t launch_schwarz_md(int la, int lb, const PairInfo* pairs, const PrimPair* prims, int first, int count,
                              const double* boys, const double* expt, double* out, int prim_mode, cudaStream_t st) {
  if (!md_class_ok(la, lb, la, lb)) return cudaErrorInvalidValue;
  if (count <= 0) return cudaSuccess;
  const MDClass c = md_class(la, lb, la, lb);
  const size_t smem = md_smem_bytes(c);
  cudaFuncSetAttribute(schwarz_md_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  schwarz_md_kernel<<<(unsigned)count, kMDThreads, smem, st>>>(c, pairs, prims, first, boys, expt, out, prim_mode);
  return cudaGetLastError();
}

cudaError_t launch_quartet_md(int la, int lb, int lc, int ld, const PairInfo* pairs, const PrimPair* prims,
                              const double* boys, const double* expt, double* out, cudaStream_t st) {
  if (!md_class_ok(la, lb, lc, ld)) return cudaErrorInvalidValue;
  const MDClass c = md_class(la, lb, lc, ld);
  const size_t smem = md_smem_bytes(c);
  cudaFuncSetAttribute(quartet_md_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  quartet_md_kernel<<<1, kMDThreads, smem, st>>>(c, pairs, prims, boys, expt, out);
  return cudaGetLastError();
}

cudaError_t launch_eri_packed_md(int la, int lb, int lc, int ld, const JKEntry* entries, const long long* prefix,
                                 int nentries, long long nwarps, const PairInfo* pairs, const double* pairQ,
                                 double thr, const PrimRec64* rec, const float* pbound, const double* boys,
                                 const double* expt, double* out, cudaStream_t st) {
  if (!md_class_ok(la, lb, lc, ld)) return cudaErrorInvalidValue;
  if (nwarps <= 0) return cudaSuccess;
  if (nwarps > 0x7fffffffLL) return cudaErrorInvalidValue;
  const MDClass c = md_class(la, lb, lc, ld);
  const size_t smem = md_smem_bytes(c);
  cudaFuncSetAttribute(eri_packed_md_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  eri_packed_md_kernel<<<(unsigned)nwarps, kMDThreads, smem, st>>>(c, entries, prefix, nentries, pairs, pairQ, thr,
                                                                   rec, pbound, boys, expt, out);
  return cudaGetLastError();
}

cudaError_t launch_jk_md(int la, int lb, int lc, int ld, const JKLaunchArgs& a, cudaStream_t st) {
  if (!md_class_ok(la, lb, lc, ld)) return cudaErrorInvalidValue;
  if (a.nchunks <= 0) return cudaSuccess;
  const MDClass c = md_class(la, lb, lc, ld);
  const size_t smem = md_smem_bytes(c);
  cudaFuncSetAttribute(jk_md_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  long long grid = a.serial ? 1 : md_resident_blocks((const void*)jk_md_kernel, smem);
  if (grid > a.nchunks) grid = a.nchunks;
  jk_md_kernel<<<(unsigned)grid, kMDThreads, smem, st>>>(c, a);
  return cudaGetLastError();
}

cudaError_t launch_grad_md(int la, int lb, int lc, int ld, const JKLaunchArgs& j, const int* ao_atom, double* grad,
                           cudaStream_t st) {
  if (!md_class_ok(la, lb, lc, ld) || la > kMDLMax - 1 || lb > kMDLMax - 1 || lc > kMDLMax - 1 || ld > kMDLMax - 1)
    return cudaErrorInvalidValue;
  if (j.nchunks <= 0) return cudaSuccess;
  const MDClass c = md_class(la, lb, lc, ld);
  GradArgs a;
  a.entries = j.entries;
  a.prefix = j.prefix;
  a.chunk_start = j.chunk_start;
  a.chunk_entry = j.chunk_entry;
  a.nchunks = j.nchunks;
  a.counter = j.counter;
  a.pairs = j.pairs;
  a.pairQ = j.pairQ;
  a.thr = j.thr;
  a.rec = j.rec64;
  a.boys = j.boys64;
  a.expt = j.expt64;
  a.P = j.Dtot;
  a.Ps = j.Dspin;
  a.nspin = j.nspin;
  a.n = j.n;
  a.ao_atom = ao_atom;
  a.grad = grad;
  const size_t smem = GradLayout(c).bytes();
  cudaFuncSetAttribute(grad_md_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  long long grid = md_resident_blocks((const void*)grad_md_kernel, smem);
  if (grid > j.nchunks) grid = j.nchunks;
  grad_md_kernel<<<(unsigned)grid, kMDThreads, smem, st>>>(c, a);
  return cudaGetLastError();
}

}  // namespace hfg
