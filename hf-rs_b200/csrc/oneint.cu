// One-electron integrals S, T, V on the device (needed by the SCF driver).
//
// McMurchie-Davidson form, as hf-rs computes them (src/integrals.rs:408-535,
// :747-793; src/scf.rs:247-271): one thread per Cartesian function pair
// mu >= nu, looping over primitive pairs; Hermite expansion coefficients
// E_t^{ij} per axis, S = E_0^x E_0^y E_0^z (pi/p)^{3/2}, T from the overlap
// recursion with lb +- 2, V = -Z 2pi/p sum E_t E_u E_v R_tuv(p, P - C) over
// nuclei.  Instantiated for shells up to d (LM = 2) and up to f (LM = 3);
// the kinetic term needs E up to lb + 2.
#include <cuda_runtime.h>

#include "boys.cuh"
#include "hfg_ctx.h"

namespace hfg {

// Hermite table extents for shells up to angular momentum LM
template <int LM> struct OneIntDims {
  static constexpr int EI = LM + 1;      // i index 0..LM
  static constexpr int EJ = LM + 3;      // j index 0..LM+2 (lb + 2)
  static constexpr int ET = 2 * LM + 3;  // t index
  static constexpr int L = 2 * LM;       // highest Boys order of V
};

struct FuncInfo {
  double c[3];
  int l[3];
  int shell;
};

struct OneIntArgs {
  const FuncInfo* funcs;
  const double* exps;   // per shell primitive exponents (shell prim_off)
  const double* coefs;  // per shell contraction coefficients (component scale applied below)
  const int* sh_off;    // shell -> prim offset
  const int* sh_K;      // shell -> primitive count
  const double* atoms;  // natom * 4: x, y, z, charge
  int natom, n;
  const double* boys;
  const double* expt;
  double *S, *T, *V;  // n x n
};

// E[i][j][t] for one axis, i <= la, j <= lb (+2 allowed), 1D MD recursion.
template <int LM>
__device__ __forceinline__ void hermite_1d(int la, int lb, double alpha, double beta, double a, double b,
                                           double E[OneIntDims<LM>::EI][OneIntDims<LM>::EJ][OneIntDims<LM>::ET]) {
  constexpr int kET = OneIntDims<LM>::ET;
  const double p = alpha + beta, inv2p = 0.5 / p;
  const double P = (alpha * a + beta * b) / p;
  const double xpa = P - a, xpb = P - b;
  const double mu = alpha * beta / p;
  for (int i = 0; i <= la; ++i)
    for (int j = 0; j <= lb; ++j)
      for (int t = 0; t < kET; ++t) E[i][j][t] = 0.0;
  E[0][0][0] = exp(-mu * (a - b) * (a - b));
  for (int i = 0; i <= la; ++i)
    for (int j = 0; j <= lb; ++j) {
      if (i == 0 && j == 0) continue;
      for (int t = 0; t <= i + j; ++t) {
        double v;
        if (i > 0) {
          v = xpa * E[i - 1][j][t];
          if (t > 0) v += inv2p * E[i - 1][j][t - 1];
          if (t + 1 <= i - 1 + j) v += (t + 1) * E[i - 1][j][t + 1];
        } else {
          v = xpb * E[i][j - 1][t];
          if (t > 0) v += inv2p * E[i][j - 1][t - 1];
          if (t + 1 <= i + j - 1) v += (t + 1) * E[i][j - 1][t + 1];
        }
        E[i][j][t] = v;
      }
    }
}

__device__ __forceinline__ double comp_norm(const int l[3]) {
  // 1/sqrt(prod (2 l_i - 1)!!)
  double d = 1.0;
  for (int k = 0; k < 3; ++k)
    for (int m = 2 * l[k] - 1; m > 1; m -= 2) d *= m;
  return rsqrt(d);
}

template <int LM>
__global__ void __launch_bounds__(128) oneint_kernel(const OneIntArgs a) {
  using Dm = OneIntDims<LM>;
  constexpr int kEI = Dm::EI, kEJ = Dm::EJ, kET = Dm::ET, kL = Dm::L;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  double* sm = reinterpret_cast<double*>(smem_raw);
  boys_stage<double, kL>(sm, a.boys, a.expt);
  __syncthreads();
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long npair = (long long)a.n * (a.n + 1) / 2;
  if (t >= npair) return;
  // t -> (mu, nu), mu >= nu
  int mu = (int)((sqrt(8.0 * (double)t + 1.0) - 1.0) * 0.5);
  while ((long long)mu * (mu + 1) / 2 > t) --mu;
  while ((long long)(mu + 1) * (mu + 2) / 2 <= t) ++mu;
  const int nu = (int)(t - (long long)mu * (mu + 1) / 2);
  const FuncInfo A = a.funcs[mu], B = a.funcs[nu];
  const double na = comp_norm(A.l), nb = comp_norm(B.l);
  const int pa = a.sh_off[A.shell], ka = a.sh_K[A.shell], pb = a.sh_off[B.shell], kb = a.sh_K[B.shell];
  double S = 0.0, Tk = 0.0, V = 0.0;
  double Ex[kEI][kEJ][kET], Ey[kEI][kEJ][kET], Ez[kEI][kEJ][kET];
  for (int i = 0; i < ka; ++i)
    for (int j = 0; j < kb; ++j) {
      const double al = a.exps[pa + i], be = a.exps[pb + j];
      const double cc = a.coefs[pa + i] * a.coefs[pb + j] * na * nb;
      const double p = al + be, inv_p = 1.0 / p;
      hermite_1d<LM>(A.l[0], B.l[0] + 2, al, be, A.c[0], B.c[0], Ex);
      hermite_1d<LM>(A.l[1], B.l[1] + 2, al, be, A.c[1], B.c[1], Ey);
      hermite_1d<LM>(A.l[2], B.l[2] + 2, al, be, A.c[2], B.c[2], Ez);
      const double pref = 5.56832799683170784528 * inv_p * sqrt(inv_p);  // (pi/p)^{3/2}
      const double sx = Ex[A.l[0]][B.l[0]][0], sy = Ey[A.l[1]][B.l[1]][0], sz = Ez[A.l[2]][B.l[2]][0];
      S += cc * pref * sx * sy * sz;
      auto t1d = [&](int li, int lj, double E[kEI][kEJ][kET]) {
        double v = be * (2.0 * lj + 1.0) * E[li][lj][0] - 2.0 * be * be * E[li][lj + 2][0];
        if (lj >= 2) v -= 0.5 * lj * (lj - 1) * E[li][lj - 2][0];
        return v;
      };
      Tk += cc * pref * (t1d(A.l[0], B.l[0], Ex) * sy * sz + sx * t1d(A.l[1], B.l[1], Ey) * sz +
                         sx * sy * t1d(A.l[2], B.l[2], Ez));
      // nuclear attraction
      const double P[3] = {(al * A.c[0] + be * B.c[0]) * inv_p, (al * A.c[1] + be * B.c[1]) * inv_p,
                           (al * A.c[2] + be * B.c[2]) * inv_p};
      const int mt = A.l[0] + B.l[0], mu_ = A.l[1] + B.l[1], mv = A.l[2] + B.l[2];
      const int L = mt + mu_ + mv;
      double vsum = 0.0;
      for (int at = 0; at < a.natom; ++at) {
        const double PC[3] = {P[0] - a.atoms[4 * at], P[1] - a.atoms[4 * at + 1], P[2] - a.atoms[4 * at + 2]};
        const double T = p * (PC[0] * PC[0] + PC[1] * PC[1] + PC[2] * PC[2]);
        double F[kL + 1];
        boys_eval<kL>(T, sm, F);
        // R^n_{tuv} for t+u+v <= L via the MD recursion, n <= L
        double R[kL + 1][kL + 1][kL + 1][kL + 1];  // [n][t][u][v]
        double m2p = 1.0;
        for (int n = 0; n <= L; ++n) {
          R[n][0][0][0] = m2p * F[n];
          m2p *= -2.0 * p;
        }
        for (int n = L - 1; n >= 0; --n)
          for (int tt = 0; tt <= L - n; ++tt)
            for (int uu = 0; uu <= L - n - tt; ++uu)
              for (int vv = 0; vv <= L - n - tt - uu; ++vv) {
                if (tt + uu + vv == 0) continue;
                double r;
                if (tt > 0) {
                  r = PC[0] * R[n + 1][tt - 1][uu][vv];
                  if (tt > 1) r += (tt - 1) * R[n + 1][tt - 2][uu][vv];
                } else if (uu > 0) {
                  r = PC[1] * R[n + 1][tt][uu - 1][vv];
                  if (uu > 1) r += (uu - 1) * R[n + 1][tt][uu - 2][vv];
                } else {
                  r = PC[2] * R[n + 1][tt][uu][vv - 1];
                  if (vv > 1) r += (vv - 1) * R[n + 1][tt][uu][vv - 2];
                }
                R[n][tt][uu][vv] = r;
              }
        double s = 0.0;
        for (int tt = 0; tt <= mt; ++tt)
          for (int uu = 0; uu <= mu_; ++uu)
            for (int vv = 0; vv <= mv; ++vv)
              s += Ex[A.l[0]][B.l[0]][tt] * Ey[A.l[1]][B.l[1]][uu] * Ez[A.l[2]][B.l[2]][vv] * R[0][tt][uu][vv];
        vsum += -a.atoms[4 * at + 3] * s;
      }
      V += cc * 2.0 * 3.14159265358979323846 * inv_p * vsum;
    }
  a.S[(size_t)mu * a.n + nu] = a.S[(size_t)nu * a.n + mu] = S;
  a.T[(size_t)mu * a.n + nu] = a.T[(size_t)nu * a.n + mu] = Tk;
  a.V[(size_t)mu * a.n + nu] = a.V[(size_t)nu * a.n + mu] = V;
}

// S, T, V (device, row-major n x n) of the context basis for the given nuclei.
int one_electron(hfg_ctx* ctx, int natom, const double* pos, const double* charge, double* dS, double* dT,
                 double* dV) {
  const int n = ctx->n;
  std::vector<FuncInfo> f(n);
  std::vector<int> off, K;
  for (size_t s = 0; s < ctx->shells.size(); ++s) {
    const Shell& sh = ctx->shells[s];
    off.push_back(sh.prim_off);
    K.push_back(sh.K);
    const int cnt = (sh.l + 1) * (sh.l + 2) / 2;
    int c = 0;
    // hf-rs component order (src/basis.rs:418-445)
    static const int d_order[6][3] = {{2, 0, 0}, {0, 2, 0}, {0, 0, 2}, {1, 1, 0}, {1, 0, 1}, {0, 1, 1}};
    for (int lx = sh.l; lx >= 0 && c < cnt; --lx)
      for (int ly = sh.l - lx; ly >= 0 && c < cnt; --ly) {
        FuncInfo& fi = f[sh.ao + c];
        for (int k = 0; k < 3; ++k) fi.c[k] = sh.c[k];
        if (sh.l == 2) {
          fi.l[0] = d_order[c][0];
          fi.l[1] = d_order[c][1];
          fi.l[2] = d_order[c][2];
        } else {
          fi.l[0] = lx;
          fi.l[1] = ly;
          fi.l[2] = sh.l - lx - ly;
        }
        fi.shell = (int)s;
        ++c;
      }
  }
  std::vector<double> at(4 * natom);
  for (int i = 0; i < natom; ++i) {
    for (int k = 0; k < 3; ++k) at[4 * i + k] = pos[3 * i + k];
    at[4 * i + 3] = charge[i];
  }
  DevBuf<FuncInfo> df;
  DevBuf<double> dex, dco, dat;
  DevBuf<int> doff, dK;
  int rc = HFG_OK;
  auto chk = [&](cudaError_t e, const char* w) {
    if (rc == HFG_OK) rc = cuda_check(ctx, e, w);
  };
  chk(df.alloc(n), "alloc");
  chk(dex.alloc(ctx->exps.size()), "alloc");
  chk(dco.alloc(ctx->coefs.size()), "alloc");
  chk(dat.alloc(at.size() + 1), "alloc");
  chk(doff.alloc(off.size()), "alloc");
  chk(dK.alloc(K.size()), "alloc");
  if (rc != HFG_OK) return rc;
  chk(cudaMemcpyAsync(df.p, f.data(), n * sizeof(FuncInfo), cudaMemcpyHostToDevice, ctx->stream), "copy");
  chk(cudaMemcpyAsync(dex.p, ctx->exps.data(), ctx->exps.size() * 8, cudaMemcpyHostToDevice, ctx->stream), "copy");
  chk(cudaMemcpyAsync(dco.p, ctx->coefs.data(), ctx->coefs.size() * 8, cudaMemcpyHostToDevice, ctx->stream), "copy");
  chk(cudaMemcpyAsync(dat.p, at.data(), at.size() * 8, cudaMemcpyHostToDevice, ctx->stream), "copy");
  chk(cudaMemcpyAsync(doff.p, off.data(), off.size() * 4, cudaMemcpyHostToDevice, ctx->stream), "copy");
  chk(cudaMemcpyAsync(dK.p, K.data(), K.size() * 4, cudaMemcpyHostToDevice, ctx->stream), "copy");
  OneIntArgs a{df.p, dex.p, dco.p, doff.p, dK.p, dat.p, natom, n, ctx->d_boys64.p, ctx->d_expt64.p, dS, dT, dV};
  const long long npair = (long long)n * (n + 1) / 2;
  const int smem = (int)boys_smem_bytes<double>();
  auto kern = ctx->lmax <= 2 ? oneint_kernel<2> : oneint_kernel<3>;
  chk(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, smem), "attr");
  if (npair > 0) kern<<<(unsigned)((npair + 127) / 128), 128, smem, ctx->stream>>>(a);
  chk(cudaGetLastError(), "oneint kernel");
  chk(cudaStreamSynchronize(ctx->stream), "oneint sync");
  return rc;
}

}  // namespace hfg
