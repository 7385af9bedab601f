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

// One-electron part of the analytic nuclear gradient, as hf-rs's
// compute_gradient_from_density (src/gradient.rs:372-455): for the basis
// derivative d/dA_x phi_mu = 2 alpha phi_{mu+1x} - l_x phi_{mu-1x} of every
// function on atom A,
//   g_A += 2 sum_nu [P_mu,nu (dT + dV)_mu,nu - W_mu,nu dS_mu,nu],
// and the operator derivative of the nuclear attraction (by translational
// invariance)  g_C -= 2 sum_mu,nu P_mu,nu (d mu | V_C | nu).  One block per
// function mu, threads over nu; per-atom sums in shared memory.
struct OneGradArgs {
  const FuncInfo* funcs;
  const double* exps;
  const double* coefs;
  const int* sh_off;
  const int* sh_K;
  const double* atoms;  // natom * 4: x, y, z, charge
  const int* func_atom;
  int natom, n;
  const double* boys;
  const double* expt;
  const double* P;  // total density
  const double* W;  // energy-weighted density
  double* grad;     // natom * 3
};

__global__ void __launch_bounds__(128) oneint_grad_kernel(const OneGradArgs a) {
  constexpr int LM = 3;
  using Dm = OneIntDims<LM>;
  constexpr int kEI = Dm::EI, kEJ = Dm::EJ, kET = Dm::ET, kL = Dm::L;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  double* sm = reinterpret_cast<double*>(smem_raw);
  double* gacc = sm + boys_smem_bytes<double>() / sizeof(double);  // natom * 3
  boys_stage<double, kL>(sm, a.boys, a.expt);
  for (int x = threadIdx.x; x < 3 * a.natom; x += blockDim.x) gacc[x] = 0.0;
  __syncthreads();
  const int mu = blockIdx.x;
  const FuncInfo A = a.funcs[mu];
  const int atA = a.func_atom[mu];
  const double na = comp_norm(A.l);
  const int pa = a.sh_off[A.shell], ka = a.sh_K[A.shell];
  for (int nu = threadIdx.x; nu < a.n; nu += blockDim.x) {
    const FuncInfo B = a.funcs[nu];
    const double Pmn = a.P[(size_t)mu * a.n + nu], Wmn = a.W[(size_t)mu * a.n + nu];
    if (Pmn == 0.0 && Wmn == 0.0) continue;
    const double nb = comp_norm(B.l);
    const int pb = a.sh_off[B.shell], kb = a.sh_K[B.shell];
    double dS[3] = {0, 0, 0}, dT[3] = {0, 0, 0}, dV[3] = {0, 0, 0};
    double Ex[kEI][kEJ][kET], Ey[kEI][kEJ][kET], Ez[kEI][kEJ][kET];
    for (int i = 0; i < ka; ++i)
      for (int j = 0; j < kb; ++j) {
        const double al = a.exps[pa + i], be = a.exps[pb + j];
        const double cc = a.coefs[pa + i] * a.coefs[pb + j] * na * nb;
        const double p = al + be, inv_p = 1.0 / p;
        hermite_1d<LM>(A.l[0] + 1, B.l[0] + 2, al, be, A.c[0], B.c[0], Ex);
        hermite_1d<LM>(A.l[1] + 1, B.l[1] + 2, al, be, A.c[1], B.c[1], Ey);
        hermite_1d<LM>(A.l[2] + 1, B.l[2] + 2, al, be, A.c[2], B.c[2], Ez);
        const double pref = 5.56832799683170784528 * inv_p * sqrt(inv_p);  // (pi/p)^{3/2}
        double (*E[3])[kEJ][kET] = {Ex, Ey, Ez};
        // overlap and kinetic factors of axis k for the a-power ia (b fixed)
        auto s1 = [&](int k, int ia) { return E[k][ia][B.l[k]][0]; };
        auto t1 = [&](int k, int ia) {
          const int lj = B.l[k];
          double v = be * (2.0 * lj + 1.0) * E[k][ia][lj][0] - 2.0 * be * be * E[k][ia][lj + 2][0];
          if (lj >= 2) v -= 0.5 * lj * (lj - 1) * E[k][ia][lj - 2][0];
          return v;
        };
        for (int tau = 0; tau < 3; ++tau)
          for (int term = 0; term < 2; ++term) {
            if (term == 1 && A.l[tau] == 0) break;
            const double f = term == 0 ? 2.0 * al : -(double)A.l[tau];
            int ap[3] = {A.l[0], A.l[1], A.l[2]};
            ap[tau] += term == 0 ? 1 : -1;
            const double sx = s1(0, ap[0]), sy = s1(1, ap[1]), sz = s1(2, ap[2]);
            dS[tau] += cc * pref * f * sx * sy * sz;
            dT[tau] += cc * pref * f * (t1(0, ap[0]) * sy * sz + sx * t1(1, ap[1]) * sz + sx * sy * t1(2, ap[2]));
          }
        // nuclear attraction: R per nucleus up to the raised total
        const double P3[3] = {(al * A.c[0] + be * B.c[0]) * inv_p, (al * A.c[1] + be * B.c[1]) * inv_p,
                              (al * A.c[2] + be * B.c[2]) * inv_p};
        const int L = A.l[0] + A.l[1] + A.l[2] + 1 + B.l[0] + B.l[1] + B.l[2];
        for (int at = 0; at < a.natom; ++at) {
          const double PC[3] = {P3[0] - a.atoms[4 * at], P3[1] - a.atoms[4 * at + 1], P3[2] - a.atoms[4 * at + 2]};
          const double T = p * (PC[0] * PC[0] + PC[1] * PC[1] + PC[2] * PC[2]);
          double F[kL + 1];
          boys_eval<kL>(T, sm, F);
          // R^{n}_{tuv} level by level (n = L .. 0), two levels held at a time;
          // level 0 ends in Ra
          double Ra[kL + 1][kL + 1][kL + 1], Rb[kL + 1][kL + 1][kL + 1];
          for (int n = L; n >= 0; --n) {
            double(*cur)[kL + 1][kL + 1] = (n & 1) ? Rb : Ra;
            double(*prev)[kL + 1][kL + 1] = (n & 1) ? Ra : Rb;
            double w = 1.0;
            for (int k = 0; k < n; ++k) w *= -2.0 * p;
            cur[0][0][0] = w * F[n];
            for (int tt = 0; tt <= L - n; ++tt)
              for (int uu = 0; uu <= L - n - tt; ++uu)
                for (int vv = 0; vv <= L - n - tt - uu; ++vv) {
                  if (tt + uu + vv == 0) continue;
                  double r;
                  if (tt > 0) {
                    r = PC[0] * prev[tt - 1][uu][vv];
                    if (tt > 1) r += (tt - 1) * prev[tt - 2][uu][vv];
                  } else if (uu > 0) {
                    r = PC[1] * prev[tt][uu - 1][vv];
                    if (uu > 1) r += (uu - 1) * prev[tt][uu - 2][vv];
                  } else {
                    r = PC[2] * prev[tt][uu][vv - 1];
                    if (vv > 1) r += (vv - 1) * prev[tt][uu][vv - 2];
                  }
                  cur[tt][uu][vv] = r;
                }
          }
          const double zf = -a.atoms[4 * at + 3] * 2.0 * 3.14159265358979323846 * inv_p * cc;
          for (int tau = 0; tau < 3; ++tau) {
            double dv = 0.0;
            for (int term = 0; term < 2; ++term) {
              if (term == 1 && A.l[tau] == 0) break;
              const double f = term == 0 ? 2.0 * al : -(double)A.l[tau];
              int ap[3] = {A.l[0], A.l[1], A.l[2]};
              ap[tau] += term == 0 ? 1 : -1;
              double sum = 0.0;
              for (int tt = 0; tt <= ap[0] + B.l[0]; ++tt)
                for (int uu = 0; uu <= ap[1] + B.l[1]; ++uu)
                  for (int vv = 0; vv <= ap[2] + B.l[2]; ++vv)
                    sum += Ex[ap[0]][B.l[0]][tt] * Ey[ap[1]][B.l[1]][uu] * Ez[ap[2]][B.l[2]][vv] * Ra[tt][uu][vv];
              dv += f * sum;
            }
            dv *= zf;
            dV[tau] += dv;
            // the operator derivative acting on nucleus `at`
            atomicAdd(&gacc[3 * at + tau], -2.0 * Pmn * dv);
          }
        }
      }
    for (int tau = 0; tau < 3; ++tau) atomicAdd(&gacc[3 * atA + tau], 2.0 * (Pmn * (dT[tau] + dV[tau]) - Wmn * dS[tau]));
  }
  __syncthreads();
  for (int x = threadIdx.x; x < 3 * a.natom; x += blockDim.x)
    if (gacc[x] != 0.0) atomicAdd(a.grad + x, gacc[x]);
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

// One-electron gradient terms (device) for nuclei (positions, charges),
// added into grad (host, natom * 3).
int one_electron_gradient(hfg_ctx* ctx, int natom, const double* pos, const double* charge, const double* P,
                          const double* W, double* grad) {
  const int n = ctx->n;
  std::vector<FuncInfo> f(n);
  std::vector<int> off, K, fatom(n);
  for (size_t s = 0; s < ctx->shells.size(); ++s) {
    const Shell& sh = ctx->shells[s];
    off.push_back(sh.prim_off);
    K.push_back(sh.K);
    const int cnt = (sh.l + 1) * (sh.l + 2) / 2;
    static const int d_order[6][3] = {{2, 0, 0}, {0, 2, 0}, {0, 0, 2}, {1, 1, 0}, {1, 0, 1}, {0, 1, 1}};
    int c = 0;
    for (int lx = sh.l; lx >= 0 && c < cnt; --lx)
      for (int ly = sh.l - lx; ly >= 0 && c < cnt; --ly) {
        FuncInfo& fi = f[sh.ao + c];
        for (int k = 0; k < 3; ++k) fi.c[k] = sh.c[k];
        if (sh.l == 2) {
          for (int k = 0; k < 3; ++k) fi.l[k] = d_order[c][k];
        } else {
          fi.l[0] = lx;
          fi.l[1] = ly;
          fi.l[2] = sh.l - lx - ly;
        }
        fi.shell = (int)s;
        fatom[sh.ao + c] = sh.atom;
        ++c;
      }
  }
  std::vector<double> at(4 * natom);
  for (int i = 0; i < natom; ++i) {
    for (int k = 0; k < 3; ++k) at[4 * i + k] = pos[3 * i + k];
    at[4 * i + 3] = charge[i];
  }
  const size_t nn = (size_t)n * n;
  DevBuf<FuncInfo> df;
  DevBuf<double> dex, dco, dat, dP, dW, dg;
  DevBuf<int> doff, dK, dfa;
  int rc = HFG_OK;
  auto chk = [&](cudaError_t e, const char* w) {
    if (rc == HFG_OK) rc = cuda_check(ctx, e, w);
  };
  chk(df.alloc(n), "alloc");
  chk(dex.alloc(ctx->exps.size()), "alloc");
  chk(dco.alloc(ctx->coefs.size()), "alloc");
  chk(dat.alloc(at.size() + 1), "alloc");
  chk(dP.alloc(nn), "alloc");
  chk(dW.alloc(nn), "alloc");
  chk(dg.alloc(3 * (size_t)natom), "alloc");
  chk(doff.alloc(off.size()), "alloc");
  chk(dK.alloc(K.size()), "alloc");
  chk(dfa.alloc(n), "alloc");
  if (rc != HFG_OK) return rc;
  cudaStream_t st = ctx->stream;
  chk(cudaMemcpyAsync(df.p, f.data(), n * sizeof(FuncInfo), cudaMemcpyHostToDevice, st), "copy");
  chk(cudaMemcpyAsync(dex.p, ctx->exps.data(), ctx->exps.size() * 8, cudaMemcpyHostToDevice, st), "copy");
  chk(cudaMemcpyAsync(dco.p, ctx->coefs.data(), ctx->coefs.size() * 8, cudaMemcpyHostToDevice, st), "copy");
  chk(cudaMemcpyAsync(dat.p, at.data(), at.size() * 8, cudaMemcpyHostToDevice, st), "copy");
  chk(cudaMemcpyAsync(dP.p, P, nn * 8, cudaMemcpyHostToDevice, st), "copy");
  chk(cudaMemcpyAsync(dW.p, W, nn * 8, cudaMemcpyHostToDevice, st), "copy");
  chk(cudaMemcpyAsync(doff.p, off.data(), off.size() * 4, cudaMemcpyHostToDevice, st), "copy");
  chk(cudaMemcpyAsync(dK.p, K.data(), K.size() * 4, cudaMemcpyHostToDevice, st), "copy");
  chk(cudaMemcpyAsync(dfa.p, fatom.data(), n * 4, cudaMemcpyHostToDevice, st), "copy");
  chk(cudaMemsetAsync(dg.p, 0, 3 * (size_t)natom * 8, st), "memset");
  OneGradArgs a{df.p, dex.p, dco.p, doff.p, dK.p, dat.p, dfa.p, natom, n, ctx->d_boys64.p, ctx->d_expt64.p,
                dP.p, dW.p, dg.p};
  const size_t smem = boys_smem_bytes<double>() + 3 * (size_t)natom * sizeof(double);
  chk(cudaFuncSetAttribute(oneint_grad_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem), "attr");
  if (n > 0) oneint_grad_kernel<<<(unsigned)n, 128, smem, st>>>(a);
  chk(cudaGetLastError(), "one-electron gradient kernel");
  std::vector<double> g(3 * (size_t)natom);
  chk(cudaMemcpyAsync(g.data(), dg.p, g.size() * 8, cudaMemcpyDeviceToHost, st), "copy");
  chk(cudaStreamSynchronize(st), "sync");
  if (rc == HFG_OK)
    for (size_t x = 0; x < g.size(); ++x) grad[x] += g[x];
  return rc;
}

}  // namespace hfg
