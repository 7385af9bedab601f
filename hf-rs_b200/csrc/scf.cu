// Device-resident SCF driver: RHF and UHF with CDIIS, the spherical AO space
// and the canonical orthogonaliser, and the mixed-precision mode with FP64
// refinement iterations.
//
// Stands in for hf-rs's run_scf_in_space_with_convergence (src/scf.rs:410-627)
// and run_uhf_in_space_with_convergence (src/scf.rs:691-979) with
// ConvAlgo::Cdiis: the same energy expression, commutator error
// X^T (FPS - SPF) X, convergence tests (|dE| < tol, max|e| < residual,
// rmsd(P - P_prev) < density), CDIIS with 8 vectors (src/diis.rs:72-219),
// UHF damping 0.7/0.3 in iterations 1-2, and the final diagonalisation of the
// true Fock matrix.  Density, Fock, DIIS history and orbitals stay on the
// device; only scalars (energies, norms, the DIIS overlap matrix) come back to
// the host each iteration.  Linear algebra: cuBLAS DGEMM, cuSOLVER Dsyevd.
//
// All matrices here are column-major (the native cuBLAS/cuSOLVER layout);
// the symmetric ones (S, H, P, F, J, K) are identical in row-major.
#include <cublas_v2.h>
#include <cuda_runtime.h>
#include <cusolverDn.h>

#include <algorithm>
#include <array>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <map>
#include <memory>
#include <vector>

#include "hfg_ctx.h"

namespace hfg {

int one_electron(hfg_ctx* ctx, int natom, const double* pos, const double* charge, double* dS, double* dT,
                 double* dV);

namespace {

__global__ void axpby_kernel(double* __restrict__ y, const double* __restrict__ x, double a, double b, long long n) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) y[i] = a * x[i] + b * y[i];
}

// out = A - A^T (n x n); the commutator FPS - SPF = FPS - (FPS)^T.
__global__ void antisym_kernel(const double* __restrict__ A, double* __restrict__ out, int n) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)n * n) return;
  const int i = (int)(t / n), j = (int)(t % n);
  out[t] = A[t] - A[(long long)j * n + i];
}

// Eigenvector phase of hf-rs (src/matrix.rs:175-189): the component of
// largest magnitude (first one on ties) made positive.  Column-major V.
__global__ void phase_kernel(double* __restrict__ V, int m, int ncols) {
  const int col = blockIdx.x;
  if (col >= ncols) return;
  double* v = V + (size_t)col * m;
  __shared__ double bv[256];
  __shared__ int bi[256];
  double best = -1.0;
  int idx = 0;
  for (int r = threadIdx.x; r < m; r += blockDim.x) {
    const double a = fabs(v[r]);
    if (a > best) {
      best = a;
      idx = r;
    }
  }
  bv[threadIdx.x] = best;
  bi[threadIdx.x] = idx;
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s) {
      const double o = bv[threadIdx.x + s];
      const int oi = bi[threadIdx.x + s];
      if (o > bv[threadIdx.x] || (o == bv[threadIdx.x] && oi < bi[threadIdx.x])) {
        bv[threadIdx.x] = o;
        bi[threadIdx.x] = oi;
      }
    }
    __syncthreads();
  }
  const double sign = v[bi[0]] < 0.0 ? -1.0 : 1.0;
  __syncthreads();
  if (sign < 0.0)
    for (int r = threadIdx.x; r < m; r += blockDim.x) v[r] = -v[r];
}

__global__ void scale_cols_kernel(double* __restrict__ V, const double* __restrict__ w, int m, int ncols,
                                  int first) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)m * ncols) return;
  const int col = (int)(t / m);
  V[t] *= rsqrt(w[first + col]);
}

inline unsigned nblk(long long n, int b = 256) { return (unsigned)((n + b - 1) / b); }

// Gaussian elimination with partial pivoting (first maximum wins), None
// below a 1e-28 pivot: the bordered CDIIS system of src/diis.rs:532-580.
bool solve_small(std::vector<double> a, std::vector<double>& x, int n) {
  for (int i = 0; i < n; ++i) {
    int mr = i;
    double mv = std::fabs(a[i * n + i]);
    for (int k = i + 1; k < n; ++k)
      if (std::fabs(a[k * n + i]) > mv) {
        mv = std::fabs(a[k * n + i]);
        mr = k;
      }
    if (mv < 1e-28) return false;
    if (mr != i) {
      std::swap(x[i], x[mr]);
      for (int c = 0; c < n; ++c) std::swap(a[i * n + c], a[mr * n + c]);
    }
    const double d = a[i * n + i];
    for (int j = i + 1; j < n; ++j) {
      const double f = a[j * n + i] / d;
      a[j * n + i] = f;
      for (int k = i + 1; k < n; ++k) a[j * n + k] -= f * a[i * n + k];
      x[j] -= f * x[i];
    }
  }
  for (int i = n - 1; i >= 0; --i) {
    double s = x[i];
    for (int k = i + 1; k < n; ++k) s -= a[i * n + k] * x[k];
    x[i] = s / a[i * n + i];
  }
  return true;
}

double dfact(int n) {
  double r = 1.0;
  for (int k = n; k > 0; k -= 2) r *= k;
  return r;
}
double fact(int n) {
  double r = 1.0;
  for (int k = 2; k <= n; ++k) r *= k;
  return r;
}

// Real solid harmonic of degree l, order m, as Cartesian polynomial
// coefficients over powers (px, py, pz): PySCF order m = -l..l, sine for
// m < 0, cosine for m > 0 (the convention of src/ao.rs:94-131).
void solid_harmonic(int l, int m, std::vector<std::pair<std::array<int, 3>, double>>& out) {
  out.clear();
  const int am = std::abs(m);
  const double norm = std::sqrt(fact(l - am) / fact(l + am)) * (am == 0 ? 1.0 : std::sqrt(2.0));
  for (int k = 0; k <= (l - am) / 2; ++k) {
    const double coef = ((k & 1) ? -1.0 : 1.0) * fact(2 * l - 2 * k) /
                        (std::pow(2.0, l) * fact(k) * fact(l - k) * fact(l - am - 2 * k));
    for (int y = 0; y <= am; ++y) {
      double phase = 0.0;
      const int r = y % 4;
      if ((m < 0 && r == 1) || (m >= 0 && r == 0)) phase = 1.0;
      else if ((m < 0 && r == 3) || (m >= 0 && r == 2)) phase = -1.0;
      if (phase == 0.0) continue;
      const double binom = fact(am) / (fact(y) * fact(am - y));
      for (int xx = 0; xx <= k; ++xx)
        for (int yy = 0; yy <= k - xx; ++yy) {
          const int zz = k - xx - yy;
          const std::array<int, 3> pw = {am - y + 2 * xx, y + 2 * yy, l - am - 2 * k + 2 * zz};
          const double mult = fact(k) / (fact(xx) * fact(yy) * fact(zz));
          bool found = false;
          for (auto& e : out)
            if (e.first == pw) {
              e.second += norm * coef * binom * phase * mult;
              found = true;
            }
          if (!found) out.push_back({pw, norm * coef * binom * phase * mult});
        }
    }
  }
}

// cuBLAS / cuSOLVER handles are created once per host thread and device and
// reused by every SCF that thread runs (handle creation costs milliseconds,
// which matters for streams of small jobs); each call binds its stream.
struct ThreadHandles {
  int device = -1;
  cublasHandle_t blas = nullptr;
  cusolverDnHandle_t solver = nullptr;
  ~ThreadHandles() {
    if (blas) cublasDestroy(blas);
    if (solver) cusolverDnDestroy(solver);
  }
};
thread_local ThreadHandles tl_handles;

struct Scf {
  hfg_ctx* ctx;
  cublasHandle_t blas = nullptr;
  cusolverDnHandle_t solver = nullptr;
  int n = 0, m = 0;
  DevBuf<double> S, H, T, V, X, W, tmp1, tmp2, evals, work;
  DevBuf<int> info;
  int lwork = 0;
  int gemm(cublasOperation_t ta, cublasOperation_t tb, int M, int N, int K, double alpha, const double* A, int lda,
           const double* B, int ldb, double beta, double* C, int ldc) {
    const cublasStatus_t s = cublasDgemm(blas, ta, tb, M, N, K, &alpha, A, lda, B, ldb, &beta, C, ldc);
    return s == CUBLAS_STATUS_SUCCESS ? HFG_OK : set_error(ctx, HFG_ERR_CUDA, "cublasDgemm failed");
  }
  double dot(const double* a, const double* b, long long len) {
    double r = 0.0;
    cublasDdot(blas, (int)len, a, 1, b, 1, &r);
    return r;
  }
  double maxabs(const double* a, long long len) {
    int i = 0;
    cublasIdamax(blas, (int)len, a, 1, &i);
    double v = 0.0;
    cudaMemcpyAsync(&v, a + (i - 1), 8, cudaMemcpyDeviceToHost, ctx->stream);
    cudaStreamSynchronize(ctx->stream);
    return std::fabs(v);
  }
  // symmetric eigendecomposition of A (m x m, column-major, overwritten by
  // the eigenvectors, ascending eigenvalues in w)
  int eigh(double* A, double* w, int dim) {
    int need = 0;
    cusolverDnDsyevd_bufferSize(solver, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_LOWER, dim, A, dim, w, &need);
    if (need > lwork) {
      int rc = cuda_check(ctx, work.alloc(need), "alloc syevd work");
      if (rc != HFG_OK) return rc;
      lwork = need;
    }
    const cusolverStatus_t s =
        cusolverDnDsyevd(solver, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_LOWER, dim, A, dim, w, work.p, lwork, info.p);
    if (s != CUSOLVER_STATUS_SUCCESS) return set_error(ctx, HFG_ERR_CUDA, "cusolverDnDsyevd failed");
    return HFG_OK;
  }
};

}  // namespace
}  // namespace hfg

namespace hfg {
namespace {
// One-electron integrals, H = T + V, and the orthogonaliser X (n x m) of the
// Cartesian or real spherical AO space with cutoff 1e-8.
int scf_setup(hfg_ctx* ctx, const hfg_scf_opts* o, Scf& s, int& m_out) {
  const int n = ctx->n;
  int rc = HFG_OK;
#define CK(call)                         \
  do {                                   \
    rc = cuda_check(ctx, (call), #call); \
    if (rc != HFG_OK) return rc;         \
  } while (0)
#define RK(call)                 \
  do {                           \
    rc = (call);                 \
    if (rc != HFG_OK) return rc; \
  } while (0)
  s.ctx = ctx;
  s.n = n;
  if (tl_handles.device != ctx->device) {
    if (tl_handles.blas) cublasDestroy(tl_handles.blas);
    if (tl_handles.solver) cusolverDnDestroy(tl_handles.solver);
    tl_handles.blas = nullptr;
    tl_handles.solver = nullptr;
    if (cublasCreate(&tl_handles.blas) != CUBLAS_STATUS_SUCCESS) return set_error(ctx, HFG_ERR_CUDA, "cublasCreate");
    if (cusolverDnCreate(&tl_handles.solver) != CUSOLVER_STATUS_SUCCESS)
      return set_error(ctx, HFG_ERR_CUDA, "cusolverDnCreate");
    tl_handles.device = ctx->device;
  }
  s.blas = tl_handles.blas;
  s.solver = tl_handles.solver;
  cublasSetStream(s.blas, ctx->stream);
  cusolverDnSetStream(s.solver, ctx->stream);
  const long long nn = (long long)n * n;
  CK(s.S.alloc(nn));
  CK(s.H.alloc(nn));
  CK(s.T.alloc(nn));
  CK(s.V.alloc(nn));
  CK(s.tmp1.alloc(nn));
  CK(s.tmp2.alloc(nn));
  CK(s.evals.alloc(n));
  CK(s.info.alloc(1));
  RK(one_electron(ctx, o->natom, o->positions, o->charges, s.S.p, s.T.p, s.V.p));
  CK(cudaMemcpyAsync(s.H.p, s.T.p, nn * 8, cudaMemcpyDeviceToDevice, ctx->stream));
  axpby_kernel<<<nblk(nn), 256, 0, ctx->stream>>>(s.H.p, s.V.p, 1.0, 1.0, nn);
  CK(cudaGetLastError());

  // Cartesian -> physical AO transform (identity or real spherical;
  // src/ao.rs:167-217), then the canonical orthogonaliser with cutoff 1e-8
  // (src/ao.rs:58-67, src/matrix.rs:329-346).
  int nsph = 0;
  for (const auto& sh : ctx->shells) nsph += o->spherical ? 2 * sh.l + 1 : (sh.l + 1) * (sh.l + 2) / 2;
  std::vector<double> Tm((size_t)n * nsph, 0.0);  // column-major n x nsph
  {
    std::vector<double> Sh;
    if (o->spherical) {
      Sh.resize(nn);
      CK(cudaMemcpyAsync(Sh.data(), s.S.p, nn * 8, cudaMemcpyDeviceToHost, ctx->stream));
      CK(cudaStreamSynchronize(ctx->stream));
    }
    int col = 0;
    std::vector<std::pair<std::array<int, 3>, double>> poly;
    for (const auto& sh : ctx->shells) {
      const int cnt = (sh.l + 1) * (sh.l + 2) / 2;
      if (!o->spherical || sh.l <= 1) {
        for (int r = 0; r < cnt; ++r) Tm[(size_t)col++ * n + sh.ao + r] = 1.0;
        continue;
      }
      // Cartesian components in hf-rs order (d: xx, yy, zz, xy, xz, yz; f and
      // above lexicographic, src/basis.rs:418-445)
      std::vector<std::array<int, 3>> comps;
      if (sh.l == 2) {
        comps = {{2, 0, 0}, {0, 2, 0}, {0, 0, 2}, {1, 1, 0}, {1, 0, 1}, {0, 1, 1}};
      } else {
        for (int lx = sh.l; lx >= 0; --lx)
          for (int ly = sh.l - lx; ly >= 0; --ly) comps.push_back({lx, ly, sh.l - lx - ly});
      }
      for (int mm = -sh.l; mm <= sh.l; ++mm) {
        solid_harmonic(sh.l, mm, poly);
        std::vector<double> c(cnt, 0.0);
        for (int r = 0; r < cnt; ++r) {
          double w = std::sqrt(dfact(2 * comps[r][0] - 1) * dfact(2 * comps[r][1] - 1) * dfact(2 * comps[r][2] - 1));
          for (auto& e : poly)
            if (e.first == comps[r]) c[r] = e.second * w;
        }
        double norm = 0.0;
        for (int i = 0; i < cnt; ++i)
          for (int j = 0; j < cnt; ++j) norm += c[i] * Sh[(size_t)(sh.ao + i) * n + sh.ao + j] * c[j];
        if (!(norm > 0)) return set_error(ctx, HFG_ERR_INTEGRAL, "invalid spherical normalization");
        for (int r = 0; r < cnt; ++r) Tm[(size_t)col * n + sh.ao + r] = c[r] / std::sqrt(norm);
        ++col;
      }
    }
  }
  DevBuf<double> dT2;
  CK(dT2.alloc(Tm.size()));
  CK(cudaMemcpyAsync(dT2.p, Tm.data(), Tm.size() * 8, cudaMemcpyHostToDevice, ctx->stream));
  // s' = T^T S T (nsph x nsph)
  RK(s.gemm(CUBLAS_OP_N, CUBLAS_OP_N, n, nsph, n, 1.0, s.S.p, n, dT2.p, n, 0.0, s.tmp1.p, n));
  RK(s.gemm(CUBLAS_OP_T, CUBLAS_OP_N, nsph, nsph, n, 1.0, dT2.p, n, s.tmp1.p, n, 0.0, s.tmp2.p, nsph));
  RK(s.eigh(s.tmp2.p, s.evals.p, nsph));
  std::vector<double> w(nsph);
  CK(cudaMemcpyAsync(w.data(), s.evals.p, nsph * 8, cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  if (w[0] < -1e-8) return set_error(ctx, HFG_ERR_INTEGRAL, "overlap has a negative eigenvalue");
  int first = 0;
  while (first < nsph && w[first] < 1e-8) ++first;
  const int m = nsph - first;
  if (m <= 0) return set_error(ctx, HFG_ERR_INTEGRAL, "overlap has zero retained rank");
  s.m = m;
  // U_keep / sqrt(w), then X = T U_keep diag(w^-1/2)  (n x m)
  phase_kernel<<<nsph, 256, 0, ctx->stream>>>(s.tmp2.p, nsph, nsph);
  scale_cols_kernel<<<nblk((long long)nsph * m), 256, 0, ctx->stream>>>(s.tmp2.p + (size_t)first * nsph, s.evals.p,
                                                                       nsph, m, first);
  CK(s.X.alloc((size_t)n * m));
  RK(s.gemm(CUBLAS_OP_N, CUBLAS_OP_N, n, m, nsph, 1.0, dT2.p, n, s.tmp2.p + (size_t)first * nsph, nsph, 0.0, s.X.p, n));

  m_out = m;
  return HFG_OK;
#undef CK
#undef RK
}

// ---------------------------------------------------------------------------
// Superposition of atomic densities (src/sad.rs:24-259): for each element
// (keyed by nuclear charge and its basis functions) a spin-averaged atomic
// RHF with fractional occupations -- degenerate levels (within 1e-6) share
// their electrons equally -- converged with CDIIS(8) and 0.5 damping for the
// first five iterations (|dE| < 1e-11, rmsd(D - D_next) < 1e-9, max|FDS - SDF|
// < 1e-8).  Hydrogen's atomic Fock operator is H alone.  Results are cached
// per element; the molecular guess is their block-diagonal superposition
// rescaled to Tr(PS) = N.
std::mutex g_sad_mu;
std::map<std::vector<double>, std::vector<double>> g_sad_cache;

std::vector<double> occupations(const std::vector<double>& eps, double nel) {
  std::vector<double> occ(eps.size(), 0.0);
  double left = nel;
  size_t i = 0;
  while (i < eps.size() && left > 1e-12) {
    size_t end = i + 1;
    while (end < eps.size() && std::fabs(eps[end] - eps[i]) < 1e-6) ++end;
    const double pop = std::min(left, 2.0 * (double)(end - i));
    for (size_t k = i; k < end; ++k) occ[k] = pop / (double)(end - i);
    left -= pop;
    i = end;
  }
  return occ;
}

__global__ void scale_cols_by(double* __restrict__ C, const double* __restrict__ w, int n, int m) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t < (long long)n * m) C[t] *= w[t / n];
}

// Atomic fractional HF density of the functions [f0, f1) of `ctx` (one atom).
int atomic_density(hfg_ctx* ctx, int f0, int f1, double Z, std::vector<double>& out) {
  const int n = f1 - f0;
  // the atom's functions at the origin, as an hfg_basis
  std::vector<double> center(3 * n, 0.0), exps, coefs;
  std::vector<int> lxyz(3 * n), atom(n, 0), off(1, 0);
  for (const auto& sh : ctx->shells) {
    if (sh.ao < f0 || sh.ao >= f1) continue;
    std::vector<std::array<int, 3>> comps;
    if (sh.l == 2) comps = {{2, 0, 0}, {0, 2, 0}, {0, 0, 2}, {1, 1, 0}, {1, 0, 1}, {0, 1, 1}};
    else
      for (int lx = sh.l; lx >= 0; --lx)
        for (int ly = sh.l - lx; ly >= 0; --ly) comps.push_back({lx, ly, sh.l - lx - ly});
    for (size_t c = 0; c < comps.size(); ++c) {
      const int f = sh.ao + (int)c - f0;
      for (int k = 0; k < 3; ++k) lxyz[3 * f + k] = comps[c][k];
      const double sc = 1.0 / std::sqrt(dfact(2 * comps[c][0] - 1) * dfact(2 * comps[c][1] - 1) * dfact(2 * comps[c][2] - 1));
      for (int q = 0; q < sh.K; ++q) {
        exps.push_back(ctx->exps[sh.prim_off + q]);
        coefs.push_back(ctx->coefs[sh.prim_off + q] * sc);
      }
      off.push_back((int)exps.size());
    }
  }
  hfg_basis b{n, center.data(), lxyz.data(), atom.data(), off.data(), exps.data(), coefs.data()};
  hfg_ctx* ac = nullptr;
  int rc = hfg_ctx_create(&b, ctx->device, ctx->stream, &ac);
  if (rc != HFG_OK) {
    if (ac) hfg_ctx_destroy(ac);
    return set_error(ctx, rc, "SAD atomic context");
  }
  std::unique_ptr<hfg_ctx, int (*)(hfg_ctx*)> guard(ac, hfg_ctx_destroy);
  hfg_scf_opts o;
  hfg_scf_opts_default(&o);
  const double origin[3] = {0.0, 0.0, 0.0};
  o.natom = 1;
  o.positions = origin;
  o.charges = &Z;
  Scf s;
  int m = 0;
  rc = scf_setup(ac, &o, s, m);
  if (rc != HFG_OK) return set_error(ctx, rc, "SAD setup: " + ac->err);
  const long long nn = (long long)n * n;
  DevBuf<double> D, Dn, F, J, K, Fp, C, E, Fh, Eh, Fx, wv;
  auto ok = [&](cudaError_t e) { return e == cudaSuccess; };
  if (!ok(D.alloc(nn)) || !ok(Dn.alloc(nn)) || !ok(F.alloc(nn)) || !ok(J.alloc(nn)) || !ok(K.alloc(nn)) ||
      !ok(Fp.alloc(nn)) || !ok(C.alloc(nn)) || !ok(E.alloc(nn)) || !ok(Fh.alloc(8 * nn)) || !ok(Eh.alloc(8 * nn)) ||
      !ok(Fx.alloc(nn)) || !ok(wv.alloc(n)))
    return set_error(ctx, HFG_ERR_OOM, "SAD buffers");
  cudaStream_t st = ac->stream;
  std::vector<double> eps(m);
  // density from a Fock-like matrix with fractional occupations
  auto dens = [&](const double* Fm, double* Dm) -> int {
    if (s.gemm(CUBLAS_OP_N, CUBLAS_OP_N, n, m, n, 1.0, Fm, n, s.X.p, n, 0.0, s.tmp1.p, n)) return HFG_ERR_CUDA;
    if (s.gemm(CUBLAS_OP_T, CUBLAS_OP_N, m, m, n, 1.0, s.X.p, n, s.tmp1.p, n, 0.0, Fp.p, m)) return HFG_ERR_CUDA;
    if (s.eigh(Fp.p, s.evals.p, m)) return HFG_ERR_CUDA;
    if (s.gemm(CUBLAS_OP_N, CUBLAS_OP_N, n, m, m, 1.0, s.X.p, n, Fp.p, m, 0.0, C.p, n)) return HFG_ERR_CUDA;
    cudaMemcpyAsync(eps.data(), s.evals.p, m * 8, cudaMemcpyDeviceToHost, st);
    cudaStreamSynchronize(st);
    std::vector<double> occ = occupations(eps, Z);
    for (auto& v : occ) v = std::sqrt(v);
    cudaMemcpyAsync(wv.p, occ.data(), m * 8, cudaMemcpyHostToDevice, st);
    scale_cols_by<<<nblk((long long)n * m), 256, 0, st>>>(C.p, wv.p, n, m);
    return s.gemm(CUBLAS_OP_N, CUBLAS_OP_T, n, n, m, 1.0, C.p, n, C.p, n, 0.0, Dm, n);
  };
  auto fock = [&](const double* Dm) -> int {
    cudaMemcpyAsync(F.p, s.H.p, nn * 8, cudaMemcpyDeviceToDevice, st);
    if (std::fabs(Z - 1.0) < 1e-12) return HFG_OK;
    hfg_jk_opts jo;
    hfg_jk_opts_default(&jo);
    int r = jk_device_locked(ac, &jo, 1, Dm, Dm, J.p, K.p);
    if (r != HFG_OK) return r;
    axpby_kernel<<<nblk(nn), 256, 0, st>>>(F.p, J.p, 1.0, 1.0, nn);
    axpby_kernel<<<nblk(nn), 256, 0, st>>>(F.p, K.p, -0.5, 1.0, nn);
    return HFG_OK;
  };
  if ((rc = dens(s.H.p, D.p)) != HFG_OK) return set_error(ctx, rc, "SAD");
  double prev = INFINITY;
  std::vector<int> slot;
  std::vector<double> Bm;
  int count = 0;
  for (int it = 1; it <= 200; ++it) {
    if ((rc = fock(D.p)) != HFG_OK) return set_error(ctx, rc, "SAD Fock");
    const double e = 0.5 * (s.dot(D.p, s.H.p, nn) + s.dot(D.p, F.p, nn));
    if ((rc = dens(F.p, Dn.p)) != HFG_OK) return set_error(ctx, rc, "SAD");
    // error FDS - SDF and rmsd(D - Dn)
    s.gemm(CUBLAS_OP_N, CUBLAS_OP_N, n, n, n, 1.0, F.p, n, D.p, n, 0.0, s.tmp1.p, n);
    s.gemm(CUBLAS_OP_N, CUBLAS_OP_N, n, n, n, 1.0, s.tmp1.p, n, s.S.p, n, 0.0, s.T.p, n);
    antisym_kernel<<<nblk(nn), 256, 0, st>>>(s.T.p, E.p, n);
    const double err = s.maxabs(E.p, nn);
    cudaMemcpyAsync(s.tmp1.p, D.p, nn * 8, cudaMemcpyDeviceToDevice, st);
    axpby_kernel<<<nblk(nn), 256, 0, st>>>(s.tmp1.p, Dn.p, -1.0, 1.0, nn);
    double nr = 0.0;
    cublasDnrm2(s.blas, (int)nn, s.tmp1.p, 1, &nr);
    const double rmsd = nr / std::sqrt((double)nn);
    if (std::fabs(e - prev) < 1e-11 && rmsd < 1e-9 && err < 1e-8) {
      out.resize(nn);
      cudaMemcpyAsync(out.data(), Dn.p, nn * 8, cudaMemcpyDeviceToHost, st);
      cudaStreamSynchronize(st);
      return HFG_OK;
    }
    prev = e;
    int sl;
    if (count < 8) {
      sl = count++;
      slot.push_back(sl);
    } else {
      sl = slot.front();
      slot.erase(slot.begin());
      slot.push_back(sl);
    }
    cudaMemcpyAsync(Fh.p + (long long)sl * nn, F.p, nn * 8, cudaMemcpyDeviceToDevice, st);
    cudaMemcpyAsync(Eh.p + (long long)sl * nn, E.p, nn * 8, cudaMemcpyDeviceToDevice, st);
    const int k = (int)slot.size();
    std::vector<double> Bn((size_t)k * k);
    const int kprev = (int)std::sqrt((double)Bm.size());
    for (int i = 0; i < k - 1; ++i)
      for (int j = 0; j < k - 1; ++j) Bn[(size_t)i * k + j] = Bm[(size_t)(kprev - (k - 1) + i) * kprev + kprev - (k - 1) + j];
    for (int i = 0; i < k; ++i) {
      const double d = s.dot(Eh.p + (long long)slot[i] * nn, Eh.p + (long long)sl * nn, nn);
      Bn[(size_t)i * k + (k - 1)] = Bn[(size_t)(k - 1) * k + i] = d;
    }
    Bm = Bn;
    const double* Fuse = F.p;
    if (k >= 2) {
      const int dim = k + 1;
      std::vector<double> A((size_t)dim * dim, 0.0), x(dim, 0.0);
      for (int i = 0; i < k; ++i) {
        for (int j = 0; j < k; ++j) A[(size_t)i * dim + j] = Bm[(size_t)i * k + j];
        A[(size_t)i * dim + k] = A[(size_t)k * dim + i] = -1.0;
      }
      x[k] = -1.0;
      if (solve_small(A, x, dim)) {
        cudaMemsetAsync(Fx.p, 0, nn * 8, st);
        for (int i = 0; i < k; ++i)
          axpby_kernel<<<nblk(nn), 256, 0, st>>>(Fx.p, Fh.p + (long long)slot[i] * nn, x[i], 1.0, nn);
        Fuse = Fx.p;
      }
    }
    if ((rc = dens(Fuse, Dn.p)) != HFG_OK) return set_error(ctx, rc, "SAD");
    if (it <= 5) axpby_kernel<<<nblk(nn), 256, 0, st>>>(D.p, Dn.p, 0.5, 0.5, nn);
    else cudaMemcpyAsync(D.p, Dn.p, nn * 8, cudaMemcpyDeviceToDevice, st);
  }
  return set_error(ctx, HFG_ERR_SCF, "fractional atomic HF did not converge");
}

// SAD density of the molecule into dP (device, n x n), rescaled to nel.
int sad_guess(hfg_ctx* ctx, const hfg_scf_opts* o, Scf& s, double nel, double* dP) {
  const int n = ctx->n;
  std::vector<double> P((size_t)n * n, 0.0);
  // functions of each atom (consecutive shells of one atom index)
  std::map<int, std::pair<int, int>> range;
  for (const auto& sh : ctx->shells) {
    auto it = range.find(sh.atom);
    const int f1 = sh.ao + (sh.l + 1) * (sh.l + 2) / 2;
    if (it == range.end()) range[sh.atom] = {sh.ao, f1};
    else {
      if (sh.ao != it->second.second) return set_error(ctx, HFG_ERR_INVALID_INPUT, "atom functions not contiguous");
      it->second.second = f1;
    }
  }
  for (auto& kv : range) {
    const int a = kv.first, f0 = kv.second.first, f1 = kv.second.second;
    if (a < 0 || a >= o->natom) return set_error(ctx, HFG_ERR_INVALID_INPUT, "atom index out of range");
    const double Z = o->charges[a];
    std::vector<double> key{Z};
    for (const auto& sh : ctx->shells)
      if (sh.ao >= f0 && sh.ao < f1) {
        key.push_back(sh.l);
        for (int q = 0; q < sh.K; ++q) {
          key.push_back(ctx->exps[sh.prim_off + q]);
          key.push_back(ctx->coefs[sh.prim_off + q]);
        }
      }
    std::vector<double> Da;
    {
      std::lock_guard<std::mutex> lk(g_sad_mu);
      auto it = g_sad_cache.find(key);
      if (it != g_sad_cache.end()) Da = it->second;
    }
    if (Da.empty()) {
      const int rc = atomic_density(ctx, f0, f1, Z, Da);
      if (rc != HFG_OK) return rc;
      std::lock_guard<std::mutex> lk(g_sad_mu);
      g_sad_cache[key] = Da;
    }
    const int na = f1 - f0;
    for (int i = 0; i < na; ++i)
      for (int j = 0; j < na; ++j) P[(size_t)(f0 + i) * n + f0 + j] = Da[(size_t)i * na + j];
  }
  cudaMemcpyAsync(dP, P.data(), P.size() * 8, cudaMemcpyHostToDevice, ctx->stream);
  const double el = s.dot(dP, s.S.p, (long long)n * n);
  if (el <= 1e-12) return set_error(ctx, HFG_ERR_SCF, "zero SAD population");
  const double scale = nel / el;
  cublasDscal(s.blas, n * n, &scale, dP, 1);
  return HFG_OK;
}
}  // namespace
}  // namespace hfg

using namespace hfg;

extern "C" {

void hfg_scf_opts_default(hfg_scf_opts* o) {
  if (!o) return;
  *o = hfg_scf_opts{};
  o->multiplicity = 1;
  o->max_iter = 100;
  o->energy_tol = 1e-10;
  o->residual_tol = std::max(std::sqrt(1e-10) * 1e-2, 1e-11);
  o->density_tol = std::min(std::max(std::sqrt(1e-10) * 0.1, 1e-12), 1e-10);
  hfg_jk_opts_default(&o->jk);
  o->refine_iters = 2;
  o->diis_size = 8;
  o->incremental_tol = 1e-12;
  o->rebuild_every = 8;
  o->refine_at = 10.0;
}

int hfg_scf(hfg_ctx* ctx, const hfg_scf_opts* o, hfg_scf_result* res, double* P_out, double* F_out, double* C_out,
            double* eps_out) {
  if (!ctx || !o || !res) return HFG_ERR_INVALID_INPUT;
  auto t_start = std::chrono::steady_clock::now();
  std::lock_guard<std::mutex> lk(ctx->mu);
  cudaSetDevice(ctx->device);
  AllocScope alloc_scope(ctx->stream);
  *res = hfg_scf_result{};
  const int n = ctx->n;
  if (o->natom <= 0 || !o->positions || !o->charges)
    return set_error(ctx, HFG_ERR_INVALID_INPUT, "SCF requires nuclei");
  if (o->max_iter <= 0 || !(o->energy_tol > 0) || !(o->residual_tol > 0) || !(o->density_tol > 0))
    return set_error(ctx, HFG_ERR_INVALID_INPUT, "SCF requires a positive tolerance and iteration limit");
  for (int a = 0; a < 3 * o->natom; ++a)
    if (!std::isfinite(o->positions[a])) return set_error(ctx, HFG_ERR_INVALID_INPUT, "non-finite geometry");
  double zsum = 0.0;
  for (int a = 0; a < o->natom; ++a) zsum += o->charges[a];
  const int nel = (int)std::lround(zsum) - o->charge;
  if (nel <= 0) return set_error(ctx, HFG_ERR_INVALID_INPUT, "invalid electron count");
  const bool uhf = o->uhf != 0;
  const int two_s = o->multiplicity - 1;
  if (o->multiplicity < 1 || two_s > nel || ((nel + two_s) & 1))
    return set_error(ctx, HFG_ERR_INVALID_INPUT, "incompatible electron count and multiplicity");
  if (!uhf && (nel & 1)) return set_error(ctx, HFG_ERR_INVALID_INPUT, "RHF requires an even number of electrons");
  const int na = uhf ? (nel + two_s) / 2 : nel / 2, nb = uhf ? (nel - two_s) / 2 : nel / 2;
  const int nspin = uhf ? 2 : 1;
  // nuclear repulsion (src/scf.rs:207-218)
  double e_nuc = 0.0;
  for (int i = 0; i < o->natom; ++i)
    for (int j = i + 1; j < o->natom; ++j) {
      const double dx = o->positions[3 * i] - o->positions[3 * j], dy = o->positions[3 * i + 1] - o->positions[3 * j + 1],
                   dz = o->positions[3 * i + 2] - o->positions[3 * j + 2];
      const double d = std::sqrt(dx * dx + dy * dy + dz * dz);
      if (d < 1e-8) return set_error(ctx, HFG_ERR_INVALID_INPUT, "coincident nuclei");
      e_nuc += o->charges[i] * o->charges[j] / d;
    }

  Scf s;
  int m = 0;
  {
    const int rcs = scf_setup(ctx, o, s, m);
    if (rcs != HFG_OK) return rcs;
  }
  if (na > m || nb > m) return set_error(ctx, HFG_ERR_INVALID_INPUT, "more occupied orbitals than retained rank");
  const long long nn = (long long)n * n;
  int rc = HFG_OK;
#define CK(call)                                    \
  do {                                              \
    rc = cuda_check(ctx, (call), #call);            \
    if (rc != HFG_OK) return rc;                    \
  } while (0)
#define RK(call)             \
  do {                       \
    rc = (call);             \
    if (rc != HFG_OK) return rc; \
  } while (0)
  // state
  const int hist = std::max(2, o->diis_size);
  DevBuf<double> P, Pprev, F, J, K, E, C, Fh, Eh, Fp;
  CK(P.alloc(nspin * nn));
  CK(Pprev.alloc(nspin * nn));
  CK(F.alloc(nspin * nn));
  CK(J.alloc(nn));
  CK(K.alloc(nspin * nn));
  const long long elen = (long long)m * m;
  CK(E.alloc(nspin * std::max(nn, elen)));
  CK(C.alloc(nspin * (long long)n * m));
  CK(Fh.alloc((long long)hist * nspin * nn));
  CK(Eh.alloc((long long)hist * nspin * elen));
  CK(Fp.alloc(std::max(nn, elen) * 1));
  CK(s.evals.alloc(std::max(n, m) * 2));
  const int nocc[2] = {na, nb};
  const double occ_scale = uhf ? 1.0 : 2.0;

  // density from a Fock-like matrix: F' = X^T F X, eigh, C = X C', P = s C_occ C_occ^T
  auto diag = [&](const double* Fm, double* Cm, double* Pm, double* eps, int no) -> int {
    RK(s.gemm(CUBLAS_OP_N, CUBLAS_OP_N, n, m, n, 1.0, Fm, n, s.X.p, n, 0.0, s.tmp1.p, n));
    RK(s.gemm(CUBLAS_OP_T, CUBLAS_OP_N, m, m, n, 1.0, s.X.p, n, s.tmp1.p, n, 0.0, Fp.p, m));
    RK(s.eigh(Fp.p, eps, m));
    phase_kernel<<<m, 256, 0, ctx->stream>>>(Fp.p, m, m);
    RK(s.gemm(CUBLAS_OP_N, CUBLAS_OP_N, n, m, m, 1.0, s.X.p, n, Fp.p, m, 0.0, Cm, n));
    if (Pm) RK(s.gemm(CUBLAS_OP_N, CUBLAS_OP_T, n, n, no, occ_scale, Cm, n, Cm, n, 0.0, Pm, n));
    return HFG_OK;
  };
  // Fock matrices from the densities with the given J/K options
  double* Ptot = s.tmp2.p;
  int builds64 = 0, buildsmix = 0;
  auto fock = [&](const hfg_jk_opts& jo) -> int {
    const double* pt = P.p;
    if (uhf) {
      CK(cudaMemcpyAsync(Ptot, P.p, nn * 8, cudaMemcpyDeviceToDevice, ctx->stream));
      axpby_kernel<<<nblk(nn), 256, 0, ctx->stream>>>(Ptot, P.p + nn, 1.0, 1.0, nn);
      pt = Ptot;
    }
    RK(jk_device_locked(ctx, &jo, nspin, pt, P.p, J.p, K.p));
    if (jo.precision == HFG_MIXED) ++buildsmix; else ++builds64;
    for (int sp = 0; sp < nspin; ++sp) {
      double* f = F.p + sp * nn;
      CK(cudaMemcpyAsync(f, s.H.p, nn * 8, cudaMemcpyDeviceToDevice, ctx->stream));
      axpby_kernel<<<nblk(nn), 256, 0, ctx->stream>>>(f, J.p, 1.0, 1.0, nn);
      axpby_kernel<<<nblk(nn), 256, 0, ctx->stream>>>(f, K.p + sp * nn, uhf ? -1.0 : -0.5, 1.0, nn);
    }
    return HFG_OK;
  };
  auto energy = [&]() -> double {
    if (!uhf) return 0.5 * (s.dot(P.p, s.H.p, nn) + s.dot(P.p, F.p, nn));
    double e = 0.0;
    for (int sp = 0; sp < 2; ++sp) e += 0.5 * (s.dot(P.p + sp * nn, s.H.p, nn) + s.dot(P.p + sp * nn, F.p + sp * nn, nn));
    return e;
  };
  // commutator error of spin sp into E (m x m when X is rectangular)
  auto error = [&](int sp, double* out) -> int {
    RK(s.gemm(CUBLAS_OP_N, CUBLAS_OP_N, n, n, n, 1.0, F.p + sp * nn, n, P.p + sp * nn, n, 0.0, s.tmp1.p, n));
    RK(s.gemm(CUBLAS_OP_N, CUBLAS_OP_N, n, n, n, 1.0, s.tmp1.p, n, s.S.p, n, 0.0, s.T.p, n));
    antisym_kernel<<<nblk(nn), 256, 0, ctx->stream>>>(s.T.p, s.V.p, n);
    if (m < n) {
      RK(s.gemm(CUBLAS_OP_N, CUBLAS_OP_N, n, m, n, 1.0, s.V.p, n, s.X.p, n, 0.0, s.tmp1.p, n));
      RK(s.gemm(CUBLAS_OP_T, CUBLAS_OP_N, m, m, n, 1.0, s.X.p, n, s.tmp1.p, n, 0.0, out, m));
    } else {
      CK(cudaMemcpyAsync(out, s.V.p, nn * 8, cudaMemcpyDeviceToDevice, ctx->stream));
    }
    return HFG_OK;
  };
  const long long elen_eff = m < n ? elen : nn;

  // initial guess (src/scf.rs:452-471 for RHF, :742-751 for UHF): the SAD
  // density (RHF starts from it; UHF from the orbitals of its Fock matrix),
  // or core Hamiltonian orbitals
  if (o->guess == 0) {
    RK(sad_guess(ctx, o, s, (double)nel, Ptot));
    if (!uhf) {
      CK(cudaMemcpyAsync(P.p, Ptot, nn * 8, cudaMemcpyDeviceToDevice, ctx->stream));
    } else {
      // Fock of the SAD density with RHF weights, then its orbitals
      hfg_jk_opts j64 = o->jk;
      j64.precision = HFG_FP64;
      RK(jk_device_locked(ctx, &j64, 1, Ptot, Ptot, J.p, K.p));
      CK(cudaMemcpyAsync(F.p, s.H.p, nn * 8, cudaMemcpyDeviceToDevice, ctx->stream));
      axpby_kernel<<<nblk(nn), 256, 0, ctx->stream>>>(F.p, J.p, 1.0, 1.0, nn);
      axpby_kernel<<<nblk(nn), 256, 0, ctx->stream>>>(F.p, K.p, -0.5, 1.0, nn);
      for (int sp = 0; sp < 2; ++sp) RK(diag(F.p, C.p + sp * (long long)n * m, P.p + sp * nn, s.evals.p, nocc[sp]));
    }
  } else {
    for (int sp = 0; sp < nspin; ++sp) RK(diag(s.H.p, C.p + sp * (long long)n * m, P.p + sp * nn, s.evals.p, nocc[sp]));
  }

  const bool mixed = o->jk.precision == HFG_MIXED;
  hfg_jk_opts jo = o->jk;
  hfg_jk_opts jo64 = o->jk;
  jo64.precision = HFG_FP64;
  // the refinement and final builds keep primitive screening at 1e-15 at most
  // (the mixed phase may use a looser, autotuned one)
  jo64.prim_threshold = std::min(jo64.prim_threshold, 1e-15);
  // Incremental builds in the mixed phase: J/K are linear in the density, so
  // J(P) = J(P_full) + J(P - P_full) summed over the builds since the last
  // full one, and the change only needs the quartets with
  // Q_ab Q_cd max|dP| >= incremental_tol (a Schwarz threshold scaled by
  // 1 / max|dP|, rounded down to a decade so that few plans are built).
  // The FP64 refinement and the final Fock matrices are full builds.
  const bool incremental = mixed && o->incremental_tol > 0.0;
  const int rebuild_every = std::max(1, o->rebuild_every);
  DevBuf<double> Jinc, Kinc, Pinc, dP;
  if (incremental) {
    CK(Jinc.alloc(nn));
    CK(Kinc.alloc(nspin * nn));
    CK(Pinc.alloc(nspin * nn));
    CK(dP.alloc((nspin + 1) * nn));
  }
  int since_full = -1, builds_inc = 0, base_prec = -1;
  // jb: the options of this build; a change of precision (the switch to the
  // FP64 refinement) starts from a full build
  auto fock_inc = [&](const hfg_jk_opts& jb) -> int {
    if (since_full < 0 || since_full >= rebuild_every || jb.precision != base_prec) {
      base_prec = jb.precision;
      RK(fock(jb));
      CK(cudaMemcpyAsync(Jinc.p, J.p, nn * 8, cudaMemcpyDeviceToDevice, ctx->stream));
      CK(cudaMemcpyAsync(Kinc.p, K.p, nspin * nn * 8, cudaMemcpyDeviceToDevice, ctx->stream));
      CK(cudaMemcpyAsync(Pinc.p, P.p, nspin * nn * 8, cudaMemcpyDeviceToDevice, ctx->stream));
      since_full = 0;
      return HFG_OK;
    }
    double dmax = 0.0;
    for (int sp = 0; sp < nspin; ++sp) {
      CK(cudaMemcpyAsync(dP.p + sp * nn, P.p + sp * nn, nn * 8, cudaMemcpyDeviceToDevice, ctx->stream));
      axpby_kernel<<<nblk(nn), 256, 0, ctx->stream>>>(dP.p + sp * nn, Pinc.p + sp * nn, -1.0, 1.0, nn);
      dmax = std::max(dmax, s.maxabs(dP.p + sp * nn, nn));
    }
    const double* dpt = dP.p;
    if (uhf) {
      CK(cudaMemcpyAsync(dP.p + 2 * nn, dP.p, nn * 8, cudaMemcpyDeviceToDevice, ctx->stream));
      axpby_kernel<<<nblk(nn), 256, 0, ctx->stream>>>(dP.p + 2 * nn, dP.p + nn, 1.0, 1.0, nn);
      dpt = dP.p + 2 * nn;
    }
    if (dmax > 0.0) {
      hfg_jk_opts ji = jb;
      double thr = std::max(o->incremental_tol / dmax, jb.schwarz_threshold);
      ji.schwarz_threshold = std::pow(10.0, std::floor(std::log10(thr) + 1e-9));
      RK(jk_device_locked(ctx, &ji, nspin, dpt, dP.p, J.p, K.p));
      if (jb.precision == HFG_MIXED) ++buildsmix; else ++builds64;
      ++builds_inc;
      axpby_kernel<<<nblk(nn), 256, 0, ctx->stream>>>(Jinc.p, J.p, 1.0, 1.0, nn);
      axpby_kernel<<<nblk(nspin * nn), 256, 0, ctx->stream>>>(Kinc.p, K.p, 1.0, 1.0, nspin * nn);
      CK(cudaMemcpyAsync(Pinc.p, P.p, nspin * nn * 8, cudaMemcpyDeviceToDevice, ctx->stream));
    }
    ++since_full;
    for (int sp = 0; sp < nspin; ++sp) {
      double* f = F.p + sp * nn;
      CK(cudaMemcpyAsync(f, s.H.p, nn * 8, cudaMemcpyDeviceToDevice, ctx->stream));
      axpby_kernel<<<nblk(nn), 256, 0, ctx->stream>>>(f, Jinc.p, 1.0, 1.0, nn);
      axpby_kernel<<<nblk(nn), 256, 0, ctx->stream>>>(f, Kinc.p + sp * nn, uhf ? -1.0 : -0.5, 1.0, nn);
    }
    return HFG_OK;
  };
  bool refining = !mixed;
  const double refine_at = o->refine_at > 1.0 ? o->refine_at : 1.0;
  int refine_done = 0;
  double prev_e = 0.0, e_tot = 0.0;
  bool converged = false;
  int it = 0, count = 0;
  std::vector<double> Bm;  // DIIS overlap matrix (count x count), host
  std::vector<int> slot;   // history slot of each stored vector, oldest first
  CK(cudaMemcpyAsync(Pprev.p, P.p, nspin * nn * 8, cudaMemcpyDeviceToDevice, ctx->stream));
  // HFG_SCF_PROFILE=1: wall time of the iteration phases (the stream is
  // synchronised at each phase boundary), printed on stderr
  static const bool profile = getenv("HFG_SCF_PROFILE") && getenv("HFG_SCF_PROFILE")[0] == '1';
  double ph_ms[4] = {0, 0, 0, 0};  // Fock build, convergence tests, DIIS, diagonalisation
  auto ph_t = std::chrono::steady_clock::now();
  auto phase = [&](int k) {
    if (!profile) return;
    cudaStreamSynchronize(ctx->stream);
    const auto t = std::chrono::steady_clock::now();
    ph_ms[k] += std::chrono::duration<double, std::milli>(t - ph_t).count();
    ph_t = t;
  };
  for (it = 1; it <= o->max_iter; ++it) {
    phase(3);
    // incremental (mixed mode): the mixed phase, then the FP64 refinement
    // from one full FP64 build
    if (incremental) RK(fock_inc(refining ? jo64 : jo));
    else RK(fock(refining ? jo64 : jo));
    phase(0);
    if (refining) ++refine_done;
    e_tot = energy() + e_nuc;
    const double de = std::fabs(e_tot - prev_e);
    prev_e = e_tot;
    double en = 0.0;
    for (int sp = 0; sp < nspin; ++sp) {
      RK(error(sp, E.p + sp * elen_eff));
      en = std::max(en, s.maxabs(E.p + sp * elen_eff, elen_eff));
    }
    // rmsd of the density change (src/matrix.rs:150-159), max over spins
    double dr = 0.0;
    for (int sp = 0; sp < nspin; ++sp) {
      CK(cudaMemcpyAsync(s.tmp1.p, P.p + sp * nn, nn * 8, cudaMemcpyDeviceToDevice, ctx->stream));
      axpby_kernel<<<nblk(nn), 256, 0, ctx->stream>>>(s.tmp1.p, Pprev.p + sp * nn, -1.0, 1.0, nn);
      double nr = 0.0;
      cublasDnrm2(s.blas, (int)nn, s.tmp1.p, 1, &nr);
      dr = std::max(dr, nr / std::sqrt((double)nn));
    }
    if (o->verbose) fprintf(stderr, "hfg scf %3d  E = %.12f  dE = %.3e  |e| = %.3e  dP = %.3e  %s\n", it, e_tot, de, en, dr,
                           refining ? "fp64" : "mixed");
    if (it > 1 && de < o->energy_tol && en < o->residual_tol && dr < o->density_tol &&
        refining && refine_done >= (mixed ? std::max(1, o->refine_iters) : 0)) {
      converged = true;
      break;
    }
    // the mixed phase ends once the measures are below refine_at x the
    // tolerances (refine_at = 1: fully converged in mixed precision)
    if (!refining && it > 1 && de < refine_at * o->energy_tol && en < refine_at * o->residual_tol &&
        dr < refine_at * o->density_tol) {
      res->energy_before_refinement = e_tot;
      refining = true;
    }
    if (mixed && !refining && it >= o->max_iter - std::max(1, o->refine_iters)) {
      res->energy_before_refinement = e_tot;
      refining = true;
    }
    CK(cudaMemcpyAsync(Pprev.p, P.p, nspin * nn * 8, cudaMemcpyDeviceToDevice, ctx->stream));
    phase(1);
    // CDIIS push (drop the oldest when full) and extrapolate
    int sl;
    if (count < hist) {
      sl = count++;
      slot.push_back(sl);
    } else {
      sl = slot.front();
      slot.erase(slot.begin());
      slot.push_back(sl);
    }
    for (int sp = 0; sp < nspin; ++sp) {
      CK(cudaMemcpyAsync(Fh.p + ((long long)sl * nspin + sp) * nn, F.p + sp * nn, nn * 8, cudaMemcpyDeviceToDevice,
                         ctx->stream));
      CK(cudaMemcpyAsync(Eh.p + ((long long)sl * nspin + sp) * elen, E.p + sp * elen_eff, elen_eff * 8,
                         cudaMemcpyDeviceToDevice, ctx->stream));
    }
    const int k = (int)slot.size();
    std::vector<double> Bn((size_t)k * k);
    // rebuild the overlap matrix in slot order (previous entries reused)
    {
      std::vector<double> newrow(k);
      for (int i = 0; i < k; ++i) {
        double d = 0.0;
        for (int sp = 0; sp < nspin; ++sp)
          d += s.dot(Eh.p + ((long long)slot[i] * nspin + sp) * elen, Eh.p + ((long long)sl * nspin + sp) * elen,
                     elen_eff);
        newrow[i] = d;
      }
      // previous matrix in previous order: entries for slots shared with the new order
      const int kprev = (int)std::sqrt((double)Bm.size());
      for (int i = 0; i < k - 1; ++i)
        for (int j = 0; j < k - 1; ++j) {
          const int oi = kprev - (k - 1) + i, oj = kprev - (k - 1) + j;
          Bn[(size_t)i * k + j] = Bm[(size_t)oi * kprev + oj];
        }
      for (int i = 0; i < k; ++i) Bn[(size_t)i * k + (k - 1)] = Bn[(size_t)(k - 1) * k + i] = newrow[i];
    }
    Bm = Bn;
    const double* Fuse[2] = {F.p, F.p + nn};
    if (k >= 2) {
      const int dim = k + 1;
      std::vector<double> A((size_t)dim * dim, 0.0), x(dim, 0.0);
      for (int i = 0; i < k; ++i) {
        for (int j = 0; j < k; ++j) A[(size_t)i * dim + j] = Bm[(size_t)i * k + j];
        A[(size_t)i * dim + k] = A[(size_t)k * dim + i] = -1.0;
      }
      x[k] = -1.0;
      if (solve_small(A, x, dim)) {
        for (int sp = 0; sp < nspin; ++sp) {
          double* out = s.T.p;
          if (sp == 1) out = s.V.p;
          CK(cudaMemsetAsync(out, 0, nn * 8, ctx->stream));
          for (int i = 0; i < k; ++i)
            axpby_kernel<<<nblk(nn), 256, 0, ctx->stream>>>(out, Fh.p + ((long long)slot[i] * nspin + sp) * nn, x[i],
                                                            1.0, nn);
          Fuse[sp] = out;
        }
      }
    }
    phase(2);
    for (int sp = 0; sp < nspin; ++sp) {
      double* Pn = uhf ? s.tmp2.p : P.p;
      RK(diag(Fuse[sp], C.p + sp * (long long)n * m, Pn, s.evals.p, nocc[sp]));
      if (uhf) {
        double* Ps = P.p + sp * nn;
        if (it <= 2) axpby_kernel<<<nblk(nn), 256, 0, ctx->stream>>>(Ps, Pn, 0.7, 0.3, nn);
        else CK(cudaMemcpyAsync(Ps, Pn, nn * 8, cudaMemcpyDeviceToDevice, ctx->stream));
      }
    }
  }
  phase(3);
  if (profile)
    fprintf(stderr, "hfg-profile scf n %d m %d iterations %d: fock %.1f ms, convergence tests %.1f ms, DIIS %.1f ms, "
                    "diagonalisation %.1f ms\n", n, m, it, ph_ms[0], ph_ms[1], ph_ms[2], ph_ms[3]);
  if (it > o->max_iter) it = o->max_iter;
  // final orbitals from the true Fock matrix (src/scf.rs:579-597)
  if (!converged) RK(fock(jo64));
  for (int sp = 0; sp < nspin; ++sp)
    RK(diag(F.p + sp * nn, C.p + sp * (long long)n * m, P.p + sp * nn, s.evals.p + sp * m, nocc[sp]));
  std::vector<double> epsh((size_t)nspin * m);
  CK(cudaMemcpyAsync(epsh.data(), s.evals.p, nspin * m * 8, cudaMemcpyDeviceToHost, ctx->stream));
  if (incremental) RK(fock_inc(jo64));
  else RK(fock(jo64));
  const double e_el = energy();
  res->energy = e_el + e_nuc;
  res->electronic = e_el;
  res->nuclear = e_nuc;
  if (!mixed) res->energy_before_refinement = res->energy;
  res->iterations = it;
  res->converged = converged ? 1 : 0;
  res->n_mo = m;
  res->fock_builds_fp64 = builds64;
  res->fock_builds_mixed = buildsmix;
  res->fock_builds_incremental = builds_inc;
  if (uhf) {
    // <S^2> = S(S+1) + N_b - sum |(C_a^T S C_b)_ij|^2 over occupied
    RK(s.gemm(CUBLAS_OP_N, CUBLAS_OP_N, n, nb > 0 ? nb : 1, n, 1.0, s.S.p, n, C.p + (long long)n * m, n, 0.0, s.tmp1.p, n));
    RK(s.gemm(CUBLAS_OP_T, CUBLAS_OP_N, na, nb > 0 ? nb : 1, n, 1.0, C.p, n, s.tmp1.p, n, 0.0, s.tmp2.p, na));
    double ov = 0.0;
    if (nb > 0) {
      std::vector<double> h((size_t)na * nb);
      CK(cudaMemcpyAsync(h.data(), s.tmp2.p, h.size() * 8, cudaMemcpyDeviceToHost, ctx->stream));
      CK(cudaStreamSynchronize(ctx->stream));
      for (double v : h) ov += v * v;
    }
    res->s2 = (two_s / 2.0) * (two_s / 2.0 + 1.0) + nb - ov;
  }
  // outputs (row-major for the caller; P and F are symmetric)
  if (P_out) CK(cudaMemcpyAsync(P_out, P.p, nspin * nn * 8, cudaMemcpyDeviceToHost, ctx->stream));
  if (F_out) CK(cudaMemcpyAsync(F_out, F.p, nspin * nn * 8, cudaMemcpyDeviceToHost, ctx->stream));
  if (C_out) {
    std::vector<double> cm((size_t)n * m);
    for (int sp = 0; sp < nspin; ++sp) {
      CK(cudaMemcpyAsync(cm.data(), C.p + sp * (long long)n * m, cm.size() * 8, cudaMemcpyDeviceToHost, ctx->stream));
      CK(cudaStreamSynchronize(ctx->stream));
      for (int i = 0; i < n; ++i)
        for (int j = 0; j < m; ++j) C_out[(size_t)sp * n * m + (size_t)i * m + j] = cm[(size_t)j * n + i];
    }
  }
  CK(cudaStreamSynchronize(ctx->stream));
  if (eps_out) std::copy(epsh.begin(), epsh.end(), eps_out);
  res->time_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t_start).count();
#undef CK
#undef RK
  return converged ? HFG_OK : set_error(ctx, HFG_ERR_SCF, "SCF did not converge within the iteration limit");
}

}  // extern "C"

extern "C" int hfg_scf_df(hfg_ctx* ctx, hfg_df* df, int mma, const hfg_scf_opts* o, hfg_scf_result* res, double* P_out,
                          double* F_out, double* J_out, double* K_out) {
  // run_factorized_rhf (src/hf_variants/ri_df_hf.rs:160-263): core guess,
  // CDIIS from the second iteration, convergence on |dE|, the residual and
  // max |P_next - P| of the density from the un-extrapolated Fock matrix.
  if (!ctx || !df || !o || !res) return HFG_ERR_INVALID_INPUT;
  if (df_is_shard(df)) return set_error(ctx, HFG_ERR_INVALID_INPUT, "DF-RHF needs the whole factor, not a shard of it");
  auto t_start = std::chrono::steady_clock::now();
  std::lock_guard<std::mutex> lk(ctx->mu);
  cudaSetDevice(ctx->device);
  AllocScope alloc_scope(ctx->stream);
  *res = hfg_scf_result{};
  const int n = ctx->n;
  double zsum = 0.0;
  for (int a = 0; a < o->natom; ++a) zsum += o->charges[a];
  const double electrons = zsum - o->charge;
  if (!(electrons > 0) || std::fabs(electrons - std::round(electrons)) > 1e-8 || ((long)std::lround(electrons) & 1))
    return set_error(ctx, HFG_ERR_INVALID_INPUT, "factorized RHF requires a positive even electron count");
  const int no = (int)std::lround(electrons) / 2;
  double e_nuc = 0.0;
  for (int i = 0; i < o->natom; ++i)
    for (int j = i + 1; j < o->natom; ++j) {
      const double dx = o->positions[3 * i] - o->positions[3 * j], dy = o->positions[3 * i + 1] - o->positions[3 * j + 1],
                   dz = o->positions[3 * i + 2] - o->positions[3 * j + 2];
      e_nuc += o->charges[i] * o->charges[j] / std::sqrt(dx * dx + dy * dy + dz * dz);
    }
  Scf s;
  int m = 0;
  {
    const int rcs = scf_setup(ctx, o, s, m);
    if (rcs != HFG_OK) return rcs;
  }
  if (no > m) return set_error(ctx, HFG_ERR_INVALID_INPUT, "factorized RHF occupied count exceeds overlap rank");
  const long long nn = (long long)n * n;
  int rc = HFG_OK;
#define CK(call)                         \
  do {                                   \
    rc = cuda_check(ctx, (call), #call); \
    if (rc != HFG_OK) return rc;         \
  } while (0)
#define RK(call)                 \
  do {                           \
    rc = (call);                 \
    if (rc != HFG_OK) return rc; \
  } while (0)
  const int hist = std::max(2, o->diis_size);
  DevBuf<double> P, Pn, F, J, K, E, C, Cn, Fh, Eh, Fp, Fx;
  const long long elen = (long long)m * m;
  const long long elen_eff = m < n ? elen : nn;
  CK(P.alloc(nn));
  CK(Pn.alloc(nn));
  CK(F.alloc(nn));
  CK(Fx.alloc(nn));
  CK(J.alloc(nn));
  CK(K.alloc(nn));
  CK(E.alloc(std::max(nn, elen)));
  CK(C.alloc((long long)n * m));
  CK(Cn.alloc((long long)n * m));
  CK(Fh.alloc((long long)hist * nn));
  CK(Eh.alloc((long long)hist * elen));
  CK(Fp.alloc(std::max(nn, elen)));
  CK(s.evals.alloc(std::max(n, m)));
  auto diag = [&](const double* Fm, double* Cm, double* Pm) -> int {
    RK(s.gemm(CUBLAS_OP_N, CUBLAS_OP_N, n, m, n, 1.0, Fm, n, s.X.p, n, 0.0, s.tmp1.p, n));
    RK(s.gemm(CUBLAS_OP_T, CUBLAS_OP_N, m, m, n, 1.0, s.X.p, n, s.tmp1.p, n, 0.0, Fp.p, m));
    RK(s.eigh(Fp.p, s.evals.p, m));
    phase_kernel<<<m, 256, 0, ctx->stream>>>(Fp.p, m, m);
    RK(s.gemm(CUBLAS_OP_N, CUBLAS_OP_N, n, m, m, 1.0, s.X.p, n, Fp.p, m, 0.0, Cm, n));
    RK(s.gemm(CUBLAS_OP_N, CUBLAS_OP_T, n, n, no, 2.0, Cm, n, Cm, n, 0.0, Pm, n));
    return HFG_OK;
  };
  // Precision phases: with a tensor-core mode (TF32 / BF16) the Fock matrix
  // carries rounding noise of the GEMMs, so the SCF first converges loosely
  // with it (|dE| <= 1e-5 and residual <= 1e-2, or 25 iterations), then
  // drops the DIIS history and refines with FP64 arithmetic on the stored
  // factor (at least two FP64 builds) to the requested criteria.  Only the
  // factor's storage rounding remains in the refined energy.
  int cur = mma == HFG_DF_FP64 ? HFG_DF_FP64 : mma;
  int builds64 = 0, builds_low = 0;
  auto fock = [&](const double* Cm) -> int {
    RK(df_jk_device(df, Cm, no, J.p, K.p, cur));
    if (cur == HFG_DF_FP64) ++builds64; else ++builds_low;
    CK(cudaMemcpyAsync(F.p, s.H.p, nn * 8, cudaMemcpyDeviceToDevice, ctx->stream));
    axpby_kernel<<<nblk(nn), 256, 0, ctx->stream>>>(F.p, J.p, 1.0, 1.0, nn);
    axpby_kernel<<<nblk(nn), 256, 0, ctx->stream>>>(F.p, K.p, -0.5, 1.0, nn);
    return HFG_OK;
  };
  auto energy = [&](const double* Pm) { return 0.5 * (s.dot(Pm, s.H.p, nn) + s.dot(Pm, F.p, nn)) + e_nuc; };
  if (o->guess == 0) {
    // SAD start (an option: run_factorized_rhf itself starts from the core
    // Hamiltonian): one FP64 four-centre build of the SAD density, whose
    // Fock matrix gives the first orbitals
    RK(sad_guess(ctx, o, s, electrons, Pn.p));
    hfg_jk_opts j64;
    hfg_jk_opts_default(&j64);
    j64.prim_threshold = 1e-15;
    RK(jk_device_locked(ctx, &j64, 1, Pn.p, Pn.p, J.p, K.p));
    CK(cudaMemcpyAsync(F.p, s.H.p, nn * 8, cudaMemcpyDeviceToDevice, ctx->stream));
    axpby_kernel<<<nblk(nn), 256, 0, ctx->stream>>>(F.p, J.p, 1.0, 1.0, nn);
    axpby_kernel<<<nblk(nn), 256, 0, ctx->stream>>>(F.p, K.p, -0.5, 1.0, nn);
    RK(diag(F.p, C.p, P.p));
  } else {
    RK(diag(s.H.p, C.p, P.p));
  }
  double last = INFINITY;
  bool converged = false;
  int it = 0, count = 0;
  std::vector<int> slot;
  std::vector<double> Bm;
  for (it = 1; it <= o->max_iter; ++it) {
    RK(fock(C.p));
    const double e = energy(P.p);
    // residual X^T (FPS - SPF) X
    RK(s.gemm(CUBLAS_OP_N, CUBLAS_OP_N, n, n, n, 1.0, F.p, n, P.p, n, 0.0, s.tmp1.p, n));
    RK(s.gemm(CUBLAS_OP_N, CUBLAS_OP_N, n, n, n, 1.0, s.tmp1.p, n, s.S.p, n, 0.0, s.T.p, n));
    antisym_kernel<<<nblk(nn), 256, 0, ctx->stream>>>(s.T.p, s.V.p, n);
    RK(s.gemm(CUBLAS_OP_N, CUBLAS_OP_N, n, m, n, 1.0, s.V.p, n, s.X.p, n, 0.0, s.tmp1.p, n));
    RK(s.gemm(CUBLAS_OP_T, CUBLAS_OP_N, m, m, n, 1.0, s.X.p, n, s.tmp1.p, n, 0.0, E.p, m));
    const double resid = s.maxabs(E.p, elen);
    RK(diag(F.p, Cn.p, Pn.p));
    CK(cudaMemcpyAsync(s.tmp1.p, Pn.p, nn * 8, cudaMemcpyDeviceToDevice, ctx->stream));
    axpby_kernel<<<nblk(nn), 256, 0, ctx->stream>>>(s.tmp1.p, P.p, -1.0, 1.0, nn);
    const double dch = s.maxabs(s.tmp1.p, nn);
    if (!std::isfinite(e) || !std::isfinite(resid)) return set_error(ctx, HFG_ERR_SCF, "DF-HF energy/residual became nonfinite");
    if (o->verbose) fprintf(stderr, "hfg df-scf %3d  E = %.12f  |e| = %.3e  dP = %.3e  %s\n", it, e, resid, dch,
                           cur == HFG_DF_FP64 ? "fp64" : "tensor");
    res->energy = e;  // the latest energy, reported if the SCF does not converge
    res->electronic = e - e_nuc;
    res->nuclear = e_nuc;
    if (cur != HFG_DF_FP64 && ((std::fabs(e - last) <= 1e-5 && resid <= 1e-2) || builds_low >= 25)) {
      res->energy_before_refinement = e;
      cur = HFG_DF_FP64;
      count = 0;
      slot.clear();
      Bm.clear();
      last = INFINITY;
      RK(diag(F.p, C.p, P.p));
      continue;
    }
    const bool enough64 = mma == HFG_DF_FP64 || builds64 >= 2;
    if (enough64 && std::fabs(e - last) <= o->energy_tol && resid <= o->residual_tol && dch <= o->density_tol) {
      RK(fock(Cn.p));
      const double ef = energy(Pn.p);
      res->energy = ef;
      res->electronic = ef - e_nuc;
      res->nuclear = e_nuc;
      if (mma == HFG_DF_FP64) res->energy_before_refinement = ef;
      converged = true;
      break;
    }
    last = e;
    int sl;
    if (count < hist) {
      sl = count++;
      slot.push_back(sl);
    } else {
      sl = slot.front();
      slot.erase(slot.begin());
      slot.push_back(sl);
    }
    CK(cudaMemcpyAsync(Fh.p + (long long)sl * nn, F.p, nn * 8, cudaMemcpyDeviceToDevice, ctx->stream));
    CK(cudaMemcpyAsync(Eh.p + (long long)sl * elen, E.p, elen * 8, cudaMemcpyDeviceToDevice, ctx->stream));
    const int k = (int)slot.size();
    std::vector<double> Bn((size_t)k * k);
    {
      const int kprev = (int)std::sqrt((double)Bm.size());
      for (int i = 0; i < k - 1; ++i)
        for (int j = 0; j < k - 1; ++j) Bn[(size_t)i * k + j] = Bm[(size_t)(kprev - (k - 1) + i) * kprev + kprev - (k - 1) + j];
      for (int i = 0; i < k; ++i) {
        const double d = s.dot(Eh.p + (long long)slot[i] * elen, Eh.p + (long long)sl * elen, elen);
        Bn[(size_t)i * k + (k - 1)] = Bn[(size_t)(k - 1) * k + i] = d;
      }
    }
    Bm = Bn;
    const double* Fuse = F.p;
    if (it >= 2 && k >= 2) {
      const int dim = k + 1;
      std::vector<double> A((size_t)dim * dim, 0.0), x(dim, 0.0);
      for (int i = 0; i < k; ++i) {
        for (int j = 0; j < k; ++j) A[(size_t)i * dim + j] = Bm[(size_t)i * k + j];
        A[(size_t)i * dim + k] = A[(size_t)k * dim + i] = -1.0;
      }
      x[k] = -1.0;
      if (solve_small(A, x, dim)) {
        CK(cudaMemsetAsync(Fx.p, 0, nn * 8, ctx->stream));
        for (int i = 0; i < k; ++i)
          axpby_kernel<<<nblk(nn), 256, 0, ctx->stream>>>(Fx.p, Fh.p + (long long)slot[i] * nn, x[i], 1.0, nn);
        Fuse = Fx.p;
      }
    }
    RK(diag(Fuse, C.p, P.p));
  }
  (void)elen_eff;
  if (it > o->max_iter) it = o->max_iter;
  res->iterations = it;
  res->converged = converged ? 1 : 0;
  res->n_mo = m;
  res->fock_builds_fp64 = builds64;
  res->fock_builds_mixed = builds_low;
  if (P_out) CK(cudaMemcpyAsync(P_out, Pn.p, nn * 8, cudaMemcpyDeviceToHost, ctx->stream));
  if (F_out) CK(cudaMemcpyAsync(F_out, F.p, nn * 8, cudaMemcpyDeviceToHost, ctx->stream));
  if (J_out) CK(cudaMemcpyAsync(J_out, J.p, nn * 8, cudaMemcpyDeviceToHost, ctx->stream));
  if (K_out) CK(cudaMemcpyAsync(K_out, K.p, nn * 8, cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  res->time_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t_start).count();
#undef CK
#undef RK
  return converged ? HFG_OK : set_error(ctx, HFG_ERR_SCF, "factorized RHF did not converge");
}
