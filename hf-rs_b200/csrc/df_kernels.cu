// Density fitting on the device: three-centre integrals (ab|P), the Coulomb
// metric (P|Q), and the unpack/convert kernels of the DF J/K contraction.
//
// hf-rs forms both with its four-centre engine and an exponent-0 unit
// partner (src/df.rs:30-78): (P|Q) = (P 1|Q 1), (P|mn) = (mn|P 1).  Here the
// same generated Obara-Saika classes EriClass<LA,LB,LC,0> evaluate them,
// with the auxiliary function and its unit partner as a one-centre "pair"
// (p = alpha_P, P = centre of P, prefactor c_P / alpha_P).
#include <cuda_bf16.h>
#include <algorithm>
#include <cuda_runtime.h>

#include "boys.cuh"
#include "df_internal.h"
#include "eri_gen.cuh"

namespace hfg {

constexpr double kTwoPiPow25df = 34.986836655249726164477;

__host__ __device__ constexpr int ncart_df(int l) { return (l + 1) * (l + 2) / 2; }

// 1/sqrt(prod (2 l_i - 1)!!) of component i of angular momentum l in hf-rs
// order (l <= 4).
__device__ __forceinline__ double comp_scale_any(int l, int i) {
  if (l < 2) return 1.0;
  int lx, ly, lz;
  if (l == 2) {
    const int t[6][3] = {{2, 0, 0}, {0, 2, 0}, {0, 0, 2}, {1, 1, 0}, {1, 0, 1}, {0, 1, 1}};
    lx = t[i][0];
    ly = t[i][1];
    lz = t[i][2];
  } else {
    int c = 0;
    lx = ly = lz = 0;
    for (int x = l; x >= 0; --x)
      for (int y = l - x; y >= 0; --y) {
        if (c == i) {
          lx = x;
          ly = y;
          lz = l - x - y;
        }
        ++c;
      }
  }
  auto df2 = [](int v) {  // (2v-1)!!
    double r = 1.0;
    for (int k = 2 * v - 1; k > 0; k -= 2) r *= k;
    return r;
  };
  return rsqrt(df2(lx) * df2(ly) * df2(lz));
}

// One block of (ab|P 1): bra pair i (orbital pair or unit-paired auxiliary
// shell), ket unit pair P.  Thread per (bra, ket) combination of one class.
template <int LA, int LB, int LC>
__global__ void __launch_bounds__(128) df3c_kernel(const Df3cArgs a) {
  using C = EriClass<LA, LB, LC, 0>;
  constexpr int NA = ncart_df(LA), NB = ncart_df(LB), NC = ncart_df(LC);
  extern __shared__ __align__(16) unsigned char smem_raw[];
  double* sm = reinterpret_cast<double*>(smem_raw);
  boys_stage<double, C::L>(sm, a.boys, a.expt);
  __syncthreads();
  const long long total = (long long)a.nbra * a.nket;
  for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < total;
       t += (long long)gridDim.x * blockDim.x) {
    const int ib = (int)(t % a.nbra), ik = (int)(t / a.nbra);
    const PairInfo bra = a.bra_pairs[a.bra_idx[ib]];
    const PairInfo ket = a.ket_pairs[a.ket_idx[ik]];
    double acc[C::NACC];
#pragma unroll
    for (int x = 0; x < C::NACC; ++x) acc[x] = 0.0;
    const double ACx = bra.Ax - ket.Ax, ACy = bra.Ay - ket.Ay, ACz = bra.Az - ket.Az;
    for (int q = 0; q < ket.npp; ++q) {
      const PrimPair Q = a.ket_prims[ket.pp_off + q];
      for (int p = 0; p < bra.npp; ++p) {
        const PrimPair P = a.bra_prims[bra.pp_off + p];
        const double pp = P.p, qq = Q.p;
        const double PQx = ACx + P.PAx - Q.PAx, PQy = ACy + P.PAy - Q.PAy, PQz = ACz + P.PAz - Q.PAz;
        const double s = pp + qq, r = rsqrt(s), inv_s = r * r;
        const double tt = pp * qq * inv_s * (PQx * PQx + PQy * PQy + PQz * PQz);
        double F[C::L + 1];
        boys_eval<C::L>(tt, sm, F);
        const double pref = kTwoPiPow25df * P.kp * Q.kp * r;
#pragma unroll
        for (int m = 0; m <= C::L; ++m) F[m] *= pref;
        const double qs = qq * inv_s, ps = pp * inv_s;
        C::prim(acc, F, P.PAx, P.PAy, P.PAz, -qs * PQx, -qs * PQy, -qs * PQz, Q.PAx, Q.PAy, Q.PAz, ps * PQx,
                ps * PQy, ps * PQz, 0.5 * P.inv_p, 0.5 * Q.inv_p, 0.5 * inv_s, qs, ps);
      }
    }
    double out[C::NOUT];
    C::hrr(acc, out, bra.ABx, bra.ABy, bra.ABz, 0.0, 0.0, 0.0);
    // write: rows = ket functions (auxiliary), columns = bra components
    const long long col0 = a.bra_col[ib];
    const int kf0 = ket.ao_a;
#pragma unroll
    for (int i = 0; i < NA; ++i)
#pragma unroll
      for (int j = 0; j < NB; ++j) {
        // unique AO pairs only: for a shell paired with itself keep i >= j
        if (bra.same && j > i) continue;
        const long long col = bra.same ? col0 + i * (i + 1) / 2 + j : col0 + i * NB + j;
        const double sab = comp_scale_any(LA, i) * comp_scale_any(LB, j);
#pragma unroll
        for (int k = 0; k < NC; ++k)
          a.out[(long long)(kf0 + k) * a.ld + col] = out[(i * NB + j) * NC + k] * sab * comp_scale_any(LC, k);
      }
  }
}

#define HFG_DF_CASE(A, B, Cc)                                                                          \
  if (la == A && lb == B && lc == Cc) {                                                                \
    cudaFuncSetAttribute(df3c_kernel<A, B, Cc>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);    \
    df3c_kernel<A, B, Cc><<<grid, 128, smem, st>>>(args);                                              \
    return cudaGetLastError();                                                                         \
  }
#define HFG_DF_KETS(A, B) \
  HFG_DF_CASE(A, B, 0) HFG_DF_CASE(A, B, 1) HFG_DF_CASE(A, B, 2) HFG_DF_CASE(A, B, 3) HFG_DF_CASE(A, B, 4)

cudaError_t launch_df3c(int la, int lb, int lc, const Df3cArgs& args, cudaStream_t st) {
  const long long total = (long long)args.nbra * args.nket;
  if (total <= 0) return cudaSuccess;
  const int smem = (int)boys_smem_bytes<double>();
  long long g = (total + 127) / 128;
  const unsigned grid = (unsigned)(g < 148 * 64 ? g : 148 * 64);
  HFG_DF_KETS(0, 0)
  HFG_DF_KETS(1, 0)
  HFG_DF_KETS(1, 1)
  HFG_DF_KETS(2, 0)
  HFG_DF_KETS(2, 1)
  HFG_DF_KETS(2, 2)
  HFG_DF_KETS(3, 0)
  HFG_DF_KETS(4, 0)
  return cudaErrorInvalidValue;
}

// Unpack rows [q0, q0+qc) of B (rank x ncol, packed unique AO pairs) into
// the dense layout out[(m * qc + q) * n + k] = B_q[m][k] (both triangles),
// converted to the GEMM input type.
template <typename TO, typename TI>
__global__ void df_unpack_kernel(const TI* __restrict__ B, long long ldb, const int2* __restrict__ colmn,
                                 long long ncol, int q0, int qc, int n, TO* __restrict__ out) {
  const long long total = ncol * qc;
  for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < total;
       t += (long long)gridDim.x * blockDim.x) {
    const int q = (int)(t / ncol);
    const long long c = t % ncol;
    const int2 mn = colmn[c];
    const TO v = (TO)(float)B[(long long)(q0 + q) * ldb + c];
    out[((long long)mn.x * qc + q) * n + mn.y] = v;
    out[((long long)mn.y * qc + q) * n + mn.x] = v;
  }
}

template <>
__global__ void df_unpack_kernel<double, double>(const double* __restrict__ B, long long ldb,
                                                 const int2* __restrict__ colmn, long long ncol, int q0, int qc,
                                                 int n, double* __restrict__ out) {
  const long long total = ncol * qc;
  for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < total;
       t += (long long)gridDim.x * blockDim.x) {
    const int q = (int)(t / ncol);
    const long long c = t % ncol;
    const int2 mn = colmn[c];
    const double v = B[(long long)(q0 + q) * ldb + c];
    out[((long long)mn.x * qc + q) * n + mn.y] = v;
    out[((long long)mn.y * qc + q) * n + mn.x] = v;
  }
}

cudaError_t launch_df_unpack(int mode, const void* B, long long ldb, const int2* colmn, long long ncol, int q0, int qc,
                             int n, void* out, cudaStream_t st) {
  const long long total = ncol * qc;
  const unsigned grid = (unsigned)std::min<long long>((total + 255) / 256, 148 * 32);
  if (total <= 0) return cudaSuccess;
  if (mode == 0)
    df_unpack_kernel<double, double><<<grid, 256, 0, st>>>((const double*)B, ldb, colmn, ncol, q0, qc, n,
                                                           (double*)out);
  else if (mode == 1)
    df_unpack_kernel<float, float><<<grid, 256, 0, st>>>((const float*)B, ldb, colmn, ncol, q0, qc, n, (float*)out);
  else if (mode == 2)
    df_unpack_kernel<__nv_bfloat16, __nv_bfloat16><<<grid, 256, 0, st>>>((const __nv_bfloat16*)B, ldb, colmn, ncol,
                                                                         q0, qc, n, (__nv_bfloat16*)out);
  else if (mode == 5)
    df_unpack_kernel<__nv_bfloat16, float><<<grid, 256, 0, st>>>((const float*)B, ldb, colmn, ncol, q0, qc, n,
                                                                  (__nv_bfloat16*)out);
  else if (mode == 3)
    df_unpack_kernel<double, float><<<grid, 256, 0, st>>>((const float*)B, ldb, colmn, ncol, q0, qc, n, (double*)out);
  else
    df_unpack_kernel<double, __nv_bfloat16><<<grid, 256, 0, st>>>((const __nv_bfloat16*)B, ldb, colmn, ncol, q0, qc,
                                                                  n, (double*)out);
  return cudaGetLastError();
}

// J contractions on a stored FP32 / BF16 factor with FP64 accumulation
// (memory-bound: each reads B once): gam[q] = sum_c B[q][c] p[c], one block
// per auxiliary index; j[c] = sum_q B[q][c] gam[q], one thread per column.
template <typename TB>
__global__ void df_gamma_kernel(const TB* __restrict__ B, long long ncol, const double* __restrict__ p,
                                double* __restrict__ gam) {
  const long long row = (long long)blockIdx.x * ncol;
  double s = 0.0;
  for (long long c = threadIdx.x; c < ncol; c += blockDim.x) s += (double)(float)B[row + c] * p[c];
  for (int off = 16; off > 0; off >>= 1) s += __shfl_xor_sync(0xffffffffu, s, off);
  __shared__ double part[8];
  if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int k = 0; k < (int)(blockDim.x >> 5); ++k) t += part[k];
    gam[blockIdx.x] = t;
  }
}

template <typename TB>
__global__ void df_jcol_kernel(const TB* __restrict__ B, long long ncol, int rank, const double* __restrict__ gam,
                               double* __restrict__ j) {
  for (long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x; c < ncol; c += (long long)gridDim.x * blockDim.x) {
    double s = 0.0;
    for (int q = 0; q < rank; ++q) s += (double)(float)B[(long long)q * ncol + c] * gam[q];
    j[c] = s;
  }
}

cudaError_t launch_df_j(int mode, const void* B, long long ncol, int rank, const double* p, double* gam, double* j,
                        cudaStream_t st) {
  if (ncol <= 0 || rank <= 0) return cudaSuccess;
  const unsigned grid = (unsigned)std::min<long long>((ncol + 255) / 256, 148 * 16);
  if (mode == 1) {
    df_gamma_kernel<float><<<rank, 256, 0, st>>>((const float*)B, ncol, p, gam);
    df_jcol_kernel<float><<<grid, 256, 0, st>>>((const float*)B, ncol, rank, gam, j);
  } else {
    df_gamma_kernel<__nv_bfloat16><<<rank, 256, 0, st>>>((const __nv_bfloat16*)B, ncol, p, gam);
    df_jcol_kernel<__nv_bfloat16><<<grid, 256, 0, st>>>((const __nv_bfloat16*)B, ncol, rank, gam, j);
  }
  return cudaGetLastError();
}

// Packed density weights p[c] = P[m][n] (m == n) or 2 P[m][n] (m != n), so
// that gamma_Q = sum_c B[Q][c] p[c] = sum_mn B_Q[m][n] P[m][n].
__global__ void df_pack_density_kernel(const double* __restrict__ P, const int2* __restrict__ colmn, long long ncol,
                                       int n, double* __restrict__ p) {
  for (long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x; c < ncol; c += (long long)gridDim.x * blockDim.x) {
    const int2 mn = colmn[c];
    const double v = P[(long long)mn.x * n + mn.y];
    p[c] = mn.x == mn.y ? v : 2.0 * v;
  }
}

// J from packed columns: J[m][n] = J[n][m] = j[c].
__global__ void df_unpack_j_kernel(const double* __restrict__ j, const int2* __restrict__ colmn, long long ncol, int n,
                                   double* __restrict__ J) {
  for (long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x; c < ncol; c += (long long)gridDim.x * blockDim.x) {
    const int2 mn = colmn[c];
    J[(long long)mn.x * n + mn.y] = j[c];
    J[(long long)mn.y * n + mn.x] = j[c];
  }
}

template <typename TO>
__global__ void convert_kernel(const double* __restrict__ in, TO* __restrict__ out, long long len) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < len; i += (long long)gridDim.x * blockDim.x)
    out[i] = (TO)(float)in[i];
}
template <>
__global__ void convert_kernel<double>(const double* __restrict__ in, double* __restrict__ out, long long len) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < len; i += (long long)gridDim.x * blockDim.x)
    out[i] = in[i];
}

cudaError_t launch_convert(int mode, const double* in, void* out, long long len, cudaStream_t st) {
  const unsigned grid = (unsigned)std::min<long long>((len + 255) / 256, 148 * 32);
  if (len <= 0) return cudaSuccess;
  if (mode == 0) convert_kernel<double><<<grid, 256, 0, st>>>(in, (double*)out, len);
  else if (mode == 1) convert_kernel<float><<<grid, 256, 0, st>>>(in, (float*)out, len);
  else convert_kernel<__nv_bfloat16><<<grid, 256, 0, st>>>(in, (__nv_bfloat16*)out, len);
  return cudaGetLastError();
}

// out[r * ldo + c0 + j] = in[r * w + j] for r < rows, j < w (a chunk of B's
// columns, FP64 GEMM output, into the stored factor)
template <typename TO>
__global__ void convert_cols_kernel(const double* __restrict__ in, int w, long long rows, TO* __restrict__ out,
                                    long long ldo, long long c0) {
  const long long len = rows * w;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < len; i += (long long)gridDim.x * blockDim.x) {
    const long long r = i / w, j = i - r * w;
    out[r * ldo + c0 + j] = (TO)(float)in[i];
  }
}

cudaError_t launch_convert_cols(int mode, const double* in, int w, long long rows, void* out, long long ldo,
                                long long c0, cudaStream_t st) {
  const long long len = rows * w;
  if (len <= 0) return cudaSuccess;
  const unsigned grid = (unsigned)std::min<long long>((len + 255) / 256, 148 * 32);
  if (mode == 1) convert_cols_kernel<float><<<grid, 256, 0, st>>>(in, w, rows, (float*)out, ldo, c0);
  else convert_cols_kernel<__nv_bfloat16><<<grid, 256, 0, st>>>(in, w, rows, (__nv_bfloat16*)out, ldo, c0);
  return cudaGetLastError();
}

// acc (FP64) += 2 * src (FP32), n x n
__global__ void accumulate_f32_kernel(double* __restrict__ acc, const float* __restrict__ src, double scale,
                                      long long len) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < len; i += (long long)gridDim.x * blockDim.x)
    acc[i] += scale * (double)src[i];
}

template <typename TO>
__global__ void convert_f32_kernel(const float* __restrict__ in, TO* __restrict__ out, long long len) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < len; i += (long long)gridDim.x * blockDim.x)
    out[i] = (TO)in[i];
}

// FP32 -> FP64 (mode 0) or BF16 (mode 2)
cudaError_t launch_convert_f32(int mode, const float* in, void* out, long long len, cudaStream_t st) {
  if (len <= 0) return cudaSuccess;
  const unsigned grid = (unsigned)std::min<long long>((len + 255) / 256, 148 * 32);
  if (mode == 0) convert_f32_kernel<double><<<grid, 256, 0, st>>>(in, (double*)out, len);
  else convert_f32_kernel<__nv_bfloat16><<<grid, 256, 0, st>>>(in, (__nv_bfloat16*)out, len);
  return cudaGetLastError();
}

cudaError_t launch_pack_density(const double* P, const int2* colmn, long long ncol, int n, double* p, cudaStream_t st) {
  if (ncol <= 0) return cudaSuccess;
  const unsigned grid = (unsigned)std::min<long long>((ncol + 255) / 256, 148 * 32);
  df_pack_density_kernel<<<grid, 256, 0, st>>>(P, colmn, ncol, n, p);
  return cudaGetLastError();
}
cudaError_t launch_unpack_j(const double* j, const int2* colmn, long long ncol, int n, double* J, cudaStream_t st) {
  if (ncol <= 0) return cudaSuccess;
  const unsigned grid = (unsigned)std::min<long long>((ncol + 255) / 256, 148 * 32);
  df_unpack_j_kernel<<<grid, 256, 0, st>>>(j, colmn, ncol, n, J);
  return cudaGetLastError();
}
cudaError_t launch_accumulate_f32(double* acc, const float* src, double scale, long long len, cudaStream_t st) {
  if (len <= 0) return cudaSuccess;
  const unsigned grid = (unsigned)std::min<long long>((len + 255) / 256, 148 * 32);
  accumulate_f32_kernel<<<grid, 256, 0, st>>>(acc, src, scale, len);
  return cudaGetLastError();
}

}  // namespace hfg
