// Generic McMurchie-Davidson shell-quartet engine (eri_md.cu) for the
// angular classes with an f shell, which the generated Obara-Saika kernels
// do not cover.
#pragma once
#include <cuda_runtime.h>

#include "hfg_internal.h"

namespace hfg {

constexpr int kMDLMax = 3;  // highest shell angular momentum of the generic engine (f)

struct MDClass {
  int la, lb, lc, ld;
  int na, nb, nc, nd;  // Cartesian components per shell
  int L, lab, lcd;
};

MDClass md_class(int la, int lb, int lc, int ld);
size_t md_smem_bytes(const MDClass& c);
bool md_class_ok(int la, int lb, int lc, int ld);

cudaError_t launch_schwarz_md(int la, int lb, const PairInfo* pairs, const PrimPair* prims, int first, int count,
                              const double* boys, const double* expt, double* out, int prim_mode, cudaStream_t st);
cudaError_t launch_quartet_md(int la, int lb, int lc, int ld, const PairInfo* pairs, const PrimPair* prims,
                              const double* boys, const double* expt, double* out, cudaStream_t st);
cudaError_t launch_eri_packed_md(int la, int lb, int lc, int ld, const JKEntry* entries, const long long* prefix,
                                 int nentries, long long nwarps, const PairInfo* pairs, const double* pairQ,
                                 double thr, const PrimRec64* rec, const float* pbound, const double* boys,
                                 const double* expt, double* out, cudaStream_t st);
// FP64 J/K over the launch's work queue (a.serial: one block, deterministic)
cudaError_t launch_jk_md(int la, int lb, int lc, int ld, const JKLaunchArgs& a, cudaStream_t st);
// Nuclear derivatives of the two-electron energy over the launch's work
// queue (densities a.Dtot, a.Dspin; shells up to d): adds into grad[atom][3]
cudaError_t launch_grad_md(int la, int lb, int lc, int ld, const JKLaunchArgs& a, const int* ao_atom, double* grad,
                           cudaStream_t st);

}  // namespace hfg
