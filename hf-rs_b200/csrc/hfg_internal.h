// Internal data layout shared by the host runtime and the kernels.
#pragma once
#include <cuda_runtime.h>
#include <cstdint>

namespace hfg {

constexpr int kLMax = 2;  // angular momentum built into the J/K kernels (s, p, d)

// One shell pair, oriented so that la >= lb (and Ka >= Kb when la == lb).
// 80 bytes.
struct PairInfo {
  double Ax, Ay, Az;     // centre of shell a
  double ABx, ABy, ABz;  // A - B
  int ao_a, ao_b;        // first Cartesian function of shell a / b
  int pp_off, npp;       // primitive pairs [pp_off, pp_off + npp) of the PrimPair table, sorted by bound
  int same;              // shells a and b are the same shell
  int cls;               // pair class index
  // compact records (PrimRec64 / PrimRec32 / bounds) of primitive pair k of
  // this shell pair: index rec_off + k * rec_stride.  The records of one pair
  // class are interleaved (stride = pairs in the class), so the lanes of a
  // warp holding consecutive pairs of a class read consecutive records.
  int rec_off, rec_stride;
};

// One primitive pair.  64 bytes.  kp = c_a c_b exp(-mu |AB|^2) / p with the
// shell contraction coefficients (component scale factored out); the
// Gaussian product centre is stored relative to centre A (P = A + PA), which
// keeps P - Q accurate in FP32 as (A - C) + PA - QC.
struct PrimPair {
  double p, inv_p;
  double PAx, PAy, PAz;
  double kp;
  double bound;  // sqrt(max_i (ab|ab)_ii) of this primitive pair alone
  double pad;
};

// Compact primitive-pair records read by the J/K kernels (next to a float
// bound array, same indexing): P - A = -bp * AB with bp = beta/p.
struct __align__(32) PrimRec64 {
  double p, inv_p, kp, bp;
};
struct __align__(16) PrimRec32 {
  float p, inv_p, kp, bp;
};

// The ket-side fields of the sorted pair table as separate arrays, so that
// the 32 lanes of a warp, which hold consecutive kets, load each field
// with coalesced 16-byte accesses (the 80-byte PairInfo records would
// spread one field over 20 cache lines).
struct KetSoA {
  const double2* a0;  // Ax, Ay
  const double2* a1;  // Az, ABx
  const double2* a2;  // ABy, ABz
  const int4* ii;     // ao_a, ao_b, rec_off, rec_stride
  const int2* nn;     // npp, same
};

// Work entry of one J/K launch: bra pair and the range of ket pairs
// [k_lo, k_hi) (global pair indices, kets of one pair class).
struct JKEntry {
  int bra, k_lo, k_hi, pad;
};

// One molecule of a batched J/K launch: its launch's work queue and the
// buffers of its context (RHF: the total density is the spin density).
struct JKJob {
  const JKEntry* entries;
  const long long* prefix;
  const long long* chunk_start;
  const int* chunk_entry;
  const PairInfo* pairs;
  const double* pairQ;
  const PrimRec64* rec64;
  const PrimRec32* rec32;
  const float* pbound;
  KetSoA kets;
  const double* Dtot;
  const float* Dtot32;  // its FP32 copy (FP32 launches)
  double* Jacc;
  double* Kacc;
  double thr, prim_eps;  // the molecule's Schwarz and primitive thresholds
  int n;
};

struct JKLaunchArgs {
  const JKEntry* entries;
  const long long* prefix;  // warp-task prefix over entries (size nentries + 1)
  const long long* chunk_start;  // work-queue steps: tasks [chunk_start[c], chunk_start[c + 1])
  const int* chunk_entry;        // entry holding the first task of each step
  int nentries;
  long long nchunks;
  long long nwarps;
  const PairInfo* pairs;
  KetSoA kets;          // ket-side fields of `pairs` (same indexing)
  const double* pairQ;  // Schwarz bound per pair; a lane's quartet counts if Q_bra Q_ket > thr
  double thr;
  const PrimRec64* rec64;
  const PrimRec32* rec32;
  const float* pbound;  // primitive-pair bounds, sorted descending within each pair
  const double* boys64;
  const float* boys32;
  const double* expt64;  // e^{-T0} per Boys grid row
  const float* expt32;
  unsigned long long* counter;  // work-queue counter of this launch (zeroed before it)
  const double* Dtot;  // n x n
  const double* Dspin; // nspin n x n
  // FP32 copies of Dtot / Dspin, read by the FP32 launches (required for
  // them)
  const float* Dtot32;
  const float* Dspin32;
  double* Jacc;        // n x n
  double* Kacc;        // nspin n x n
  int n, nspin;
  double prim_eps;
  // deterministic mode: one warp takes the steps in order and each task runs
  // once per lane with only that lane's quartet active, so every atomic add
  // lands in a fixed order
  int serial;
  // batched launches: molecule table and the first step of each molecule
  const JKJob* jobs;
  const long long* job_steps;
  int njobs;
};

}  // namespace hfg
