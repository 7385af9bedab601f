/*
 * hfg.h -- C ABI of the B200 Fock-build library (libhfg.so).
 *
 * Drop-in replacement, at the C level, for hf-rs's integral and Fock-build
 * calls.  Each entry point names the hf-rs function it stands in for
 * (paths relative to the hf-rs project root).  All host matrices are
 * row-major doubles owned by the caller; device state lives behind the
 * opaque handles.  Every call returns an hfg_status; hfg_last_error()
 * gives the message of the last failure on a context.
 *
 * Threading: one context per CUDA stream.  Calls on one context are
 * serialised by the context; different contexts may run concurrently.
 */
#ifndef HFG_H
#define HFG_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes; the first four mirror HfError (src/error.rs:6-15). */
typedef enum {
  HFG_OK = 0,
  HFG_ERR_INVALID_INPUT = 1, /* HfError::InvalidInput */
  HFG_ERR_INTEGRAL = 2,      /* HfError::Integral */
  HFG_ERR_SCF = 3,           /* HfError::Scf (and the SCF drivers' Err(String)) */
  HFG_ERR_OOM = 4,           /* device memory or admission budget exhausted */
  HFG_ERR_TIMEOUT = 5,       /* a bounded device wait gave up */
  HFG_ERR_CUDA = 6,          /* CUDA runtime / library failure */
  HFG_ERR_UNSUPPORTED = 7    /* angular momentum or shape not built into this library */
} hfg_status;

/*
 * A list of Cartesian contracted Gaussians, laid out exactly like hf-rs's
 * Vec<ContractedGaussian> (src/basis.rs:87-100): per function its centre
 * (bohr), Cartesian powers, atom index and primitives whose coefficients are
 * fully normalised for that component (src/basis.rs:455-496).  Functions of
 * one shell must be consecutive and complete, as build_basis emits them
 * (src/ao.rs:133-164).
 */
typedef struct {
  int n;                /* number of Cartesian functions */
  const double* center; /* [n][3] */
  const int* lxyz;      /* [n][3] */
  const int* atom;      /* [n] */
  const int* prim_off;  /* [n+1] offsets into exps/coefs */
  const double* exps;   /* [prim_off[n]] */
  const double* coefs;  /* [prim_off[n]] */
} hfg_basis;

typedef enum { HFG_FP64 = 0, HFG_MIXED = 1 } hfg_precision;

typedef struct {
  double schwarz_threshold; /* keep (ab|cd) iff Q_ab*Q_cd > this; hf-rs uses 1e-12
                               (src/shell_integrals.rs:184) */
  double prim_threshold;    /* drop primitive quartets whose Cauchy-Schwarz bound is
                               below this; 0 reproduces hf-rs's quartet set exactly */
  int precision;            /* hfg_precision */
  int deterministic;        /* 1: bitwise reproducible J/K for debugging (one warp
                               runs the work queue in order and its lanes add
                               into J/K one at a time; slow); 0: atomics in
                               arrival order (default) */
  double mixed_threshold;   /* HFG_MIXED: quartets with Q_ab*Q_cd below this are
                               evaluated in FP32 and accumulated in FP64 */
  int tile;                 /* quartet tile of the work queue: a warp takes up to
                               `tile` tasks of 32 shell quartets per step, and
                               steps are sized for tile/8 tasks of average cost
                               per resident warp (0: 64) */
} hfg_jk_opts;

typedef struct hfg_ctx hfg_ctx;

/* Default options: Schwarz 1e-12, no primitive screening, FP64, atomic
   (not deterministic) accumulation, tile 64. */
void hfg_jk_opts_default(hfg_jk_opts* opts);

/*
 * Creates a context for one basis on one device: groups the functions into
 * shells, builds the shell-pair and primitive-pair tables and the Schwarz
 * bounds Q_ab = sqrt(max_i (ab|ab)_ii) on the device (src/shell_integrals.rs:
 * 156-173).  `stream` is a cudaStream_t (NULL = a stream owned by the
 * context).
 */
int hfg_ctx_create(const hfg_basis* basis, int device, void* stream, hfg_ctx** out);
int hfg_ctx_destroy(hfg_ctx* ctx);
const char* hfg_last_error(const hfg_ctx* ctx);

/* Basic sizes: Cartesian functions, shells, shell pairs. */
int hfg_ctx_sizes(const hfg_ctx* ctx, int* n_ao, int* n_shell, long* n_pair);

/* Schwarz bounds in hf-rs shell-pair order (a >= b, row by row). */
int hfg_schwarz(hfg_ctx* ctx, double* bounds, long n);

/*
 * Stands in for compute_shell_quartet (src/shell_integrals.rs:138-151):
 * the contracted Cartesian block (ab|cd) for shells a,b,c,d of the context
 * basis, a,b,c,d row-major.  `out` holds n_a*n_b*n_c*n_d doubles.
 */
int hfg_shell_quartet(hfg_ctx* ctx, int a, int b, int c, int d, double* out);

/*
 * compute_eri_tensor (src/scf.rs:275-333, built by compute_shell_eri_tensor,
 * src/shell_integrals.rs:156-240): the packed 8-fold tensor of Cartesian
 * integrals, slot c(c(mu,nu), c(lam,sig)) with c(i,j) = i(i+1)/2 + j for
 * i >= j (src/scf.rs:222-235); shell quartets with Q_ab Q_cd <= threshold
 * stay zero (hf-rs uses 1e-12).  len must be n_p (n_p + 1) / 2 with
 * n_p = n (n + 1) / 2.  hfg_eri_packed fills a host array (the tensor is
 * built on the device, which needs len doubles of device memory);
 * hfg_eri_packed_device fills a device array on the context stream.
 */
int hfg_eri_packed(hfg_ctx* ctx, double schwarz_threshold, double* out, size_t len);
int hfg_eri_packed_device(hfg_ctx* ctx, double schwarz_threshold, double* d_out, size_t len);

/*
 * Stands in for compute_eri_tensor (src/scf.rs:275) followed by
 * contract_jk (src/scf.rs:337-364), without storing the integrals: a direct
 * J/K build from densities.  P_total (n x n) gives J; P_spin holds nspin
 * n x n densities giving nspin K matrices (nspin = 1: RHF, K from P_total
 * passed again; nspin = 2: UHF alpha/beta).  Host pointers; the call copies
 * inputs to the device, builds, and copies J and K back.
 */
int hfg_jk(hfg_ctx* ctx, const hfg_jk_opts* opts, int nspin, const double* P_total, const double* P_spin,
           double* J, double* K);

/*
 * One shard of a J/K build for a multi-GPU Fock build (no hf-rs counterpart:
 * hf-rs parallelises one process with Rayon).  Every launch's work queue is
 * cut into `nshards` ranges of equal nominal cost and this call runs range
 * `shard`, so J and K of all shards sum to hfg_jk_device's (J/K are linear in
 * the integrals).  Device pointers, context stream; each rank of a
 * multi-GPU build calls it with its own shard and then sums J and K over the
 * ranks (one all-reduce of (1 + nspin) n^2 doubles).
 */
int hfg_jk_device_shard(hfg_ctx* ctx, const hfg_jk_opts* opts, int nspin, const double* d_P_total,
                        const double* d_P_spin, double* d_J, double* d_K, int shard, int nshards);

/* As hfg_jk with device pointers, on the context stream, without copies. */
int hfg_jk_device(hfg_ctx* ctx, const hfg_jk_opts* opts, int nspin, const double* d_P_total,
                  const double* d_P_spin, double* d_J, double* d_K);

/*
 * No counterpart in hf-rs.  As hfg_jk_device, but allocates no device
 * memory at all, for callers that cannot allocate while they run:
 * latency-bound loops that cannot take cudaMalloc's device synchronisation,
 * and host programs whose own allocator has reserved all device memory.
 * The J'/K' accumulators and work-queue counters live in one 8 MiB device
 * array that the library reserves when it is loaded, so (1 + nspin) * n^2
 * doubles plus 8 bytes per launch of the plan (rounded up to 256), and in
 * mixed precision (1 + nspin) * n^2 floats of FP32 density copies, must fit:
 * n <= 724 (RHF), n <= 591 (UHF) in FP64, n <= 591 (RHF), n <= 482 (UHF) in
 * mixed precision; larger systems return HFG_ERR_INVALID_INPUT.  The launch plan for `opts` must already exist on
 * the context (one earlier hfg_jk or hfg_jk_device call with the same
 * options builds it).  The first call on a device looks up the array's
 * device address; make that first call before any stream capture.  All calls
 * on a device share the array, which keeps the last call's contents (each
 * call clears what it uses first): calls that overlap on the GPU race and
 * must be serialised by the caller.
 */
int hfg_jk_device_noalloc(hfg_ctx* ctx, const hfg_jk_opts* opts, int nspin, const double* d_P_total,
                          const double* d_P_spin, double* d_J, double* d_K);

/*
 * No counterpart in hf-rs, which builds one molecule's J and K per call
 * (contract_jk, src/scf.rs:337-364).  RHF J and K of n_jobs molecules, one
 * context each (no context twice, all on one device), in one pass: for each
 * angular class and precision one launch covers the work queues of every
 * molecule, so a batch of small molecules fills the GPU where their
 * separate builds would each leave it mostly idle.  d_P[j], d_J[j], d_K[j]
 * are molecule j's n_j x n_j device matrices; results equal hfg_jk_device's
 * per molecule up to FP64 summation order.  Runs on `stream` (NULL: the
 * first context's stream), after the work already queued on every context
 * stream, and every context stream waits for it.  Does not synchronise.
 */
int hfg_jk_device_batch(hfg_ctx* const* ctxs, int n_jobs, const hfg_jk_opts* opts, const double* const* d_P,
                        double* const* d_J, double* const* d_K, void* stream);

/*
 * Stands in for contract_eri_derivatives with the RHF / UHF densities of
 * compute_gradient_from_density (src/gradient.rs:33-69, :287-301) and the
 * UHF driver: the two-electron part of the analytic nuclear gradient,
 * grad[3 * atom + axis] = dE2/dR, E2 = 1/2 sum (ab|cd) (P_ab P_cd - x
 * (P_ac P_bd + P_ad P_bc)) with x = 1/4 on P_total (nspin 1, P_spin =
 * P_total) or x = 1/2 per spin density (nspin 2).  Host pointers; `natom`
 * must exceed every basis function's atom index.  Shells up to d (the
 * derivative integrals raise one shell to f); quartets with Q_ab Q_cd <=
 * schwarz_threshold are skipped.
 */
int hfg_eri_gradient(hfg_ctx* ctx, double schwarz_threshold, int nspin, const double* P_total, const double* P_spin,
                     int natom, double* grad);

/*
 * Stands in for compute_gradient_from_density (src/gradient.rs:287-455), as
 * compute_rhf_gradient / compute_uhf_gradient call it: the analytic nuclear
 * gradient dE/dR (grad[3 * atom + axis], hartree/bohr) of an SCF solution
 * given its total density P_total, its spin densities as hfg_eri_gradient
 * takes them, and the energy-weighted density W = sum_occ eps_i C_i C_i^T
 * (x 2 for a closed shell), all host n x n in the Cartesian basis: nuclear
 * repulsion, the one-electron terms (basis derivatives of S, T, V and the
 * operator derivative of V) and the two-electron terms.  Nuclei as in
 * hfg_scf_opts (bohr).  Shells up to d.
 */
int hfg_gradient(hfg_ctx* ctx, int natom, const double* positions, const double* charges, int nspin,
                 const double* P_total, const double* P_spin, const double* W, double schwarz_threshold,
                 double* grad);

/* Stands in for build_fock_matrix (src/scf.rs:366-369): F = H + J - K/2. */
int hfg_fock_rhf(hfg_ctx* ctx, const hfg_jk_opts* opts, const double* H, const double* P, double* F);

/* Stands in for build_uhf_fock_matrices (src/scf.rs:371-375):
   F_a = H + J - K_a, F_b = H + J - K_b with J from P_a + P_b. */
int hfg_fock_uhf(hfg_ctx* ctx, const hfg_jk_opts* opts, const double* H, const double* Pa, const double* Pb,
                 double* Fa, double* Fb);

/* Work counters of the last J/K build on this context: shell quartets and
   primitive quartets evaluated in FP64 and FP32, and W_MD-weighted flops
   (the McMurchie-Davidson count per primitive quartet of each class). */
typedef struct {
  double quartets_fp64, quartets_fp32;
  double prim_quartets_fp64, prim_quartets_fp32;
  double wmd_flops_fp64, wmd_flops_fp32;
  int launches;
} hfg_jk_stats;
int hfg_jk_last_stats(const hfg_ctx* ctx, hfg_jk_stats* stats);

/*
 * Autotuner of the mixed-precision J/K build (no hf-rs counterpart: hf-rs
 * has a single FP64 path).  For the given densities (device pointers, as
 * hfg_jk_device) it builds J/K once in plain FP64 (Schwarz screening only,
 * the reference's arithmetic) and then, for every pair of FP32 threshold
 * and primitive threshold in the candidate lists, times `repeats` mixed
 * builds on the device (CUDA events on the context stream; the first build
 * of each candidate, which makes its plan, is not timed) and evaluates the
 * energy error of the build,
 *   dE = 1/2 sum P_total (J - J64) - w sum_s P_s (K_s - K64_s),
 * w = 1/4 for RHF (nspin 1) and 1/2 for UHF.  The fastest candidate with
 * |dE| <= max_energy_error is returned in `best` (schwarz_threshold from
 * `base`); if none qualifies, `best` is the FP64 options of `base` and
 * `found` is 0.  Then the best pair is timed with each quartet tile of
 * `tiles` (hfg_jk_opts.tile) and the fastest within the budget kept.  Empty
 * candidate lists use 1e-7, 1e-6, 1e-5, 1e-4 (FP32), 1e-15, 1e-14, 1e-13
 * (primitives) and tiles 8, 16, 32, 256 (beside the default 64); the default budget
 * is 5e-9 Eh.
 */
typedef struct {
  double fp32_thresholds[8];
  int n_fp32;
  double prim_thresholds[8];
  int n_prim;
  double max_energy_error;
  int repeats;
  int tiles[4]; /* quartet tiles tried on the best threshold pair (hfg_jk_opts.tile) */
  int n_tile;
} hfg_autotune_opts;
typedef struct {
  hfg_jk_opts best;
  int found;
  double best_ms, best_energy_error;
  double fp64_ms;                   /* the plain FP64 build */
  int evaluated;
  double ms[64], energy_error[64];  /* per candidate: FP32-threshold-major order,
                                       then one per tile on the best pair */
} hfg_autotune_result;
void hfg_autotune_opts_default(hfg_autotune_opts* opts);
int hfg_jk_autotune(hfg_ctx* ctx, const hfg_jk_opts* base, int nspin, const double* d_P_total,
                    const double* d_P_spin, const hfg_autotune_opts* opts, hfg_autotune_result* result);

/* Density fitting (src/df.rs, src/hf_variants/ri_df_hf.rs). */
typedef enum { HFG_DF_FP64 = 0, HFG_DF_FP32 = 1, HFG_DF_BF16 = 2 } hfg_df_precision;
typedef struct hfg_df hfg_df;

/*
 * Stands in for DfTensor::build (src/df.rs:89-127, Cartesian auxiliary
 * space): the Coulomb metric (P|Q), its canonical orthogonaliser with
 * `metric_cutoff` (src/df.rs:16-28), the three-centre integrals (P|mn) and
 * B = X^T (P|mn), all on the device.  B keeps the unique AO pairs of the
 * shell pairs whose Schwarz bound exceeds `pair_threshold` (0 keeps all, as
 * hf-rs) and is stored in `storage` precision (hfg_df_precision).
 */
int hfg_df_build(hfg_ctx* ctx, const hfg_basis* aux, double metric_cutoff, double pair_threshold, int storage,
                 hfg_df** out);
/*
 * No counterpart in hf-rs (one process, Rayon over Q, src/df.rs:143-173).
 * As hfg_df_build, but the factor holds only rows [R shard / nshards,
 * R (shard + 1) / nshards) of the R whitened auxiliary functions: one rank's
 * share of a multi-GPU DF build.  Every rank evaluates the three-centre
 * integrals of all auxiliary functions; the B GEMM, the factor's memory and
 * the J/K built from it (hfg_df_jk and its variants, which then give that
 * rank's partial J and K, to be summed over the ranks) are divided.
 * hfg_df_sizes reports the shard's rows.  DF-RHF and RI-MP2 need the whole
 * factor and refuse a shard.
 */
int hfg_df_build_shard(hfg_ctx* ctx, const hfg_basis* aux, double metric_cutoff, double pair_threshold, int storage,
                       int shard, int nshards, hfg_df** out);
int hfg_df_destroy(hfg_df* df);
int hfg_df_sizes(const hfg_df* df, int* naux, int* rank, long long* ncol);
/* The metric (P|Q) as built (naux x naux, row-major). */
int hfg_df_metric(hfg_df* df, double* M);
/*
 * Stands in for three_center_integrals (src/df.rs:60-78): (P|mu nu) of every
 * auxiliary function P of `aux` (rows) and every AO pair mu >= nu of the
 * context's basis (packed columns compound_index(mu, nu), src/scf.rs:222),
 * row-major, len = n_aux * n (n + 1) / 2, unscreened.  Meant for inspection
 * and small systems (the factor build never forms this matrix whole).
 */
int hfg_df_three_center(hfg_ctx* ctx, const hfg_basis* aux, double* out, size_t len);
/*
 * Stands in for DfTensor::coulomb_exchange_rhf (src/df.rs:133-174): J and K
 * of the density 2 C_occ C_occ^T, C_occ row-major n x nocc (host).  `mma`
 * selects the K GEMMs: FP64, TF32 (FP32 storage) or BF16 tensor cores with
 * FP32 accumulation, summed into FP64.
 */
int hfg_df_jk(hfg_df* df, const double* C_occ, int nocc, double* J, double* K, int mma);
/*
 * One shard of hfg_df_jk for a multi-GPU DF build (no hf-rs counterpart:
 * hf-rs's loop over the auxiliary index Q is one Rayon map-reduce,
 * src/df.rs:143-173).  Shard s of N sums J and K over the auxiliary functions
 * [s R / N, (s + 1) R / N) of the factor's R; the shards' J and K add up to
 * hfg_df_jk's (one all-reduce of 2 n^2 doubles).  Host buffers as hfg_df_jk.
 */
int hfg_df_jk_shard(hfg_df* df, const double* C_occ, int nocc, double* J, double* K, int mma, int shard,
                    int nshards);
/*
 * As hfg_df_jk_shard with device pointers on the context stream: d_C is the
 * occupied block column-major (n x nocc, leading dimension n), d_J and d_K
 * are n x n.
 */
int hfg_df_jk_device_shard(hfg_df* df, const double* d_C, int nocc, double* d_J, double* d_K, int mma, int shard,
                           int nshards);
/*
 * Stands in for DfTensor::transform (src/df.rs:182-210): the factor in the MO
 * basis C (host, row-major n x m, hf-rs's Matrix with m MO columns),
 * out[Q][compound_index(p, q)] = (C^T B_Q C)[p][q] for p >= q, row-major
 * rank x m (m + 1) / 2 (len must equal that).  FP64 on the stored factor.
 */
int hfg_df_transform(hfg_df* df, const double* C, int m, double* out, size_t len);
/*
 * Stands in for DfTensor::transform(C) followed by mp2_energy(eps, n_occ,
 * n_frozen) (src/df.rs:182-236): the closed-shell RI-MP2 correlation energy
 * in the canonical MO basis C (row-major n x m) with orbital energies eps[m]
 * and the n_frozen lowest occupied orbitals frozen.  Rejects an invalid
 * partition (HFG_ERR_INVALID_INPUT) and a denominator within 1e-12 of zero
 * (HFG_ERR_SCF, hf-rs's HfError::Response).
 */
int hfg_df_mp2(hfg_df* df, const double* C, const double* eps, int m, int n_occ, int n_frozen, double* energy);
/*
 * Stands in for pivoted_cholesky_eri (src/cholesky.rs:42-190): the pivoted
 * Cholesky vectors of the AO ERI supermatrix, (pq|rs) ~ sum_K L_K(pq) L_K(rs),
 * to a largest residual diagonal <= threshold, as a factor handle over every
 * packed AO pair (hfg_df_jk and hfg_scf_df then run Cholesky-factorised RHF,
 * run_cd_hf).  The pivot is the largest residual diagonal, ties within 1e-12
 * relative going to the smallest packed index.  `budget` bounds the stored
 * vectors' bytes (hf-rs's CD_HF_FACTOR_BUDGET is 512 MiB); the supermatrix
 * itself is held on the device (n_p (n_p + 1) / 2 doubles, n_p = n (n + 1) / 2).
 * Outputs the largest residual diagonal, the pivots in selection order (up
 * to max_pivots of them) and their count.
 */
int hfg_cholesky_eri(hfg_ctx* ctx, double threshold, size_t budget, hfg_df** out, double* max_residual,
                     long long* pivots, int max_pivots, int* n_pivots);
/*
 * No counterpart in hf-rs.  Device time (ms) of the exchange (K) of the last
 * tensor-core hfg_df_jk on this factor, the tensor-core flops it executed
 * (both GEMMs, zero tiles skipped, lower triangle of K only), and the share
 * of the 128-row tiles of the unpacked B_Q that hold any stored AO pair.
 */
int hfg_df_last_stats(hfg_df* df, double* k_ms, double* k_flops, double* tiles_fraction);

/* Options of hfg_scf: nuclei, electrons, AO space and convergence controls of
   run_scf_in_space_with_convergence / run_uhf_in_space_with_convergence
   (src/scf.rs:410, :691; RhfConvergence src/scf.rs:400-407). */
typedef struct {
  int natom;
  const double* positions; /* [natom][3] bohr */
  const double* charges;   /* [natom] nuclear charges */
  int charge;              /* molecular charge */
  int multiplicity;        /* 2S + 1 */
  int uhf;                 /* 0: RHF, 1: UHF */
  int spherical;           /* 1: real spherical AO space (BasisKind::Spherical, src/ao.rs:14-27) */
  int max_iter;
  double energy_tol, residual_tol, density_tol;
  hfg_jk_opts jk;          /* J/K options; HFG_MIXED runs FP32 quartets until converged,
                              then FP64 iterations (refine_iters at least) to convergence */
  int refine_iters;
  int diis_size;           /* CDIIS subspace (hf-rs: 8, src/scf.rs:479) */
  int verbose;             /* iteration table on stderr */
  int guess;               /* 0: superposition of atomic densities (hf-rs's default, src/sad.rs),
                              1: core Hamiltonian */
  double incremental_tol;  /* HFG_MIXED phase only: J/K built from the density change dP since the
                              last full build, skipping shell quartets with Q_ab Q_cd max|dP| below
                              this (1e-12 by default; 0: a full build every iteration) */
  int rebuild_every;       /* full build after this many incremental ones (default 8) */
  double refine_at;        /* HFG_MIXED: the FP64 refinement starts once the three convergence
                              measures are below refine_at times their tolerances (default 10;
                              1: the mixed phase converges fully first) */
} hfg_scf_opts;

typedef struct {
  double energy, electronic, nuclear;
  double energy_before_refinement; /* HFG_MIXED: energy when the mixed phase converged */
  double s2;                       /* UHF <S^2> */
  int iterations, converged, n_mo;
  int fock_builds_fp64, fock_builds_mixed;
  double time_ms;
  int fock_builds_incremental;     /* of the mixed builds, those from a density change */
} hfg_scf_result;

/* Defaults: RHF singlet, 100 iterations, tolerances derived from 1e-10 as
   run_scf_in_space does (src/scf.rs:393-399), FP64 J/K, 2 refinement
   iterations, CDIIS(8), incremental mixed builds at 1e-12 with a full
   build every 8. */
void hfg_scf_opts_default(hfg_scf_opts* opts);

/*
 * Stands in for run_scf_in_space_with_convergence (src/scf.rs:410-627) and
 * run_uhf_in_space_with_convergence (src/scf.rs:691-979) with CDIIS: a
 * direct SCF whose one-electron integrals, Fock builds, DIIS and
 * diagonalisations all run on the device.  Initial guess as hf-rs: the
 * superposition of cached atomic fractional-occupation HF densities
 * (src/sad.rs:56-259), or the core Hamiltonian on request.
 * Optional outputs (NULL to skip), row-major: P and F (nspin x n x n),
 * C (nspin x n x n_mo, Cartesian rows), orbital energies (nspin x n_mo).
 * Returns HFG_ERR_SCF if not converged within max_iter (results still set).
 */
int hfg_scf(hfg_ctx* ctx, const hfg_scf_opts* opts, hfg_scf_result* result, double* P, double* F, double* C,
            double* eps);

/*
 * Stands in for run_df_hf_with_aux / run_factorized_rhf
 * (src/hf_variants/ri_df_hf.rs:122-263): DF-RHF with the DF tensor `df`
 * built on this context.  Uses the nuclei, charge, AO space, iteration
 * limit, tolerances and DIIS size of `opts`, and its guess: 1 = the core
 * Hamiltonian, as run_factorized_rhf; 0 = orbitals of the Fock matrix of
 * the SAD density (one FP64 four-centre build).  `mma` HFG_DF_FP32 (TF32)
 * or HFG_DF_BF16 runs tensor-core J/K until loosely converged, then FP64
 * arithmetic on the stored factor to the tolerances; HFG_DF_FP64 runs FP64
 * throughout.  Optional outputs (row-major n x n, NULL to skip): P, F, J, K
 * at convergence.
 */
int hfg_scf_df(hfg_ctx* ctx, hfg_df* df, int mma, const hfg_scf_opts* opts, hfg_scf_result* result, double* P,
               double* F, double* J, double* K);

/* ---- Serving: a request loop for streams of SCF jobs (no hf-rs counterpart;
   each job runs the hfg_scf equivalent of run_scf_in_space_with_convergence /
   run_uhf_in_space_with_convergence). ---- */
typedef struct {
  hfg_basis basis;          /* copied at submit */
  int natom;
  const double* positions;  /* [natom][3] bohr, copied */
  const double* charges;    /* [natom], copied */
  int charge, multiplicity, uhf, spherical;
  int max_iter;
  double energy_tol, residual_tol, density_tol;
  hfg_jk_opts jk;
  long long tag;            /* caller's identifier, returned with the result */
} hfg_job;

typedef struct {
  long long tag;
  int status, iterations, converged, n_ao;
  double energy, energy_before_refinement;
  double submit_ms, start_ms, end_ms; /* since hfg_server_create */
  long long footprint_bytes;
} hfg_job_result;

typedef struct hfg_server hfg_server;

/* `slots` worker slots (host threads with their own CUDA streams) on one
   device; jobs are admitted first in, first out when a slot is free and their
   estimated device footprint fits in `hbm_budget_bytes` minus the running
   jobs' footprints. */
int hfg_server_create(int device, int slots, long long hbm_budget_bytes, hfg_server** out);
/* Queue a job (non-blocking; inputs are copied).  HFG_ERR_OOM if the job
   alone exceeds the budget. */
int hfg_server_submit(hfg_server* server, const hfg_job* job);
/* Up to `max` completed jobs; with wait_for_one, blocks until one completes
   or nothing is pending or running. */
int hfg_server_poll(hfg_server* server, hfg_job_result* out, int max, int* n_out, int wait_for_one);
int hfg_server_stats(hfg_server* server, int* pending, int* running, long long* in_use_bytes);
/* Jobs submitted with HFG_MIXED J/K options but fewer than n_ao basis
   functions run FP64 (primitive screening at 1e-15 at most): on small jobs
   the refinement builds cost more than FP32 saves.  Default 256. */
int hfg_server_set_mixed_min_ao(hfg_server* server, int n_ao);
/* Fock builds of RHF jobs with fewer than max_ao functions are batched
   across the running jobs (hfg_jk_device_batch's launches): a batch takes
   the builds submitted within window_us of its first one, or fewer when
   every batching job has one queued.  max_ao = 0 turns batching off.
   Defaults: 256 functions, 300 us. */
int hfg_server_set_batching(hfg_server* server, int max_ao, double window_us);
/* Builds that went through batches, and the number of batches. */
int hfg_server_batch_stats(hfg_server* server, long long* batched_builds, long long* batches);
/* Finishes the queued jobs, then stops the workers. */
int hfg_server_destroy(hfg_server* server);

/* Measured FMA-pipe peak of the device in TFLOP/s (FP64 when fp32 == 0):
   independent FMA chains in registers on every SM.  The roofline
   denominator of the ERI kernels, which are bound by these pipes. */
int hfg_fma_peak(int device, int fp32, double* tflops);

#ifdef __cplusplus
}
#endif

#endif /* HFG_H */
