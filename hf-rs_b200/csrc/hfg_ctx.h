// Host-side context of libhfg: the basis as shells, the shell-pair and
// primitive-pair tables (device resident), and cached J/K launch plans.
#pragma once
#include <cuda_runtime.h>

#include <map>
#include <set>
#include <tuple>
#include <memory>
#include <mutex>
#include <string>
#include <tuple>
#include <vector>

#include "../../include/hfg.h"
#include "hfg_internal.h"

namespace hfg {

struct Shell {
  double c[3];
  int l, K, ao, atom;
  int prim_off;  // into hfg_ctx::exps / coefs (shell contraction coefficients)
};

struct PairClass {
  int la, lb, Ka, Kb;
  int first, count;  // range of the sorted global pair table
  // Schwarz-bound buckets (factor 4, descending) of the class: bucket j holds
  // pairs [first + bstart[j], first + bstart[j + 1]), ordered by AO index,
  // with largest bound bqmax[j]
  std::vector<int> bstart;
  std::vector<double> bqmax;
};

struct Launch {
  int la, lb, lc, ld;
  cudaStream_t st = nullptr;  // stream of the entries/prefix allocations
  bool fp32;
  double quartets = 0, prims = 0;  // shell quartets and primitive quartets (after screening) of this launch
  std::vector<JKEntry> entries;
  std::vector<long long> prefix;
  JKEntry* d_entries = nullptr;
  long long* d_prefix = nullptr;
  int* d_chunk = nullptr;             // entry of the first task of every work-queue step
  long long* d_cstart = nullptr;      // first task of every step (nchunks + 1)
  long long nchunks = 0;
  std::vector<double> cost_prefix;  // nominal cost of steps [0, c) (nchunks + 1)
};

struct Plan {
  std::vector<Launch> launches;
  hfg_jk_stats stats{};  // nominal counts until `counted`
  double thr = 0.0, prim_eps = 0.0;
  bool counted = false;  // exact shell/primitive-quartet counts made (on the first stats request)
};

// Stream on which DevBuf allocations of the current host thread are made
// (stream-ordered cudaMallocAsync / cudaFreeAsync, so that jobs running on
// different streams never synchronise the device through cudaFree).  Each
// C-ABI entry point sets it to its context's stream for its duration.
extern thread_local cudaStream_t tl_alloc_stream;
struct AllocScope {
  cudaStream_t prev;
  explicit AllocScope(cudaStream_t s) : prev(tl_alloc_stream) { tl_alloc_stream = s; }
  ~AllocScope() { tl_alloc_stream = prev; }
};

// Device buffer (stream-ordered when allocated under an AllocScope).
template <typename T> struct DevBuf {
  T* p = nullptr;
  size_t n = 0;
  cudaStream_t st = nullptr;
  cudaError_t alloc(size_t count) {
    if (count <= n) return cudaSuccess;
    release();
    st = tl_alloc_stream;
    cudaError_t e = st ? cudaMallocAsync((void**)&p, count * sizeof(T), st) : cudaMalloc(&p, count * sizeof(T));
    if (e == cudaSuccess) n = count; else p = nullptr;
    return e;
  }
  void release() {
    if (p) {
      if (st) cudaFreeAsync(p, st); else cudaFree(p);
    }
    p = nullptr;
    n = 0;
  }
  ~DevBuf() { release(); }
  DevBuf() = default;
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
  DevBuf(DevBuf&& o) noexcept : p(o.p), n(o.n), st(o.st) {
    o.p = nullptr;
    o.n = 0;
  }
};

}  // namespace hfg

namespace hfg {
// side streams on which a J/K build's class launches run next to the
// context stream
constexpr int kJKSideStreams = 3;
// Collects the RHF J/K builds of several contexts into batched builds
// (server.cu); a context with one set routes its builds through it.
struct JKBatcher;
}  // namespace hfg

struct hfg_ctx {
  int device = 0;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  // fork / join of a J/K build's class launches (created on first use)
  cudaStream_t side[hfg::kJKSideStreams] = {};
  hfg::JKBatcher* batcher = nullptr;  // RHF builds go through this batcher when set
  cudaEvent_t ev_fork = nullptr, ev_join[hfg::kJKSideStreams] = {};
  cudaError_t ensure_side_streams() {
    if (ev_fork) return cudaSuccess;
    // the side streams take the context stream's priority
    int prio = 0;
    if (stream && cudaStreamGetPriority(stream, &prio) != cudaSuccess) prio = 0;
    for (auto& x : side) {
      const cudaError_t e = cudaStreamCreateWithPriority(&x, cudaStreamNonBlocking, prio);
      if (e != cudaSuccess) return e;
    }
    for (auto& x : ev_join) {
      const cudaError_t e = cudaEventCreateWithFlags(&x, cudaEventDisableTiming);
      if (e != cudaSuccess) return e;
    }
    return cudaEventCreateWithFlags(&ev_fork, cudaEventDisableTiming);
  }
  std::mutex mu;
  std::string err;

  int n = 0;     // Cartesian functions
  int lmax = 0;  // highest shell angular momentum
  std::vector<hfg::Shell> shells;
  std::vector<double> exps, coefs;
  std::vector<std::pair<int, int>> ref_pairs;  // hf-rs order: (a, b), a >= b
  std::vector<int> ref_to_sorted;             // hf-rs pair index -> sorted pair index
  // J/K builds replayed as CUDA graphs, keyed by plan and buffers
  using GraphKey = std::tuple<const void*, int, const void*, const void*, const void*, const void*, const void*,
                              const void*, const void*>;
  bool use_graphs = true;
  hfg::Plan* last_plan = nullptr;  // plan of the last J/K build (for hfg_jk_last_stats)
  std::map<GraphKey, cudaGraphExec_t> graphs;
  std::set<GraphKey> graph_seen, graph_failed;
  std::vector<double> sorted_Q;               // Schwarz bound per sorted pair
  hfg::DevBuf<double> d_pairQ;                // the same on the device (per-lane screening)
  std::vector<hfg::PairInfo> h_pairs;         // sorted pair table
  std::vector<hfg::PrimPair> h_prims;
  std::vector<hfg::PairClass> classes;

  hfg::DevBuf<hfg::PairInfo> d_pairs;
  // ket-side fields of d_pairs as separate arrays (hfg::KetSoA)
  hfg::DevBuf<double2> d_ka0, d_ka1, d_ka2;
  hfg::DevBuf<int4> d_kii;
  hfg::DevBuf<int2> d_knn;
  hfg::KetSoA kets() const { return hfg::KetSoA{d_ka0.p, d_ka1.p, d_ka2.p, d_kii.p, d_knn.p}; }
  hfg::DevBuf<hfg::PrimPair> d_prims;
  hfg::DevBuf<hfg::PrimRec64> d_rec64;
  hfg::DevBuf<hfg::PrimRec32> d_rec32;
  hfg::DevBuf<float> d_pbound;
  hfg::DevBuf<double> d_boys64, d_expt64;
  hfg::DevBuf<float> d_boys32, d_expt32;
  hfg::DevBuf<unsigned long long> d_counters;  // one work-queue counter per J/K launch
  hfg::DevBuf<double> d_D, d_Ds, d_Jacc, d_Kacc, d_J, d_K, d_tmp;
  hfg::DevBuf<float> d_D32;  // FP32 copies of a build's densities (3 n^2)

  // launch plans by (Schwarz, FP32 and primitive thresholds, precision, tile)
  std::map<std::tuple<double, double, double, int, int>, std::unique_ptr<hfg::Plan>> plans;
  hfg_jk_stats last{};

  ~hfg_ctx();
};

struct hfg_df;

namespace hfg {
// Implemented in df.cu: DF J/K from column-major occupied coefficients,
// summed over the auxiliary functions [q_lo, q_hi) of the factor (q_hi < 0:
// all of them).
int df_jk_device(hfg_df* df, const double* dC, int nocc, double* dJ, double* dK, int mma, int q_lo = 0,
                 int q_hi = -1);
// Implemented in df.cu: the factor holds only a shard of the auxiliary rows.
bool df_is_shard(const hfg_df* df);
// Implemented in ctx.cu, used by scf.cu.
// shard / nshards: only the shard's cost-balanced range of work-queue steps
// of every launch (the partial J/K of all shards sum to the full build)
int jk_device_locked(hfg_ctx* ctx, const hfg_jk_opts* opts, int nspin, const double* dPt, const double* dPs,
                     double* dJ, double* dK, int shard = 0, int nshards = 1);
int set_error(hfg_ctx* ctx, int code, const std::string& msg);
// Pinned host memory for a batched build's tables, reused once `ev` (the
// previous copy out of it) has completed.
struct BatchStaging {
  void* host = nullptr;
  size_t bytes = 0;
  cudaEvent_t ev = nullptr;
};
// Implemented in ctx.cu: RHF J/K of several contexts in one pass of batched
// launches on `st` (molecule j with its own options opts[j]).  The caller
// owns every context (their locks held, or their owners blocked).
int jk_batch_locked(hfg_ctx* const* ctxs, int n_jobs, const hfg_jk_opts* opts, const double* const* dP,
                    double* const* dJ, double* const* dK, cudaStream_t st, BatchStaging* staging);
// Implemented in server.cu: queue one RHF build with the batcher and wait
// until the batch that takes it has been enqueued.
int batcher_submit(JKBatcher* b, hfg_ctx* ctx, const hfg_jk_opts& o, const double* dP, double* dJ, double* dK);
// Implemented in ctx.cu: the packed 8-fold ERI tensor on the device (length
// n_p (n_p + 1) / 2), quartets with Q_ab Q_cd > thr; the context lock held.
int eri_packed_locked(hfg_ctx* ctx, double thr, double* d_out, size_t len);
int build_shell_list(hfg_ctx* ctx, const hfg_basis* b, int lmax);
// Implemented in oneint.cu: the one-electron terms of the nuclear gradient
// (basis derivatives of S, T, V against W and P, and the operator derivative
// of V) added into grad (host, natom x 3); the context lock held.
int one_electron_gradient(hfg_ctx* ctx, int natom, const double* pos, const double* charge, const double* P,
                          const double* W, double* grad);
void make_pair(const hfg_ctx* ctx, int a, int b, PairInfo& pi, std::vector<PrimPair>& pp, int owner);
int cuda_check(hfg_ctx* ctx, cudaError_t e, const char* what);
}  // namespace hfg
