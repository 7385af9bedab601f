// hfg_jk_device_noalloc: the direct J/K build without any device allocation.
//
// Who needs this: callers that must not allocate device memory while they
// run -- latency-bound loops that cannot afford cudaMalloc's implicit device
// synchronisation, and host programs whose device memory is entirely handed
// out by their own allocator (a framework's caching pool that reserves the
// GPU up front), where a cudaMalloc from this library would fail or steal
// memory the host has promised elsewhere.  hfg_jk_device keeps its
// unsymmetrised J'/K' accumulators and work-queue counters in buffers it
// allocates on first use; this entry point keeps them instead in one
// file-scope device array, reserved when the library is loaded and held by
// every GPU that loads it until the process exits.
//
// Limit: the array holds 8 MiB: the plan's work-queue counters (8 bytes per
// launch, rounded up to 256 bytes) plus (1 + nspin) * n^2 doubles of
// accumulators, and for plans with FP32 launches (mixed precision)
// (1 + nspin) * n^2 floats of FP32 density copies.  So n <= 724 for RHF and
// n <= 591 for UHF in FP64, n <= 591 and n <= 482 in mixed precision (for
// plans of up to 224 launches; an s/p/d basis needs at most 42).  Larger
// systems are rejected with HFG_ERR_INVALID_INPUT.
//
// The first call on a device looks up the array's device address (once per
// device, with that device current); make that first call before any stream
// capture.  Every call on a device shares the one array and it keeps the
// previous call's contents, so each call clears the counters and
// accumulators first; calls that overlap on the GPU (several host threads, or
// several streams) race on the array and must be serialised by the caller.
#include <cuda_runtime.h>

#include <mutex>

#include "hfg_ctx.h"
#include "jk_dispatch.h"

namespace {

constexpr size_t kScratchBytes = 8u << 20;
constexpr int kMaxDevices = 64;

static __device__ __align__(256) unsigned char g_jk_scratch[kScratchBytes];

std::mutex g_setup_mu;
void* g_scratch_ptr[kMaxDevices] = {};

// Device address of g_jk_scratch on the current device.  Host code may not
// use the symbol itself as a pointer (it names a host-side stand-in), so the
// address is looked up once per device, with that device current.
int scratch_address(hfg_ctx* ctx, int device, void** out) {
  if (device < 0 || device >= kMaxDevices) return hfg::set_error(ctx, HFG_ERR_INVALID_INPUT, "device index");
  std::lock_guard<std::mutex> lk(g_setup_mu);
  if (!g_scratch_ptr[device]) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_jk_scratch);
    if (e != cudaSuccess || !p) return hfg::cuda_check(ctx, e == cudaSuccess ? cudaErrorUnknown : e, "scratch address");
    g_scratch_ptr[device] = p;
  }
  *out = g_scratch_ptr[device];
  return HFG_OK;
}

__global__ void symmetrize_noalloc(const double* __restrict__ acc, double* __restrict__ out, int n, int nmat) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long nn = (long long)n * n;
  if (t >= nn * nmat) return;
  const long long m = t / nn, r = t % nn;
  const int i = (int)(r / n), j = (int)(r % n);
  out[t] = 0.5 * (acc[m * nn + (long long)i * n + j] + acc[m * nn + (long long)j * n + i]);
}

// FP32 copies of the densities for the FP32 launches of a mixed plan.
__global__ void densities_f32_noalloc(const double* __restrict__ Pt, const double* __restrict__ Ps,
                                      float* __restrict__ out, long long nn, int nspin) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nn * (1 + nspin)) return;
  out[t] = (float)(t < nn ? Pt[t] : Ps[t - nn]);
}

}  // namespace

extern "C" int hfg_jk_device_noalloc(hfg_ctx* ctx, const hfg_jk_opts* opts, int nspin, const double* dPt,
                                     const double* dPs, double* dJ, double* dK) {
  if (!ctx) return HFG_ERR_INVALID_INPUT;
  if (!dPt || !dPs || !dJ || !dK) return hfg::set_error(ctx, HFG_ERR_INVALID_INPUT, "null pointer");
  if (nspin < 1 || nspin > 2) return hfg::set_error(ctx, HFG_ERR_INVALID_INPUT, "nspin must be 1 or 2");
  hfg_jk_opts o;
  if (opts) o = *opts; else hfg_jk_opts_default(&o);
  // the same checks as hfg_jk_device, before the plan lookup (a NaN key
  // would break the ordering of the plan map)
  if (!(o.schwarz_threshold >= 0.0) || !(o.prim_threshold >= 0.0) ||
      (o.precision != HFG_FP64 && o.precision != HFG_MIXED) ||
      (o.precision == HFG_MIXED && !(o.mixed_threshold >= 0.0)) || o.tile < 0 || o.tile > 4096)
    return hfg::set_error(ctx, HFG_ERR_INVALID_INPUT, "invalid J/K options");
  const size_t nn = (size_t)ctx->n * ctx->n;
  const char* too_big =
      "hfg_jk_device_noalloc: (1 + nspin) * n^2 doubles (and in mixed precision (1 + nspin) * n^2 floats) and the "
      "work-queue counters exceed its 8 MiB scratch (n <= 724 for RHF, n <= 591 for UHF; mixed precision n <= 591 "
      "and n <= 482); use hfg_jk_device";
  if (256 + (size_t)(1 + nspin) * nn * sizeof(double) > kScratchBytes)
    return hfg::set_error(ctx, HFG_ERR_INVALID_INPUT, too_big);
  std::lock_guard<std::mutex> lk(ctx->mu);
  auto it = ctx->plans.find(std::make_tuple(o.schwarz_threshold, o.precision == HFG_MIXED ? o.mixed_threshold : 0.0,
                                            o.prim_threshold, o.precision, o.tile > 0 ? o.tile : 64));
  if (it == ctx->plans.end())
    return hfg::set_error(ctx, HFG_ERR_INVALID_INPUT,
                          "hfg_jk_device_noalloc: no launch plan for these options on this context; call hfg_jk or "
                          "hfg_jk_device once with them first (that call allocates the plan)");
  const hfg::Plan& plan = *it->second;
  // counters first (one per launch, rounded up to keep the accumulators
  // 256-byte aligned), then J' and K'
  const size_t counter_bytes = (plan.launches.size() * sizeof(unsigned long long) + 255) / 256 * 256;
  const size_t acc_bytes = (size_t)(1 + nspin) * nn * sizeof(double);
  bool any32 = false;
  for (const hfg::Launch& L : plan.launches) any32 = any32 || L.fp32;
  const size_t f32_bytes = any32 ? (size_t)(1 + nspin) * nn * sizeof(float) : 0;
  const size_t need = counter_bytes + acc_bytes + f32_bytes;
  if (need > kScratchBytes) return hfg::set_error(ctx, HFG_ERR_INVALID_INPUT, too_big);
  if (cudaSetDevice(ctx->device) != cudaSuccess) return hfg::set_error(ctx, HFG_ERR_CUDA, "cudaSetDevice");
  void* base = nullptr;
  int rc = scratch_address(ctx, ctx->device, &base);
  if (rc != HFG_OK) return rc;
  unsigned char* b = static_cast<unsigned char*>(base);
  unsigned long long* counters = reinterpret_cast<unsigned long long*>(b);
  double* Jacc = reinterpret_cast<double*>(b + counter_bytes);
  double* Kacc = Jacc + nn;
  float* D32 = reinterpret_cast<float*>(b + counter_bytes + acc_bytes);
  // the array keeps the last call's contents: clear counters and accumulators
  rc = hfg::cuda_check(ctx, cudaMemsetAsync(b, 0, counter_bytes + acc_bytes, ctx->stream), "scratch clear");
  if (rc != HFG_OK) return rc;
  if (any32) {
    const long long tot = (long long)nn * (1 + nspin);
    densities_f32_noalloc<<<(unsigned)((tot + 255) / 256), 256, 0, ctx->stream>>>(dPt, dPs, D32, (long long)nn,
                                                                                  nspin);
    rc = hfg::cuda_check(ctx, cudaGetLastError(), "FP32 densities");
    if (rc != HFG_OK) return rc;
  }
  hfg::JKLaunchArgs a{};
  a.pairs = ctx->d_pairs.p;
  a.kets = ctx->kets();
  a.pairQ = ctx->d_pairQ.p;
  a.thr = o.schwarz_threshold;
  a.rec64 = ctx->d_rec64.p;
  a.rec32 = ctx->d_rec32.p;
  a.pbound = ctx->d_pbound.p;
  a.boys64 = ctx->d_boys64.p;
  a.boys32 = ctx->d_boys32.p;
  a.expt64 = ctx->d_expt64.p;
  a.expt32 = ctx->d_expt32.p;
  a.Dtot = dPt;
  a.Dspin = dPs;
  a.Dtot32 = any32 ? D32 : nullptr;
  a.Dspin32 = any32 ? D32 + nn : nullptr;
  a.Jacc = Jacc;
  a.Kacc = Kacc;
  a.n = ctx->n;
  a.nspin = nspin;
  a.prim_eps = o.prim_threshold;
  a.serial = o.deterministic != 0;
  for (size_t l = 0; l < plan.launches.size(); ++l) {
    const hfg::Launch& L = plan.launches[l];
    a.counter = counters + l;
    a.entries = L.d_entries;
    a.prefix = L.d_prefix;
    a.chunk_entry = L.d_chunk;
    a.chunk_start = L.d_cstart;
    a.nchunks = L.nchunks;
    a.nentries = (int)L.prefix[0];
    a.nwarps = L.prefix[1];
    rc = hfg::cuda_check(ctx, hfg::launch_jk(L.la, L.lb, L.lc, L.ld, L.fp32, a, ctx->stream), "J/K launch");
    if (rc != HFG_OK) return rc;
  }
  const int blk = 256;
  symmetrize_noalloc<<<(unsigned)((nn + blk - 1) / blk), blk, 0, ctx->stream>>>(Jacc, dJ, ctx->n, 1);
  symmetrize_noalloc<<<(unsigned)((nspin * nn + blk - 1) / blk), blk, 0, ctx->stream>>>(Kacc, dK, ctx->n, nspin);
  rc = hfg::cuda_check(ctx, cudaGetLastError(), "symmetrize");
  if (rc != HFG_OK) return rc;
  ctx->last = plan.stats;
  ctx->last_plan = it->second.get();
  return HFG_OK;
}
