// Serving loop for streams of SCF jobs (continuous batching at job level).
//
// Jobs arrive through hfg_server_submit as callers receive them.  A fixed set
// of worker slots, each a host thread with its own CUDA stream, take jobs in
// arrival order; a job is admitted when a slot is free and its estimated
// device footprint fits in what the budget has left, so that requests which
// arrive while others are running start as soon as a slot and memory free
// up.  Every admitted job keeps its density, Fock, DIIS history and orbitals
// on the device for its whole SCF (hfg_scf), and the kernels of the running
// jobs overlap on the GPU through their streams (all device memory of a job
// is stream-ordered, so no job synchronises the device).  Completed jobs
// are reported with their submit / start / end times for latency
// percentiles.  hf-rs has no serving layer; this is the request loop that
// calls the hf-rs-equivalent SCF entry point for each job.
//
// Fock builds of small RHF jobs are batched across jobs: their contexts
// route every J/K build to the server's batcher, which collects the builds
// that the running jobs submit within a short window (or until every
// batching job has one queued) and runs them as one batched build
// (jk_batch_locked: one launch per angular class over all their work
// queues).  A small molecule's own build is a few dozen launches of a few
// blocks each, which leave most of the GPU idle; a batch fills it.  Larger
// jobs, whose own launches fill the GPU, and UHF jobs build alone on their
// streams.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <memory>
#include <mutex>
#include <thread>
#include <vector>

#include "hfg_ctx.h"

namespace {

struct JobCopy {
  long long tag;
  std::vector<double> center, exps, coefs, positions, charges;
  std::vector<int> lxyz, atom, prim_off;
  int n;
  hfg_job spec;  // scalar fields; pointers re-bound to the copies above
  long long footprint;
  double submit_ms;
};

}  // namespace

namespace hfg {

struct JKBatcher {
  struct Req {
    hfg_ctx* ctx;
    hfg_jk_opts o;
    const double* P;
    double* J;
    double* K;
    int rc;
    bool done;
  };
  int device = 0;
  double window_us = 300.0;
  std::mutex mu;
  std::condition_variable cv;
  std::vector<Req*> open;  // builds of the batch being collected
  int participants = 0;    // running jobs whose builds come here
  long long batches = 0, builds = 0;
  // one batch enqueues at a time, on the batcher's stream, with its tables
  // staged through a ring of pinned buffers
  std::mutex exec_mu;
  cudaStream_t stream = nullptr;
  static constexpr int kSlots = 4;
  static constexpr size_t kSlotBytes = 1 << 20;
  BatchStaging slots[kSlots];
  int next_slot = 0;

  explicit JKBatcher(int dev) : device(dev) {
    cudaSetDevice(dev);
    cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking);
    for (auto& x : slots) {
      if (cudaMallocHost(&x.host, kSlotBytes) == cudaSuccess) x.bytes = kSlotBytes; else x.host = nullptr;
      cudaEventCreateWithFlags(&x.ev, cudaEventDisableTiming);
    }
    cudaGetLastError();
  }
  ~JKBatcher() {
    cudaSetDevice(device);
    if (stream) cudaStreamSynchronize(stream);
    for (auto& x : slots) {
      if (x.host) cudaFreeHost(x.host);
      if (x.ev) cudaEventDestroy(x.ev);
    }
    if (stream) cudaStreamDestroy(stream);
  }
  void join() {
    std::lock_guard<std::mutex> lk(mu);
    ++participants;
  }
  void leave() {
    {
      std::lock_guard<std::mutex> lk(mu);
      --participants;
    }
    cv.notify_all();  // a collecting batch may now be complete
  }
};

// The first build of a batch leads it: it waits until every participant has
// a build queued or the window has passed, takes the queue and enqueues the
// batch; the others wait until their batch has been enqueued.  Nothing waits
// on the device here: each context's stream waits for its batch by event.
int batcher_submit(JKBatcher* b, hfg_ctx* ctx, const hfg_jk_opts& o, const double* dP, double* dJ, double* dK) {
  JKBatcher::Req r{ctx, o, dP, dJ, dK, HFG_OK, false};
  std::unique_lock<std::mutex> lk(b->mu);
  b->open.push_back(&r);
  if (b->open.size() > 1) {
    b->cv.notify_all();
    b->cv.wait(lk, [&] { return r.done; });
    return r.rc;
  }
  const auto deadline = std::chrono::steady_clock::now() + std::chrono::microseconds((long long)b->window_us);
  b->cv.wait_until(lk, deadline, [&] { return (int)b->open.size() >= b->participants; });
  std::vector<JKBatcher::Req*> batch;
  batch.swap(b->open);
  lk.unlock();
  int rc = HFG_OK;
  {
    std::lock_guard<std::mutex> ex(b->exec_mu);
    const int m = (int)batch.size();
    std::vector<hfg_ctx*> ctxs(m);
    std::vector<hfg_jk_opts> opts(m);
    std::vector<const double*> P(m);
    std::vector<double*> J(m), K(m);
    for (int j = 0; j < m; ++j) {
      ctxs[j] = batch[j]->ctx;
      opts[j] = batch[j]->o;
      P[j] = batch[j]->P;
      J[j] = batch[j]->J;
      K[j] = batch[j]->K;
    }
    BatchStaging* slot = &b->slots[b->next_slot];
    b->next_slot = (b->next_slot + 1) % JKBatcher::kSlots;
    cudaSetDevice(b->device);
    rc = jk_batch_locked(ctxs.data(), m, opts.data(), P.data(), J.data(), K.data(), b->stream, slot);
  }
  lk.lock();
  ++b->batches;
  b->builds += (long long)batch.size();
  for (JKBatcher::Req* q : batch) {
    q->rc = rc;
    q->done = true;
  }
  lk.unlock();
  b->cv.notify_all();
  return rc;
}

}  // namespace hfg

struct hfg_server {
  int device = 0;
  long long budget = 0, in_use = 0;
  int mixed_min_ao = 256;  // mixed-precision jobs below this size run FP64
  int batch_max_ao = 256;  // RHF jobs below this size batch their Fock builds (0: none)
  std::unique_ptr<hfg::JKBatcher> batcher;
  std::chrono::steady_clock::time_point t0;
  std::mutex mu;
  std::condition_variable cv_work, cv_done;
  std::deque<JobCopy> pending;
  std::vector<hfg_job_result> done;
  std::vector<std::thread> workers;
  bool stopping = false;
  int running = 0;
  double now_ms() const {
    return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
  }
};

namespace {

// Device bytes a job needs: shell-pair and primitive-pair tables, launch
// plans, the SCF matrices (S, H, scratch, X, P, F, J, K, error vectors and
// a DIIS history of 8 Fock / error pairs per spin) and the J/K accumulators.
long long estimate_footprint(const hfg_basis* b, int uhf) {
  // shells: consecutive functions of one centre and total l
  std::vector<int> K;
  for (int i = 0; i < b->n;) {
    const int l = b->lxyz[3 * i] + b->lxyz[3 * i + 1] + b->lxyz[3 * i + 2];
    K.push_back(b->prim_off[i + 1] - b->prim_off[i]);
    i += (l + 1) * (l + 2) / 2;
  }
  const long long ns = (long long)K.size(), npair = ns * (ns + 1) / 2;
  long long kk = 0, ksum = 0;
  for (int k : K) ksum += k;
  kk = ksum * ksum / 2 + ksum;
  const long long n = b->n, nn = n * n, nspin = uhf ? 2 : 1;
  long long bytes = npair * 64 + kk * (64 + 32 + 16 + 4);
  bytes += npair * 21 * 2 * 24;                 // plan entries and prefixes (both precisions)
  bytes += nn * 8 * (12 + nspin * (6 + 2 * 8));  // SCF matrices and DIIS history
  bytes += nn * 8 * (1 + 2 * nspin);             // J/K accumulators
  return bytes + (4 << 20);
}

void worker(hfg_server* s) {
  cudaSetDevice(s->device);
  cudaStream_t st;
  cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking);
  for (;;) {
    JobCopy job;
    {
      std::unique_lock<std::mutex> lk(s->mu);
      // FIFO admission: the oldest job starts once a slot is free (this
      // thread) and its footprint fits in what the budget has left
      s->cv_work.wait(lk, [&] {
        if (s->pending.empty()) return s->stopping;
        return s->in_use + s->pending.front().footprint <= s->budget || s->running == 0;
      });
      if (s->pending.empty()) break;
      job = std::move(s->pending.front());
      s->pending.pop_front();
      s->in_use += job.footprint;
      ++s->running;
    }
    hfg_job_result r{};
    r.tag = job.tag;
    r.submit_ms = job.submit_ms;
    r.start_ms = s->now_ms();
    r.footprint_bytes = job.footprint;
    hfg_basis b{job.n, job.center.data(), job.lxyz.data(), job.atom.data(), job.prim_off.data(), job.exps.data(),
                job.coefs.data()};
    hfg_ctx* ctx = nullptr;
    int rc = hfg_ctx_create(&b, s->device, st, &ctx);
    bool batched = false;
    if (rc == HFG_OK && !job.spec.uhf && job.n < s->batch_max_ao && s->batcher && ctx->lmax <= hfg::kLMax) {
      ctx->batcher = s->batcher.get();
      s->batcher->join();
      batched = true;
    }
    if (rc == HFG_OK) {
      hfg_scf_opts o;
      hfg_scf_opts_default(&o);
      o.natom = (int)job.charges.size();
      o.positions = job.positions.data();
      o.charges = job.charges.data();
      o.charge = job.spec.charge;
      o.multiplicity = job.spec.multiplicity;
      o.uhf = job.spec.uhf;
      o.spherical = job.spec.spherical;
      o.max_iter = job.spec.max_iter;
      o.energy_tol = job.spec.energy_tol;
      o.residual_tol = job.spec.residual_tol;
      o.density_tol = job.spec.density_tol;
      // precision policy: mixed precision pays only on larger jobs (FP32
      // quartets, then FP64 refinement builds and extra plans); smaller ones
      // run FP64 with primitive screening at 1e-15 at most
      o.jk = job.spec.jk;
      if (o.jk.precision == HFG_MIXED && job.n < s->mixed_min_ao) {
        o.jk.precision = HFG_FP64;
        o.jk.prim_threshold = std::min(o.jk.prim_threshold, 1e-15);
      }
      o.refine_iters = 2;
      hfg_scf_result res{};
      rc = hfg_scf(ctx, &o, &res, nullptr, nullptr, nullptr, nullptr);
      r.energy = res.energy;
      r.energy_before_refinement = res.energy_before_refinement;
      r.iterations = res.iterations;
      r.converged = res.converged;
      r.n_ao = job.n;
    }
    if (batched) s->batcher->leave();
    if (ctx) hfg_ctx_destroy(ctx);
    cudaStreamSynchronize(st);
    r.status = rc;
    r.end_ms = s->now_ms();
    {
      std::lock_guard<std::mutex> lk(s->mu);
      s->in_use -= job.footprint;
      --s->running;
      s->done.push_back(r);
    }
    s->cv_work.notify_all();
    s->cv_done.notify_all();
  }
  cudaStreamDestroy(st);
}

}  // namespace

extern "C" {

int hfg_server_create(int device, int slots, long long hbm_budget_bytes, hfg_server** out) {
  if (!out || slots < 1 || slots > 256 || hbm_budget_bytes <= 0) return HFG_ERR_INVALID_INPUT;
  if (cudaSetDevice(device) != cudaSuccess) return HFG_ERR_CUDA;
  auto s = new hfg_server();
  s->device = device;
  s->budget = hbm_budget_bytes;
  s->t0 = std::chrono::steady_clock::now();
  s->batcher = std::make_unique<hfg::JKBatcher>(device);
  for (int i = 0; i < slots; ++i) s->workers.emplace_back(worker, s);
  *out = s;
  return HFG_OK;
}

int hfg_server_submit(hfg_server* s, const hfg_job* job) {
  if (!s || !job || job->basis.n <= 0 || job->natom <= 0) return HFG_ERR_INVALID_INPUT;
  JobCopy c;
  const hfg_basis& b = job->basis;
  c.tag = job->tag;
  c.n = b.n;
  c.center.assign(b.center, b.center + 3 * b.n);
  c.lxyz.assign(b.lxyz, b.lxyz + 3 * b.n);
  c.atom.assign(b.atom, b.atom + b.n);
  c.prim_off.assign(b.prim_off, b.prim_off + b.n + 1);
  c.exps.assign(b.exps, b.exps + b.prim_off[b.n]);
  c.coefs.assign(b.coefs, b.coefs + b.prim_off[b.n]);
  c.positions.assign(job->positions, job->positions + 3 * job->natom);
  c.charges.assign(job->charges, job->charges + job->natom);
  c.spec = *job;
  c.footprint = estimate_footprint(&b, job->uhf);
  {
    std::lock_guard<std::mutex> lk(s->mu);
    if (c.footprint > s->budget) return HFG_ERR_OOM;
    c.submit_ms = s->now_ms();
    s->pending.push_back(std::move(c));
  }
  s->cv_work.notify_all();
  return HFG_OK;
}

int hfg_server_poll(hfg_server* s, hfg_job_result* out, int max, int* n_out, int wait_for_one) {
  if (!s || !n_out || (max > 0 && !out)) return HFG_ERR_INVALID_INPUT;
  std::unique_lock<std::mutex> lk(s->mu);
  if (wait_for_one)
    s->cv_done.wait(lk, [&] { return !s->done.empty() || (s->pending.empty() && s->running == 0); });
  const int k = std::min<int>(max, (int)s->done.size());
  for (int i = 0; i < k; ++i) out[i] = s->done[i];
  s->done.erase(s->done.begin(), s->done.begin() + k);
  *n_out = k;
  return HFG_OK;
}

int hfg_server_set_mixed_min_ao(hfg_server* s, int n_ao) {
  if (!s || n_ao < 0) return HFG_ERR_INVALID_INPUT;
  std::lock_guard<std::mutex> lk(s->mu);
  s->mixed_min_ao = n_ao;
  return HFG_OK;
}

int hfg_server_set_batching(hfg_server* s, int max_ao, double window_us) {
  if (!s || max_ao < 0 || !(window_us >= 0.0) || window_us > 1e6) return HFG_ERR_INVALID_INPUT;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    s->batch_max_ao = max_ao;
  }
  std::lock_guard<std::mutex> lk(s->batcher->mu);
  s->batcher->window_us = window_us;
  return HFG_OK;
}

int hfg_server_batch_stats(hfg_server* s, long long* batched_builds, long long* batches) {
  if (!s) return HFG_ERR_INVALID_INPUT;
  std::lock_guard<std::mutex> lk(s->batcher->mu);
  if (batched_builds) *batched_builds = s->batcher->builds;
  if (batches) *batches = s->batcher->batches;
  return HFG_OK;
}

int hfg_server_stats(hfg_server* s, int* pending, int* running, long long* in_use_bytes) {
  if (!s) return HFG_ERR_INVALID_INPUT;
  std::lock_guard<std::mutex> lk(s->mu);
  if (pending) *pending = (int)s->pending.size();
  if (running) *running = s->running;
  if (in_use_bytes) *in_use_bytes = s->in_use;
  return HFG_OK;
}

int hfg_server_destroy(hfg_server* s) {
  if (!s) return HFG_OK;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    s->stopping = true;
  }
  s->cv_work.notify_all();
  for (auto& t : s->workers) t.join();
  delete s;
  return HFG_OK;
}

}  // extern "C"
