// libhfg host runtime: context creation (shells, shell pairs, primitive
// pairs, Schwarz bounds on the device), J/K launch plans, and the C-ABI
// entry points declared in include/hfg.h.
#include <cuda_runtime.h>

#include <algorithm>
#include <array>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <numeric>

#include "boys.cuh"
#include "eri_md.h"
#include "hfg_ctx.h"
#include "jk_dispatch.h"

using namespace hfg;

namespace hfg {

thread_local cudaStream_t tl_alloc_stream = nullptr;

int set_error(hfg_ctx* ctx, int code, const std::string& msg) {
  if (ctx) ctx->err = msg;
  return code;
}

int cuda_check(hfg_ctx* ctx, cudaError_t e, const char* what) {
  if (e == cudaSuccess) return HFG_OK;
  const int code = (e == cudaErrorMemoryAllocation) ? HFG_ERR_OOM : HFG_ERR_CUDA;
  return set_error(ctx, code, std::string(what) + ": " + cudaGetErrorString(e));
}

#define HFG_CUDA(ctx, call)                               \
  do {                                                    \
    int _rc = cuda_check((ctx), (call), #call);           \
    if (_rc != HFG_OK) return _rc;                        \
  } while (0)

// McMurchie-Davidson flop count per primitive quartet of each class, from
// hf-rs's loops (src/shell_integrals.rs:101-131, src/integrals.rs:70-101,
// 259-346, 905-971); the work unit of the roofline.
static double wmd_flops(int la, int lb, int lc, int ld) {
  static const std::map<std::tuple<int, int, int, int>, double> t = {
      {{0, 0, 0, 0}, 61},     {{1, 0, 0, 0}, 126},    {{1, 0, 1, 0}, 333},    {{1, 1, 0, 0}, 327},
      {{1, 1, 1, 0}, 1072},   {{1, 1, 1, 1}, 3916},   {{2, 0, 0, 0}, 256},    {{2, 0, 1, 0}, 771},
      {{2, 0, 1, 1}, 2683},   {{2, 0, 2, 0}, 1872},   {{2, 1, 0, 0}, 747},    {{2, 1, 1, 0}, 2647},
      {{2, 1, 1, 1}, 9994},   {{2, 1, 2, 0}, 6751},   {{2, 1, 2, 1}, 25570},  {{2, 2, 0, 0}, 1776},
      {{2, 2, 1, 0}, 6607},   {{2, 2, 1, 1}, 25354},  {{2, 2, 2, 0}, 16978},  {{2, 2, 2, 1}, 64681},
      {{2, 2, 2, 2}, 162643}};
  auto it = t.find({la, lb, lc, ld});
  return it == t.end() ? 0.0 : it->second;
}

// Boys grid values F_0..F_{kBoysCols-1} at T = idx * 0.05, by the series at
// the highest tabulated order (47) and downward recursion, as hf-rs builds
// its table (src/integrals.rs:27-57).
const std::vector<double>& boys_table_host() {
  static std::vector<double> table;
  static std::once_flag once;
  std::call_once(once, [] {
    const int M = 47;
    table.assign((size_t)kBoysRows * kBoysCols, 0.0);
    std::vector<double> row(M + 1);
    for (int idx = 0; idx < kBoysRows; ++idx) {
      const double t = idx * kBoysStep;
      const double et = std::exp(-t);
      double term = 1.0 / (2 * M + 1), sum = term;
      for (long i = 1; i <= 10000; ++i) {
        term *= 2.0 * t / (double)(2 * M + 2 * i + 1);
        sum += term;
        if (term < sum * 1e-17) break;
      }
      row[M] = et * sum;
      for (int m = M - 1; m >= 0; --m) row[m] = (2.0 * t * row[m + 1] + et) / (2 * m + 1);
      for (int m = 0; m < kBoysCols; ++m) table[(size_t)idx * kBoysCols + m] = row[m];
    }
  });
  return table;
}

static int ncart(int l) { return (l + 1) * (l + 2) / 2; }

// hf-rs Cartesian component order (src/basis.rs:418-445, :179-188).
static void cart_order(int l, std::vector<std::array<int, 3>>& out) {
  out.clear();
  if (l == 2) {
    out = {{2, 0, 0}, {0, 2, 0}, {0, 0, 2}, {1, 1, 0}, {1, 0, 1}, {0, 1, 1}};
    return;
  }
  for (int lx = l; lx >= 0; --lx)
    for (int ly = l - lx; ly >= 0; --ly) out.push_back({lx, ly, l - lx - ly});
}

static double dfact(int n) {  // (n)!! with n <= 0 -> 1
  double r = 1.0;
  for (int k = n; k > 0; k -= 2) r *= k;
  return r;
}

static double comp_scale_host(const std::array<int, 3>& l) {
  return 1.0 / std::sqrt(dfact(2 * l[0] - 1) * dfact(2 * l[1] - 1) * dfact(2 * l[2] - 1));
}

// Groups the Cartesian functions into shells with the semantics of hf-rs's
// shell_ranges (src/ao.rs:133-164) and recovers the shell contraction
// coefficients (component coefficient / component scale).
int build_shell_list(hfg_ctx* ctx, const hfg_basis* b, int lmax) {
  if (!b || b->n <= 0 || !b->center || !b->lxyz || !b->atom || !b->prim_off || !b->exps || !b->coefs)
    return set_error(ctx, HFG_ERR_INVALID_INPUT, "empty or incomplete basis description");
  const int n = b->n;
  ctx->n = n;
  std::vector<std::array<int, 3>> order;
  int start = 0;
  while (start < n) {
    const int* l0 = b->lxyz + 3 * start;
    const int l = l0[0] + l0[1] + l0[2];
    if (l < 0 || l > 7) return set_error(ctx, HFG_ERR_INVALID_INPUT, "invalid angular momentum");
    if (l > lmax) return set_error(ctx, HFG_ERR_UNSUPPORTED, "angular momentum not built into the kernels");
    const int cnt = ncart(l);
    if (start + cnt > n) return set_error(ctx, HFG_ERR_INVALID_INPUT, "incomplete Cartesian shell");
    const int K = b->prim_off[start + 1] - b->prim_off[start];
    if (K <= 0) return set_error(ctx, HFG_ERR_INVALID_INPUT, "function without primitives");
    cart_order(l, order);
    Shell sh{};
    for (int k = 0; k < 3; ++k) {
      sh.c[k] = b->center[3 * start + k];
      if (!std::isfinite(sh.c[k])) return set_error(ctx, HFG_ERR_INVALID_INPUT, "non-finite geometry");
    }
    sh.l = l;
    sh.K = K;
    sh.ao = start;
    sh.atom = b->atom[start];
    sh.prim_off = (int)ctx->exps.size();
    const int p0 = b->prim_off[start];
    const double s0 = comp_scale_host(order[0]);
    for (int q = 0; q < K; ++q) {
      const double e = b->exps[p0 + q], c = b->coefs[p0 + q];
      if (!(e > 0.0) || !std::isfinite(e) || !std::isfinite(c))
        return set_error(ctx, HFG_ERR_INVALID_INPUT, "invalid primitive");
      ctx->exps.push_back(e);
      ctx->coefs.push_back(c / s0);
    }
    for (int f = 0; f < cnt; ++f) {
      const int g = start + f;
      const int* lg = b->lxyz + 3 * g;
      if (lg[0] != order[f][0] || lg[1] != order[f][1] || lg[2] != order[f][2])
        return set_error(ctx, HFG_ERR_UNSUPPORTED, "Cartesian components not in hf-rs build_basis order");
      if (b->atom[g] != sh.atom || b->prim_off[g + 1] - b->prim_off[g] != K)
        return set_error(ctx, HFG_ERR_INVALID_INPUT, "noncontiguous or incomplete Cartesian shell");
      for (int k = 0; k < 3; ++k)
        if (b->center[3 * g + k] != sh.c[k])
          return set_error(ctx, HFG_ERR_INVALID_INPUT, "noncontiguous or incomplete Cartesian shell");
      const double sg = comp_scale_host(order[f]);
      for (int q = 0; q < K; ++q) {
        if (b->exps[b->prim_off[g] + q] != ctx->exps[sh.prim_off + q])
          return set_error(ctx, HFG_ERR_INVALID_INPUT, "noncontiguous or incomplete Cartesian shell");
        const double c = b->coefs[b->prim_off[g] + q] / sg;
        const double ref = ctx->coefs[sh.prim_off + q];
        if (std::fabs(c - ref) > 1e-12 * std::max(1.0, std::fabs(ref)))
          return set_error(ctx, HFG_ERR_UNSUPPORTED, "component coefficients do not share one contraction");
      }
    }
    ctx->shells.push_back(sh);
    ctx->lmax = std::max(ctx->lmax, l);
    start += cnt;
  }
  return HFG_OK;
}

// Oriented pair (la >= lb, Ka >= Kb on ties) with its primitive pairs.
void make_pair(const hfg_ctx* ctx, int a, int b, PairInfo& pi, std::vector<PrimPair>& pp, int owner) {
  const Shell& A = ctx->shells[a];
  const Shell& B = ctx->shells[b];
  pi.Ax = A.c[0];
  pi.Ay = A.c[1];
  pi.Az = A.c[2];
  pi.ABx = A.c[0] - B.c[0];
  pi.ABy = A.c[1] - B.c[1];
  pi.ABz = A.c[2] - B.c[2];
  pi.ao_a = A.ao;
  pi.ao_b = B.ao;
  pi.same = (a == b);
  pi.pp_off = (int)pp.size();
  pi.npp = A.K * B.K;
  const double ab2 = pi.ABx * pi.ABx + pi.ABy * pi.ABy + pi.ABz * pi.ABz;
  for (int i = 0; i < A.K; ++i)
    for (int j = 0; j < B.K; ++j) {
      const double al = ctx->exps[A.prim_off + i], be = ctx->exps[B.prim_off + j];
      const double p = al + be, inv_p = 1.0 / p;
      PrimPair q{};
      q.p = p;
      q.inv_p = inv_p;
      // P - A = beta (B - A) / p
      q.PAx = -be * pi.ABx * inv_p;
      q.PAy = -be * pi.ABy * inv_p;
      q.PAz = -be * pi.ABz * inv_p;
      q.kp = ctx->coefs[A.prim_off + i] * ctx->coefs[B.prim_off + j] * std::exp(-al * be * inv_p * ab2) * inv_p;
      q.bound = 0.0;
      q.pad = (double)owner;
      pp.push_back(q);
    }
}

static bool oriented_swap(const Shell& A, const Shell& B) { return A.l < B.l || (A.l == B.l && A.K < B.K); }

static int build_pairs(hfg_ctx* ctx) {
  const int ns = (int)ctx->shells.size();
  ctx->ref_pairs.clear();
  for (int a = 0; a < ns; ++a)
    for (int b = 0; b <= a; ++b) ctx->ref_pairs.push_back({a, b});
  const long np = (long)ctx->ref_pairs.size();
  // class of each oriented pair
  std::map<std::tuple<int, int, int, int>, std::vector<long>> by_class;
  for (long r = 0; r < np; ++r) {
    auto [a, b] = ctx->ref_pairs[r];
    if (oriented_swap(ctx->shells[a], ctx->shells[b])) std::swap(a, b);
    by_class[{ctx->shells[a].l, ctx->shells[b].l, ctx->shells[a].K, ctx->shells[b].K}].push_back(r);
  }
  // grouped (unsorted) tables for the bound computation
  std::vector<PairInfo> gp;
  std::vector<PrimPair> gprim;
  std::vector<long> grouped_ref;
  std::vector<PairClass> cls;
  for (auto& [key, refs] : by_class) {
    PairClass c{std::get<0>(key), std::get<1>(key), std::get<2>(key), std::get<3>(key), (int)gp.size(),
                (int)refs.size()};
    for (long r : refs) {
      auto [a, b] = ctx->ref_pairs[r];
      if (oriented_swap(ctx->shells[a], ctx->shells[b])) std::swap(a, b);
      PairInfo pi{};
      make_pair(ctx, a, b, pi, gprim, (int)gp.size());
      pi.cls = (int)cls.size();
      gp.push_back(pi);
      grouped_ref.push_back(r);
    }
    cls.push_back(c);
  }
  // device bounds
  HFG_CUDA(ctx, ctx->d_pairs.alloc(gp.size()));
  HFG_CUDA(ctx, ctx->d_prims.alloc(gprim.size()));
  HFG_CUDA(ctx, cudaMemcpyAsync(ctx->d_pairs.p, gp.data(), gp.size() * sizeof(PairInfo), cudaMemcpyHostToDevice,
                                ctx->stream));
  HFG_CUDA(ctx, cudaMemcpyAsync(ctx->d_prims.p, gprim.data(), gprim.size() * sizeof(PrimPair),
                                cudaMemcpyHostToDevice, ctx->stream));
  DevBuf<double> dq, dpb;
  HFG_CUDA(ctx, dq.alloc(gp.size()));
  HFG_CUDA(ctx, dpb.alloc(gprim.size()));
  for (const auto& c : cls) {
    HFG_CUDA(ctx, launch_schwarz(c.la, c.lb, ctx->d_pairs.p, ctx->d_prims.p, c.first, c.count, ctx->d_boys64.p,
                                 ctx->d_expt64.p, dq.p + c.first, 0, ctx->stream));
    const int p0 = gp[c.first].pp_off;
    const int p1 = gp[c.first + c.count - 1].pp_off + gp[c.first + c.count - 1].npp;
    HFG_CUDA(ctx, launch_schwarz(c.la, c.lb, ctx->d_pairs.p, ctx->d_prims.p, p0, p1 - p0, ctx->d_boys64.p,
                                 ctx->d_expt64.p, dpb.p + p0, 1, ctx->stream));
  }
  std::vector<double> Q(gp.size()), PB(gprim.size());
  HFG_CUDA(ctx, cudaMemcpyAsync(Q.data(), dq.p, Q.size() * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
  HFG_CUDA(ctx, cudaMemcpyAsync(PB.data(), dpb.p, PB.size() * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
  HFG_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  dq.release();
  dpb.release();
  for (size_t i = 0; i < gprim.size(); ++i) gprim[i].bound = PB[i];
  // Sort each class into Schwarz-bound buckets of a factor 4 (descending)
  // and, within a bucket, by the AO index of its shells: the 32 kets of a
  // warp then lie close together, so the digestion's density loads and K
  // atomics along the bra's rows hit few cache lines.  The significant kets
  // of a bra are whole buckets plus, in the last one, those passing the
  // exact per-lane test.  Primitives are sorted by bound.
  ctx->h_pairs.clear();
  ctx->h_prims.clear();
  ctx->sorted_Q.clear();
  ctx->ref_to_sorted.assign(np, -1);
  ctx->classes = cls;
  for (auto& c : ctx->classes) {
    std::vector<int> idx(c.count);
    std::iota(idx.begin(), idx.end(), c.first);
    auto bucket = [&](int x) { return Q[x] > 0.0 ? (int)std::floor(0.5 * std::log2(Q[x])) : -(1 << 20); };
    std::stable_sort(idx.begin(), idx.end(), [&](int x, int y) {
      const int bx = bucket(x), by = bucket(y);
      if (bx != by) return bx > by;
      if (gp[x].ao_a != gp[y].ao_a) return gp[x].ao_a < gp[y].ao_a;
      return gp[x].ao_b < gp[y].ao_b;
    });
    c.bstart.clear();
    c.bqmax.clear();
    for (int k = 0; k < c.count; ++k) {
      if (k == 0 || bucket(idx[k]) != bucket(idx[k - 1])) {
        c.bstart.push_back(k);
        c.bqmax.push_back(0.0);
      }
      c.bqmax.back() = std::max(c.bqmax.back(), Q[idx[k]]);
    }
    c.bstart.push_back(c.count);
    c.first = (int)ctx->h_pairs.size();
    for (int g : idx) {
      PairInfo pi = gp[g];
      std::vector<PrimPair> pr(gprim.begin() + pi.pp_off, gprim.begin() + pi.pp_off + pi.npp);
      std::stable_sort(pr.begin(), pr.end(), [](const PrimPair& x, const PrimPair& y) { return x.bound > y.bound; });
      pi.pp_off = (int)ctx->h_prims.size();
      for (auto& q : pr) {
        q.pad = (double)ctx->h_pairs.size();
        ctx->h_prims.push_back(q);
      }
      ctx->ref_to_sorted[grouped_ref[g]] = (int)ctx->h_pairs.size();
      ctx->h_pairs.push_back(pi);
      ctx->sorted_Q.push_back(Q[g]);
    }
  }
  HFG_CUDA(ctx, ctx->d_pairQ.alloc(ctx->sorted_Q.size()));
  HFG_CUDA(ctx, cudaMemcpyAsync(ctx->d_pairQ.p, ctx->sorted_Q.data(), ctx->sorted_Q.size() * sizeof(double),
                                cudaMemcpyHostToDevice, ctx->stream));
  HFG_CUDA(ctx, cudaMemcpyAsync(ctx->d_pairs.p, ctx->h_pairs.data(), ctx->h_pairs.size() * sizeof(PairInfo),
                                cudaMemcpyHostToDevice, ctx->stream));
  HFG_CUDA(ctx, cudaMemcpyAsync(ctx->d_prims.p, ctx->h_prims.data(), ctx->h_prims.size() * sizeof(PrimPair),
                                cudaMemcpyHostToDevice, ctx->stream));
  // compact records for the J/K kernels, interleaved within each pair class:
  // record k of the class's pair p at base + k * count + p (all pairs of a
  // class have the same primitive count)
  const size_t npp = ctx->h_prims.size();
  std::vector<PrimRec64> r64(npp);
  std::vector<PrimRec32> r32(npp);
  std::vector<float> pb(npp);
  {
    size_t base = 0;
    for (const auto& c : ctx->classes) {
      for (int p = 0; p < c.count; ++p) {
        PairInfo& pi = ctx->h_pairs[c.first + p];
        pi.rec_off = (int)(base + p);
        pi.rec_stride = c.count;
        const double ab2 = pi.ABx * pi.ABx + pi.ABy * pi.ABy + pi.ABz * pi.ABz;
        for (int k = 0; k < pi.npp; ++k) {
          const PrimPair& q = ctx->h_prims[pi.pp_off + k];
          // P - A = -(beta/p) AB; recover beta/p from the stored P - A
          double bp = 0.0;
          if (ab2 > 0.0) bp = -(q.PAx * pi.ABx + q.PAy * pi.ABy + q.PAz * pi.ABz) / ab2;
          const size_t r = base + (size_t)k * c.count + p;
          r64[r] = {q.p, q.inv_p, q.kp, bp};
          r32[r] = {(float)q.p, (float)q.inv_p, (float)q.kp, (float)bp};
          pb[r] = (float)q.bound;
        }
      }
      base += (size_t)c.count * (size_t)c.Ka * c.Kb;
    }
  }
  HFG_CUDA(ctx, cudaMemcpyAsync(ctx->d_pairs.p, ctx->h_pairs.data(), ctx->h_pairs.size() * sizeof(PairInfo),
                                cudaMemcpyHostToDevice, ctx->stream));
  {
    const size_t np2 = ctx->h_pairs.size();
    std::vector<double2> a0(np2), a1(np2), a2(np2);
    std::vector<int4> ii(np2);
    std::vector<int2> nn(np2);
    for (size_t k = 0; k < np2; ++k) {
      const PairInfo& q = ctx->h_pairs[k];
      a0[k] = make_double2(q.Ax, q.Ay);
      a1[k] = make_double2(q.Az, q.ABx);
      a2[k] = make_double2(q.ABy, q.ABz);
      ii[k] = make_int4(q.ao_a, q.ao_b, q.rec_off, q.rec_stride);
      nn[k] = make_int2(q.npp, q.same);
    }
    HFG_CUDA(ctx, ctx->d_ka0.alloc(np2));
    HFG_CUDA(ctx, ctx->d_ka1.alloc(np2));
    HFG_CUDA(ctx, ctx->d_ka2.alloc(np2));
    HFG_CUDA(ctx, ctx->d_kii.alloc(np2));
    HFG_CUDA(ctx, ctx->d_knn.alloc(np2));
    HFG_CUDA(ctx, cudaMemcpyAsync(ctx->d_ka0.p, a0.data(), np2 * sizeof(double2), cudaMemcpyHostToDevice, ctx->stream));
    HFG_CUDA(ctx, cudaMemcpyAsync(ctx->d_ka1.p, a1.data(), np2 * sizeof(double2), cudaMemcpyHostToDevice, ctx->stream));
    HFG_CUDA(ctx, cudaMemcpyAsync(ctx->d_ka2.p, a2.data(), np2 * sizeof(double2), cudaMemcpyHostToDevice, ctx->stream));
    HFG_CUDA(ctx, cudaMemcpyAsync(ctx->d_kii.p, ii.data(), np2 * sizeof(int4), cudaMemcpyHostToDevice, ctx->stream));
    HFG_CUDA(ctx, cudaMemcpyAsync(ctx->d_knn.p, nn.data(), np2 * sizeof(int2), cudaMemcpyHostToDevice, ctx->stream));
    // the host vectors go out of scope: the copies must have read them
    HFG_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  }
  HFG_CUDA(ctx, ctx->d_rec64.alloc(npp));
  HFG_CUDA(ctx, ctx->d_rec32.alloc(npp));
  HFG_CUDA(ctx, ctx->d_pbound.alloc(npp));
  HFG_CUDA(ctx, cudaMemcpyAsync(ctx->d_rec64.p, r64.data(), npp * sizeof(PrimRec64), cudaMemcpyHostToDevice,
                                ctx->stream));
  HFG_CUDA(ctx, cudaMemcpyAsync(ctx->d_rec32.p, r32.data(), npp * sizeof(PrimRec32), cudaMemcpyHostToDevice,
                                ctx->stream));
  HFG_CUDA(ctx, cudaMemcpyAsync(ctx->d_pbound.p, pb.data(), npp * sizeof(float), cudaMemcpyHostToDevice, ctx->stream));
  HFG_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return HFG_OK;
}

// Launch plan for (Schwarz threshold, FP32 threshold, precision): for every
// pair of pair classes (bra class >= ket class) and every bra pair, the
// significant kets form a prefix of the ket class (kets sorted by Q); in
// mixed precision the kets below the FP32 threshold form the tail of it.
static int build_plan(hfg_ctx* ctx, double thr, double mixed, double prim_eps, int precision, int tile,
                      Plan*& out) {
  if (tile <= 0) tile = 64;
  auto key = std::make_tuple(thr, precision == HFG_MIXED ? mixed : 0.0, prim_eps, precision, tile);
  auto it = ctx->plans.find(key);
  if (it != ctx->plans.end()) {
    out = it->second.get();
    return HFG_OK;
  }
  auto plan = std::make_unique<Plan>();
  std::map<std::tuple<int, int, int, int, int>, int> lidx;
  auto get_launch = [&](int la, int lb, int lc, int ld, bool fp32) -> Launch& {
    auto k = std::make_tuple(la, lb, lc, ld, (int)fp32);
    auto f = lidx.find(k);
    if (f != lidx.end()) return plan->launches[f->second];
    lidx[k] = (int)plan->launches.size();
    Launch L;
    L.la = la;
    L.lb = lb;
    L.lc = lc;
    L.ld = ld;
    L.fp32 = fp32;
    L.prefix.push_back(0);
    plan->launches.push_back(std::move(L));
    return plan->launches.back();
  };
  const auto& Q = ctx->sorted_Q;
  // cumulative primitive-pair counts for the nominal primitive-quartet totals
  std::vector<double> cum(ctx->h_pairs.size() + 1, 0.0);
  for (size_t i = 0; i < ctx->h_pairs.size(); ++i) cum[i + 1] = cum[i] + ctx->h_pairs[i].npp;
  hfg_jk_stats st{};
  const int nc = (int)ctx->classes.size();
  for (int cb = 0; cb < nc; ++cb) {
    const PairClass& B = ctx->classes[cb];
    for (int ck = 0; ck <= cb; ++ck) {
      const PairClass& Kc = ctx->classes[ck];
      const double w = wmd_flops(B.la, B.lb, Kc.la, Kc.lb);
      for (int i = B.first; i < B.first + B.count; ++i) {
        const double qi = Q[i];
        // kets in the buckets that can hold qi * qj > thr (whole buckets;
        // the kernels test each quartet exactly)
        const int nb = (int)Kc.bqmax.size();
        int jb = 0;
        while (jb < nb && qi * Kc.bqmax[jb] > thr) ++jb;
        int nsig = Kc.bstart[jb];
        if (cb == ck) nsig = std::min(nsig, i - B.first + 1);
        if (nsig <= 0) continue;
        int n64 = nsig;
        // classes with an f shell run on the generic engine, FP64 only
        const bool generic = B.la > kLMax || B.lb > kLMax || Kc.la > kLMax || Kc.lb > kLMax;
        if (precision == HFG_MIXED && !generic) {
          // FP32 only for buckets whose every ket has qi * qj < mixed
          int jm = 0;
          while (jm < nb && qi * Kc.bqmax[jm] >= mixed) ++jm;
          n64 = std::min(nsig, Kc.bstart[jm]);
        }
        const int ranges[2][2] = {{0, n64}, {n64, nsig}};
        for (int r = 0; r < 2; ++r) {
          const int a0 = ranges[r][0], a1 = ranges[r][1];
          if (a1 <= a0) continue;
          Launch& L = get_launch(B.la, B.lb, Kc.la, Kc.lb, r == 1);
          L.entries.push_back({i, Kc.first + a0, Kc.first + a1, 0});
          L.prefix.push_back(L.prefix.back() + (a1 - a0 + 31) / 32);
          const double nq = a1 - a0;
          const double npr = ctx->h_pairs[i].npp * (cum[Kc.first + a1] - cum[Kc.first + a0]);
          L.quartets += nq;
          L.prims += npr;
          if (r == 0) {
            st.quartets_fp64 += nq;
            st.prim_quartets_fp64 += npr;
            st.wmd_flops_fp64 += npr * w;
          } else {
            st.quartets_fp32 += nq;
            st.prim_quartets_fp32 += npr;
            st.wmd_flops_fp32 += npr * w;
          }
        }
      }
    }
  }
  // most expensive launches first
  std::sort(plan->launches.begin(), plan->launches.end(), [](const Launch& x, const Launch& y) {
    return std::make_tuple(x.la + x.lb + x.lc + x.ld, x.fp32) > std::make_tuple(y.la + y.lb + y.lc + y.ld, y.fp32);
  });
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ctx->device);
  for (auto& L : plan->launches) {
    L.st = ctx->stream;
    // Work-queue steps.  Entries are ordered by the nominal cost of one of
    // their warp tasks (bra x ket primitive pairs, before primitive
    // screening), most expensive first, so that the cheap tasks form the
    // tail of the launch; consecutive tasks are cut into steps of about equal
    // nominal cost and at most `tile` tasks (the quartet tile: at the
    // default 64, about eight steps per resident warp, up to 32 warps per
    // SM; the step cost scales with the tile).  Each step's first task and
    // its entry are tabulated, so no warp searches the prefix.
    std::vector<double> cost;
    {
      const size_t ne = L.entries.size();
      cost.resize(ne);
      for (size_t e = 0; e < ne; ++e)
        cost[e] = (double)ctx->h_pairs[L.entries[e].bra].npp * ctx->h_pairs[L.entries[e].k_lo].npp;
      std::vector<size_t> ord(ne);
      std::iota(ord.begin(), ord.end(), 0);
      std::stable_sort(ord.begin(), ord.end(), [&](size_t x, size_t y) { return cost[x] > cost[y]; });
      std::vector<JKEntry> ents(ne);
      std::vector<double> c2(ne);
      L.prefix.assign(1, 0);
      for (size_t i = 0; i < ne; ++i) {
        ents[i] = L.entries[ord[i]];
        c2[i] = cost[ord[i]];
        L.prefix.push_back(L.prefix.back() + (ents[i].k_hi - ents[i].k_lo + 31) / 32);
      }
      L.entries.swap(ents);
      cost.swap(c2);
    }
    const long long nw_total = L.prefix.back();
    std::vector<long long> cstart;
    std::vector<int> chunk_entry;
    {
      double total = 0.0;
      for (size_t e = 0; e < L.entries.size(); ++e) total += cost[e] * (double)(L.prefix[e + 1] - L.prefix[e]);
      const double target = total / ((double)sms * 32 * 8) * ((double)tile / 64.0);
      size_t e = 0;
      long long t = 0;
      L.cost_prefix.assign(1, 0.0);
      while (t < nw_total) {
        while (L.prefix[e + 1] <= t) ++e;
        cstart.push_back(t);
        chunk_entry.push_back((int)e);
        double acc = 0.0;
        long long k = 0;
        size_t ee = e;
        while (t < nw_total && k < tile && (k == 0 || acc < target)) {
          while (L.prefix[ee + 1] <= t) ++ee;
          acc += cost[ee];
          ++t;
          ++k;
        }
        L.cost_prefix.push_back(L.cost_prefix.back() + acc);
      }
      cstart.push_back(nw_total);
      if (chunk_entry.empty()) chunk_entry.push_back(0);
    }
    L.nchunks = (long long)cstart.size() - 1;
    HFG_CUDA(ctx, cudaMallocAsync((void**)&L.d_entries, L.entries.size() * sizeof(JKEntry), ctx->stream));
    HFG_CUDA(ctx, cudaMallocAsync((void**)&L.d_prefix, L.prefix.size() * sizeof(long long), ctx->stream));
    HFG_CUDA(ctx, cudaMallocAsync((void**)&L.d_cstart, cstart.size() * sizeof(long long), ctx->stream));
    HFG_CUDA(ctx, cudaMemcpyAsync(L.d_cstart, cstart.data(), cstart.size() * sizeof(long long),
                                  cudaMemcpyHostToDevice, ctx->stream));
    HFG_CUDA(ctx, cudaMallocAsync((void**)&L.d_chunk, chunk_entry.size() * sizeof(int), ctx->stream));
    HFG_CUDA(ctx, cudaMemcpyAsync(L.d_entries, L.entries.data(), L.entries.size() * sizeof(JKEntry),
                                  cudaMemcpyHostToDevice, ctx->stream));
    HFG_CUDA(ctx, cudaMemcpyAsync(L.d_prefix, L.prefix.data(), L.prefix.size() * sizeof(long long),
                                  cudaMemcpyHostToDevice, ctx->stream));
    HFG_CUDA(ctx, cudaMemcpyAsync(L.d_chunk, chunk_entry.data(), chunk_entry.size() * sizeof(int),
                                  cudaMemcpyHostToDevice, ctx->stream));
    HFG_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    // the host copies are no longer needed beyond the counts
    const size_t ne = L.entries.size();
    const long long nw = L.prefix.back();
    L.entries.clear();
    L.entries.shrink_to_fit();
    L.prefix.assign({(long long)ne, nw});
  }
  plan->thr = thr;
  plan->prim_eps = prim_eps;
  st.launches = (int)plan->launches.size();
  plan->stats = st;
  out = plan.get();
  ctx->plans[key] = std::move(plan);
  return HFG_OK;
}

// Exact shell- and primitive-quartet counts of a plan (the per-lane Schwarz
// test and primitive screening of the kernels): the work unit of the
// roofline.  Made on the first stats request only, since an SCF builds
// plans it never reports on.
static int count_plan(hfg_ctx* ctx, Plan* plan) {
  if (plan->counted) return HFG_OK;
  const double thr = plan->thr, prim_eps = plan->prim_eps;
  hfg_jk_stats& st = plan->stats;
  {
    DevBuf<unsigned long long> cnt;
    const size_t nl = plan->launches.size();
    HFG_CUDA(ctx, cnt.alloc(2 * nl));
    HFG_CUDA(ctx, cudaMemsetAsync(cnt.p, 0, 2 * nl * 8, ctx->stream));
    for (size_t l = 0; l < nl; ++l) {
      const Launch& L = plan->launches[l];
      HFG_CUDA(ctx, launch_count(L.d_entries, L.d_prefix, (int)L.prefix[0], L.prefix[1], ctx->d_pairs.p,
                                 ctx->d_pairQ.p, thr, ctx->d_pbound.p, prim_eps, cnt.p + 2 * l, ctx->stream));
    }
    std::vector<unsigned long long> h(2 * nl);
    HFG_CUDA(ctx, cudaMemcpyAsync(h.data(), cnt.p, h.size() * 8, cudaMemcpyDeviceToHost, ctx->stream));
    HFG_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    cnt.release();
    st.prim_quartets_fp64 = st.prim_quartets_fp32 = st.wmd_flops_fp64 = st.wmd_flops_fp32 = 0.0;
    st.quartets_fp64 = st.quartets_fp32 = 0.0;
    for (size_t l = 0; l < nl; ++l) {
      Launch& L = plan->launches[l];
      L.prims = (double)h[2 * l];
      L.quartets = (double)h[2 * l + 1];
      const double w = wmd_flops(L.la, L.lb, L.lc, L.ld);
      if (L.fp32) {
        st.prim_quartets_fp32 += L.prims;
        st.quartets_fp32 += L.quartets;
        st.wmd_flops_fp32 += L.prims * w;
      } else {
        st.prim_quartets_fp64 += L.prims;
        st.quartets_fp64 += L.quartets;
        st.wmd_flops_fp64 += L.prims * w;
      }
    }
  }
  plan->counted = true;
  return HFG_OK;
}

__global__ void symmetrize_kernel(const double* __restrict__ acc, double* __restrict__ out, int n, int nmat) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long nn = (long long)n * n;
  if (t >= nn * nmat) return;
  const long long m = t / nn, r = t % nn;
  const int i = (int)(r / n), j = (int)(r % n);
  out[t] = 0.5 * (acc[m * nn + (long long)i * n + j] + acc[m * nn + (long long)j * n + i]);
}

// FP32 copies of the densities for the FP32 launches: out[0, nn) = Pt,
// out[nn, nn + nspin nn) = Ps.
__global__ void densities_to_f32_kernel(const double* __restrict__ Pt, const double* __restrict__ Ps,
                                        float* __restrict__ out, long long nn, int nspin) {
  const long long total = nn * (1 + nspin);
  for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < total;
       t += (long long)gridDim.x * blockDim.x)
    out[t] = (float)(t < nn ? Pt[t] : Ps[t - nn]);
}

// One matrix of a batched build: its accumulator and (symmetrised) output.
struct BatchMat {
  double* acc;
  double* out;
  int n;
};

// Over the matrices of a batched build (blockIdx.y): zero the accumulators
// (sym = 0) or write out = (acc + acc^T) / 2 (sym = 1).
__global__ void batch_mats_kernel(const BatchMat* __restrict__ mats, int sym) {
  const BatchMat m = mats[blockIdx.y];
  const long long nn = (long long)m.n * m.n;
  for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < nn; t += (long long)gridDim.x * blockDim.x) {
    if (!sym) {
      m.acc[t] = 0.0;
    } else {
      const long long i = t / m.n, j = t % m.n;
      m.out[t] = 0.5 * (m.acc[t] + m.acc[j * m.n + i]);
    }
  }
}

// a -= b
__global__ void axpy_sub_kernel(double* __restrict__ a, const double* __restrict__ b, long long len) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t < len) a[t] -= b[t];
}

// out += w * sum a[i] b[i] (one atomic per block of 256 threads)
__global__ void wdot_kernel(const double* __restrict__ a, const double* __restrict__ b, long long len, double w,
                            double* __restrict__ out) {
  double s = 0.0;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < len; i += (long long)gridDim.x * blockDim.x)
    s += a[i] * b[i];
  for (int off = 16; off > 0; off >>= 1) s += __shfl_xor_sync(0xffffffffu, s, off);
  __shared__ double part[8];
  if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int k = 0; k < (int)(blockDim.x >> 5); ++k) t += part[k];
    atomicAdd(out, t * w);
  }
}

static unsigned nblk(long long len) { return (unsigned)((len + 255) / 256); }

__global__ void fock_kernel(const double* __restrict__ H, const double* __restrict__ J, const double* __restrict__ K,
                            double* __restrict__ F, double kscale, long long nn) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t < nn) F[t] = H[t] + J[t] - kscale * K[t];
}

int jk_device_locked(hfg_ctx* ctx, const hfg_jk_opts* opts, int nspin, const double* dPt, const double* dPs,
                     double* dJ, double* dK, int shard, int nshards) {
  if (nshards < 1 || shard < 0 || shard >= nshards) return set_error(ctx, HFG_ERR_INVALID_INPUT, "invalid shard");
  hfg_jk_opts o;
  if (opts) o = *opts; else hfg_jk_opts_default(&o);
  if (nspin < 1 || nspin > 2) return set_error(ctx, HFG_ERR_INVALID_INPUT, "nspin must be 1 or 2");
  // (a NaN threshold would break the ordering of the plan map)
  if (!(o.schwarz_threshold >= 0.0) || !(o.prim_threshold >= 0.0) ||
      (o.precision != HFG_FP64 && o.precision != HFG_MIXED) ||
      (o.precision == HFG_MIXED && !(o.mixed_threshold >= 0.0)) || o.tile < 0 || o.tile > 4096)
    return set_error(ctx, HFG_ERR_INVALID_INPUT, "invalid J/K options");
  // a context served with others hands its RHF builds to their batcher
  if (ctx->batcher && nspin == 1 && nshards == 1 && dPs == dPt && !o.deterministic)
    return batcher_submit(ctx->batcher, ctx, o, dPt, dJ, dK);
  Plan* plan = nullptr;
  int rc = build_plan(ctx, o.schwarz_threshold, o.mixed_threshold, o.prim_threshold, o.precision, o.tile, plan);
  if (rc != HFG_OK) return rc;
  const size_t nn = (size_t)ctx->n * ctx->n;
  HFG_CUDA(ctx, ctx->d_Jacc.alloc(nn));
  HFG_CUDA(ctx, ctx->d_Kacc.alloc(2 * nn));
  HFG_CUDA(ctx, ctx->d_counters.alloc(plan->launches.size() + 1));
  // FP32 launches read FP32 copies of the densities, made at the start of
  // the build; the buffer is sized for UHF from the first use on, so it never
  // moves under a captured graph
  bool any32 = false;
  for (const Launch& L : plan->launches) any32 = any32 || L.fp32;
  if (any32) HFG_CUDA(ctx, ctx->d_D32.alloc(3 * nn));
  // HFG_PROFILE=1: per-launch device time (CUDA events) on stderr
  static const bool profile = getenv("HFG_PROFILE") && getenv("HFG_PROFILE")[0] == '1';
  // The build is a fixed sequence (clears, one launch per class, two
  // symmetrisations) whose arguments depend only on the plan and the
  // buffers.  A sequence seen for the second time is captured into a CUDA
  // graph and replayed from then on (an SCF reuses its buffers every
  // iteration); the first build of a sequence always runs eagerly, so the
  // kernels' one-time attribute and occupancy set-up happens outside any
  // capture.  Shards and profiled builds run eagerly.
  const bool graphs_on = ctx->use_graphs && nshards == 1 && !profile && !o.deterministic;
  const hfg_ctx::GraphKey key{plan, nspin, dPt, dPs, dJ, dK, ctx->d_Jacc.p, ctx->d_Kacc.p, ctx->d_counters.p};
  if (graphs_on) {
    auto it = ctx->graphs.find(key);
    if (it != ctx->graphs.end()) {
      HFG_CUDA(ctx, cudaGraphLaunch(it->second, ctx->stream));
      ctx->last = plan->stats;
      ctx->last_plan = plan;
      return HFG_OK;
    }
  }
  JKLaunchArgs a{};
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
  a.Dtot32 = any32 ? ctx->d_D32.p : nullptr;
  a.Dspin32 = any32 ? ctx->d_D32.p + nn : nullptr;
  a.Jacc = ctx->d_Jacc.p;
  a.Kacc = ctx->d_Kacc.p;
  a.n = ctx->n;
  a.nspin = nspin;
  a.prim_eps = o.prim_threshold;
  a.serial = o.deterministic != 0;
  auto enqueue = [&]() -> int {
  if (any32) {
    const long long tot = (long long)nn * (1 + nspin);
    densities_to_f32_kernel<<<(unsigned)std::min<long long>((tot + 255) / 256, 148 * 8), 256, 0, ctx->stream>>>(
        dPt, dPs, ctx->d_D32.p, (long long)nn, nspin);
    HFG_CUDA(ctx, cudaGetLastError());
  }
  HFG_CUDA(ctx, cudaMemsetAsync(ctx->d_Jacc.p, 0, nn * sizeof(double), ctx->stream));
  HFG_CUDA(ctx, cudaMemsetAsync(ctx->d_Kacc.p, 0, nspin * nn * sizeof(double), ctx->stream));
  HFG_CUDA(ctx, cudaMemsetAsync(ctx->d_counters.p, 0, (plan->launches.size() + 1) * 8, ctx->stream));
  std::vector<cudaEvent_t> ev;
  if (profile) {
    HFG_CUDA(ctx, count_plan(ctx, plan) == HFG_OK ? cudaSuccess : cudaErrorUnknown);
    ev.resize(plan->launches.size() + 1);
    for (auto& x : ev) cudaEventCreate(&x);
    cudaEventRecord(ev[0], ctx->stream);
  }
  // The class launches are independent (each adds into J', K' with atomics):
  // they are spread over the context stream and its side streams so that
  // they run concurrently (parallel branches when captured into a graph).  A
  // small molecule's build then costs about its slowest class instead of the
  // sum over classes; a large one's persistent grids fill the GPU either way.
  // Profiled builds stay on one stream (per-launch events).
  const int nstreams = (profile || a.serial) ? 1 : 1 + kJKSideStreams;
  if (nstreams > 1) {
    HFG_CUDA(ctx, ctx->ensure_side_streams());
    HFG_CUDA(ctx, cudaEventRecord(ctx->ev_fork, ctx->stream));
    for (int k = 0; k < kJKSideStreams; ++k) HFG_CUDA(ctx, cudaStreamWaitEvent(ctx->side[k], ctx->ev_fork, 0));
  }
  for (size_t l = 0; l < plan->launches.size(); ++l) {
    const Launch& L = plan->launches[l];
    const int si = (int)(l % (size_t)nstreams);
    cudaStream_t ls = si == 0 ? ctx->stream : ctx->side[si - 1];
    a.counter = ctx->d_counters.p + l;
    a.entries = L.d_entries;
    a.prefix = L.d_prefix;
    // shard: steps [c0, c1) with about shard/nshards .. (shard+1)/nshards of
    // the launch's nominal cost
    long long c0 = 0, c1 = L.nchunks;
    if (nshards > 1) {
      const double tot = L.cost_prefix.back();
      auto cut = [&](int k) -> long long {
        if (k <= 0) return 0;
        if (k >= nshards) return L.nchunks;
        const double target = tot * (double)k / (double)nshards;
        return (long long)(std::lower_bound(L.cost_prefix.begin(), L.cost_prefix.end(), target) -
                           L.cost_prefix.begin());
      };
      c0 = std::min(cut(shard), L.nchunks);
      c1 = std::min(std::max(cut(shard + 1), c0), L.nchunks);
    }
    a.chunk_entry = L.d_chunk + c0;
    a.chunk_start = L.d_cstart + c0;
    a.nchunks = c1 - c0;
    a.nentries = (int)L.prefix[0];
    a.nwarps = L.prefix[1];
    HFG_CUDA(ctx, launch_jk(L.la, L.lb, L.lc, L.ld, L.fp32, a, ls));
    if (profile) cudaEventRecord(ev[l + 1], ctx->stream);
  }
  if (nstreams > 1) {
    for (int k = 0; k < kJKSideStreams; ++k) {
      HFG_CUDA(ctx, cudaEventRecord(ctx->ev_join[k], ctx->side[k]));
      HFG_CUDA(ctx, cudaStreamWaitEvent(ctx->stream, ctx->ev_join[k], 0));
    }
  }
  if (profile) {
    cudaEventSynchronize(ev.back());
    double tot = 0;
    for (size_t l = 0; l < plan->launches.size(); ++l) {
      float ms = 0;
      cudaEventElapsedTime(&ms, ev[l], ev[l + 1]);
      tot += ms;
      const Launch& L = plan->launches[l];
      fprintf(stderr, "hfg-profile (%d%d|%d%d) %s entries %8lld warps %10lld quartets %.3e prims %.3e  %9.3f ms  %.3e prim/s\n",
              L.la, L.lb, L.lc, L.ld, L.fp32 ? "fp32" : "fp64", L.prefix[0], L.prefix[1], L.quartets, L.prims, ms,
              L.prims / (ms * 1e-3));
    }
    fprintf(stderr, "hfg-profile total %.3f ms\n", tot);
    for (auto& x : ev) cudaEventDestroy(x);
  }
  const int blk = 256;
  HFG_CUDA(ctx, (symmetrize_kernel<<<(unsigned)((nn + blk - 1) / blk), blk, 0, ctx->stream>>>(ctx->d_Jacc.p, dJ,
                                                                                              ctx->n, 1),
                 cudaGetLastError()));
  HFG_CUDA(ctx, (symmetrize_kernel<<<(unsigned)((nspin * nn + blk - 1) / blk), blk, 0, ctx->stream>>>(
                     ctx->d_Kacc.p, dK, ctx->n, nspin),
                 cudaGetLastError()));
  return HFG_OK;
  };
  if (graphs_on && !ctx->graph_failed.count(key)) {
    if (ctx->graph_seen.count(key)) {
      // second build of this sequence: capture it, then launch the graph
      cudaGraph_t g = nullptr;
      cudaGraphExec_t ge = nullptr;
      if (cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal) == cudaSuccess) {
        const int erc = enqueue();
        const cudaError_t ec = cudaStreamEndCapture(ctx->stream, &g);
        if (erc == HFG_OK && ec == cudaSuccess && g && cudaGraphInstantiate(&ge, g, 0) == cudaSuccess)
          ctx->graphs.emplace(key, ge);
        if (g) cudaGraphDestroy(g);
      }
      cudaGetLastError();  // a failed capture leaves an error; the build then runs eagerly
      auto it = ctx->graphs.find(key);
      if (it != ctx->graphs.end()) {
        HFG_CUDA(ctx, cudaGraphLaunch(it->second, ctx->stream));
        ctx->last = plan->stats;
        ctx->last_plan = plan;
        return HFG_OK;
      }
      ctx->graph_failed.insert(key);
    } else {
      ctx->graph_seen.insert(key);
    }
  }
  rc = enqueue();
  if (rc != HFG_OK) return rc;
  ctx->last = plan->stats;
  ctx->last_plan = plan;
  return HFG_OK;
}

}  // namespace hfg

hfg_ctx::~hfg_ctx() {
  for (auto& kv : plans)
    for (auto& L : kv.second->launches) {
      if (L.d_entries) cudaFreeAsync(L.d_entries, L.st);
      if (L.d_prefix) cudaFreeAsync(L.d_prefix, L.st);
      if (L.d_chunk) cudaFreeAsync(L.d_chunk, L.st);
      if (L.d_cstart) cudaFreeAsync(L.d_cstart, L.st);
    }
  for (auto& kv : graphs) cudaGraphExecDestroy(kv.second);
  // every device buffer is released here, before the context's stream is
  // destroyed (their frees are ordered on it)
  d_pairQ.release();
  d_pairs.release();
  d_ka0.release();
  d_ka1.release();
  d_ka2.release();
  d_kii.release();
  d_knn.release();
  d_prims.release();
  d_rec64.release();
  d_rec32.release();
  d_pbound.release();
  d_boys64.release();
  d_boys32.release();
  d_expt64.release();
  d_expt32.release();
  d_counters.release();
  d_D.release();
  d_Ds.release();
  d_D32.release();
  d_Jacc.release();
  d_Kacc.release();
  d_J.release();
  d_K.release();
  d_tmp.release();
  for (auto& x : side)
    if (x) cudaStreamDestroy(x);
  if (ev_fork) cudaEventDestroy(ev_fork);
  for (auto& x : ev_join)
    if (x) cudaEventDestroy(x);
  if (own_stream && stream) cudaStreamDestroy(stream);
}

extern "C" {

void hfg_jk_opts_default(hfg_jk_opts* o) {
  if (!o) return;
  o->schwarz_threshold = 1e-12;
  o->prim_threshold = 0.0;
  o->precision = HFG_FP64;
  o->deterministic = 0;
  o->mixed_threshold = 1e-7;
  o->tile = 0;
}

int hfg_ctx_create(const hfg_basis* basis, int device, void* stream, hfg_ctx** out) {
  if (!out) return HFG_ERR_INVALID_INPUT;
  *out = nullptr;
  auto ctx = std::make_unique<hfg_ctx>();
  ctx->device = device;
  // HFG_NO_GRAPHS=1: every J/K build launches eagerly
  ctx->use_graphs = !(getenv("HFG_NO_GRAPHS") && getenv("HFG_NO_GRAPHS")[0] == '1');
  int rc = cuda_check(ctx.get(), cudaSetDevice(device), "cudaSetDevice");
  if (rc == HFG_OK) {
    if (stream) ctx->stream = (cudaStream_t)stream;
    else {
      rc = cuda_check(ctx.get(), cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking), "stream");
      ctx->own_stream = true;
    }
  }
  if (rc == HFG_OK) {
    // keep freed stream-ordered memory in the pool for reuse
    static std::once_flag pool_once[64];
    if (device >= 0 && device < 64)
      std::call_once(pool_once[device], [device] {
        cudaMemPool_t pool;
        if (cudaDeviceGetDefaultMemPool(&pool, device) == cudaSuccess) {
          unsigned long long thr = ~0ull;
          cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr);
        }
      });
  }
  AllocScope alloc_scope(rc == HFG_OK ? ctx->stream : nullptr);
  // s, p, d on the generated kernels; f on the generic engine
  if (rc == HFG_OK) rc = build_shell_list(ctx.get(), basis, kMDLMax);
  if (rc == HFG_OK) {
    const auto& t = boys_table_host();
    std::vector<float> tf(t.begin(), t.end());
    rc = cuda_check(ctx.get(), ctx->d_boys64.alloc(t.size()), "alloc boys");
    if (rc == HFG_OK) rc = cuda_check(ctx.get(), ctx->d_boys32.alloc(tf.size()), "alloc boys32");
    if (rc == HFG_OK)
      rc = cuda_check(ctx.get(), cudaMemcpy(ctx->d_boys64.p, t.data(), t.size() * 8, cudaMemcpyHostToDevice), "boys");
    if (rc == HFG_OK)
      rc = cuda_check(ctx.get(), cudaMemcpy(ctx->d_boys32.p, tf.data(), tf.size() * 4, cudaMemcpyHostToDevice),
                      "boys32");
    std::vector<double> e64(kBoysRows);
    std::vector<float> e32(kBoysRows);
    for (int i = 0; i < kBoysRows; ++i) {
      e64[i] = std::exp(-i * kBoysStep);
      e32[i] = (float)e64[i];
    }
    if (rc == HFG_OK) rc = cuda_check(ctx.get(), ctx->d_expt64.alloc(kBoysRows), "alloc expt");
    if (rc == HFG_OK) rc = cuda_check(ctx.get(), ctx->d_expt32.alloc(kBoysRows), "alloc expt32");
    if (rc == HFG_OK)
      rc = cuda_check(ctx.get(), cudaMemcpy(ctx->d_expt64.p, e64.data(), kBoysRows * 8, cudaMemcpyHostToDevice),
                      "expt");
    if (rc == HFG_OK)
      rc = cuda_check(ctx.get(), cudaMemcpy(ctx->d_expt32.p, e32.data(), kBoysRows * 4, cudaMemcpyHostToDevice),
                      "expt32");
  }
  if (rc == HFG_OK) rc = build_pairs(ctx.get());
  if (rc != HFG_OK) {
    // keep the message for the caller through a minimal context
    *out = ctx.release();
    return rc;
  }
  *out = ctx.release();
  return HFG_OK;
}

int hfg_ctx_destroy(hfg_ctx* ctx) {
  if (!ctx) return HFG_OK;
  cudaSetDevice(ctx->device);
  AllocScope alloc_scope(ctx->stream);
  if (ctx->stream) cudaStreamSynchronize(ctx->stream);
  delete ctx;
  return HFG_OK;
}

const char* hfg_last_error(const hfg_ctx* ctx) { return ctx ? ctx->err.c_str() : "null context"; }

int hfg_ctx_sizes(const hfg_ctx* ctx, int* n_ao, int* n_shell, long* n_pair) {
  if (!ctx) return HFG_ERR_INVALID_INPUT;
  if (n_ao) *n_ao = ctx->n;
  if (n_shell) *n_shell = (int)ctx->shells.size();
  if (n_pair) *n_pair = (long)ctx->ref_pairs.size();
  return HFG_OK;
}

int hfg_schwarz(hfg_ctx* ctx, double* bounds, long n) {
  if (!ctx || !bounds || n != (long)ctx->ref_pairs.size()) return set_error(ctx, HFG_ERR_INVALID_INPUT, "size");
  for (long r = 0; r < n; ++r) bounds[r] = ctx->sorted_Q[ctx->ref_to_sorted[r]];
  return HFG_OK;
}

int hfg_shell_quartet(hfg_ctx* ctx, int a, int b, int c, int d, double* out) {
  if (!ctx || !out) return HFG_ERR_INVALID_INPUT;
  std::lock_guard<std::mutex> lk(ctx->mu);
  AllocScope alloc_scope(ctx->stream);
  const int ns = (int)ctx->shells.size();
  for (int s : {a, b, c, d})
    if (s < 0 || s >= ns) return set_error(ctx, HFG_ERR_INVALID_INPUT, "shell index out of range");
  cudaSetDevice(ctx->device);
  // orient each pair la >= lb; remember swaps to permute the block back
  const bool sab = ctx->shells[a].l < ctx->shells[b].l, scd = ctx->shells[c].l < ctx->shells[d].l;
  const int A = sab ? b : a, B = sab ? a : b, C = scd ? d : c, D = scd ? c : d;
  PairInfo pi[2];
  std::vector<PrimPair> pp;
  make_pair(ctx, A, B, pi[0], pp, 0);
  make_pair(ctx, C, D, pi[1], pp, 1);
  const int na = ncart(ctx->shells[A].l), nb = ncart(ctx->shells[B].l), nc = ncart(ctx->shells[C].l),
            nd = ncart(ctx->shells[D].l);
  const size_t tot = (size_t)na * nb * nc * nd;
  DevBuf<PairInfo> dpi;
  DevBuf<PrimPair> dpp;
  DevBuf<double> dout;
  HFG_CUDA(ctx, dpi.alloc(2));
  HFG_CUDA(ctx, dpp.alloc(pp.size()));
  HFG_CUDA(ctx, dout.alloc(tot));
  HFG_CUDA(ctx, cudaMemcpyAsync(dpi.p, pi, sizeof(pi), cudaMemcpyHostToDevice, ctx->stream));
  HFG_CUDA(ctx, cudaMemcpyAsync(dpp.p, pp.data(), pp.size() * sizeof(PrimPair), cudaMemcpyHostToDevice, ctx->stream));
  HFG_CUDA(ctx, launch_quartet(ctx->shells[A].l, ctx->shells[B].l, ctx->shells[C].l, ctx->shells[D].l, dpi.p, dpp.p,
                               ctx->d_boys64.p, ctx->d_expt64.p, dout.p, ctx->stream));
  std::vector<double> blk(tot);
  HFG_CUDA(ctx, cudaMemcpyAsync(blk.data(), dout.p, tot * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
  HFG_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  dpi.release();
  dpp.release();
  dout.release();
  // permute (A B | C D) back to (a b | c d)
  const int oa = ncart(ctx->shells[a].l), ob = ncart(ctx->shells[b].l), oc = ncart(ctx->shells[c].l),
            od = ncart(ctx->shells[d].l);
  for (int i = 0; i < oa; ++i)
    for (int j = 0; j < ob; ++j)
      for (int k = 0; k < oc; ++k)
        for (int l = 0; l < od; ++l) {
          const int I = sab ? j : i, J = sab ? i : j, K = scd ? l : k, L = scd ? k : l;
          out[((i * ob + j) * oc + k) * od + l] = blk[((I * nb + J) * nc + K) * nd + L];
        }
  return HFG_OK;
}

int hfg_jk_device_shard(hfg_ctx* ctx, const hfg_jk_opts* opts, int nspin, const double* dPt, const double* dPs,
                        double* dJ, double* dK, int shard, int nshards) {
  if (!ctx || !dPt || !dPs || !dJ || !dK) return set_error(ctx, HFG_ERR_INVALID_INPUT, "null pointer");
  std::lock_guard<std::mutex> lk(ctx->mu);
  AllocScope alloc_scope(ctx->stream);
  cudaSetDevice(ctx->device);
  return jk_device_locked(ctx, opts, nspin, dPt, dPs, dJ, dK, shard, nshards);
}

int hfg_jk_device(hfg_ctx* ctx, const hfg_jk_opts* opts, int nspin, const double* dPt, const double* dPs, double* dJ,
                  double* dK) {
  if (!ctx || !dPt || !dPs || !dJ || !dK) return set_error(ctx, HFG_ERR_INVALID_INPUT, "null pointer");
  std::lock_guard<std::mutex> lk(ctx->mu);
  AllocScope alloc_scope(ctx->stream);
  cudaSetDevice(ctx->device);
  return jk_device_locked(ctx, opts, nspin, dPt, dPs, dJ, dK);
}

int hfg_jk(hfg_ctx* ctx, const hfg_jk_opts* opts, int nspin, const double* Pt, const double* Ps, double* J,
           double* K) {
  if (!ctx || !Pt || !Ps || !J || !K) return set_error(ctx, HFG_ERR_INVALID_INPUT, "null pointer");
  if (nspin < 1 || nspin > 2) return set_error(ctx, HFG_ERR_INVALID_INPUT, "nspin must be 1 or 2");
  std::lock_guard<std::mutex> lk(ctx->mu);
  AllocScope alloc_scope(ctx->stream);
  cudaSetDevice(ctx->device);
  const size_t nn = (size_t)ctx->n * ctx->n;
  HFG_CUDA(ctx, ctx->d_D.alloc(nn));
  HFG_CUDA(ctx, ctx->d_Ds.alloc(2 * nn));
  HFG_CUDA(ctx, ctx->d_J.alloc(nn));
  HFG_CUDA(ctx, ctx->d_K.alloc(2 * nn));
  HFG_CUDA(ctx, cudaMemcpyAsync(ctx->d_D.p, Pt, nn * 8, cudaMemcpyHostToDevice, ctx->stream));
  // RHF callers pass the same matrix twice: copy it once
  const bool same = (nspin == 1 && Ps == Pt);
  if (!same) HFG_CUDA(ctx, cudaMemcpyAsync(ctx->d_Ds.p, Ps, nspin * nn * 8, cudaMemcpyHostToDevice, ctx->stream));
  int rc = jk_device_locked(ctx, opts, nspin, ctx->d_D.p, same ? ctx->d_D.p : ctx->d_Ds.p, ctx->d_J.p, ctx->d_K.p);
  if (rc != HFG_OK) return rc;
  HFG_CUDA(ctx, cudaMemcpyAsync(J, ctx->d_J.p, nn * 8, cudaMemcpyDeviceToHost, ctx->stream));
  HFG_CUDA(ctx, cudaMemcpyAsync(K, ctx->d_K.p, nspin * nn * 8, cudaMemcpyDeviceToHost, ctx->stream));
  HFG_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return HFG_OK;
}

int hfg_jk_device_batch(hfg_ctx* const* ctxs, int n_jobs, const hfg_jk_opts* opts, const double* const* d_P,
                        double* const* d_J, double* const* d_K, void* stream) {
  if (!ctxs || n_jobs < 1 || !ctxs[0]) return HFG_ERR_INVALID_INPUT;
  hfg_ctx* c0 = ctxs[0];
  if (!d_P || !d_J || !d_K) return set_error(c0, HFG_ERR_INVALID_INPUT, "null pointer");
  for (int j = 0; j < n_jobs; ++j)
    if (!ctxs[j]) return set_error(c0, HFG_ERR_INVALID_INPUT, "null pointer");
  // each context's accumulators serve one molecule: no context twice
  std::vector<hfg_ctx*> order(ctxs, ctxs + n_jobs);
  std::sort(order.begin(), order.end());
  if (std::adjacent_find(order.begin(), order.end()) != order.end())
    return set_error(c0, HFG_ERR_INVALID_INPUT, "a context appears twice in the batch");
  hfg_jk_opts o;
  if (opts) o = *opts; else hfg_jk_opts_default(&o);
  std::vector<hfg_jk_opts> per(n_jobs, o);
  // lock in address order, so that concurrent batches cannot deadlock
  std::vector<std::unique_lock<std::mutex>> locks;
  locks.reserve(order.size());
  for (hfg_ctx* c : order) locks.emplace_back(c->mu);
  cudaSetDevice(c0->device);
  return jk_batch_locked(ctxs, n_jobs, per.data(), d_P, d_J, d_K, stream ? (cudaStream_t)stream : c0->stream,
                         nullptr);
}

}  // extern "C"

namespace hfg {

int jk_batch_locked(hfg_ctx* const* ctxs, int n_jobs, const hfg_jk_opts* opts, const double* const* d_P,
                    double* const* d_J, double* const* d_K, cudaStream_t st, BatchStaging* staging) {
  hfg_ctx* c0 = ctxs[0];
  // an error of the batch is reported on every context of it
  auto fail = [&](int rc, const std::string& msg) {
    for (int j = 0; j < n_jobs; ++j) set_error(ctxs[j], rc, msg);
    return rc;
  };
  auto cuda = [&](cudaError_t e, const char* what) {
    return e == cudaSuccess ? HFG_OK : fail(HFG_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
  };
#define BK(call)                                  \
  do {                                            \
    const int _rc = cuda((call), #call);          \
    if (_rc != HFG_OK) return _rc;                \
  } while (0)
  if (n_jobs < 1 || n_jobs > 32767) return fail(HFG_ERR_INVALID_INPUT, "a batch holds 1 to 32767 molecules");
  for (int j = 0; j < n_jobs; ++j) {
    const hfg_jk_opts& o = opts[j];
    if (!d_P[j] || !d_J[j] || !d_K[j]) return fail(HFG_ERR_INVALID_INPUT, "null pointer");
    if (ctxs[j]->device != c0->device) return fail(HFG_ERR_INVALID_INPUT, "the contexts of a batch must share one device");
    if (ctxs[j]->lmax > kLMax) return fail(HFG_ERR_UNSUPPORTED, "batched builds cover s, p and d shells");
    if (!(o.schwarz_threshold >= 0.0) || !(o.prim_threshold >= 0.0) ||
        (o.precision != HFG_FP64 && o.precision != HFG_MIXED) ||
        (o.precision == HFG_MIXED && !(o.mixed_threshold >= 0.0)) || o.tile < 0 || o.tile > 4096)
      return fail(HFG_ERR_INVALID_INPUT, "invalid J/K options");
  }
  // per molecule: its plan (built once, cached on its context) and its
  // accumulators, allocated on its own stream; then the batch stream waits
  // for each context stream
  std::vector<Plan*> plans(n_jobs, nullptr);
  for (int j = 0; j < n_jobs; ++j) {
    hfg_ctx* c = ctxs[j];
    AllocScope alloc_scope(c->stream);
    const hfg_jk_opts& o = opts[j];
    const int rc =
        build_plan(c, o.schwarz_threshold, o.mixed_threshold, o.prim_threshold, o.precision, o.tile, plans[j]);
    if (rc != HFG_OK) return fail(rc, c->err);
    const size_t nn = (size_t)c->n * c->n;
    BK(c->d_Jacc.alloc(nn));
    BK(c->d_Kacc.alloc(2 * nn));
    for (const Launch& L : plans[j]->launches)
      if (L.fp32) {
        BK(c->d_D32.alloc(3 * nn));
        break;
      }
    BK(c->ensure_side_streams());
    if (c->stream != st) {
      BK(cudaEventRecord(c->ev_fork, c->stream));
      BK(cudaStreamWaitEvent(st, c->ev_fork, 0));
    }
  }
  // launch groups: the molecules' launches of one class and precision
  struct Member {
    int job;
    const Launch* L;
  };
  using GroupKey = std::tuple<int, int, int, int, int>;
  std::map<GroupKey, std::vector<Member>> groups;
  for (int j = 0; j < n_jobs; ++j)
    for (const Launch& L : plans[j]->launches)
      if (L.nchunks > 0) groups[std::make_tuple(L.la, L.lb, L.lc, L.ld, (int)L.fp32)].push_back({j, &L});
  std::vector<std::pair<GroupKey, const std::vector<Member>*>> glist;
  for (const auto& kv : groups) glist.push_back({kv.first, &kv.second});
  // most expensive classes first
  std::stable_sort(glist.begin(), glist.end(), [](const auto& x, const auto& y) {
    const auto& [a0, a1, a2, a3, a4] = x.first;
    const auto& [b0, b1, b2, b3, b4] = y.first;
    return std::make_tuple(a0 + a1 + a2 + a3, a4) > std::make_tuple(b0 + b1 + b2 + b3, b4);
  });
  // one device table for the call: counters, matrices, then per group its
  // molecule table and first steps
  const int ng = (int)glist.size();
  auto align = [](size_t x) { return (x + 15) & ~(size_t)15; };
  const size_t counters_bytes = sizeof(unsigned long long) * std::max(ng, 1);
  size_t off = align(counters_bytes);
  const size_t mats_off = off;
  off = align(off + sizeof(BatchMat) * 2 * n_jobs);
  std::vector<size_t> jobs_off(ng), steps_off(ng);
  std::vector<long long> total(ng, 0);
  for (int g = 0; g < ng; ++g) {
    jobs_off[g] = off;
    off = align(off + sizeof(JKJob) * glist[g].second->size());
    steps_off[g] = off;
    off = align(off + sizeof(long long) * glist[g].second->size());
  }
  // the tables go to pinned staging when they fit (an asynchronous copy),
  // else through pageable memory
  std::vector<unsigned char> pageable;
  unsigned char* blob = nullptr;
  if (staging && staging->host && off <= staging->bytes) {
    BK(cudaEventSynchronize(staging->ev));
    blob = static_cast<unsigned char*>(staging->host);
  } else {
    pageable.resize(off);
    blob = pageable.data();
  }
  std::memset(blob, 0, off);
  int maxn = 0;
  {
    BatchMat* mats = reinterpret_cast<BatchMat*>(blob + mats_off);
    for (int j = 0; j < n_jobs; ++j) {
      mats[2 * j] = {ctxs[j]->d_Jacc.p, d_J[j], ctxs[j]->n};
      mats[2 * j + 1] = {ctxs[j]->d_Kacc.p, d_K[j], ctxs[j]->n};
      maxn = std::max(maxn, ctxs[j]->n);
    }
  }
  for (int g = 0; g < ng; ++g) {
    JKJob* jt = reinterpret_cast<JKJob*>(blob + jobs_off[g]);
    long long* stp = reinterpret_cast<long long*>(blob + steps_off[g]);
    const auto& mem = *glist[g].second;
    for (size_t k = 0; k < mem.size(); ++k) {
      const int j = mem[k].job;
      const hfg_ctx* c = ctxs[j];
      const Launch& L = *mem[k].L;
      JKJob& x = jt[k];
      x.entries = L.d_entries;
      x.prefix = L.d_prefix;
      x.chunk_start = L.d_cstart;
      x.chunk_entry = L.d_chunk;
      x.pairs = c->d_pairs.p;
      x.kets = c->kets();
      x.pairQ = c->d_pairQ.p;
      x.rec64 = c->d_rec64.p;
      x.rec32 = c->d_rec32.p;
      x.pbound = c->d_pbound.p;
      x.Dtot = d_P[j];
      x.Dtot32 = c->d_D32.p;
      x.Jacc = c->d_Jacc.p;
      x.Kacc = c->d_Kacc.p;
      x.thr = opts[j].schwarz_threshold;
      x.prim_eps = opts[j].prim_threshold;
      x.n = c->n;
      stp[k] = total[g];
      total[g] += L.nchunks;
    }
  }
  unsigned char* dev = nullptr;
  BK(cudaMallocAsync((void**)&dev, off, st));
  // released (stream-ordered, after the launches) on every return path
  struct FreeAfter {
    void* p;
    cudaStream_t s;
    ~FreeAfter() { cudaFreeAsync(p, s); }
  } free_after{dev, st};
  BK(cudaMemcpyAsync(dev, blob, off, cudaMemcpyHostToDevice, st));
  if (blob != pageable.data()) BK(cudaEventRecord(staging->ev, st));
  const BatchMat* d_mats = reinterpret_cast<const BatchMat*>(dev + mats_off);
  const long long nnmax = (long long)maxn * maxn;
  const dim3 mgrid((unsigned)std::min<long long>((nnmax + 255) / 256, 64), (unsigned)(2 * n_jobs));
  batch_mats_kernel<<<mgrid, 256, 0, st>>>(d_mats, 0);
  BK(cudaGetLastError());
  // FP32 copies of the densities of the molecules with FP32 launches
  for (int j = 0; j < n_jobs; ++j) {
    bool any32 = false;
    for (const Launch& L : plans[j]->launches) any32 = any32 || (L.fp32 && L.nchunks > 0);
    if (!any32) continue;
    const long long nn = (long long)ctxs[j]->n * ctxs[j]->n;
    densities_to_f32_kernel<<<(unsigned)std::min<long long>((nn + 255) / 256, 148 * 8), 256, 0, st>>>(
        d_P[j], d_P[j], ctxs[j]->d_D32.p, nn, 0);
    BK(cudaGetLastError());
  }
  // the groups run concurrently over the first context's side streams
  BK(cudaEventRecord(c0->ev_fork, st));
  for (int k = 0; k < kJKSideStreams; ++k) BK(cudaStreamWaitEvent(c0->side[k], c0->ev_fork, 0));
  const int nstreams = 1 + kJKSideStreams;
  for (int g = 0; g < ng; ++g) {
    const auto& [la, lb, lc, ld, f32] = glist[g].first;
    JKLaunchArgs a{};
    a.boys64 = c0->d_boys64.p;
    a.boys32 = c0->d_boys32.p;
    a.expt64 = c0->d_expt64.p;
    a.expt32 = c0->d_expt32.p;
    a.nspin = 1;
    a.counter = reinterpret_cast<unsigned long long*>(dev) + g;
    a.jobs = reinterpret_cast<const JKJob*>(dev + jobs_off[g]);
    a.job_steps = reinterpret_cast<const long long*>(dev + steps_off[g]);
    a.njobs = (int)glist[g].second->size();
    a.nchunks = total[g];
    const int si = g % nstreams;
    BK(launch_jk_batch(la, lb, lc, ld, f32 != 0, a, si == 0 ? st : c0->side[si - 1]));
  }
  for (int k = 0; k < kJKSideStreams; ++k) {
    BK(cudaEventRecord(c0->ev_join[k], c0->side[k]));
    BK(cudaStreamWaitEvent(st, c0->ev_join[k], 0));
  }
  batch_mats_kernel<<<mgrid, 256, 0, st>>>(d_mats, 1);
  BK(cudaGetLastError());
  // each context's later work (and reuse of its accumulators) follows the batch
  cudaEvent_t done = nullptr;
  BK(cudaEventCreateWithFlags(&done, cudaEventDisableTiming));
  cudaError_t e = cudaEventRecord(done, st);
  for (int j = 0; j < n_jobs && e == cudaSuccess; ++j)
    if (ctxs[j]->stream != st) e = cudaStreamWaitEvent(ctxs[j]->stream, done, 0);
  cudaEventDestroy(done);
  BK(e);
  for (int j = 0; j < n_jobs; ++j) {
    ctxs[j]->last = plans[j]->stats;
    ctxs[j]->last_plan = plans[j];
  }
#undef BK
  return HFG_OK;
}

}  // namespace hfg

extern "C" {

int hfg_eri_gradient(hfg_ctx* ctx, double schwarz_threshold, int nspin, const double* P_total, const double* P_spin,
                     int natom, double* grad) {
  if (!ctx) return HFG_ERR_INVALID_INPUT;
  if (!P_total || !P_spin || !grad) return set_error(ctx, HFG_ERR_INVALID_INPUT, "null pointer");
  if (nspin < 1 || nspin > 2) return set_error(ctx, HFG_ERR_INVALID_INPUT, "nspin must be 1 or 2");
  if (!(schwarz_threshold >= 0.0)) return set_error(ctx, HFG_ERR_INVALID_INPUT, "Schwarz threshold must be >= 0");
  std::lock_guard<std::mutex> lk(ctx->mu);
  AllocScope alloc_scope(ctx->stream);
  cudaSetDevice(ctx->device);
  // the derivative integrals raise one shell by one: shells up to d
  if (ctx->lmax > kLMax)
    return set_error(ctx, HFG_ERR_UNSUPPORTED, "ERI derivatives cover s, p and d shells");
  std::vector<int> ao_atom(ctx->n);
  for (const Shell& sh : ctx->shells) {
    if (sh.atom < 0 || sh.atom >= natom)
      return set_error(ctx, HFG_ERR_INVALID_INPUT, "natom must exceed every basis function's atom index");
    for (int k = 0; k < ncart(sh.l); ++k) ao_atom[sh.ao + k] = sh.atom;
  }
  Plan* plan = nullptr;
  int rc = build_plan(ctx, schwarz_threshold, 0.0, 0.0, HFG_FP64, 0, plan);
  if (rc != HFG_OK) return rc;
  const size_t nn = (size_t)ctx->n * ctx->n;
  HFG_CUDA(ctx, ctx->d_D.alloc(nn));
  HFG_CUDA(ctx, ctx->d_Ds.alloc(2 * nn));
  HFG_CUDA(ctx, ctx->d_counters.alloc(plan->launches.size() + 1));
  DevBuf<int> d_atom;
  DevBuf<double> d_grad;
  HFG_CUDA(ctx, d_atom.alloc(ctx->n));
  HFG_CUDA(ctx, d_grad.alloc((size_t)3 * natom));
  HFG_CUDA(ctx, cudaMemcpyAsync(ctx->d_D.p, P_total, nn * 8, cudaMemcpyHostToDevice, ctx->stream));
  HFG_CUDA(ctx, cudaMemcpyAsync(ctx->d_Ds.p, P_spin, nspin * nn * 8, cudaMemcpyHostToDevice, ctx->stream));
  HFG_CUDA(ctx, cudaMemcpyAsync(d_atom.p, ao_atom.data(), ctx->n * sizeof(int), cudaMemcpyHostToDevice, ctx->stream));
  HFG_CUDA(ctx, cudaMemsetAsync(d_grad.p, 0, (size_t)3 * natom * sizeof(double), ctx->stream));
  HFG_CUDA(ctx, cudaMemsetAsync(ctx->d_counters.p, 0, (plan->launches.size() + 1) * 8, ctx->stream));
  JKLaunchArgs a{};
  a.pairs = ctx->d_pairs.p;
  a.kets = ctx->kets();
  a.pairQ = ctx->d_pairQ.p;
  a.thr = schwarz_threshold;
  a.rec64 = ctx->d_rec64.p;
  a.boys64 = ctx->d_boys64.p;
  a.expt64 = ctx->d_expt64.p;
  a.Dtot = ctx->d_D.p;
  a.Dspin = ctx->d_Ds.p;
  a.n = ctx->n;
  a.nspin = nspin;
  for (size_t l = 0; l < plan->launches.size(); ++l) {
    const Launch& L = plan->launches[l];
    a.counter = ctx->d_counters.p + l;
    a.entries = L.d_entries;
    a.prefix = L.d_prefix;
    a.chunk_entry = L.d_chunk;
    a.chunk_start = L.d_cstart;
    a.nchunks = L.nchunks;
    HFG_CUDA(ctx, launch_grad_md(L.la, L.lb, L.lc, L.ld, a, d_atom.p, d_grad.p, ctx->stream));
  }
  HFG_CUDA(ctx, cudaMemcpyAsync(grad, d_grad.p, (size_t)3 * natom * sizeof(double), cudaMemcpyDeviceToHost,
                                ctx->stream));
  HFG_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return HFG_OK;
}

int hfg_gradient(hfg_ctx* ctx, int natom, const double* positions, const double* charges, int nspin,
                 const double* P_total, const double* P_spin, const double* W, double schwarz_threshold,
                 double* grad) {
  if (!ctx) return HFG_ERR_INVALID_INPUT;
  if (!positions || !charges || !P_total || !P_spin || !W || !grad)
    return set_error(ctx, HFG_ERR_INVALID_INPUT, "null pointer");
  if (natom < 1 || natom > 4096) return set_error(ctx, HFG_ERR_INVALID_INPUT, "natom must be in 1..4096");
  // two-electron part (its own lock and checks)
  std::vector<double> g2(3 * (size_t)natom, 0.0);
  int rc = hfg_eri_gradient(ctx, schwarz_threshold, nspin, P_total, P_spin, natom, g2.data());
  if (rc != HFG_OK) return rc;
  std::vector<double> g(3 * (size_t)natom, 0.0);
  {
    std::lock_guard<std::mutex> lk(ctx->mu);
    AllocScope alloc_scope(ctx->stream);
    cudaSetDevice(ctx->device);
    rc = one_electron_gradient(ctx, natom, positions, charges, P_total, W, g.data());
    if (rc != HFG_OK) return rc;
  }
  // nuclear repulsion: -sum_B Z_A Z_B (R_A - R_B) / |R_A - R_B|^3
  for (int A = 0; A < natom; ++A)
    for (int B = 0; B < natom; ++B) {
      if (A == B) continue;
      const double d[3] = {positions[3 * A] - positions[3 * B], positions[3 * A + 1] - positions[3 * B + 1],
                           positions[3 * A + 2] - positions[3 * B + 2]};
      const double r2 = d[0] * d[0] + d[1] * d[1] + d[2] * d[2];
      if (!(r2 > 0.0)) return set_error(ctx, HFG_ERR_INVALID_INPUT, "coincident nuclei");
      const double f = -charges[A] * charges[B] / (r2 * std::sqrt(r2));
      for (int k = 0; k < 3; ++k) g[3 * A + k] += f * d[k];
    }
  for (size_t x = 0; x < g.size(); ++x) grad[x] = g[x] + g2[x];
  return HFG_OK;
}

// Packed tensor on the device: every quartet of the FP64 plan without
// primitive screening (the plan holds each unique significant shell quartet
// once), stored by eri_packed_kernel.
}  // extern "C"

namespace hfg {
int eri_packed_locked(hfg_ctx* ctx, double thr, double* d_out, size_t len) {
  const size_t n = (size_t)ctx->n, np = n * (n + 1) / 2;
  if (len != np * (np + 1) / 2)
    return set_error(ctx, HFG_ERR_INVALID_INPUT, "packed length must be n_p (n_p + 1) / 2 with n_p = n (n + 1) / 2");
  if (!(thr >= 0.0)) return set_error(ctx, HFG_ERR_INVALID_INPUT, "Schwarz threshold must be >= 0");
  Plan* plan = nullptr;
  int rc = build_plan(ctx, thr, 0.0, 0.0, HFG_FP64, 0, plan);
  if (rc != HFG_OK) return rc;
  HFG_CUDA(ctx, cudaMemsetAsync(d_out, 0, len * sizeof(double), ctx->stream));
  for (const Launch& L : plan->launches) {
    if (L.la > kLMax || L.lb > kLMax || L.lc > kLMax || L.ld > kLMax) {
      HFG_CUDA(ctx, launch_eri_packed_md(L.la, L.lb, L.lc, L.ld, L.d_entries, L.d_prefix, (int)L.prefix[0],
                                         L.prefix[1], ctx->d_pairs.p, ctx->d_pairQ.p, thr, ctx->d_rec64.p,
                                         ctx->d_pbound.p, ctx->d_boys64.p, ctx->d_expt64.p, d_out, ctx->stream));
      continue;
    }
    HFG_CUDA(ctx, launch_eri_packed(L.la, L.lb, L.lc, L.ld, L.d_entries, L.d_prefix, (int)L.prefix[0], L.prefix[1],
                                    ctx->d_pairs.p, ctx->d_pairQ.p, thr, ctx->d_rec64.p, ctx->d_boys64.p, ctx->d_expt64.p, d_out,
                                    ctx->stream));
  }
  return HFG_OK;
}
}  // namespace hfg

extern "C" {

int hfg_eri_packed_device(hfg_ctx* ctx, double schwarz_threshold, double* d_out, size_t len) {
  if (!ctx) return HFG_ERR_INVALID_INPUT;
  if (!d_out) return set_error(ctx, HFG_ERR_INVALID_INPUT, "null pointer");
  std::lock_guard<std::mutex> lk(ctx->mu);
  AllocScope alloc_scope(ctx->stream);
  cudaSetDevice(ctx->device);
  return eri_packed_locked(ctx, schwarz_threshold, d_out, len);
}

int hfg_eri_packed(hfg_ctx* ctx, double schwarz_threshold, double* out, size_t len) {
  if (!ctx) return HFG_ERR_INVALID_INPUT;
  if (!out) return set_error(ctx, HFG_ERR_INVALID_INPUT, "null pointer");
  std::lock_guard<std::mutex> lk(ctx->mu);
  AllocScope alloc_scope(ctx->stream);
  cudaSetDevice(ctx->device);
  DevBuf<double> buf;
  if (buf.alloc(len) != cudaSuccess) {
    cudaGetLastError();
    return set_error(ctx, HFG_ERR_OOM, "packed tensor does not fit in device memory");
  }
  int rc = eri_packed_locked(ctx, schwarz_threshold, buf.p, len);
  if (rc != HFG_OK) return rc;
  HFG_CUDA(ctx, cudaMemcpyAsync(out, buf.p, len * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
  HFG_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return HFG_OK;
}

static int fock_common(hfg_ctx* ctx, const hfg_jk_opts* opts, const double* H, const double* Pa, const double* Pb,
                       double* Fa, double* Fb, int uhf) {
  if (!ctx || !H || !Pa || !Fa || (uhf && (!Pb || !Fb))) return set_error(ctx, HFG_ERR_INVALID_INPUT, "null pointer");
  std::lock_guard<std::mutex> lk(ctx->mu);
  AllocScope alloc_scope(ctx->stream);
  cudaSetDevice(ctx->device);
  const size_t nn = (size_t)ctx->n * ctx->n;
  HFG_CUDA(ctx, ctx->d_D.alloc(nn));
  HFG_CUDA(ctx, ctx->d_Ds.alloc(2 * nn));
  HFG_CUDA(ctx, ctx->d_J.alloc(nn));
  HFG_CUDA(ctx, ctx->d_K.alloc(2 * nn));
  HFG_CUDA(ctx, ctx->d_tmp.alloc(3 * nn));
  double* dH = ctx->d_tmp.p;
  double* dF = ctx->d_tmp.p + nn;
  HFG_CUDA(ctx, cudaMemcpyAsync(dH, H, nn * 8, cudaMemcpyHostToDevice, ctx->stream));
  const int nspin = uhf ? 2 : 1;
  HFG_CUDA(ctx, cudaMemcpyAsync(ctx->d_Ds.p, Pa, nn * 8, cudaMemcpyHostToDevice, ctx->stream));
  if (uhf) {
    HFG_CUDA(ctx, cudaMemcpyAsync(ctx->d_Ds.p + nn, Pb, nn * 8, cudaMemcpyHostToDevice, ctx->stream));
  }
  const double* dPt = ctx->d_Ds.p;
  if (uhf) {
    // P_total = Pa + Pb (the Fock kernel with a zero K weight)
    fock_kernel<<<(unsigned)((nn + 255) / 256), 256, 0, ctx->stream>>>(ctx->d_Ds.p, ctx->d_Ds.p + nn, ctx->d_Ds.p,
                                                                        ctx->d_D.p, 0.0, (long long)nn);
    HFG_CUDA(ctx, cudaGetLastError());
    dPt = ctx->d_D.p;
  }
  int rc = jk_device_locked(ctx, opts, nspin, dPt, ctx->d_Ds.p, ctx->d_J.p, ctx->d_K.p);
  if (rc != HFG_OK) return rc;
  const double ks = uhf ? 1.0 : 0.5;
  for (int s = 0; s < nspin; ++s) {
    fock_kernel<<<(unsigned)((nn + 255) / 256), 256, 0, ctx->stream>>>(dH, ctx->d_J.p, ctx->d_K.p + s * nn, dF, ks,
                                                                        (long long)nn);
    HFG_CUDA(ctx, cudaGetLastError());
    HFG_CUDA(ctx, cudaMemcpyAsync(s == 0 ? Fa : Fb, dF, nn * 8, cudaMemcpyDeviceToHost, ctx->stream));
    HFG_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  }
  return HFG_OK;
}

int hfg_fock_rhf(hfg_ctx* ctx, const hfg_jk_opts* opts, const double* H, const double* P, double* F) {
  return fock_common(ctx, opts, H, P, nullptr, F, nullptr, 0);
}

int hfg_fock_uhf(hfg_ctx* ctx, const hfg_jk_opts* opts, const double* H, const double* Pa, const double* Pb,
                 double* Fa, double* Fb) {
  return fock_common(ctx, opts, H, Pa, Pb, Fa, Fb, 1);
}

void hfg_autotune_opts_default(hfg_autotune_opts* o) {
  *o = hfg_autotune_opts{};
  const double f[4] = {1e-7, 1e-6, 1e-5, 1e-4}, p[3] = {1e-15, 1e-14, 1e-13};
  for (int i = 0; i < 4; ++i) o->fp32_thresholds[i] = f[i];
  o->n_fp32 = 4;
  for (int i = 0; i < 3; ++i) o->prim_thresholds[i] = p[i];
  o->n_prim = 3;
  o->max_energy_error = 5e-9;
  o->repeats = 2;
  o->tiles[0] = 8;
  o->tiles[1] = 16;
  o->tiles[2] = 32;
  o->tiles[3] = 256;
  o->n_tile = 4;
}

int hfg_jk_autotune(hfg_ctx* ctx, const hfg_jk_opts* base, int nspin, const double* dPt, const double* dPs,
                    const hfg_autotune_opts* opts, hfg_autotune_result* res) {
  if (!ctx) return HFG_ERR_INVALID_INPUT;
  if (!dPt || !dPs || !res) return set_error(ctx, HFG_ERR_INVALID_INPUT, "null pointer");
  if (nspin < 1 || nspin > 2) return set_error(ctx, HFG_ERR_INVALID_INPUT, "nspin must be 1 or 2");
  hfg_autotune_opts o;
  hfg_autotune_opts_default(&o);
  if (opts) {
    if (opts->n_fp32 < 0 || opts->n_fp32 > 8 || opts->n_prim < 0 || opts->n_prim > 8)
      return set_error(ctx, HFG_ERR_INVALID_INPUT, "at most 8 candidates per list");
    if (opts->n_fp32 > 0) {
      o.n_fp32 = opts->n_fp32;
      for (int i = 0; i < o.n_fp32; ++i) o.fp32_thresholds[i] = opts->fp32_thresholds[i];
    }
    if (opts->n_prim > 0) {
      o.n_prim = opts->n_prim;
      for (int i = 0; i < o.n_prim; ++i) o.prim_thresholds[i] = opts->prim_thresholds[i];
    }
    if (opts->max_energy_error > 0.0) o.max_energy_error = opts->max_energy_error;
    if (opts->repeats > 0) o.repeats = opts->repeats;
    if (opts->n_tile < 0 || opts->n_tile > 4) return set_error(ctx, HFG_ERR_INVALID_INPUT, "at most 4 tiles");
    if (opts->n_tile > 0) {
      o.n_tile = opts->n_tile;
      for (int i = 0; i < o.n_tile; ++i) o.tiles[i] = opts->tiles[i];
    }
  }
  for (int i = 0; i < o.n_tile; ++i)
    if (o.tiles[i] < 1 || o.tiles[i] > 4096) return set_error(ctx, HFG_ERR_INVALID_INPUT, "tiles must be in 1..4096");
  hfg_jk_opts b;
  if (base) b = *base; else hfg_jk_opts_default(&b);
  std::lock_guard<std::mutex> lk(ctx->mu);
  AllocScope alloc_scope(ctx->stream);
  cudaSetDevice(ctx->device);
  const long long nn = (long long)ctx->n * ctx->n;
  DevBuf<double> J64, K64, J, K, e;
  HFG_CUDA(ctx, J64.alloc(nn));
  HFG_CUDA(ctx, K64.alloc(nspin * nn));
  HFG_CUDA(ctx, J.alloc(nn));
  HFG_CUDA(ctx, K.alloc(nspin * nn));
  HFG_CUDA(ctx, e.alloc(1));
  struct Events {
    cudaEvent_t a = nullptr, b = nullptr;
    Events() {
      cudaEventCreate(&a);
      cudaEventCreate(&b);
    }
    ~Events() {
      cudaEventDestroy(a);
      cudaEventDestroy(b);
    }
  } ev;
  // a build with options jo into (dJ, dK): one untimed build (it makes the
  // plan), then the minimum device time over `reps` builds
  auto run = [&](const hfg_jk_opts& jo, double* dJ, double* dK, int reps, double& ms) -> int {
    int rc = jk_device_locked(ctx, &jo, nspin, dPt, dPs, dJ, dK);
    if (rc != HFG_OK) return rc;
    ms = 1e300;
    for (int r = 0; r < reps; ++r) {
      cudaEventRecord(ev.a, ctx->stream);
      rc = jk_device_locked(ctx, &jo, nspin, dPt, dPs, dJ, dK);
      if (rc != HFG_OK) return rc;
      cudaEventRecord(ev.b, ctx->stream);
      HFG_CUDA(ctx, cudaEventSynchronize(ev.b));
      float t = 0.f;
      cudaEventElapsedTime(&t, ev.a, ev.b);
      ms = std::min(ms, (double)t);
    }
    return HFG_OK;
  };
  // energy error of (J, K) against (J64, K64); overwrites J and K
  auto energy_error = [&](double& dE) -> int {
    HFG_CUDA(ctx, cudaMemsetAsync(e.p, 0, sizeof(double), ctx->stream));
    axpy_sub_kernel<<<nblk(nn), 256, 0, ctx->stream>>>(J.p, J64.p, nn);
    axpy_sub_kernel<<<nblk(nspin * nn), 256, 0, ctx->stream>>>(K.p, K64.p, nspin * nn);
    wdot_kernel<<<296, 256, 0, ctx->stream>>>(dPt, J.p, nn, 0.5, e.p);
    wdot_kernel<<<296, 256, 0, ctx->stream>>>(dPs, K.p, nspin * nn, nspin == 1 ? -0.25 : -0.5, e.p);
    HFG_CUDA(ctx, cudaGetLastError());
    HFG_CUDA(ctx, cudaMemcpyAsync(&dE, e.p, sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    HFG_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return HFG_OK;
  };
  *res = hfg_autotune_result{};
  hfg_jk_opts j64 = b;
  j64.precision = HFG_FP64;
  j64.prim_threshold = 0.0;
  int rc = run(j64, J64.p, K64.p, 1, res->fp64_ms);
  if (rc != HFG_OK) return rc;
  res->best = j64;
  res->best_ms = 1e300;
  int k = 0;
  for (int i = 0; i < o.n_fp32; ++i)
    for (int j = 0; j < o.n_prim; ++j, ++k) {
      hfg_jk_opts c = b;
      c.precision = HFG_MIXED;
      c.mixed_threshold = o.fp32_thresholds[i];
      c.prim_threshold = o.prim_thresholds[j];
      double ms = 0.0, dE = 0.0;
      rc = run(c, J.p, K.p, o.repeats, ms);
      if (rc != HFG_OK) return rc;
      rc = energy_error(dE);
      if (rc != HFG_OK) return rc;
      res->ms[k] = ms;
      res->energy_error[k] = dE;
      if (std::fabs(dE) <= o.max_energy_error && ms < res->best_ms) {
        res->best = c;
        res->best_ms = ms;
        res->best_energy_error = dE;
        res->found = 1;
      }
    }
  // the quartet tile, on the best threshold pair
  if (res->found) {
    const hfg_jk_opts pair = res->best;
    for (int i = 0; i < o.n_tile && k < 64; ++i, ++k) {
      hfg_jk_opts c = pair;
      c.tile = o.tiles[i];
      double ms = 0.0, dE = 0.0;
      rc = run(c, J.p, K.p, o.repeats, ms);
      if (rc != HFG_OK) return rc;
      rc = energy_error(dE);
      if (rc != HFG_OK) return rc;
      res->ms[k] = ms;
      res->energy_error[k] = dE;
      if (std::fabs(dE) <= o.max_energy_error && ms < res->best_ms) {
        res->best = c;
        res->best_ms = ms;
        res->best_energy_error = dE;
      }
    }
  }
  res->evaluated = k;
  if (!res->found) res->best_ms = res->fp64_ms;
  return HFG_OK;
}

int hfg_fma_peak(int device, int fp32, double* tflops) {
  if (!tflops) return HFG_ERR_INVALID_INPUT;
  if (cudaSetDevice(device) != cudaSuccess) return HFG_ERR_CUDA;
  return fma_peak(fp32, tflops) == cudaSuccess ? HFG_OK : HFG_ERR_CUDA;
}

int hfg_jk_last_stats(const hfg_ctx* cctx, hfg_jk_stats* st) {
  if (!cctx || !st) return HFG_ERR_INVALID_INPUT;
  hfg_ctx* ctx = const_cast<hfg_ctx*>(cctx);  // the exact counts are made on first request
  std::lock_guard<std::mutex> lk(ctx->mu);
  if (!ctx->last_plan) {
    *st = ctx->last;
    return HFG_OK;
  }
  AllocScope alloc_scope(ctx->stream);
  cudaSetDevice(ctx->device);
  const int rc = count_plan(ctx, ctx->last_plan);
  if (rc != HFG_OK) return rc;
  *st = ctx->last_plan->stats;
  return HFG_OK;
}

}  // extern "C"
