// CPU oracle for the hf-rs Fock-build path.  TEST INFRASTRUCTURE ONLY.
//
// This file restates, in plain C++ (OpenMP for the embarrassingly parallel
// loops), the integral and Fock-digestion arithmetic of hf-rs v0.3.2 so that
// the CUDA product can be checked against it.  Nothing in the product links
// or calls this library: only tests/, __graft_entry__.smoke() and the
// cpu_baseline leg of bench.py may load it, and only as the checker.
//
// Each function names the reference lines it follows (paths are relative to
// the hf-rs project root).  The restatement is pinned against the reference's
// own golden vectors (tests/data/boys_reference.json, the 160,000 PySCF
// Cartesian ERIs of spherical_reference.json["spdf_integrals"], the SCF
// energies of scf_reference.json and the DF fixtures); see tests/test_oracle_*.
//
// Floating-point contraction is disabled at build time (-ffp-contract=off)
// because the Rust reference never fuses multiply-adds.

#include <algorithm>
#include <array>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <mutex>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

// ---------------------------------------------------------------- Boys ----
// src/integrals.rs:20-36 (constants, lazily built Taylor table),
// :39-57 (boys_reference_downward), :70-101 (boys_array).
constexpr int kBoysMaxM = 40;
constexpr int kTaylor = 7;
constexpr int kTableM = kBoysMaxM + kTaylor;  // 47
constexpr double kGridStep = 0.05;
constexpr double kTSwitch = 50.0;
constexpr int kGridSize = 1002;
constexpr double kTwoPiPow25 = 34.986836655249726164477;
constexpr double kPiPow15 = 5.56832799683170784528;
constexpr double kHalfSqrtPi = 0.88622692545275801365;

void boys_reference_downward(int max_n, double t, double* out) {
  const double exp_t = std::exp(-t);
  double term = 1.0 / (double)(2 * max_n + 1);
  double sum = term;
  long i = 1;
  for (;;) {
    term *= 2.0 * t / (double)(2 * max_n + 2 * i + 1);
    sum += term;
    if (term < sum * 1e-17 || i > 10000) break;
    ++i;
  }
  out[max_n] = exp_t * sum;
  for (int m = max_n - 1; m >= 0; --m)
    out[m] = (2.0 * t * out[m + 1] + exp_t) / (double)(2 * m + 1);
}

std::vector<double>& boys_table() {
  static std::vector<double> table;
  static std::once_flag once;
  std::call_once(once, [] {
    table.assign((size_t)kGridSize * (kTableM + 1), 0.0);
    for (int idx = 0; idx < kGridSize; ++idx)
      boys_reference_downward(kTableM, idx * kGridStep, &table[(size_t)idx * (kTableM + 1)]);
  });
  return table;
}

void boys_array(int max_n, double t, double* out) {
  if (t > kTSwitch) {
    const double exp_t = std::exp(-t);
    const double inv_2t = 0.5 / t;
    out[0] = kHalfSqrtPi * std::erf(std::sqrt(t)) / std::sqrt(t);
    for (int n = 1; n <= max_n; ++n) out[n] = ((double)(2 * n - 1) * out[n - 1] - exp_t) * inv_2t;
    return;
  }
  const size_t idx = (size_t)std::round(t * (1.0 / kGridStep));
  const double t0 = (double)idx * kGridStep;
  const double dt = t - t0;
  const double* row = &boys_table()[idx * (kTableM + 1)];
  double coeff[kTaylor + 1];
  coeff[0] = 1.0;
  for (int k = 1; k <= kTaylor; ++k) coeff[k] = coeff[k - 1] * (-dt) / (double)k;
  for (int n = 0; n <= max_n; ++n) {
    double acc = 0.0;
    for (int k = kTaylor; k >= 0; --k) acc += coeff[k] * row[n + k];
    out[n] = acc;
  }
}

double boys(int n, double t) {
  double out[kBoysMaxM + 1];
  boys_array(n, t, out);
  return out[n];
}

// ------------------------------------------------------ Hermite E_t^{ij} --
// src/integrals.rs:135-191 (compute_hermite_coeffs).  E is stored flat as
// E[(i*(lb+1)+j)*(la+lb+1)+t].
struct Hermite1D {
  int la = 0, lb = 0;
  std::vector<double> e;
  double get(int i, int j, int t) const { return e[((size_t)i * (lb + 1) + j) * (la + lb + 1) + t]; }
};

void hermite_coeffs(int la, int lb, double alpha, double beta, double a, double b, Hermite1D& out) {
  out.la = la;
  out.lb = lb;
  const int st = la + lb + 1;
  out.e.assign((size_t)(la + 1) * (lb + 1) * st, 0.0);
  auto E = [&](int i, int j, int t) -> double& { return out.e[((size_t)i * (lb + 1) + j) * st + t]; };
  const double p = alpha + beta;
  const double inv_p = 1.0 / p;
  const double pc = (alpha * a + beta * b) * inv_p;
  const double x_pa = pc - a, x_pb = pc - b;
  const double mu = (alpha * beta) * inv_p;
  const int max_t = la + lb;
  const double inv_2p = 0.5 * inv_p;
  const double diff = a - b;
  E(0, 0, 0) = std::exp(-mu * diff * diff);
  for (int i = 0; i <= la; ++i)
    for (int j = 0; j <= lb; ++j)
      for (int t = 0; t <= i + j; ++t) {
        if (i == 0 && j == 0) continue;
        if (i > 0) {
          double t1 = t > 0 ? E(i - 1, j, t - 1) * inv_2p : 0.0;
          double t2 = x_pa * E(i - 1, j, t);
          double t3 = t < max_t ? ((double)t + 1.0) * E(i - 1, j, t + 1) : 0.0;
          E(i, j, t) = t1 + t2 + t3;
        } else {
          double t1 = t > 0 ? E(i, j - 1, t - 1) * inv_2p : 0.0;
          double t2 = x_pb * E(i, j - 1, t);
          double t3 = t < max_t ? ((double)t + 1.0) * E(i, j - 1, t + 1) : 0.0;
          E(i, j, t) = t1 + t2 + t3;
        }
      }
}

// ------------------------------------------------------ R_{tuv}^n --------
// src/integrals.rs:253-346 (coulomb_auxiliary_integrals_total).
void coulomb_aux_total(int max_t, int max_u, int max_v, int max_n, double p, const double pc[3],
                       double* r) {
  const double x = pc[0], y = pc[1], z = pc[2];
  const double r2 = x * x + y * y + z * z;
  const size_t sv = max_n + 1, su = (max_v + 1) * sv, st = (max_u + 1) * su;
  double f[kBoysMaxM + 1];
  boys_array(max_n, p * r2, f);
  const double neg_2p = -2.0 * p;
  double pw = 1.0;
  for (int n = 0; n <= max_n; ++n) {
    r[n] = pw * f[n];
    pw *= neg_2p;
  }
  for (int t = 0; t < std::min(max_t, max_n); ++t) {
    size_t cur = t * st, prev = t > 0 ? (t - 1) * st : 0, next = (t + 1) * st;
    int limit = max_n - t - 1;
    for (int n = 0; n <= limit; ++n)
      r[next + n] = t > 0 ? (double)t * r[prev + n + 1] + x * r[cur + n + 1] : x * r[cur + n + 1];
  }
  for (int t = 0; t <= std::min(max_t, max_n); ++t) {
    size_t to = t * st;
    for (int u = 0; u < std::min(max_u, max_n - t); ++u) {
      size_t cur = to + u * su, prev = u > 0 ? to + (u - 1) * su : 0, next = to + (u + 1) * su;
      int limit = max_n - t - u - 1;
      for (int n = 0; n <= limit; ++n)
        r[next + n] = u > 0 ? (double)u * r[prev + n + 1] + y * r[cur + n + 1] : y * r[cur + n + 1];
    }
  }
  for (int t = 0; t <= std::min(max_t, max_n); ++t) {
    size_t to = t * st;
    for (int u = 0; u <= std::min(max_u, max_n - t); ++u) {
      size_t tuo = to + u * su;
      for (int v = 0; v < std::min(max_v, max_n - t - u); ++v) {
        size_t cur = tuo + v * sv, prev = v > 0 ? tuo + (v - 1) * sv : 0, next = tuo + (v + 1) * sv;
        int limit = max_n - t - u - v - 1;
        for (int n = 0; n <= limit; ++n)
          r[next + n] = v > 0 ? (double)v * r[prev + n + 1] + z * r[cur + n + 1] : z * r[cur + n + 1];
      }
    }
  }
}

// src/integrals.rs:905-971 (evaluate_eri_contraction_pairs).
double eri_contraction_pairs(int tab, int uab, int vab, int tcd, int ucd, int vcd, size_t st, size_t su,
                             size_t sv, const double* exab, const double* eyab, const double* ezab,
                             const double* excd, const double* eycd, const double* ezcd, const double* r,
                             double prefactor) {
  const int mt = tab + tcd, mu = uab + ucd, mv = vab + vcd;
  double cx[kBoysMaxM + 1] = {0}, cy[kBoysMaxM + 1] = {0}, cz[kBoysMaxM + 1] = {0};
  for (int t = 0; t <= tab; ++t) {
    double et = exab[t];
    if (et == 0.0) continue;
    for (int tp = 0; tp <= tcd; ++tp) cx[t + tp] += et * ((tp & 1) ? -excd[tp] : excd[tp]);
  }
  for (int u = 0; u <= uab; ++u) {
    double eu = eyab[u];
    if (eu == 0.0) continue;
    for (int up = 0; up <= ucd; ++up) cy[u + up] += eu * ((up & 1) ? -eycd[up] : eycd[up]);
  }
  for (int v = 0; v <= vab; ++v) {
    double ev = ezab[v];
    if (ev == 0.0) continue;
    for (int vp = 0; vp <= vcd; ++vp) cz[v + vp] += ev * ((vp & 1) ? -ezcd[vp] : ezcd[vp]);
  }
  double sum = 0.0;
  for (int t = 0; t <= mt; ++t) {
    double cxt = cx[t];
    if (cxt == 0.0) continue;
    size_t to = t * st;
    for (int u = 0; u <= mu; ++u) {
      double cyu = cy[u];
      if (cyu == 0.0) continue;
      size_t idx = to + u * su;
      double cxy = cxt * cyu;
      for (int v = 0; v <= mv; ++v) {
        double czv = cz[v];
        if (czv != 0.0) sum += cxy * czv * r[idx];
        idx += sv;
      }
    }
  }
  return prefactor * sum;
}

// ---------------------------------------------------------- basis input --
// A Cartesian contracted Gaussian exactly as hf-rs's ContractedGaussian
// (src/basis.rs:87-100): center, powers, atom index, primitives with the
// fully normalised coefficient of this component (src/basis.rs:455-496).
struct CG {
  double c[3];
  int l[3];
  int atom;
  std::vector<double> exps, coefs;
  int L() const { return l[0] + l[1] + l[2]; }
};

}  // namespace

extern "C" {
// Flat description of a list of Cartesian functions.
typedef struct {
  int n;
  const double* center;  // [n*3]
  const int* lxyz;       // [n*3]
  const int* atom;       // [n]
  const int* prim_off;   // [n+1]
  const double* exps;    // [prim_off[n]]
  const double* coefs;   // [prim_off[n]]
} orc_basis;
}

namespace {

std::vector<CG> unpack(const orc_basis* b) {
  std::vector<CG> out(b->n);
  for (int i = 0; i < b->n; ++i) {
    CG& g = out[i];
    for (int k = 0; k < 3; ++k) {
      g.c[k] = b->center[3 * i + k];
      g.l[k] = b->lxyz[3 * i + k];
    }
    g.atom = b->atom[i];
    g.exps.assign(b->exps + b->prim_off[i], b->exps + b->prim_off[i + 1]);
    g.coefs.assign(b->coefs + b->prim_off[i], b->coefs + b->prim_off[i + 1]);
  }
  return out;
}

CG constant_function(const double c[3]) {
  // src/df.rs:30-40: exponent-0 unit function used to make a 3- or 2-centre
  // integral out of the 4-centre engine.
  CG g;
  for (int k = 0; k < 3; ++k) {
    g.c[k] = c[k];
    g.l[k] = 0;
  }
  g.atom = 0;
  g.exps = {0.0};
  g.coefs = {1.0};
  return g;
}

// ----------------------------------------------- scalar ERI engine -------
// src/integrals.rs:820-900 (PrimitivePairData, BasisPairData::new, with the
// 1e-15 coefficient and 1e-13 coefficient*overlap cuts), :973-1043
// (primitive_eri_from_pairs), :1043-1059 (evaluate_pair_eri, 1e-13 cut),
// :1062-1072 (contracted_eri).
struct PrimPair {
  double p, inv_p, P[3], coeff;
  int tm, um, vm;
  std::vector<double> ex, ey, ez;
};

std::vector<PrimPair> basis_pair(const CG& a, const CG& b) {
  std::vector<PrimPair> prims;
  const double dx = a.c[0] - b.c[0], dy = a.c[1] - b.c[1], dz = a.c[2] - b.c[2];
  const double d2 = dx * dx + dy * dy + dz * dz;
  Hermite1D hx, hy, hz;
  for (size_t ia = 0; ia < a.exps.size(); ++ia)
    for (size_t ib = 0; ib < b.exps.size(); ++ib) {
      const double coeff = a.coefs[ia] * b.coefs[ib];
      if (std::fabs(coeff) < 1e-15) continue;
      const double al = a.exps[ia], be = b.exps[ib];
      const double p = al + be, inv_p = 1.0 / p, mu = (al * be) * inv_p;
      const double ef = std::exp(-mu * d2);
      if (std::fabs(coeff * ef) < 1e-13) continue;
      PrimPair q;
      q.p = p;
      q.inv_p = inv_p;
      for (int k = 0; k < 3; ++k) q.P[k] = (al * a.c[k] + be * b.c[k]) * inv_p;
      q.coeff = coeff;
      hermite_coeffs(a.l[0], b.l[0], al, be, a.c[0], b.c[0], hx);
      hermite_coeffs(a.l[1], b.l[1], al, be, a.c[1], b.c[1], hy);
      hermite_coeffs(a.l[2], b.l[2], al, be, a.c[2], b.c[2], hz);
      q.tm = a.l[0] + b.l[0];
      q.um = a.l[1] + b.l[1];
      q.vm = a.l[2] + b.l[2];
      for (int t = 0; t <= q.tm; ++t) q.ex.push_back(hx.get(a.l[0], b.l[0], t));
      for (int t = 0; t <= q.um; ++t) q.ey.push_back(hy.get(a.l[1], b.l[1], t));
      for (int t = 0; t <= q.vm; ++t) q.ez.push_back(hz.get(a.l[2], b.l[2], t));
      prims.push_back(std::move(q));
    }
  return prims;
}

double primitive_eri_from_pairs(const PrimPair& ab, const PrimPair& cd, std::vector<double>& rbuf) {
  const double p = ab.p, q = cd.p, ppq = p + q;
  const double ap = (p * q) / ppq;
  const double pq[3] = {ab.P[0] - cd.P[0], ab.P[1] - cd.P[1], ab.P[2] - cd.P[2]};
  const int mt = ab.tm + cd.tm, mu = ab.um + cd.um, mv = ab.vm + cd.vm;
  const int mn = mt + mu + mv;
  const double r2 = pq[0] * pq[0] + pq[1] * pq[1] + pq[2] * pq[2];
  const double pref = kTwoPiPow25 / (p * q * std::sqrt(ppq));
  if (mn == 0) {
    double f0 = boys(0, ap * r2);
    return pref * (ab.ex[0] * ab.ey[0] * ab.ez[0]) * (cd.ex[0] * cd.ey[0] * cd.ez[0]) * f0;
  }
  const size_t sv = mn + 1, su = (mv + 1) * sv, st = (mu + 1) * su;
  const size_t total = (mt + 1) * st;
  if (rbuf.size() < total) rbuf.resize(total);
  coulomb_aux_total(mt, mu, mv, mt + mu + mv, ap, pq, rbuf.data());
  return eri_contraction_pairs(ab.tm, ab.um, ab.vm, cd.tm, cd.um, cd.vm, st, su, sv, ab.ex.data(), ab.ey.data(),
                               ab.ez.data(), cd.ex.data(), cd.ey.data(), cd.ez.data(), rbuf.data(), pref);
}

double evaluate_pair_eri(const std::vector<PrimPair>& ab, const std::vector<PrimPair>& cd,
                         std::vector<double>& rbuf) {
  double val = 0.0;
  for (const auto& x : ab)
    for (const auto& y : cd) {
      const double tc = x.coeff * y.coeff;
      if (std::fabs(tc) < 1e-13) continue;
      val += tc * primitive_eri_from_pairs(x, y, rbuf);
    }
  return val;
}

double contracted_eri(const CG& a, const CG& b, const CG& c, const CG& d) {
  std::vector<double> rbuf(8192);
  return evaluate_pair_eri(basis_pair(a, b), basis_pair(c, d), rbuf);
}

// ------------------------------------------------- shell ERI engine ------
// src/ao.rs:133-164 (shell_ranges: consecutive complete Cartesian shells).
bool shell_ranges(const std::vector<CG>& basis, std::vector<std::pair<int, int>>& out) {
  out.clear();
  size_t start = 0;
  while (start < basis.size()) {
    const CG& a = basis[start];
    const int l = a.L();
    const size_t count = (size_t)(l + 1) * (l + 2) / 2;
    if (l > 7 || start + count > basis.size()) return false;
    for (size_t k = start; k < start + count; ++k) {
      const CG& b = basis[k];
      if (b.atom != a.atom || b.c[0] != a.c[0] || b.c[1] != a.c[1] || b.c[2] != a.c[2] || b.L() != l ||
          b.exps.size() != a.exps.size())
        return false;
      for (size_t q = 0; q < a.exps.size(); ++q)
        if (b.exps[q] != a.exps[q]) return false;
      for (size_t q = start; q < k; ++q)
        if (basis[q].l[0] == b.l[0] && basis[q].l[1] == b.l[1] && basis[q].l[2] == b.l[2]) return false;
    }
    out.push_back({(int)start, (int)count});
    start += count;
  }
  return true;
}

// src/shell_integrals.rs:12-90 (PairPrimitive, ShellPair::new, expansion).
struct PairPrim {
  double exponent, center[3];
  std::vector<double> hermite[3];  // [(i*(lb+1)+j)*(la+lb+1)+t]
  std::vector<double> coefficients;  // per component pair ij = i*nb+j
};
struct ShellPair {
  const CG* a;
  int na;
  const CG* b;
  int nb;
  int la, lb;
  std::vector<PairPrim> prims;
  int len() const { return na * nb; }
  const double* expansion(const PairPrim& p, int axis, int i, int j) const {
    const int stride = la + lb + 1;
    const size_t off = ((size_t)a[i].l[axis] * (lb + 1) + b[j].l[axis]) * stride;
    return &p.hermite[axis][off];
  }
};

ShellPair make_shell_pair(const CG* a, int na, const CG* b, int nb) {
  ShellPair sp{a, na, b, nb, a[0].L(), b[0].L(), {}};
  const int la = sp.la, lb = sp.lb;
  const int stride = (lb + 1) * (la + lb + 1);
  Hermite1D h;
  for (size_t ia = 0; ia < a[0].exps.size(); ++ia)
    for (size_t ib = 0; ib < b[0].exps.size(); ++ib) {
      PairPrim pp;
      const double ea = a[0].exps[ia], eb = b[0].exps[ib];
      const double p = ea + eb;
      pp.exponent = p;
      for (int k = 0; k < 3; ++k) pp.center[k] = (ea * a[0].c[k] + eb * b[0].c[k]) / p;
      for (int axis = 0; axis < 3; ++axis) {
        hermite_coeffs(la, lb, ea, eb, a[0].c[axis], b[0].c[axis], h);
        pp.hermite[axis].assign((size_t)(la + 1) * stride, 0.0);
        for (int i = 0; i <= la; ++i)
          for (int j = 0; j <= lb; ++j)
            for (int t = 0; t <= i + j; ++t)
              pp.hermite[axis][(size_t)i * stride + j * (la + lb + 1) + t] = h.get(i, j, t);
      }
      for (int i = 0; i < na; ++i)
        for (int j = 0; j < nb; ++j) pp.coefficients.push_back(a[i].coefs[ia] * b[j].coefs[ib]);
      sp.prims.push_back(std::move(pp));
    }
  return sp;
}

// src/shell_integrals.rs:92-135 (quartet).
void quartet(const ShellPair& ab, const ShellPair& cd, bool diagonal_only, std::vector<double>& result,
             std::vector<double>& r) {
  const int nab = ab.len(), ncd = cd.len();
  result.assign(diagonal_only ? nab : (size_t)nab * ncd, 0.0);
  const int order = ab.la + ab.lb + cd.la + cd.lb;
  const size_t sv = order + 1, su = sv * sv, st = su * sv;
  r.assign(st * sv, 0.0);
  for (const auto& p : ab.prims)
    for (const auto& q : cd.prims) {
      const double rho = p.exponent * q.exponent / (p.exponent + q.exponent);
      const double delta[3] = {p.center[0] - q.center[0], p.center[1] - q.center[1], p.center[2] - q.center[2]};
      coulomb_aux_total(order, order, order, order, rho, delta, r.data());
      const double pref = kTwoPiPow25 / (p.exponent * q.exponent * std::sqrt(p.exponent + q.exponent));
      for (int ij = 0; ij < nab; ++ij) {
        const int i = ij / ab.nb, j = ij % ab.nb;
        const double* eab[3];
        int lab[3];
        for (int k = 0; k < 3; ++k) {
          eab[k] = ab.expansion(p, k, i, j);
          lab[k] = ab.a[i].l[k] + ab.b[j].l[k];
        }
        const int start = diagonal_only ? ij : 0, end = diagonal_only ? ij + 1 : ncd;
        for (int kl = start; kl < end; ++kl) {
          const int k = kl / cd.nb, l = kl % cd.nb;
          const double* ecd[3];
          int lcd[3];
          for (int x = 0; x < 3; ++x) {
            ecd[x] = cd.expansion(q, x, k, l);
            lcd[x] = cd.a[k].l[x] + cd.b[l].l[x];
          }
          const double value = eri_contraction_pairs(lab[0], lab[1], lab[2], lcd[0], lcd[1], lcd[2], st, su, sv,
                                                     eab[0], eab[1], eab[2], ecd[0], ecd[1], ecd[2], r.data(), pref);
          const size_t index = diagonal_only ? ij : (size_t)ij * ncd + kl;
          result[index] += p.coefficients[ij] * q.coefficients[kl] * value;
        }
      }
    }
}

inline size_t compound_index(size_t i, size_t j) { return i >= j ? i * (i + 1) / 2 + j : j * (j + 1) / 2 + i; }
inline size_t eri_index(size_t i, size_t j, size_t k, size_t l) {
  return compound_index(compound_index(i, j), compound_index(k, l));
}

// Shell pairs (a>=b) in the order of src/shell_integrals.rs:158-161 and their
// Schwarz bounds Q_ab = sqrt(max diag (ab|ab)) (:165-173).
struct PairTable {
  std::vector<std::pair<int, int>> shells;       // ranges
  std::vector<std::pair<int, int>> shell_pairs;  // (a,b), a>=b
  std::vector<ShellPair> pairs;
  std::vector<double> bounds;
};

bool build_pairs(const std::vector<CG>& basis, PairTable& t, int nthreads) {
  if (!shell_ranges(basis, t.shells)) return false;
  const int ns = (int)t.shells.size();
  for (int a = 0; a < ns; ++a)
    for (int b = 0; b <= a; ++b) t.shell_pairs.push_back({a, b});
  const size_t np = t.shell_pairs.size();
  t.pairs.resize(np);
  t.bounds.assign(np, 0.0);
#pragma omp parallel for schedule(dynamic, 4) num_threads(nthreads)
  for (long ij = 0; ij < (long)np; ++ij) {
    auto [a, b] = t.shell_pairs[ij];
    t.pairs[ij] = make_shell_pair(&basis[t.shells[a].first], t.shells[a].second, &basis[t.shells[b].first],
                                  t.shells[b].second);
    std::vector<double> res, r;
    quartet(t.pairs[ij], t.pairs[ij], true, res, r);
    double m = 0.0;
    for (double v : res) m = std::max(m, v);
    t.bounds[ij] = std::sqrt(m);
  }
  return true;
}

// src/scf.rs:337-364 (contract_jk): digestion of one unique AO quartet with
// the pair/bra/ket flips of the 8-fold symmetry.
inline void digest(size_t n, size_t mu, size_t nu, size_t lam, size_t sig, double value, const double* tot,
                   int nspin, const double* spins, double* J, double* K) {
  const size_t ij = compound_index(mu, nu), kl = compound_index(lam, sig);
  for (int pf = 0; pf < (ij == kl ? 1 : 2); ++pf) {
    size_t aa, bb, cc, dd;
    if (pf == 0) {
      aa = mu; bb = nu; cc = lam; dd = sig;
    } else {
      aa = lam; bb = sig; cc = mu; dd = nu;
    }
    for (int abf = 0; abf < (aa == bb ? 1 : 2); ++abf) {
      const size_t a = abf == 0 ? aa : bb, b = abf == 0 ? bb : aa;
      for (int cdf = 0; cdf < (cc == dd ? 1 : 2); ++cdf) {
        const size_t c = cdf == 0 ? cc : dd, d = cdf == 0 ? dd : cc;
        J[a * n + b] += tot[c * n + d] * value;
        for (int s = 0; s < nspin; ++s) K[s * n * n + a * n + c] += spins[s * n * n + b * n + d] * value;
      }
    }
  }
}

}  // namespace

extern "C" {

// ---------------------------------------------------------------- API ----
void orc_boys_array(int max_n, double t, double* out) { boys_array(max_n, t, out); }

double orc_contracted_eri(const orc_basis* b, int i, int j, int k, int l) {
  auto basis = unpack(b);
  return contracted_eri(basis[i], basis[j], basis[k], basis[l]);
}

// Contracted ERIs for an explicit list of function index quartets, each drawn
// from its own basis list (used for the SPDF golden block, which spans four
// single-atom bases).
void orc_contracted_eri_list(const orc_basis* b0, const orc_basis* b1, const orc_basis* b2, const orc_basis* b3,
                             long count, const int* idx, double* out, int nthreads) {
  auto B0 = unpack(b0), B1 = unpack(b1), B2 = unpack(b2), B3 = unpack(b3);
#pragma omp parallel for schedule(dynamic, 64) num_threads(nthreads)
  for (long q = 0; q < count; ++q)
    out[q] = contracted_eri(B0[idx[4 * q]], B1[idx[4 * q + 1]], B2[idx[4 * q + 2]], B3[idx[4 * q + 3]]);
}

// src/shell_integrals.rs:138-151 (compute_shell_quartet): four single-shell
// bases, a,b,c,d row-major block.  Returns the block length or -1.
long orc_shell_quartet(const orc_basis* b0, const orc_basis* b1, const orc_basis* b2, const orc_basis* b3,
                       double* out) {
  auto B0 = unpack(b0), B1 = unpack(b1), B2 = unpack(b2), B3 = unpack(b3);
  std::vector<std::pair<int, int>> r;
  for (auto* B : {&B0, &B1, &B2, &B3})
    if (!shell_ranges(*B, r) || r.size() != 1) return -1;
  auto ab = make_shell_pair(B0.data(), (int)B0.size(), B1.data(), (int)B1.size());
  auto cd = make_shell_pair(B2.data(), (int)B2.size(), B3.data(), (int)B3.size());
  std::vector<double> res, rr;
  quartet(ab, cd, false, res, rr);
  std::memcpy(out, res.data(), res.size() * sizeof(double));
  return (long)res.size();
}

// Shell ranges (start, count) of a basis; returns the shell count or -1.
int orc_shell_ranges(const orc_basis* b, int* starts, int* counts) {
  auto basis = unpack(b);
  std::vector<std::pair<int, int>> r;
  if (!shell_ranges(basis, r)) return -1;
  for (size_t i = 0; i < r.size(); ++i) {
    if (starts) starts[i] = r[i].first;
    if (counts) counts[i] = r[i].second;
  }
  return (int)r.size();
}

// Schwarz bounds of every shell pair a>=b in reference order; returns the pair
// count or -1.
long orc_schwarz(const orc_basis* b, double* bounds, int nthreads) {
  auto basis = unpack(b);
  PairTable t;
  if (!build_pairs(basis, t, nthreads)) return -1;
  if (bounds) std::memcpy(bounds, t.bounds.data(), t.bounds.size() * sizeof(double));
  return (long)t.bounds.size();
}

// src/shell_integrals.rs:156-240 (compute_shell_eri_tensor): packed 8-fold
// tensor with shell Schwarz screening at 1e-12.  out has n_p(n_p+1)/2 slots.
int orc_eri_packed(const orc_basis* b, double* out, size_t len, int nthreads) {
  auto basis = unpack(b);
  const size_t n = basis.size(), npair = n * (n + 1) / 2;
  if (len != npair * (npair + 1) / 2) return -2;
  PairTable t;
  if (!build_pairs(basis, t, nthreads)) return -1;
  std::memset(out, 0, len * sizeof(double));
  const long np = (long)t.pairs.size();
#pragma omp parallel for schedule(dynamic, 1) num_threads(nthreads)
  for (long ij = 0; ij < np; ++ij) {
    std::vector<double> block, r;
    for (long kl = 0; kl <= ij; ++kl) {
      if (t.bounds[ij] * t.bounds[kl] <= 1e-12) continue;
      quartet(t.pairs[ij], t.pairs[kl], false, block, r);
      auto [a, bb] = t.shell_pairs[ij];
      auto [c, d] = t.shell_pairs[kl];
      const ShellPair &AB = t.pairs[ij], &CD = t.pairs[kl];
      for (int i = 0; i < AB.na; ++i)
        for (int j = 0; j < AB.nb; ++j) {
          const size_t mu = t.shells[a].first + i, nu = t.shells[bb].first + j;
          if (mu < nu) continue;
          for (int k = 0; k < CD.na; ++k)
            for (int l = 0; l < CD.nb; ++l) {
              const size_t lam = t.shells[c].first + k, sig = t.shells[d].first + l;
              if (lam < sig) continue;
              // Distinct (ij,kl) shell quartets never share a packed slot; the
              // ij==kl block writes each slot twice with equal values.
              out[eri_index(mu, nu, lam, sig)] = block[((size_t)i * AB.nb + j) * CD.len() + k * CD.nb + l];
            }
        }
    }
  }
  return 0;
}

// src/scf.rs:337-375: J and K_s from the packed tensor.  spins holds nspin
// n x n row-major matrices; K receives nspin matrices.
void orc_contract_jk(int n_, const double* eri, const double* tot, int nspin, const double* spins, double* J,
                     double* K) {
  const size_t n = n_;
  std::memset(J, 0, n * n * sizeof(double));
  std::memset(K, 0, nspin * n * n * sizeof(double));
  std::vector<std::pair<size_t, size_t>> pairs;
  for (size_t i = 0; i < n; ++i)
    for (size_t j = 0; j <= i; ++j) pairs.push_back({i, j});
  for (size_t ij = 0; ij < pairs.size(); ++ij) {
    const double* row = eri + ij * (ij + 1) / 2;
    for (size_t kl = 0; kl <= ij; ++kl) {
      const double v = row[kl];
      if (v == 0.0) continue;
      digest(n, pairs[ij].first, pairs[ij].second, pairs[kl].first, pairs[kl].second, v, tot, nspin, spins, J, K);
    }
  }
}

// Direct form of compute_shell_eri_tensor followed by contract_jk: the same
// screened shell quartets and the same integral values, digested into J/K
// without storing the tensor.  If rows != NULL only the listed bra shell
// pairs ij are processed (a bounded sample for CPU timing).  Returns 0 or -1.
int orc_direct_jk(const orc_basis* b, const double* tot, int nspin, const double* spins, double* J, double* K,
                  double thresh, const long* rows, long nrows, int nthreads) {
  auto basis = unpack(b);
  const size_t n = basis.size();
  PairTable t;
  if (!build_pairs(basis, t, nthreads)) return -1;
  const long np = (long)t.pairs.size();
  std::vector<long> work;
  if (rows) work.assign(rows, rows + nrows);
  else
    for (long ij = np - 1; ij >= 0; --ij) work.push_back(ij);
  std::memset(J, 0, n * n * sizeof(double));
  std::memset(K, 0, nspin * n * n * sizeof(double));
#pragma omp parallel num_threads(nthreads)
  {
    std::vector<double> Jl(n * n, 0.0), Kl(nspin * n * n, 0.0), block, r;
#pragma omp for schedule(dynamic, 1)
    for (long w = 0; w < (long)work.size(); ++w) {
      const long ij = work[w];
      for (long kl = 0; kl <= ij; ++kl) {
        if (t.bounds[ij] * t.bounds[kl] <= thresh) continue;
        quartet(t.pairs[ij], t.pairs[kl], false, block, r);
        auto [a, bb] = t.shell_pairs[ij];
        auto [c, d] = t.shell_pairs[kl];
        const ShellPair &AB = t.pairs[ij], &CD = t.pairs[kl];
        for (int i = 0; i < AB.na; ++i)
          for (int j = 0; j < AB.nb; ++j) {
            const size_t mu = t.shells[a].first + i, nu = t.shells[bb].first + j;
            if (mu < nu) continue;
            for (int k = 0; k < CD.na; ++k)
              for (int l = 0; l < CD.nb; ++l) {
                const size_t lam = t.shells[c].first + k, sig = t.shells[d].first + l;
                if (lam < sig) continue;
                if (ij == kl && compound_index(mu, nu) < compound_index(lam, sig)) continue;
                const double v = block[((size_t)i * AB.nb + j) * CD.len() + k * CD.nb + l];
                if (v == 0.0) continue;
                digest(n, mu, nu, lam, sig, v, tot, nspin, spins, Jl.data(), Kl.data());
              }
          }
      }
    }
#pragma omp critical
    {
      for (size_t x = 0; x < n * n; ++x) J[x] += Jl[x];
      for (size_t x = 0; x < nspin * n * n; ++x) K[x] += Kl[x];
    }
  }
  return 0;
}

// src/integrals.rs:408-425 (primitive_overlap), :427-470 (primitive_kinetic),
// :472-535 (primitive_nuclear_attraction), :747-793 (contractions), and
// src/scf.rs:247-271 (compute_one_electron_integrals).
void orc_one_electron(const orc_basis* b, int natom, const double* apos, const double* acharge, double* S,
                      double* T, double* V, int nthreads) {
  auto basis = unpack(b);
  const long n = (long)basis.size();
#pragma omp parallel for schedule(dynamic, 1) num_threads(nthreads)
  for (long i = 0; i < n; ++i) {
    std::vector<double> rbuf;
    Hermite1D ex, ey, ez;
    for (long j = 0; j <= i; ++j) {
      const CG &A = basis[i], &B = basis[j];
      double s = 0, t = 0, v = 0;
      for (size_t ia = 0; ia < A.exps.size(); ++ia)
        for (size_t ib = 0; ib < B.exps.size(); ++ib) {
          const double al = A.exps[ia], be = B.exps[ib], cc = A.coefs[ia] * B.coefs[ib];
          const double p = al + be, inv_p = 1.0 / p;
          // overlap
          hermite_coeffs(A.l[0], B.l[0], al, be, A.c[0], B.c[0], ex);
          hermite_coeffs(A.l[1], B.l[1], al, be, A.c[1], B.c[1], ey);
          hermite_coeffs(A.l[2], B.l[2], al, be, A.c[2], B.c[2], ez);
          s += cc * (ex.get(A.l[0], B.l[0], 0) * ey.get(A.l[1], B.l[1], 0) * ez.get(A.l[2], B.l[2], 0) *
                     (kPiPow15 * inv_p * std::sqrt(inv_p)));
          // kinetic: E with lb+2
          {
            Hermite1D kx, ky, kz;
            hermite_coeffs(A.l[0], B.l[0] + 2, al, be, A.c[0], B.c[0], kx);
            hermite_coeffs(A.l[1], B.l[1] + 2, al, be, A.c[1], B.c[1], ky);
            hermite_coeffs(A.l[2], B.l[2] + 2, al, be, A.c[2], B.c[2], kz);
            auto t1d = [&](int li, int lj, const Hermite1D& h) {
              double a1 = be * (2.0 * lj + 1.0) * h.get(li, lj, 0);
              double a2 = -2.0 * be * be * h.get(li, lj + 2, 0);
              double a3 = lj >= 2 ? -0.5 * (double)(lj * (lj - 1)) * h.get(li, lj - 2, 0) : 0.0;
              return a1 + a2 + a3;
            };
            const double tx = t1d(A.l[0], B.l[0], kx), ty = t1d(A.l[1], B.l[1], ky), tz = t1d(A.l[2], B.l[2], kz);
            const double sx = kx.get(A.l[0], B.l[0], 0), sy = ky.get(A.l[1], B.l[1], 0), sz = kz.get(A.l[2], B.l[2], 0);
            const double pref = kPiPow15 * inv_p * std::sqrt(inv_p);
            t += cc * (pref * (tx * sy * sz + sx * ty * sz + sx * sy * tz));
          }
          // nuclear attraction
          if (std::fabs(cc) >= 1e-15) {
            const double P[3] = {(al * A.c[0] + be * B.c[0]) * inv_p, (al * A.c[1] + be * B.c[1]) * inv_p,
                                 (al * A.c[2] + be * B.c[2]) * inv_p};
            const int mt = A.l[0] + B.l[0], mu = A.l[1] + B.l[1], mv = A.l[2] + B.l[2];
            const int mn = mt + mu + mv;
            const size_t sv = mn + 1, su = (mv + 1) * sv, st = (mu + 1) * su;
            rbuf.assign((mt + 1) * st, 0.0);
            const double pref = 2.0 * M_PI * inv_p;
            for (int at = 0; at < natom; ++at) {
              const double pc[3] = {P[0] - apos[3 * at], P[1] - apos[3 * at + 1], P[2] - apos[3 * at + 2]};
              coulomb_aux_total(mt, mu, mv, mn, p, pc, rbuf.data());
              double sum = 0.0;
              for (int it = 0; it <= mt; ++it) {
                double et = ex.get(A.l[0], B.l[0], it);
                if (et == 0.0) continue;
                for (int iu = 0; iu <= mu; ++iu) {
                  double eu = ey.get(A.l[1], B.l[1], iu);
                  if (eu == 0.0) continue;
                  for (int iv = 0; iv <= mv; ++iv) {
                    double ev = ez.get(A.l[2], B.l[2], iv);
                    if (ev == 0.0) continue;
                    sum += et * eu * ev * rbuf[it * st + iu * su + iv * sv];
                  }
                }
              }
              v += cc * (-acharge[at] * pref * sum);
            }
          }
        }
      S[i * n + j] = S[j * n + i] = s;
      T[i * n + j] = T[j * n + i] = t;
      V[i * n + j] = V[j * n + i] = v;
    }
  }
}

// src/df.rs:43-57 (coulomb_metric): (P|Q) with unit exponent-0 partners.
void orc_df_metric(const orc_basis* aux, double* M, int nthreads) {
  auto A = unpack(aux);
  const long n = (long)A.size();
#pragma omp parallel for schedule(dynamic, 1) num_threads(nthreads)
  for (long p = 0; p < n; ++p) {
    CG one_p = constant_function(A[p].c);
    for (long q = 0; q < n; ++q) {
      CG one_q = constant_function(A[q].c);
      M[p * n + q] = contracted_eri(A[p], one_p, A[q], one_q);
    }
  }
}

// src/df.rs:60-78 (three_center_integrals): (P|mu nu), aux rows, packed
// compound_index(mu,nu) columns.
void orc_df_three(const orc_basis* b, const orc_basis* aux, double* out, int nthreads) {
  auto B = unpack(b);
  auto A = unpack(aux);
  const long na = (long)A.size();
  const size_t n = B.size(), np = n * (n + 1) / 2;
#pragma omp parallel for schedule(dynamic, 1) num_threads(nthreads)
  for (long p = 0; p < na; ++p) {
    CG one = constant_function(A[p].c);
    for (size_t mu = 0; mu < n; ++mu)
      for (size_t nu = 0; nu <= mu; ++nu) out[p * np + compound_index(mu, nu)] = contracted_eri(B[mu], B[nu], A[p], one);
  }
}

}  // extern "C"
