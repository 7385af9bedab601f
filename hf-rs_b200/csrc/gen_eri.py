"""Generate the per-angular-class ERI code (eri_gen.cuh).

For every class (la lb|lc ld) with la >= lb, lc >= ld and l <= LMAX this
emits a specialisation of `EriClass<LA,LB,LC,LD>` with two device functions:

  prim(acc, F, geometry...)  one primitive quartet: Obara-Saika vertical
      recursion (Obara & Saika, J. Chem. Phys. 84, 3963 (1986); the
      Head-Gordon-Pople form, J. Chem. Phys. 89, 5777 (1988)) from the scaled
      Boys values F[m] = pref * F_m(T) up to [e0|f0]^(0) for |e| in
      [la, la+lb], |f| in [lc, lc+ld], added into the contracted
      accumulators `acc`;
  hrr(acc, out, AB, CD)  the horizontal recursion
      (a,b+1_i| = (a+1_i,b| + AB_i (a,b|, and its ket analogue, on the
      contracted accumulators, giving the Cartesian block (ab|cd) in a,b,c,d
      row-major order with hf-rs's component order (s; x,y,z;
      xx,yy,zz,xy,xz,yz; src/basis.rs:418-445).

The vertical recursion used, with W = (pP+qQ)/(p+q), rho = pq/(p+q):

  [a|c+1_i]^m = QC_i [a|c]^m + WQ_i [a|c]^{m+1}
              + c_i/(2q) ([a|c-1_i]^m - rho/q [a|c-1_i]^{m+1})
              + a_i/(2(p+q)) [a-1_i|c]^{m+1}
  [a+1_i|0]^m = PA_i [a|0]^m + WP_i [a|0]^{m+1}
              + a_i/(2p) ([a-1_i|0]^m - rho/p [a-1_i|0]^{m+1})

Run:  python gen_eri.py [LMAX]   (writes eri_gen.cuh next to this file)
"""
import os
import sys

AX = "xyz"


def cart(l):
    """Cartesian components of angular momentum l in hf-rs order."""
    if l == 0:
        return [(0, 0, 0)]
    if l == 1:
        return [(1, 0, 0), (0, 1, 0), (0, 0, 1)]
    if l == 2:
        return [(2, 0, 0), (0, 2, 0), (0, 0, 2), (1, 1, 0), (1, 0, 1), (0, 1, 1)]
    out = []
    for lx in range(l, -1, -1):
        for ly in range(l - lx, -1, -1):
            out.append((lx, ly, l - lx - ly))
    return out


def sub(t, i, k=1):
    t = list(t)
    t[i] -= k
    return tuple(t)


def add(t, i, k=1):
    t = list(t)
    t[i] += k
    return tuple(t)


def nz(t):
    return all(x >= 0 for x in t)


class Vrr:
    """Builds straight-line code for [a|c]^(m) intermediates."""

    def __init__(self, L):
        self.L = L
        self.names = {}
        self.lines = []
        self.count = 0

    def get(self, a, c, m):
        key = (a, c, m)
        if key in self.names:
            return self.names[key]
        if sum(a) == 0 and sum(c) == 0:
            name = "F[%d]" % m
            self.names[key] = name
            return name
        terms = []
        if sum(c) > 0:
            i = next(k for k in range(3) if c[k] > 0)
            c1 = sub(c, i)
            terms.append("QC%s*%s" % (AX[i], self.get(a, c1, m)))
            terms.append("WQ%s*%s" % (AX[i], self.get(a, c1, m + 1)))
            if c1[i] > 0:
                c2 = sub(c1, i)
                terms.append("T(%d)*i2q*(%s - rq*%s)" % (c1[i], self.get(a, c2, m), self.get(a, c2, m + 1)))
            if a[i] > 0:
                terms.append("T(%d)*i2s*%s" % (a[i], self.get(sub(a, i), c1, m + 1)))
        else:
            i = next(k for k in range(3) if a[k] > 0)
            a1 = sub(a, i)
            terms.append("PA%s*%s" % (AX[i], self.get(a1, c, m)))
            terms.append("WP%s*%s" % (AX[i], self.get(a1, c, m + 1)))
            if a1[i] > 0:
                a2 = sub(a1, i)
                terms.append("T(%d)*i2p*(%s - rp*%s)" % (a1[i], self.get(a2, c, m), self.get(a2, c, m + 1)))
        name = "v%d" % self.count
        self.count += 1
        self.lines.append("const T %s = %s;" % (name, " + ".join(terms)))
        self.names[key] = name
        return name


def gen_class(la, lb, lc, ld):
    L = la + lb + lc + ld
    erange = [e for l in range(la, la + lb + 1) for e in cart(l)]
    frange = [f for l in range(lc, lc + ld + 1) for f in cart(l)]
    eidx = {e: k for k, e in enumerate(erange)}
    fidx = {f: k for k, f in enumerate(frange)}
    nacc = len(erange) * len(frange)
    v = Vrr(L)
    acc_lines = []
    for e in erange:
        for f in frange:
            name = v.get(e, f, 0)
            acc_lines.append("acc[%d] += %s;" % (eidx[e] * len(frange) + fidx[f], name))
    # HRR bra: for each f, (a,b| from (e,0|
    hl = []
    cnt = [0]

    def newv():
        cnt[0] += 1
        return "h%d" % cnt[0]

    bra_memo = {}

    def bra(a, b, f):
        key = (a, b, f)
        if key in bra_memo:
            return bra_memo[key]
        if sum(b) == 0:
            r = "acc[%d]" % (eidx[a] * len(frange) + fidx[f])
        else:
            i = next(k for k in range(3) if b[k] > 0)
            b1 = sub(b, i)
            x1 = bra(add(a, i), b1, f)
            x2 = bra(a, b1, f)
            r = newv()
            hl.append("const T %s = %s + AB%s*%s;" % (r, x1, AX[i], x2))
        bra_memo[key] = r
        return r

    ket_memo = {}

    def ket(a, b, c, d):
        key = (a, b, c, d)
        if key in ket_memo:
            return ket_memo[key]
        if sum(d) == 0:
            r = bra(a, b, c)
        else:
            i = next(k for k in range(3) if d[k] > 0)
            d1 = sub(d, i)
            x1 = ket(a, b, add(c, i), d1)
            x2 = ket(a, b, c, d1)
            r = newv()
            hl.append("const T %s = %s + CD%s*%s;" % (r, x1, AX[i], x2))
        ket_memo[key] = r
        return r

    out_lines = []
    n = 0
    for a in cart(la):
        for b in cart(lb):
            for c in cart(lc):
                for d in cart(ld):
                    out_lines.append("out[%d] = %s;" % (n, ket(a, b, c, d)))
                    n += 1
    s = []
    s.append("template <> struct EriClass<%d, %d, %d, %d> {" % (la, lb, lc, ld))
    s.append("  static constexpr int L = %d;" % L)
    s.append("  static constexpr int NACC = %d;" % nacc)
    s.append("  static constexpr int NOUT = %d;" % n)
    s.append("  template <typename T>")
    s.append("  __device__ __forceinline__ static void prim(T* __restrict__ acc, const T* __restrict__ F,")
    s.append("      T PAx, T PAy, T PAz, T WPx, T WPy, T WPz, T QCx, T QCy, T QCz, T WQx, T WQy, T WQz,")
    s.append("      T i2p, T i2q, T i2s, T rp, T rq) {")
    s.append("    (void)PAx; (void)PAy; (void)PAz; (void)WPx; (void)WPy; (void)WPz;")
    s.append("    (void)QCx; (void)QCy; (void)QCz; (void)WQx; (void)WQy; (void)WQz;")
    s.append("    (void)i2p; (void)i2q; (void)i2s; (void)rp; (void)rq;")
    for ln in v.lines:
        s.append("    " + ln)
    for ln in acc_lines:
        s.append("    " + ln)
    s.append("  }")
    s.append("  template <typename T>")
    s.append("  __device__ __forceinline__ static void hrr(const T* __restrict__ acc, T* __restrict__ out,")
    s.append("      T ABx, T ABy, T ABz, T CDx, T CDy, T CDz) {")
    s.append("    (void)ABx; (void)ABy; (void)ABz; (void)CDx; (void)CDy; (void)CDz;")
    for ln in hl:
        s.append("    " + ln)
    for ln in out_lines:
        s.append("    " + ln)
    s.append("  }")
    s.append("};")
    return "\n".join(s), v.count, len(hl)


def class_list(lmax):
    """Four-centre classes with l <= lmax, plus the density-fitting classes
    (la lb|lc 0): orbital pairs (la, lb <= 2) or an auxiliary function with a
    unit partner (la <= 4, lb = 0) against an auxiliary function (lc <= 4)."""
    out = []
    for la in range(lmax + 1):
        for lb in range(la + 1):
            for lc in range(lmax + 1):
                for ld in range(lc + 1):
                    out.append((la, lb, lc, ld))
    bras = [(la, lb) for la in range(3) for lb in range(la + 1)] + [(3, 0), (4, 0)]
    for la, lb in bras:
        for lc in range(5):
            if (la, lb, lc, 0) not in out:
                out.append((la, lb, lc, 0))
    return out


def render(lmax):
    """The text of eri_gen.cuh for classes up to lmax, and per-class counts
    of recursion temporaries."""
    parts = ["// Generated by gen_eri.py -- do not edit.  Obara-Saika VRR + HRR per class.",
             "#pragma once",
             "namespace hfg {",
             "template <int LA, int LB, int LC, int LD> struct EriClass;",
             "#define T(n) static_cast<T>(n)"]
    stats = []
    for la, lb, lc, ld in class_list(lmax):
        code, nv, nh = gen_class(la, lb, lc, ld)
        parts.append(code)
        stats.append((la, lb, lc, ld, nv, nh))
    parts.append("#undef T")
    parts.append("}  // namespace hfg")
    return "\n".join(parts) + "\n", stats


def main():
    lmax = int(sys.argv[1]) if len(sys.argv) > 1 else 2
    here = os.path.dirname(os.path.abspath(__file__))
    text, stats = render(lmax)
    with open(os.path.join(here, "eri_gen.cuh"), "w") as f:
        f.write(text)
    for s in stats:
        print("class (%d%d|%d%d): %d vrr temps, %d hrr temps" % s)


if __name__ == "__main__":
    main()
