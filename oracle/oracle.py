"""CPU oracle for the hf-rs Fock-build path.  TEST INFRASTRUCTURE ONLY.

Python side of the oracle: a restatement of hf-rs's basis construction,
spherical AO space, SCF drivers (RHF/UHF with CDIIS, SAD guess) and DF-RHF,
on top of the C++ integral restatement in hf_oracle.cpp (loaded through
ctypes).  Only tests/, __graft_entry__.smoke() and the cpu_baseline leg of
bench.py may import this module, and only as the checker; the product never
does.

Reference lines followed (paths relative to the hf-rs project root):
  src/basis.rs:107-132 (double_factorial, primitive_norm), :296-357
  (try_parse_gaussian94), :402-496 (build_basis, make_contracted_gaussian)
  src/ao.rs:14-27 (BasisKind), :58-67 (orthogonalizer), :94-217
  (real solid harmonics, spherical_transform)
  src/matrix.rs:107-110, :150-159, :162-191 (eigh phase convention), :329-346
  src/diis.rs:53-137 (CDIIS), :140-219 (UHF CDIIS), :532-580 (LU solve)
  src/scf.rs:207-218, :377-627 (RHF), :691-979 (UHF)
  src/sad.rs:24-259 (SAD guess)
  src/df.rs:16-28, :81-174 and src/hf_variants/ri_df_hf.rs:66-263 (DF-RHF)
"""
import ctypes
import math
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "liboracle.so")
BASIS_DIR = os.path.join(os.path.dirname(HERE), "hf-rs_b200", "hfgpu", "basis_data")
ANG_TO_BOHR = 1.8897261246257702  # src/basis.rs:39

SYMBOLS = ["H", "He", "Li", "Be", "B", "C", "N", "O", "F", "Ne", "Na", "Mg", "Al", "Si", "P", "S", "Cl", "Ar"]


def build_library():
    subprocess.check_call(["make", "-s", "-C", HERE])


_lib = None


class OrcBasis(ctypes.Structure):
    _fields_ = [
        ("n", ctypes.c_int),
        ("center", ctypes.POINTER(ctypes.c_double)),
        ("lxyz", ctypes.POINTER(ctypes.c_int)),
        ("atom", ctypes.POINTER(ctypes.c_int)),
        ("prim_off", ctypes.POINTER(ctypes.c_int)),
        ("exps", ctypes.POINTER(ctypes.c_double)),
        ("coefs", ctypes.POINTER(ctypes.c_double)),
    ]


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build_library()
        L = ctypes.CDLL(LIB_PATH)
        dp = ctypes.POINTER(ctypes.c_double)
        bp = ctypes.POINTER(OrcBasis)
        L.orc_boys_array.argtypes = [ctypes.c_int, ctypes.c_double, dp]
        L.orc_contracted_eri.restype = ctypes.c_double
        L.orc_contracted_eri.argtypes = [bp, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int]
        L.orc_contracted_eri_list.argtypes = [bp, bp, bp, bp, ctypes.c_long, ctypes.POINTER(ctypes.c_int), dp, ctypes.c_int]
        L.orc_shell_quartet.restype = ctypes.c_long
        L.orc_shell_quartet.argtypes = [bp, bp, bp, bp, dp]
        L.orc_shell_ranges.restype = ctypes.c_int
        L.orc_shell_ranges.argtypes = [bp, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int)]
        L.orc_schwarz.restype = ctypes.c_long
        L.orc_schwarz.argtypes = [bp, dp, ctypes.c_int]
        L.orc_eri_packed.restype = ctypes.c_int
        L.orc_eri_packed.argtypes = [bp, dp, ctypes.c_size_t, ctypes.c_int]
        L.orc_contract_jk.argtypes = [ctypes.c_int, dp, dp, ctypes.c_int, dp, dp, dp]
        L.orc_direct_jk.restype = ctypes.c_int
        L.orc_direct_jk.argtypes = [bp, dp, ctypes.c_int, dp, dp, dp, ctypes.c_double,
                                    ctypes.POINTER(ctypes.c_long), ctypes.c_long, ctypes.c_int]
        L.orc_one_electron.argtypes = [bp, ctypes.c_int, dp, dp, dp, dp, dp, ctypes.c_int]
        L.orc_df_metric.argtypes = [bp, dp, ctypes.c_int]
        L.orc_df_three.argtypes = [bp, bp, dp, ctypes.c_int]
        _lib = L
    return _lib


def _dp(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _ip(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_int))


def nthreads():
    return int(os.environ.get("ORACLE_THREADS", os.cpu_count() or 1))


# ------------------------------------------------------------------ basis --
def double_factorial(n):
    # src/basis.rs:107-121: (2n-1)!! with (-1)!! = 1
    if n <= 0:
        return 1.0
    r, k = 1.0, n
    while k > 0:
        r *= k
        k -= 2
    return r


def primitive_norm(alpha, l):
    # src/basis.rs:123-132
    lt = sum(l)
    pref = (2.0 * alpha / math.pi) ** 0.75
    num = (4.0 * alpha) ** lt
    den = double_factorial(2 * l[0] - 1) * double_factorial(2 * l[1] - 1) * double_factorial(2 * l[2] - 1)
    return pref * math.sqrt(num / den)


def parse_number(tok):
    return float(tok.replace("D", "E").replace("d", "E"))


SHELL_L = {"S": 0, "P": 1, "D": 2, "F": 3, "G": 4, "H": 5, "I": 6, "K": 7}


def parse_gaussian94(text):
    """src/basis.rs:296-357: element -> list of (type, exps, coefs, pcoefs)."""
    lines = [ln.split("!")[0].split("#")[0].strip() for ln in text.splitlines()]
    lines = [ln for ln in lines if ln]
    out, elem, i = {}, None, 0
    while i < len(lines):
        if lines[i] == "****":
            elem = None
            i += 1
            continue
        tok = lines[i].split()
        if elem is None:
            elem = tok[0].upper()
            out.setdefault(elem, [])
            i += 1
            continue
        st = tok[0].upper()
        n = int(tok[1])
        scale = parse_number(tok[2])
        exps, cols = [], None
        for row in range(n):
            i += 1
            vals = [parse_number(t) for t in lines[i].split()]
            if row == 0:
                cols = [[] for _ in range(len(vals) - 1)]
            exps.append(vals[0] * scale * scale)
            for c, v in zip(cols, vals[1:]):
                c.append(v)
        if st == "SP":
            for k in range(0, len(cols), 2):
                out[elem].append(("SP", exps, cols[k], cols[k + 1]))
        else:
            for c in cols:
                out[elem].append((st, exps, c, None))
        i += 1
    return out


def load_basis(name):
    fn = {"sto-3g": "sto-3g.gbs", "6-31g*": "6-31gstar.gbs", "6-31g": "6-31g.gbs", "cc-pvdz": "cc-pvdz.gbs",
          "def2-universal-jkfit": "def2-universal-jkfit.gbs", "def2-svp-ri": "def2-svp-ri.gbs"}[name.lower()]
    with open(os.path.join(BASIS_DIR, fn)) as f:
        return parse_gaussian94(f.read())


def cartesian_components(l):
    # src/basis.rs:430-445 (d order xx,yy,zz,xy,xz,yz) and cartesian_components_for_l
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


def make_cg(atom_index, center, l, exps, coefs):
    # src/basis.rs:455-496
    prims = [(e, c * primitive_norm(e, l)) for e, c in zip(exps, coefs)]
    so = 0.0
    for e1, c1 in prims:
        for e2, c2 in prims:
            p = e1 + e2
            sxyz = ((math.pi / p) ** 1.5
                    * (double_factorial(2 * l[0] - 1) / (2.0 * p) ** l[0])
                    * (double_factorial(2 * l[1] - 1) / (2.0 * p) ** l[1])
                    * (double_factorial(2 * l[2] - 1) / (2.0 * p) ** l[2]))
            so += c1 * c2 * sxyz
    nf = 1.0 / math.sqrt(so)
    return {"atom": atom_index, "center": tuple(center), "l": tuple(l),
            "exps": [e for e, _ in prims], "coefs": [c * nf for _, c in prims]}


def build_basis(atoms, bmap):
    """src/basis.rs:402-452.  atoms: list of (symbol, (x,y,z) bohr)."""
    basis = []
    for ai, (sym, pos) in enumerate(atoms):
        for st, exps, coefs, pcoefs in bmap[sym.upper()]:
            if st == "SP":
                basis.append(make_cg(ai, pos, (0, 0, 0), exps, coefs))
                for comp in cartesian_components(1):
                    basis.append(make_cg(ai, pos, comp, exps, pcoefs))
            else:
                for comp in cartesian_components(SHELL_L[st]):
                    basis.append(make_cg(ai, pos, comp, exps, coefs))
    return basis


class FlatBasis:
    """Keeps the numpy arrays alive behind an OrcBasis struct."""

    def __init__(self, basis):
        n = len(basis)
        self.n = n
        self.center = np.array([g["center"] for g in basis], dtype=np.float64).reshape(n, 3)
        self.lxyz = np.array([g["l"] for g in basis], dtype=np.int32).reshape(n, 3)
        self.atom = np.array([g["atom"] for g in basis], dtype=np.int32)
        off = [0]
        for g in basis:
            off.append(off[-1] + len(g["exps"]))
        self.prim_off = np.array(off, dtype=np.int32)
        self.exps = np.array([e for g in basis for e in g["exps"]], dtype=np.float64)
        self.coefs = np.array([c for g in basis for c in g["coefs"]], dtype=np.float64)
        self.s = OrcBasis(n, _dp(self.center), _ip(self.lxyz), _ip(self.atom), _ip(self.prim_off),
                          _dp(self.exps), _dp(self.coefs))

    def ref(self):
        return ctypes.byref(self.s)


# ------------------------------------------------------------ integrals ----
def boys_array(max_n, t):
    out = np.zeros(max_n + 1)
    lib().orc_boys_array(max_n, t, _dp(out))
    return out


def shell_ranges(basis):
    fb = FlatBasis(basis)
    st = np.zeros(len(basis), dtype=np.int32)
    ct = np.zeros(len(basis), dtype=np.int32)
    ns = lib().orc_shell_ranges(fb.ref(), _ip(st), _ip(ct))
    if ns < 0:
        raise ValueError("incomplete Cartesian shell")
    return [(int(st[i]), int(ct[i])) for i in range(ns)]


def shell_quartet(b0, b1, b2, b3):
    fbs = [FlatBasis(b) for b in (b0, b1, b2, b3)]
    out = np.zeros(len(b0) * len(b1) * len(b2) * len(b3))
    n = lib().orc_shell_quartet(fbs[0].ref(), fbs[1].ref(), fbs[2].ref(), fbs[3].ref(), _dp(out))
    if n < 0:
        raise ValueError("one shell per quartet slot is required")
    return out


def contracted_eri_list(b0, b1, b2, b3, idx):
    fbs = [FlatBasis(b) for b in (b0, b1, b2, b3)]
    idx = np.ascontiguousarray(idx, dtype=np.int32)
    out = np.zeros(len(idx))
    lib().orc_contracted_eri_list(fbs[0].ref(), fbs[1].ref(), fbs[2].ref(), fbs[3].ref(), len(idx), _ip(idx),
                                  _dp(out), nthreads())
    return out


def schwarz(basis):
    fb = FlatBasis(basis)
    ns = len(shell_ranges(basis))
    out = np.zeros(ns * (ns + 1) // 2)
    lib().orc_schwarz(fb.ref(), _dp(out), nthreads())
    return out


def eri_packed(basis):
    fb = FlatBasis(basis)
    n = len(basis)
    npair = n * (n + 1) // 2
    out = np.zeros(npair * (npair + 1) // 2)
    rc = lib().orc_eri_packed(fb.ref(), _dp(out), out.size, nthreads())
    if rc != 0:
        raise ValueError("eri_packed failed %d" % rc)
    return out


def contract_jk(eri, total, spins):
    n = total.shape[0]
    tot = np.ascontiguousarray(total, dtype=np.float64)
    sp = np.ascontiguousarray(np.stack(spins), dtype=np.float64)
    J = np.zeros((n, n))
    K = np.zeros((len(spins), n, n))
    lib().orc_contract_jk(n, _dp(np.ascontiguousarray(eri)), _dp(tot), len(spins), _dp(sp), _dp(J), _dp(K))
    return J, K


def direct_jk(basis, total, spins, thresh=1e-12, rows=None, fb=None):
    fb = fb or FlatBasis(basis)
    n = fb.n
    tot = np.ascontiguousarray(total, dtype=np.float64)
    sp = np.ascontiguousarray(np.stack(spins), dtype=np.float64)
    J = np.zeros((n, n))
    K = np.zeros((len(spins), n, n))
    if rows is not None:
        rows = np.ascontiguousarray(rows, dtype=np.int64)
        rp, nr = rows.ctypes.data_as(ctypes.POINTER(ctypes.c_long)), len(rows)
    else:
        rp, nr = None, 0
    rc = lib().orc_direct_jk(fb.ref(), _dp(tot), len(spins), _dp(sp), _dp(J), _dp(K), thresh, rp, nr, nthreads())
    if rc != 0:
        raise ValueError("direct_jk failed")
    return J, K


def one_electron(basis, atoms):
    fb = FlatBasis(basis)
    n = len(basis)
    pos = np.array([p for _, p in atoms], dtype=np.float64).reshape(-1, 3)
    chg = np.array([float(SYMBOLS.index(s.capitalize()) + 1) for s, _ in atoms])
    S, T, V = np.zeros((n, n)), np.zeros((n, n)), np.zeros((n, n))
    lib().orc_one_electron(fb.ref(), len(atoms), _dp(pos), _dp(chg), _dp(S), _dp(T), _dp(V), nthreads())
    return S, T, V


def df_metric(aux):
    fb = FlatBasis(aux)
    M = np.zeros((len(aux), len(aux)))
    lib().orc_df_metric(fb.ref(), _dp(M), nthreads())
    return M


def df_three(basis, aux):
    fb, fa = FlatBasis(basis), FlatBasis(aux)
    n = len(basis)
    out = np.zeros((len(aux), n * (n + 1) // 2))
    lib().orc_df_three(fb.ref(), fa.ref(), _dp(out), nthreads())
    return out


def nuclear_repulsion(atoms):
    # src/scf.rs:207-218
    e = 0.0
    for i in range(len(atoms)):
        for j in range(i + 1, len(atoms)):
            zi = SYMBOLS.index(atoms[i][0].capitalize()) + 1
            zj = SYMBOLS.index(atoms[j][0].capitalize()) + 1
            d = math.sqrt(sum((atoms[i][1][k] - atoms[j][1][k]) ** 2 for k in range(3)))
            e += zi * zj / d
    return e


# ----------------------------------------------------------- lin. algebra --
def eigh(a):
    """src/matrix.rs:162-191: ascending eigenvalues; each eigenvector's
    largest-|component| entry made positive (first maximum wins)."""
    w, v = np.linalg.eigh(a)
    order = np.argsort(w, kind="stable")
    w, v = w[order], v[:, order].copy()
    for c in range(v.shape[1]):
        k = int(np.argmax(np.abs(v[:, c])))
        if v[k, c] < 0:
            v[:, c] = -v[:, c]
    return w, v


def canonical_orthogonalizer(s, cutoff):
    # src/matrix.rs:329-346
    w, v = eigh(s)
    if w[0] < -cutoff:
        raise ValueError("overlap has negative eigenvalue")
    keep = [i for i in range(len(w)) if w[i] >= cutoff]
    return v[:, keep] / np.sqrt(w[keep])


def _fact(n):
    return float(math.factorial(n))


def solid_harmonic(l, m):
    # src/ao.rs:94-131: real solid harmonic as {powers: coefficient}
    am = abs(m)
    out = {}
    norm = math.sqrt(_fact(l - am) / _fact(l + am)) * (1.0 if am == 0 else math.sqrt(2.0))
    for k in range((l - am) // 2 + 1):
        coef = (-1.0) ** k * _fact(2 * l - 2 * k) / (2.0 ** l * _fact(k) * _fact(l - k) * _fact(l - am - 2 * k))
        for y in range(am + 1):
            r = y % 4
            if (m < 0 and r == 1) or (m >= 0 and r == 0):
                phase = 1.0
            elif (m < 0 and r == 3) or (m >= 0 and r == 2):
                phase = -1.0
            else:
                continue
            binom = _fact(am) / (_fact(y) * _fact(am - y))
            for xx in range(k + 1):
                for yy in range(k - xx + 1):
                    zz = k - xx - yy
                    powers = (am - y + 2 * xx, y + 2 * yy, l - am - 2 * k + 2 * zz)
                    mult = _fact(k) / (_fact(xx) * _fact(yy) * _fact(zz))
                    out[powers] = out.get(powers, 0.0) + norm * coef * binom * phase * mult
    return out


def spherical_transform(basis, S):
    """src/ao.rs:167-217: Cartesian -> real spherical (PySCF order)."""
    shells = shell_ranges(basis)
    nsph = sum(2 * sum(basis[s]["l"]) + 1 for s, _ in shells)
    T = np.zeros((len(basis), nsph))
    col = 0
    for start, cnt in shells:
        l = sum(basis[start]["l"])
        rng = range(start, start + cnt)
        if l <= 1:
            for r in rng:
                T[r, col] = 1.0
                col += 1
            continue
        ov = S[start:start + cnt, start:start + cnt]
        for m in range(-l, l + 1):
            p = solid_harmonic(l, m)
            coef = []
            for r in rng:
                lx = basis[r]["l"]
                w = math.sqrt(double_factorial(2 * lx[0] - 1) * double_factorial(2 * lx[1] - 1)
                              * double_factorial(2 * lx[2] - 1))
                coef.append(p.get(tuple(lx), 0.0) * w)
            coef = np.array(coef)
            norm = float(coef @ ov @ coef)
            T[start:start + cnt, col] = coef / math.sqrt(norm)
            col += 1
    return T


def orthogonalizer(S, cart_to_ao):
    # src/ao.rs:58-67
    s = cart_to_ao.T @ S @ cart_to_ao
    return cart_to_ao @ canonical_orthogonalizer(s, 1e-8)


def solve_linear_system(a, b):
    """src/diis.rs:532-580: Gaussian elimination with partial pivoting;
    None when a pivot falls below 1e-28."""
    n = a.shape[0]
    m = a.astype(np.float64).copy()
    x = np.array(b, dtype=np.float64)
    for i in range(n):
        # first maximum wins (strict >), as the reference loop does
        best, mr = abs(m[i, i]), i
        for k in range(i + 1, n):
            if abs(m[k, i]) > best:
                best, mr = abs(m[k, i]), k
        if best < 1e-28:
            return None
        if mr != i:
            m[[i, mr]] = m[[mr, i]]
            x[[i, mr]] = x[[mr, i]]
        d = m[i, i]
        for j in range(i + 1, n):
            f = m[j, i] / d
            m[j, i:] -= f * m[i, i:]
            x[j] -= f * x[i]
    out = np.zeros(n)
    for i in range(n - 1, -1, -1):
        s = x[i] - m[i, i + 1:] @ out[i + 1:]
        out[i] = s / m[i, i]
    return out


class Cdiis:
    """src/diis.rs:72-137 (and the joint UHF form :140-219 when two spins)."""

    def __init__(self, size=8):
        self.size = max(size, 2)
        self.focks, self.errors = [], []

    def push(self, focks, errors):
        if len(self.focks) >= self.size:
            self.focks.pop(0)
            self.errors.pop(0)
        self.focks.append([f.copy() for f in focks])
        self.errors.append([e.copy() for e in errors])

    def extrapolate(self):
        m = len(self.errors)
        if m < 2:
            return None
        B = np.zeros((m + 1, m + 1))
        for i in range(m):
            for j in range(i + 1):
                d = sum(float(np.sum(a * b)) for a, b in zip(self.errors[i], self.errors[j]))
                B[i, j] = B[j, i] = d
            B[i, m] = B[m, i] = -1.0
        rhs = np.zeros(m + 1)
        rhs[m] = -1.0
        c = solve_linear_system(B, rhs)
        if c is None:
            return None
        return [sum(c[i] * self.focks[i][s] for i in range(m)) for s in range(len(self.focks[0]))]


def diis_error(F, P, S):
    # src/diis.rs:53-57
    return F @ P @ S - S @ P @ F


def occupied_density(C, nocc, scale):
    co = C[:, :nocc]
    return scale * (co @ co.T)


# ------------------------------------------------------------------ SAD ----
def _occupations(eps, nel):
    # src/sad.rs:24-44
    occ = np.zeros(len(eps))
    left, i = nel, 0
    while i < len(eps) and left > 1e-12:
        end = i + 1
        while end < len(eps) and abs(eps[end] - eps[i]) < 1e-6:
            end += 1
        pop = min(left, 2.0 * (end - i))
        occ[i:end] = pop / (end - i)
        left -= pop
        i = end
    return occ


def _frac_density(C, occ):
    w = C * np.sqrt(occ)[None, :]
    return w @ w.T


_sad_cache = {}


def atomic_fractional_hf(sym, local_basis):
    """src/sad.rs:56-158: spin-averaged fractional-occupation atomic RHF."""
    key = (sym, tuple((tuple(g["l"]), tuple(g["exps"]), tuple(g["coefs"])) for g in local_basis))
    if key in _sad_cache:
        return _sad_cache[key]
    basis = [dict(g, center=(0.0, 0.0, 0.0), atom=0) for g in local_basis]
    atoms = [(sym, (0.0, 0.0, 0.0))]
    S, T, V = one_electron(basis, atoms)
    H = T + V
    X = canonical_orthogonalizer(S, 1e-8)
    Z = float(SYMBOLS.index(sym.capitalize()) + 1)
    eri = eri_packed(basis)

    def fock(P):
        if abs(Z - 1.0) < 1e-12:
            return H.copy()
        J, K = contract_jk(eri, P, [P])
        return H + J - 0.5 * K[0]

    eps, cp = eigh(X.T @ H @ X)
    D = _frac_density(X @ cp, _occupations(eps, Z))
    prev = math.inf
    diis = Cdiis(8)
    for it in range(1, 201):
        F = fock(D)
        e = 0.5 * float(np.sum(D * (H + F)))
        eps, cp = eigh(X.T @ F @ X)
        nxt = _frac_density(X @ cp, _occupations(eps, Z))
        err = diis_error(F, D, S)
        if abs(e - prev) < 1e-11 and rmsd(D, nxt) < 1e-9 and np.max(np.abs(err)) < 1e-8:
            _sad_cache[key] = nxt
            return nxt
        prev = e
        diis.push([F], [err])
        ext = diis.extrapolate()
        fuse = ext[0] if ext is not None else F
        eps, cp = eigh(X.T @ fuse @ X)
        nxt = _frac_density(X @ cp, _occupations(eps, Z))
        D = 0.5 * D + 0.5 * nxt if it <= 5 else nxt
    raise RuntimeError("fractional atomic HF did not converge for " + sym)


def sad_density(atoms, basis, charge, S):
    """src/sad.rs:217-259."""
    n = len(basis)
    target = sum(SYMBOLS.index(s.capitalize()) + 1 for s, _ in atoms) - charge
    D = np.zeros((n, n))
    for a, (sym, _) in enumerate(atoms):
        idx = [i for i, g in enumerate(basis) if g["atom"] == a]
        Da = atomic_fractional_hf(sym, [basis[i] for i in idx])
        D[np.ix_(idx, idx)] = Da
    el = float(np.sum(D * S))
    return D * (target / el)


def rmsd(a, b):
    # src/matrix.rs:150-159
    return math.sqrt(float(np.sum((a - b) ** 2)) / a.size)


# ------------------------------------------------------------------- SCF ---
def convergence_from_tol(tol):
    # src/scf.rs:393-399
    return tol, max(math.sqrt(tol) * 1e-2, 1e-11), min(max(math.sqrt(tol) * 0.1, 1e-12), 1e-10)


class JKPacked:
    """Conventional J/K (the reference's stored-ERI path)."""

    def __init__(self, basis):
        self.eri = eri_packed(basis)

    def __call__(self, total, spins):
        return contract_jk(self.eri, total, spins)


class JKDirect:
    """Same integrals and digestion as JKPacked, without storing the tensor."""

    def __init__(self, basis, thresh=1e-12):
        self.fb = FlatBasis(basis)
        self.basis = basis
        self.thresh = thresh

    def __call__(self, total, spins):
        return direct_jk(self.basis, total, spins, self.thresh, fb=self.fb)


def rhf(atoms, basis, charge=0, max_iter=100, tol=1e-10, spherical=False, jk=None, guess="sad",
        verbose=False):
    """src/scf.rs:410-627 with ConvAlgo::Cdiis."""
    e_tol, r_tol, d_tol = convergence_from_tol(tol)
    n = len(basis)
    nel = sum(SYMBOLS.index(s.capitalize()) + 1 for s, _ in atoms) - charge
    nocc = nel // 2
    e_nuc = nuclear_repulsion(atoms)
    S, T, V = one_electron(basis, atoms)
    H = T + V
    cart_to_ao = spherical_transform(basis, S) if spherical else np.eye(n)
    X = orthogonalizer(S, cart_to_ao)
    jk = jk or JKPacked(basis)

    def fock(P):
        J, K = jk(P, [P])
        return H + J - 0.5 * K[0]

    if guess == "sad":
        P = sad_density(atoms, basis, charge, S)
        F0 = fock(P)
        _, cp = eigh(X.T @ F0 @ X)
        C = X @ cp
    else:
        _, cp = eigh(X.T @ H @ X)
        C = X @ cp
        P = occupied_density(C, nocc, 2.0)
    prev_e, converged = 0.0, False
    diis = Cdiis(8)
    prevP = P.copy()
    it = 0
    history = []
    for it in range(1, max_iter + 1):
        F = fock(P)
        e_tot = 0.5 * float(np.sum(P * (H + F))) + e_nuc
        de = abs(e_tot - prev_e)
        prev_e = e_tot
        err = diis_error(F, P, S)
        if X.shape[1] < n:
            err = X.T @ err @ X
        en = float(np.max(np.abs(err)))
        history.append(e_tot)
        if verbose:
            print(it, e_tot, de, en)
        if it > 1 and de < e_tol and en < r_tol and rmsd(P, prevP) < d_tol:
            converged = True
            break
        prevP = P.copy()
        diis.push([F], [err])
        ext = diis.extrapolate()
        fuse = ext[0] if ext is not None else F
        _, cp = eigh(X.T @ fuse @ X)
        C = X @ cp
        P = occupied_density(C, nocc, 2.0)
    if not converged:
        F = fock(P)
    eps, cp = eigh(X.T @ F @ X)
    C = X @ cp
    P = occupied_density(C, nocc, 2.0)
    F = fock(P)
    e_el = 0.5 * float(np.sum(P * (H + F)))
    return {"energy": e_el + e_nuc, "electronic": e_el, "nuclear": e_nuc, "eps": eps, "C": C, "P": P, "F": F,
            "S": S, "H": H, "X": X, "iterations": it, "converged": converged, "history": history}


def uhf(atoms, basis, charge=0, multiplicity=1, max_iter=100, tol=1e-10, spherical=False, jk=None):
    """src/scf.rs:691-979 (no broken-symmetry start)."""
    e_tol, r_tol, d_tol = convergence_from_tol(tol)
    n = len(basis)
    nel = sum(SYMBOLS.index(s.capitalize()) + 1 for s, _ in atoms) - charge
    two_s = multiplicity - 1
    na, nb = (nel + two_s) // 2, (nel - two_s) // 2
    e_nuc = nuclear_repulsion(atoms)
    S, T, V = one_electron(basis, atoms)
    H = T + V
    cart_to_ao = spherical_transform(basis, S) if spherical else np.eye(n)
    X = orthogonalizer(S, cart_to_ao)
    nmo = X.shape[1]
    jk = jk or JKPacked(basis)

    def focks(Pa, Pb):
        J, K = jk(Pa + Pb, [Pa, Pb])
        return H + J - K[0], H + J - K[1]

    sad = sad_density(atoms, basis, charge, S)
    Jg, Kg = jk(sad, [sad])
    gF = H + Jg - 0.5 * Kg[0]
    _, cp = eigh(X.T @ gF @ X)
    Ca = X @ cp
    Cb = Ca.copy()
    Pa, Pb = occupied_density(Ca, na, 1.0), occupied_density(Cb, nb, 1.0)
    prev_e, converged = 0.0, False
    diis = Cdiis(8)
    pa_prev, pb_prev = Pa.copy(), Pb.copy()
    it = 0
    for it in range(1, max_iter + 1):
        Fa, Fb = focks(Pa, Pb)
        e_tot = 0.5 * float(np.sum((Pa + Pb) * H + Pa * Fa + Pb * Fb)) + e_nuc
        de = abs(e_tot - prev_e)
        prev_e = e_tot
        ea, eb = diis_error(Fa, Pa, S), diis_error(Fb, Pb, S)
        if nmo < n:
            ea, eb = X.T @ ea @ X, X.T @ eb @ X
        en = max(float(np.max(np.abs(ea))), float(np.max(np.abs(eb))))
        if it > 1 and de < e_tol and en < r_tol and max(rmsd(Pa, pa_prev), rmsd(Pb, pb_prev)) < d_tol:
            converged = True
            break
        pa_prev, pb_prev = Pa.copy(), Pb.copy()
        diis.push([Fa, Fb], [ea, eb])
        ext = diis.extrapolate()
        fa_use, fb_use = (ext if ext is not None else (Fa, Fb))
        _, ca = eigh(X.T @ fa_use @ X)
        _, cb = eigh(X.T @ fb_use @ X)
        Ca, Cb = X @ ca, X @ cb
        na_new, nb_new = occupied_density(Ca, na, 1.0), occupied_density(Cb, nb, 1.0)
        if it <= 2:
            Pa, Pb = 0.7 * na_new + 0.3 * Pa, 0.7 * nb_new + 0.3 * Pb
        else:
            Pa, Pb = na_new, nb_new
    if not converged:
        Fa, Fb = focks(Pa, Pb)
    epa, ca = eigh(X.T @ Fa @ X)
    epb, cb = eigh(X.T @ Fb @ X)
    Ca, Cb = X @ ca, X @ cb
    Pa, Pb = occupied_density(Ca, na, 1.0), occupied_density(Cb, nb, 1.0)
    Fa, Fb = focks(Pa, Pb)
    e_el = 0.5 * float(np.sum((Pa + Pb) * H + Pa * Fa + Pb * Fb))
    mo = Ca.T @ S @ Cb
    s2 = (two_s / 2.0) * (two_s / 2.0 + 1.0) + nb - float(np.sum(mo[:na, :nb] ** 2))
    return {"energy": e_el + e_nuc, "Pa": Pa, "Pb": Pb, "Fa": Fa, "Fb": Fb, "s2": s2, "iterations": it,
            "converged": converged, "S": S, "H": H, "X": X}


# -------------------------------------------------------------------- DF ---
def df_tensor(basis, aux, cutoff=1e-10):
    """src/df.rs:16-28, :81-127 (Cartesian metric space): B = X^T (P|mn)."""
    M = df_metric(aux)
    Xm = canonical_orthogonalizer(M, cutoff)
    return Xm.T @ df_three(basis, aux)


def unpack_pairs(Bq, n):
    """Packed compound_index columns -> n x n symmetric matrices, per row."""
    out = np.zeros((Bq.shape[0], n, n))
    ii, jj = np.tril_indices(n)
    idx = ii * (ii + 1) // 2 + jj
    out[:, ii, jj] = Bq[:, idx]
    out[:, jj, ii] = Bq[:, idx]
    return out


def df_jk(B, Cocc, n):
    """src/df.rs:133-174 (coulomb_exchange_rhf)."""
    Bm = unpack_pairs(B, n)
    A = np.einsum("qpr,ri->qpi", Bm, Cocc)
    charge = 2.0 * np.einsum("qpi,pi->q", A, Cocc)
    J = np.einsum("q,qpr->pr", charge, Bm)
    K = 2.0 * np.einsum("qpi,qri->pr", A, A)
    return J, K


def df_rhf(atoms, basis, aux, charge=0, max_iter=100, e_tol=1e-12, r_tol=1e-10, d_tol=1e-10, cutoff=1e-10,
           spherical=False):
    """src/hf_variants/ri_df_hf.rs:122-263 (run_df_hf_with_aux ->
    run_factorized_rhf)."""
    return factorized_rhf(atoms, basis, df_tensor(basis, aux, cutoff), charge, max_iter, e_tol, r_tol, d_tol,
                          spherical)


def pivoted_cholesky(basis, threshold, budget=512 * 1024 * 1024):
    """src/cholesky.rs:42-190: pivoted Cholesky vectors L (rank x n_pair, packed
    compound_index columns) of the ERI supermatrix, the pivots and the
    largest residual diagonal.  Columns of a pivot's shell pair come from
    complete shell quartets with Q_ab Q_cd > 1e-15; the largest residual
    diagonal is the pivot, ties within 1e-12 (relative) going to the smallest
    packed index."""
    n = len(basis)
    shells = shell_ranges(basis)
    ns = len(shells)
    npair = n * (n + 1) // 2
    shell_of = np.zeros(n, dtype=int)
    for s, (st, ct) in enumerate(shells):
        shell_of[st:st + ct] = s
    sl = [basis[st:st + ct] for st, ct in shells]
    sp_index = lambda a, b: a * (a + 1) // 2 + b
    diag = np.zeros(npair)
    for a in range(ns):
        for b in range(a + 1):
            blk = shell_quartet(sl[a], sl[b], sl[a], sl[b])
            na, nb = shells[a][1], shells[b][1]
            for i in range(na):
                for j in range(nb):
                    p, q = shells[a][0] + i, shells[b][0] + j
                    if p < q:
                        continue
                    ij = i * nb + j
                    diag[p * (p + 1) // 2 + q] = blk[ij * na * nb + ij]
    scale = max(float(diag.max()), 1.0)
    if np.any(diag < -1e-12 * scale):
        raise ValueError("negative ERI diagonal")
    schw = np.zeros(ns * (ns + 1) // 2)
    for p in range(n):
        for q in range(p + 1):
            k = sp_index(shell_of[p], shell_of[q])
            schw[k] = max(schw[k], math.sqrt(max(diag[p * (p + 1) // 2 + q], 0.0)))
    pairs = [(a, b) for a in range(ns) for b in range(a + 1)]

    def columns(spi):
        r, s_ = pairs[spi]
        cols = {}
        for pq, (a, b) in enumerate(pairs):
            if not schw[pq] * schw[spi] > 1e-15:
                continue
            blk = shell_quartet(sl[a], sl[b], sl[r], sl[s_])
            na, nb, nr, nss = shells[a][1], shells[b][1], shells[r][1], shells[s_][1]
            for k in range(nr):
                for l in range(nss):
                    rr, ss = shells[r][0] + k, shells[s_][0] + l
                    if rr < ss:
                        continue
                    col = cols.setdefault(rr * (rr + 1) // 2 + ss, np.zeros(npair))
                    for i in range(na):
                        for j in range(nb):
                            p, q = shells[a][0] + i, shells[b][0] + j
                            if p >= q:
                                col[p * (p + 1) // 2 + q] = blk[((i * nb + j) * nr + k) * nss + l]
        return cols

    factors, pivots, cache = [], [], (None, None)
    while True:
        largest = float(diag.max())
        pivot = int(np.nonzero(diag >= largest - 1e-12 * abs(largest))[0][0])
        maximum = float(diag[pivot])
        if maximum <= threshold or len(factors) == npair:
            max_res = max(maximum, 0.0)
            break
        if 8 * npair * (len(factors) + 2) > budget:
            raise ValueError("factor storage exceeds the memory budget")
        p = int((math.isqrt(8 * pivot + 1) - 1) // 2)
        q = pivot - p * (p + 1) // 2
        spi = sp_index(max(shell_of[p], shell_of[q]), min(shell_of[p], shell_of[q]))
        if cache[0] != spi:
            cache = (spi, columns(spi))
        col = cache[1].get(pivot, np.zeros(npair))
        root = math.sqrt(maximum)
        L = np.array(factors) if factors else np.zeros((0, npair))
        row = (col - (L[:, pivot] @ L if len(factors) else 0.0)) / root
        row[pivot] = root
        diag = diag - row * row
        if np.any(diag < -1e-10 * scale):
            raise ValueError("nonpositive residual Coulomb diagonal")
        diag = np.maximum(diag, 0.0)
        factors.append(row)
        pivots.append(pivot)
    if not factors:
        raise ValueError("threshold exceeds every ERI diagonal")
    return np.array(factors), pivots, max_res


def factorized_rhf(atoms, basis, B, charge=0, max_iter=100, e_tol=1e-12, r_tol=1e-10, d_tol=1e-10, spherical=False):
    """src/hf_variants/ri_df_hf.rs:160-263 (run_factorized_rhf) on a given
    factor B (DF or Cholesky vectors)."""
    n = len(basis)
    nel = sum(SYMBOLS.index(s.capitalize()) + 1 for s, _ in atoms) - charge
    no = nel // 2
    S, T, V = one_electron(basis, atoms)
    H = T + V
    cart_to_ao = spherical_transform(basis, S) if spherical else np.eye(n)
    X = orthogonalizer(S, cart_to_ao)
    enuc = nuclear_repulsion(atoms)

    def diag(F):
        eps, c = eigh(X.T @ F @ X)
        return eps, X @ c

    def fock(co):
        J, K = df_jk(B, co, n)
        return H + J - 0.5 * K, J, K

    _, C = diag(H)
    co = C[:, :no]
    P = 2.0 * co @ co.T
    diis = Cdiis(8)
    last = math.inf
    for it in range(1, max_iter + 1):
        F, _, _ = fock(co)
        e = 0.5 * float(np.sum(P * (H + F))) + enuc
        err = X.T @ diis_error(F, P, S) @ X
        res = float(np.max(np.abs(err)))
        eps, nc = diag(F)
        nco = nc[:, :no]
        nP = 2.0 * nco @ nco.T
        dchg = float(np.max(np.abs(nP - P)))
        if abs(e - last) <= e_tol and res <= r_tol and dchg <= d_tol:
            Ff, J, K = fock(nco)
            ef = 0.5 * float(np.sum(nP * (H + Ff))) + enuc
            return {"energy": ef, "P": nP, "F": Ff, "J": J, "K": K, "eps": eps, "iterations": it,
                    "converged": True, "n_aux": B.shape[0], "B": B}
        last = e
        diis.push([F], [err])
        ext = diis.extrapolate() if it >= 2 else None
        fuse = ext[0] if ext is not None else F
        _, C = diag(fuse)
        co = C[:, :no]
        P = 2.0 * co @ co.T
    raise RuntimeError("factorized RHF did not converge")


# --------------------------------------------------------- water clusters --
WATER_BOHR = [("O", (0.0, 0.0, 0.2217)), ("H", (0.0, 1.4309, -0.8867)), ("H", (0.0, -1.4309, -0.8867))]
