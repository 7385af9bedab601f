"""Basis input for libhfg: Gaussian-94 parsing and Cartesian function lists.

Produces, for a molecule, the flat Cartesian-function arrays the C ABI takes
(hfg_basis in include/hfg.h) with the same content as hf-rs's
build_basis (src/basis.rs:402-452): one entry per Cartesian component in
hf-rs order (s; x,y,z; xx,yy,zz,xy,xz,yz; then lx, ly descending), each with
its primitives' coefficients fully normalised -- contraction coefficient x
primitive norm (2a/pi)^(3/4) sqrt((4a)^L / prod(2l_i-1)!!) x the shell's
self-overlap normalisation (src/basis.rs:123-132, 455-496).
"""
import math
import os

import numpy as np

DATA = os.path.join(os.path.dirname(os.path.abspath(__file__)), "basis_data")
SYMBOLS = ["H", "He", "Li", "Be", "B", "C", "N", "O", "F", "Ne", "Na", "Mg", "Al", "Si", "P", "S", "Cl", "Ar"]
SHELL_L = {"S": 0, "P": 1, "D": 2, "F": 3, "G": 4, "H": 5, "I": 6, "K": 7}
FILES = {"sto-3g": "sto-3g.gbs", "6-31g*": "6-31gstar.gbs", "6-31g": "6-31g.gbs", "cc-pvdz": "cc-pvdz.gbs",
         "def2-universal-jkfit": "def2-universal-jkfit.gbs", "def2-svp-ri": "def2-svp-ri.gbs"}


def atomic_number(sym):
    return SYMBOLS.index(sym.capitalize()) + 1


def read_gaussian94(text):
    """{ELEMENT: [(l or 'SP', exponents, coefficients, p_coefficients)]}."""
    rows = []
    for ln in text.splitlines():
        ln = ln.split("!")[0].split("#")[0].strip()
        if ln:
            rows.append(ln)
    out, elem, i = {}, None, 0

    def num(t):
        return float(t.replace("D", "E").replace("d", "E"))

    while i < len(rows):
        if rows[i] == "****":
            elem, i = None, i + 1
            continue
        tok = rows[i].split()
        if elem is None:
            elem = tok[0].upper()
            out.setdefault(elem, [])
            i += 1
            continue
        kind, nprim, scale = tok[0].upper(), int(tok[1]), num(tok[2])
        block = np.array([[num(t) for t in rows[i + 1 + r].split()] for r in range(nprim)])
        exps = block[:, 0] * scale * scale
        cols = block[:, 1:].T
        if kind == "SP":
            for k in range(0, len(cols), 2):
                out[elem].append(("SP", exps, cols[k], cols[k + 1]))
        else:
            for c in cols:
                out[elem].append((SHELL_L[kind], exps, c, None))
        i += 1 + nprim
    return out


def builtin(name):
    with open(os.path.join(DATA, FILES[name.lower()])) as f:
        return read_gaussian94(f.read())


def cartesian_components(l):
    if l == 2:
        return [(2, 0, 0), (0, 2, 0), (0, 0, 2), (1, 1, 0), (1, 0, 1), (0, 1, 1)]
    return [(lx, ly, l - lx - ly) for lx in range(l, -1, -1) for ly in range(l - lx, -1, -1)]


def _dfact(n):
    r = 1.0
    while n > 0:
        r *= n
        n -= 2
    return r


def _component_coefs(l, lxyz, exps, coefs):
    norm = (2.0 * exps / math.pi) ** 0.75 * np.sqrt((4.0 * exps) ** l / np.prod([_dfact(2 * x - 1) for x in lxyz]))
    c = coefs * norm
    p = exps[:, None] + exps[None, :]
    sxyz = (math.pi / p) ** 1.5
    for x in lxyz:
        sxyz = sxyz * (_dfact(2 * x - 1) / (2.0 * p) ** x)
    so = float(np.sum(c[:, None] * c[None, :] * sxyz))
    return c / math.sqrt(so)


class CartesianBasis:
    """Flat Cartesian function list of a molecule (hfg_basis content)."""

    def __init__(self, atoms, basis_map):
        centers, lxyz, atom, off, exps, coefs, shells = [], [], [], [0], [], [], []
        for ai, (sym, pos) in enumerate(atoms):
            for kind, e, c, pc in basis_map[sym.upper()]:
                parts = [(0, c), (1, pc)] if kind == "SP" else [(kind, c)]
                for l, cc in parts:
                    shells.append((len(centers), l, ai))
                    for comp in cartesian_components(l):
                        centers.append(pos)
                        lxyz.append(comp)
                        atom.append(ai)
                        exps.extend(e)
                        coefs.extend(_component_coefs(l, comp, np.asarray(e), np.asarray(cc)))
                        off.append(off[-1] + len(e))
        self.atoms = atoms
        self.n = len(centers)
        self.center = np.ascontiguousarray(centers, dtype=np.float64).reshape(self.n, 3)
        self.lxyz = np.ascontiguousarray(lxyz, dtype=np.int32).reshape(self.n, 3)
        self.atom = np.ascontiguousarray(atom, dtype=np.int32)
        self.prim_off = np.ascontiguousarray(off, dtype=np.int32)
        self.exps = np.ascontiguousarray(exps, dtype=np.float64)
        self.coefs = np.ascontiguousarray(coefs, dtype=np.float64)
        self.shells = shells  # (first function, l, atom)

    @classmethod
    def build(cls, atoms, name):
        return cls(atoms, builtin(name))

    def nuclear_charges(self):
        return np.array([float(atomic_number(s)) for s, _ in self.atoms])

    def positions(self):
        return np.array([p for _, p in self.atoms], dtype=np.float64).reshape(-1, 3)

    def n_electrons(self, charge=0):
        return int(round(self.nuclear_charges().sum())) - charge
