"""Write the SCF energies of the SPDF problem (spdf_scf.json) from the oracle.

The molecule and basis are those of hf-rs's SPDF integral fixture, as held
in spdf_eri.npz: He, Li, Be and B at the fixture's (bohr) positions, each
with one s, p, d and f shell of two primitives (80 Cartesian, 64 spherical
functions, 14 electrons, closed shell).  The oracle's RHF restatement (SAD
guess, CDIIS(8), hf-rs's convergence criteria at tol 1e-10, direct J/K from
the McMurchie-Davidson shell engine) runs in the Cartesian and in the real
spherical AO space.

Run from the repository root (about 6 minutes on 16 cores):
    python tests/golden/make_spdf_scf.py
"""
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))


def main():
    import oracle as O
    g = np.load(os.path.join(HERE, "spdf_eri.npz"))
    atoms = [(str(s), tuple(float(x) for x in p)) for s, p in zip(g["symbols"], g["geometry"])]
    ob = O.build_basis(atoms, O.parse_gaussian94(str(g["basis"])))
    out = {"tol": 1e-10}
    for name, sph in (("cartesian", False), ("spherical", True)):
        r = O.rhf(atoms, ob, tol=1e-10, spherical=sph, jk=O.JKDirect(ob))
        assert r["converged"]
        out[name] = {"energy": r["energy"], "iterations": r["iterations"]}
        print(name, r["energy"], r["iterations"], flush=True)
    with open(os.path.join(HERE, "spdf_scf.json"), "w") as f:
        json.dump(out, f, indent=1)


if __name__ == "__main__":
    main()
