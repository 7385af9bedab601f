"""Write the (H2O)16 cc-pVDZ J/K fixture (config1_jk.npz) from the oracle.

The synthetic water cluster (H2O)16 (seed 20261203, 48 atoms, 400 Cartesian
functions) in cc-pVDZ, one direct J/K build by the oracle's restatement of
hf-rs's shell engine and contract_jk (oracle/hf_oracle.cpp: Schwarz 1e-12,
McMurchie-Davidson integrals, 8-fold digestion).

The densities are the oracle's SAD guess P (hf-rs src/sad.rs:217-259) split
into two spin densities Pa = P/2 + D, Pb = P/2 - D with a seeded symmetric
D (0.02 x standard normal, symmetrised), so that every shell block of the
spin densities is non-zero.  One build with the two spin densities gives J
(from P), Ka and Kb; by linearity the closed-shell K of P is Ka + Kb.  The
matrices are stored as upper triangles (all are symmetric).

Run from the repository root (about 15-20 minutes on 8 cores):
    python tests/golden/make_config1.py
"""
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.join(ROOT, "hf-rs_b200"))

WATERS = 16
SEED = 20261203
SCHWARZ = 1e-12


def main():
    import oracle as O
    from hfgpu.clusters import water_cluster

    atoms = water_cluster(WATERS, seed=SEED)
    basis = O.build_basis(atoms, O.load_basis("cc-pvdz"))
    n = len(basis)
    S, _, _ = O.one_electron(basis, atoms)
    P = O.sad_density(atoms, basis, 0, S)
    rng = np.random.default_rng(SEED)
    R = rng.standard_normal((n, n)) * 0.02
    D = 0.5 * (R + R.T)
    Pa, Pb = 0.5 * P + D, 0.5 * P - D
    t0 = time.time()
    J, K = O.direct_jk(basis, P, [Pa, Pb], SCHWARZ)
    dt = time.time() - t0
    iu = np.triu_indices(n)
    np.savez_compressed(os.path.join(HERE, "config1_jk.npz"), waters=WATERS, seed=SEED, schwarz=SCHWARZ, n=n,
                        P=P[iu], D=D[iu], J=J[iu], Ka=K[0][iu], Kb=K[1][iu])
    print("config1_jk.npz: n = %d, oracle build %.0f s" % (n, dt))


if __name__ == "__main__":
    main()
