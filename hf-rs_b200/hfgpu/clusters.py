"""Seeded synthetic water clusters (H2O)_n for the Fock-build workloads.

Monomer: the hf-rs test geometry of water in bohr, O (0, 0, 0.2217),
H (0, +-1.4309, -0.8867) (hf-rs tests/data/scf_reference.json "h2o").
Cluster: sites on a cubic lattice of 3.0 Angstrom spacing, k = ceil(n^(1/3))
sites per edge, filled x-fastest until n waters are placed; each water is
rotated about its oxygen by a Haar-uniform rotation (Shoemake's quaternion
from three uniforms) and its oxygen displaced by a uniform jitter in
[-0.2, 0.2] Angstrom per axis.  Angstrom -> bohr uses 1.8897261246257702
(hf-rs src/basis.rs:39).  One numpy PCG64 stream per cluster, seeded by
`seed` (default 20261203), so every cluster is reproducible.
"""
import math

import numpy as np

ANG_TO_BOHR = 1.8897261246257702
WATER = [("O", (0.0, 0.0, 0.2217)), ("H", (0.0, 1.4309, -0.8867)), ("H", (0.0, -1.4309, -0.8867))]
DEFAULT_SEED = 20261203


def _quat_rotation(u1, u2, u3):
    a = math.sqrt(1.0 - u1)
    b = math.sqrt(u1)
    q = (a * math.sin(2 * math.pi * u2), a * math.cos(2 * math.pi * u2),
         b * math.sin(2 * math.pi * u3), b * math.cos(2 * math.pi * u3))
    x, y, z, w = q
    return np.array([
        [1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)],
        [2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)],
        [2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)],
    ])


def water_cluster(n, seed=DEFAULT_SEED, spacing_ang=3.0, jitter_ang=0.2):
    """Atoms [(symbol, (x, y, z) bohr)] of a neutral closed-shell (H2O)_n."""
    if n < 1:
        raise ValueError("n must be >= 1")
    if n == 1:
        return [(s, tuple(p)) for s, p in WATER]
    rng = np.random.default_rng(seed)
    k = 1
    while k ** 3 < n:
        k += 1
    o = np.array(WATER[0][1])
    atoms = []
    for w in range(n):
        ix, iy, iz = w % k, (w // k) % k, w // (k * k)
        site = np.array([ix, iy, iz], dtype=np.float64) * spacing_ang * ANG_TO_BOHR
        u = rng.random(3)
        rot = _quat_rotation(*u)
        jit = (rng.random(3) * 2.0 - 1.0) * jitter_ang * ANG_TO_BOHR
        for s, p in WATER:
            r = rot @ (np.array(p) - o) + site + jit
            atoms.append((s, (float(r[0]), float(r[1]), float(r[2]))))
    for i in range(len(atoms)):
        for j in range(i):
            d = math.dist(atoms[i][1], atoms[j][1])
            if d < 1e-6:
                raise ValueError("coincident nuclei")
    return atoms
