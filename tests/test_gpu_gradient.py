"""The two-electron part of the analytic nuclear gradient (hfg_eri_gradient).

For a density held fixed in the AO basis, E2(R) = 1/2 tr(P J) - 1/4 tr(P K)
(closed shell) or 1/2 tr(P J) - 1/2 sum_s tr(P_s K_s) (two spin densities)
depends on the nuclei only through the integrals, so its derivative is the
ERI-derivative contraction that hf-rs's contract_eri_derivatives makes
(src/gradient.rs:33-69).  The analytic values are checked against
fourth-order central differences of E2 from J/K builds at displaced
geometries, and against translational invariance.
"""
import numpy as np
import pytest

from hfgpu import CartesianBasis, Context, HfgError
from hfgpu.clusters import water_cluster

pytestmark = pytest.mark.gpu


def e2(atoms, name, P, spins):
    ctx = Context(CartesianBasis.build(atoms, name))
    J, K = ctx.jk(P, spins)
    ctx.close()
    if spins is None:
        return 0.5 * np.sum(P * J) - 0.25 * np.sum(P * K[0])
    return 0.5 * np.sum(P * J) - 0.5 * sum(np.sum(s * k) for s, k in zip(spins, K))


def shifted(atoms, at, ax, d):
    out = [(s, list(p)) for s, p in atoms]
    out[at][1][ax] += d
    return [(s, tuple(p)) for s, p in out]


@pytest.mark.parametrize("name,nw,open_shell", [("cc-pvdz", 2, False), ("6-31g*", 2, True), ("sto-3g", 3, False)])
def test_eri_gradient_matches_finite_differences(name, nw, open_shell):
    atoms = water_cluster(nw)
    ctx = Context(CartesianBasis.build(atoms, name))
    P = ctx.scf(spherical=False, tol=1e-8, max_iter=6, want=("P",))["P"][0]
    spins = None
    if open_shell:
        rng = np.random.default_rng(4)
        D = rng.standard_normal(P.shape) * 0.01
        D = D + D.T
        spins = [0.5 * P + D, 0.5 * P - D]
    g = ctx.eri_gradient(P, spins)
    ctx.close()
    assert g.shape == (len(atoms), 3)
    scale = np.max(np.abs(g))
    # translational invariance
    assert np.max(np.abs(g.sum(axis=0))) < 1e-9 * max(1.0, scale)
    h = 1e-3
    for at in (0, 1, len(atoms) - 1):
        for ax in range(3):
            f = {k: e2(shifted(atoms, at, ax, k * h), name, P, spins) for k in (-2, -1, 1, 2)}
            fd = (8.0 * (f[1] - f[-1]) - (f[2] - f[-2])) / (12.0 * h)
            assert abs(fd - g[at, ax]) < 2e-7 * max(1.0, scale), (at, ax, fd, g[at, ax])


def test_eri_gradient_rejects_too_few_atoms():
    from hfgpu.lib import _dp
    ctx = Context(CartesianBasis.build(water_cluster(1), "sto-3g"))
    P = np.eye(ctx.n)
    g = np.zeros((1, 3))
    rc = ctx.lib.hfg_eri_gradient(ctx.h, 1e-12, 1, _dp(P), _dp(P), 1, _dp(g))
    assert rc != 0 and b"natom" in ctx.lib.hfg_last_error(ctx.h)
    ctx.close()


def scf_energy(atoms, name, spherical, charge=0, multiplicity=1, uhf=False):
    ctx = Context(CartesianBasis.build(atoms, name))
    r = ctx.scf(charge=charge, multiplicity=multiplicity, uhf=uhf, spherical=spherical, tol=1e-11, want=())
    ctx.close()
    assert r["converged"]
    return r["energy"]


@pytest.mark.parametrize("name,nw,spherical,uhf", [("cc-pvdz", 1, True, False), ("6-31g*", 2, False, False),
                                                   ("6-31g*", 1, False, True)])
def test_full_gradient_matches_finite_differences_of_the_scf_energy(name, nw, spherical, uhf):
    # hfg_gradient (nuclear repulsion + one-electron + two-electron terms) of
    # a converged SCF against fourth-order central differences of the SCF
    # energy itself: RHF in the spherical and Cartesian spaces, and the UHF
    # doublet cation
    atoms = water_cluster(nw)
    charge, mult = (1, 2) if uhf else (0, 1)
    ctx = Context(CartesianBasis.build(atoms, name))
    r, g = ctx.scf_gradient(charge=charge, multiplicity=mult, uhf=uhf, spherical=spherical, tol=1e-11)
    ctx.close()
    assert r["converged"] and g.shape == (len(atoms), 3)
    assert np.max(np.abs(g.sum(axis=0))) < 1e-8
    h = 2e-3
    for at, ax in ((0, 0), (0, 2), (1, 1), (len(atoms) - 1, 0)):
        f = {k: scf_energy(shifted(atoms, at, ax, k * h), name, spherical, charge, mult, uhf) for k in (-2, -1, 1, 2)}
        fd = (8.0 * (f[1] - f[-1]) - (f[2] - f[-2])) / (12.0 * h)
        assert abs(fd - g[at, ax]) < 1e-6, (at, ax, fd, g[at, ax])
