"""GPU SCF (hfg_scf) against hf-rs's golden energies and the CPU oracle."""
import json
import os

import numpy as np
import pytest

import oracle as O
from hfgpu import CartesianBasis, Context, JKOptions
from hfgpu.clusters import water_cluster

pytestmark = pytest.mark.gpu


def test_scf_energies_match_golden(golden_dir):
    # hf-rs tests/scf_reference_test.rs:72-94: |dE| < 1e-8 Eh vs PySCF (CDIIS, tol 1e-12)
    d = json.load(open(os.path.join(golden_dir, "scf_energies.json")))
    for c in d["cases"]:
        atoms = [(a[0], tuple(a[1])) for a in c["atoms"]]
        ctx = Context(CartesianBasis.build(atoms, c["basis"]))
        r = ctx.scf(charge=c["charge"], multiplicity=c["spin_2s"] + 1, uhf=c["spin_2s"] > 0, tol=1e-12, max_iter=200)
        assert r["converged"], c
        assert abs(r["energy"] - c["energy"]) < 1e-8, (c["name"], c["basis"], r["energy"], c["energy"])
        ctx.close()


def test_sad_guess_and_cdiis_follow_the_reference_iterations():
    # same SAD guess and CDIIS as hf-rs -> same iteration history as the oracle
    for name in ("sto-3g", "6-31g*", "cc-pvdz"):
        atoms = water_cluster(2)
        ctx = Context(CartesianBasis.build(atoms, name))
        r = ctx.scf(tol=1e-10, spherical=(name == "cc-pvdz"))
        ref = O.rhf(atoms, O.build_basis(atoms, O.load_basis(name)), tol=1e-10, spherical=(name == "cc-pvdz"))
        assert r["converged"] and abs(r["energy"] - ref["energy"]) <= 1e-10
        assert abs(r["iterations"] - ref["iterations"]) <= 1, (name, r["iterations"], ref["iterations"])


def test_water_ccpvdz_spherical_golden(golden_dir):
    # hf-rs tests/spherical_basis_test.rs:135-166 (24 retained MOs, 1e-9 Eh)
    d = json.load(open(os.path.join(golden_dir, "water_ccpvdz.json")))
    atoms = [(a[0], tuple(a[1])) for a in d["atoms"]]
    ctx = Context(CartesianBasis.build(atoms, "cc-pvdz"))
    r = ctx.scf(spherical=True, tol=1e-13, max_iter=150)
    assert r["converged"] and r["n_mo"] == 24
    assert abs(r["energy"] - d["energy"]) < 1e-9


def test_config0_water_ccpvdz_energy_and_fock_vs_oracle():
    # H2O cc-pVDZ at the hf-rs test geometry, spherical AO space, tol 1e-10:
    # |dE| <= 1e-10 Eh and Cartesian Fock elements within 1e-11 of the oracle
    atoms = water_cluster(1)
    ctx = Context(CartesianBasis.build(atoms, "cc-pvdz"))
    r = ctx.scf(spherical=True, tol=1e-10)
    ref = O.rhf(atoms, O.build_basis(atoms, O.load_basis("cc-pvdz")), tol=1e-10, spherical=True)
    assert r["converged"] and ref["converged"]
    assert abs(r["energy"] - ref["energy"]) <= 1e-10
    # same density -> same Fock: compare the reference digestion on our density
    P = r["P"][0]
    eri = O.eri_packed(O.build_basis(atoms, O.load_basis("cc-pvdz")))
    J, K = O.contract_jk(eri, P, [P])
    assert np.max(np.abs(r["F"][0] - (ref["H"] + J - 0.5 * K[0]))) < 1e-11
    assert np.max(np.abs(r["P"][0] - ref["P"])) < 1e-6


@pytest.mark.parametrize("nw", [2, 4])
def test_water_cluster_rhf_vs_oracle(nw):
    atoms = water_cluster(nw)
    ctx = Context(CartesianBasis.build(atoms, "cc-pvdz"))
    r = ctx.scf(spherical=True, tol=1e-10)
    ob = O.build_basis(atoms, O.load_basis("cc-pvdz"))
    ref = O.rhf(atoms, ob, tol=1e-10, spherical=True, jk=O.JKDirect(ob))
    assert r["converged"]
    assert abs(r["energy"] - ref["energy"]) <= 1e-10


@pytest.mark.parametrize("incremental", [0.0, 1e-12])
def test_mixed_precision_scf_refines_to_fp64(incremental):
    # mixed phase (full or incremental builds) then FP64 refinement: the
    # energy of the plain FP64 SCF within 1e-8 Eh
    atoms = water_cluster(4)
    ctx = Context(CartesianBasis.build(atoms, "cc-pvdz"))
    e64 = ctx.scf(spherical=True, tol=1e-10)["energy"]
    r = ctx.scf(spherical=True, tol=1e-10, jk=JKOptions.make(prim=1e-15, mixed=1e-7), incremental=incremental)
    assert r["converged"] and r["fock_builds_mixed"] > 0 and r["fock_builds_fp64"] >= 2
    assert (r["fock_builds_incremental"] > 0) == (incremental > 0)
    assert abs(r["energy"] - e64) <= 1e-8


def test_mixed_incremental_uhf_doublet():
    atoms = water_cluster(2)
    ctx = Context(CartesianBasis.build(atoms, "6-31g*"))
    e64 = ctx.scf(charge=1, multiplicity=2, uhf=True, tol=1e-10, max_iter=200)
    r = ctx.scf(charge=1, multiplicity=2, uhf=True, tol=1e-10, max_iter=200,
                jk=JKOptions.make(prim=1e-15, mixed=1e-7))
    assert e64["converged"] and r["converged"] and r["fock_builds_incremental"] > 0
    assert abs(r["energy"] - e64["energy"]) <= 1e-8
    assert abs(r["s2"] - e64["s2"]) < 1e-6


def test_uhf_doublet_cation_vs_oracle():
    atoms = water_cluster(1)
    ob = O.build_basis(atoms, O.load_basis("6-31g*"))
    ctx = Context(CartesianBasis.build(atoms, "6-31g*"))
    r = ctx.scf(charge=1, multiplicity=2, uhf=True, tol=1e-10, max_iter=200)
    ref = O.uhf(atoms, ob, charge=1, multiplicity=2, tol=1e-10, max_iter=200)
    assert r["converged"] and ref["converged"]
    assert abs(r["energy"] - ref["energy"]) <= 1e-9
    assert abs(r["s2"] - ref["s2"]) < 1e-6
