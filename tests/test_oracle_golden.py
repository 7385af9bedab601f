"""Pins the CPU oracle against hf-rs's own golden vectors (tests/golden/,
copied from hf-rs tests/data by tests/golden/make_golden.py)."""
import json
import os

import numpy as np
import pytest

import oracle as O


@pytest.fixture(scope="module", autouse=True)
def _built():
    O.build_library()


def test_boys_matches_mpmath_fixture(golden_dir):
    # hf-rs tests/boys_test.rs:11-40: rel <= 1e-14 for n <= 40, T in [0, 200]
    d = json.load(open(os.path.join(golden_dir, "boys.json")))
    worst = 0.0
    for row in d["rows"]:
        out = O.boys_array(40, row["t"])
        ref = np.array(row["f"])
        worst = max(worst, float(np.max(np.abs((out - ref) / ref))))
    assert worst <= 1e-14, worst


def test_boys_spot_values():
    # hf-rs src/integrals.rs:1078-1084
    assert abs(O.boys_array(1, 0.0)[0] - 1.0) < 1e-12
    assert abs(O.boys_array(1, 0.0)[1] - 1.0 / 3.0) < 1e-12
    assert abs(O.boys_array(1, 1.0)[0] - 0.746824) < 1e-5
    assert abs(O.boys_array(1, 1.0)[1] - 0.189472) < 1e-5


def spdf_problem(golden_dir):
    g = np.load(os.path.join(golden_dir, "spdf_eri.npz"))
    atoms = [(str(s), tuple(p)) for s, p in zip(g["symbols"], g["geometry"])]
    basis = O.build_basis(atoms, O.parse_gaussian94(str(g["basis"])))
    return g, basis


def test_spdf_shell_quartets_match_pyscf(golden_dir):
    # hf-rs tests/shell_eri_test.rs:216-277: every (s,p,d,f)^4 class, 2e-10 abs
    g, basis = spdf_problem(golden_dir)
    assert len(basis) == 80
    subs = [basis[20 * a:20 * a + 20] for a in range(4)]
    ranges = [(0, 1), (1, 4), (4, 10), (10, 20)]
    lookup = {tuple(x): v for x, v in zip(g["ijkl"].tolist(), g["eri"])}
    worst, checked = 0.0, 0
    for blk in range(256):
        ang = [blk // 64, blk // 16 % 4, blk // 4 % 4, blk % 4]
        sh = [subs[a][ranges[ang[a]][0]:ranges[ang[a]][1]] for a in range(4)]
        q = O.shell_quartet(*sh)
        cnt = 0
        for i in range(*ranges[ang[0]]):
            for j in range(*ranges[ang[1]]):
                for k in range(*ranges[ang[2]]):
                    for l in range(*ranges[ang[3]]):
                        v = lookup.get((i, j, k, l))
                        if v is not None:
                            worst = max(worst, abs(q[cnt] - v))
                            checked += 1
                        cnt += 1
    assert checked == len(g["eri"])
    assert worst < 2e-10, worst


def test_spdf_scalar_engine_matches_pyscf(golden_dir):
    g, basis = spdf_problem(golden_dir)
    subs = [basis[20 * a:20 * a + 20] for a in range(4)]
    sel = np.arange(0, len(g["eri"]), 37)
    v = O.contracted_eri_list(*subs, g["ijkl"][sel])
    assert np.max(np.abs(v - g["eri"][sel])) < 2e-10


def test_packed_tensor_matches_scalar_engine():
    # hf-rs tests/shell_eri_test.rs:333-349
    atoms = [("H", (0.2, 0.1, -0.5)), ("H", (-0.1, 0.3, 0.8))]
    basis = O.build_basis(atoms, O.parse_gaussian94("H 0\nS 1 1\n0.8 1\nP 1 1\n0.7 1\nD 1 1\n0.6 1\n****"))
    eri = O.eri_packed(basis)
    n = len(basis)
    idx = []
    for i in range(n):
        for j in range(i + 1):
            for k in range(n):
                for l in range(k + 1):
                    if i * (i + 1) // 2 + j >= k * (k + 1) // 2 + l:
                        idx.append((i, j, k, l))
    idx = np.array(idx)
    ref = O.contracted_eri_list(basis, basis, basis, basis, idx)
    ij = idx[:, 0] * (idx[:, 0] + 1) // 2 + idx[:, 1]
    kl = idx[:, 2] * (idx[:, 2] + 1) // 2 + idx[:, 3]
    got = eri[ij * (ij + 1) // 2 + kl]
    assert np.max(np.abs(got - ref)) < 2e-11


def test_fock_digestion_known_answer():
    # hf-rs tests/fock_contraction_test.rs:1-44 (synthetic packed ERI)
    for n in range(1, 8):
        npair = n * (n + 1) // 2
        eri = np.sin((np.arange(npair * (npair + 1) // 2) + 1) * 0.37)
        h, pa, pb = np.zeros((n, n)), np.zeros((n, n)), np.zeros((n, n))
        for i in range(n):
            for j in range(i + 1):
                h[i, j] = h[j, i] = np.cos(i + j + 1)
                pa[i, j] = pa[j, i] = np.sin(i * 3 + j + 1)
                pb[i, j] = pb[j, i] = np.cos(i + j * 2 + 1)

        def ci(i, j):
            return i * (i + 1) // 2 + j if i >= j else j * (j + 1) // 2 + i

        def ei(a, b, c, d):
            return ci(ci(a, b), ci(c, d))

        J, K = O.contract_jk(eri, pa, [pa])
        R = h + J - 0.5 * K[0]
        Ju, Ku = O.contract_jk(eri, pa + pb, [pa, pb])
        for a in range(n):
            for b in range(n):
                r = h[a, b]
                u = [r, r]
                for c in range(n):
                    for d in range(n):
                        co, ex = eri[ei(a, b, c, d)], eri[ei(a, c, b, d)]
                        r += pa[c, d] * (co - 0.5 * ex)
                        u[0] += (pa[c, d] + pb[c, d]) * co - pa[c, d] * ex
                        u[1] += (pa[c, d] + pb[c, d]) * co - pb[c, d] * ex
                assert abs(R[a, b] - r) < 1e-12
                assert abs(h[a, b] + Ju[a, b] - Ku[0][a, b] - u[0]) < 1e-12
                assert abs(h[a, b] + Ju[a, b] - Ku[1][a, b] - u[1]) < 1e-12


def test_direct_jk_equals_packed_contraction():
    atoms = O.WATER_BOHR
    basis = O.build_basis(atoms, O.load_basis("cc-pvdz"))
    rng = np.random.default_rng(1)
    A = rng.standard_normal((len(basis), len(basis)))
    P = A + A.T
    Pb = rng.standard_normal(P.shape)
    Pb = Pb + Pb.T
    J1, K1 = O.JKPacked(basis)(P + Pb, [P, Pb])
    J2, K2 = O.JKDirect(basis)(P + Pb, [P, Pb])
    assert np.max(np.abs(J1 - J2)) < 1e-12
    assert np.max(np.abs(K1 - K2)) < 1e-12


def test_scf_energies_match_pyscf(golden_dir):
    # hf-rs tests/scf_reference_test.rs:72-94 (CDIIS, tol 1e-12, 1e-8 Eh)
    d = json.load(open(os.path.join(golden_dir, "scf_energies.json")))
    for c in d["cases"]:
        atoms = [(a[0], tuple(a[1])) for a in c["atoms"]]
        basis = O.build_basis(atoms, O.load_basis(c["basis"]))
        assert len(basis) == c["n_ao"]
        if c["spin_2s"] == 0:
            r = O.rhf(atoms, basis, charge=c["charge"], tol=1e-12, max_iter=200)
        else:
            r = O.uhf(atoms, basis, charge=c["charge"], multiplicity=c["spin_2s"] + 1, tol=1e-12, max_iter=200)
        assert r["converged"]
        assert abs(r["energy"] - c["energy"]) < 1e-8, (c["name"], c["basis"], r["energy"], c["energy"])


def test_water_ccpvdz_spherical_energy(golden_dir):
    # hf-rs tests/spherical_basis_test.rs:135-166 (1e-9 Eh, 24 MO columns)
    d = json.load(open(os.path.join(golden_dir, "water_ccpvdz.json")))
    atoms = [(a[0], tuple(a[1])) for a in d["atoms"]]
    basis = O.build_basis(atoms, O.load_basis("cc-pvdz"))
    r = O.rhf(atoms, basis, tol=1e-13, max_iter=150, spherical=True)
    assert r["converged"] and r["X"].shape[1] == 24
    assert abs(r["energy"] - d["energy"]) < 1e-9


def test_df_metric_three_centre_and_dfhf(golden_dir):
    # hf-rs tests/df_test.rs:22-71 and tests/df_hf_test.rs:28-163
    g = np.load(os.path.join(golden_dir, "df.npz"))
    atoms = [("O", (0.0, 0.0, 0.0)), ("H", (1.43, 0.2, 1.1)), ("H", (-1.2, -0.3, 1.3))]
    basis = O.build_basis(atoms, O.load_basis("sto-3g"))
    aux = O.build_basis(atoms, O.load_basis("def2-svp-ri"))
    assert len(aux) == 85
    assert np.max(np.abs(O.df_metric(aux) - g["metric"])) < 2e-9
    three = O.df_three(basis, aux)
    for i in range(7):
        for j in range(i + 1):
            assert np.max(np.abs(three[:, i * (i + 1) // 2 + j] - g["three"][i][j])) < 2e-10
    watoms = [(a[0], tuple(a[1])) for a in json.loads(str(g["water_atoms"]))]
    basis = O.build_basis(watoms, O.load_basis("sto-3g"))
    aux = O.build_basis(watoms, O.load_basis("def2-svp-ri"))
    r = O.df_rhf(watoms, basis, aux)
    assert abs(r["energy"] - float(g["e_scf"])) < 1e-9
    for k in ("P", "F", "J", "K"):
        assert np.max(np.abs(r[k] - g[k])) < 1e-9, k


def test_pivoted_cholesky_and_cd_hf_match_golden(golden_dir):
    # hf-rs tests/cd_hf_test.rs:42-70: pivot sequence, vector count and
    # largest residual (1e-12) of the pivoted Cholesky ERI factor, and the
    # CD-HF energy (run_cd_hf, tol 1e-12) within 1e-9 Eh
    d = json.load(open(os.path.join(golden_dir, "cd_hf.json")))
    for c in d["cases"]:
        atoms = [(a[0], tuple(a[1])) for a in c["atoms"]]
        basis = O.build_basis(atoms, O.load_basis(c["basis"]))
        for t in c["thresholds"]:
            L, piv, mres = O.pivoted_cholesky(basis, t["threshold"])
            assert L.shape[0] == t["n_vectors"], (c["name"], t["threshold"])
            assert piv == t["pivots"], (c["name"], t["threshold"])
            assert mres <= t["threshold"] and abs(mres - t["max_residual"]) < 1e-12
            tol = 1e-12
            r = O.factorized_rhf(atoms, basis, L, max_iter=300, e_tol=tol, r_tol=max(tol ** 0.5 * 1e-2, 1e-11),
                                 d_tol=min(max(tol ** 0.5 * 0.1, 1e-12), 1e-10))
            assert abs(r["energy"] - t["e_cd_hf"]) < 1e-9, (c["name"], t["threshold"], r["energy"], t["e_cd_hf"])
