"""GPU density fitting against hf-rs's DF golden vectors and the oracle."""
import json
import os

import numpy as np
import pytest

import oracle as O
from hfgpu import CartesianBasis, Context
from hfgpu.clusters import water_cluster
from hfgpu.lib import HFG_DF_BF16, HFG_DF_FP32, HFG_DF_FP64, DFTensor

pytestmark = pytest.mark.gpu

ATOMS = [("O", (0.0, 0.0, 0.0)), ("H", (1.43, 0.2, 1.1)), ("H", (-1.2, -0.3, 1.3))]


def test_df_metric_matches_golden(golden_dir):
    # hf-rs tests/df_test.rs:22-71 (2e-9)
    g = np.load(os.path.join(golden_dir, "df.npz"))
    ctx = Context(CartesianBasis.build(ATOMS, "sto-3g"))
    df = DFTensor(ctx, CartesianBasis.build(ATOMS, "def2-svp-ri"))
    assert df.sizes()[0] == 85
    assert np.max(np.abs(df.metric() - g["metric"])) < 2e-9


def occ_coeffs(n, nocc, seed):
    q, _ = np.linalg.qr(np.random.default_rng(seed).standard_normal((n, n)))
    return np.ascontiguousarray(q[:, :nocc]) * 0.5


@pytest.mark.parametrize("nw,orb,auxname", [(1, "sto-3g", "def2-svp-ri"), (2, "cc-pvdz", "def2-universal-jkfit")])
def test_df_jk_fp64_matches_oracle(nw, orb, auxname):
    atoms = water_cluster(nw)
    ctx = Context(CartesianBasis.build(atoms, orb))
    df = DFTensor(ctx, CartesianBasis.build(atoms, auxname))
    C = occ_coeffs(ctx.n, 5 * nw, 3)
    J, K = df.jk(C)
    B = O.df_tensor(O.build_basis(atoms, O.load_basis(orb)), O.build_basis(atoms, O.load_basis(auxname)))
    Jr, Kr = O.df_jk(B, C, ctx.n)
    assert np.max(np.abs(J - Jr)) < 1e-10
    assert np.max(np.abs(K - Kr)) < 1e-10
    # tensor-core forms: stated error bounds for these O(1) test matrices
    for storage, mma, tol in [(HFG_DF_FP32, HFG_DF_FP32, 5e-3), (HFG_DF_BF16, HFG_DF_BF16, 5e-2)]:
        d2 = DFTensor(ctx, CartesianBasis.build(atoms, auxname), storage=storage)
        J2, K2 = d2.jk(C, mma=mma)
        assert np.max(np.abs(J2 - Jr)) < tol and np.max(np.abs(K2 - Kr)) < tol, storage


def test_df_rhf_matches_golden_water(golden_dir):
    # hf-rs tests/df_hf_test.rs:28-163: energy and every P, F, J, K element, 1e-9
    g = np.load(os.path.join(golden_dir, "df.npz"))
    atoms = [(a[0], tuple(a[1])) for a in json.loads(str(g["water_atoms"]))]
    ctx = Context(CartesianBasis.build(atoms, "sto-3g"))
    df = DFTensor(ctx, CartesianBasis.build(atoms, "def2-svp-ri"))
    r = ctx.scf_df(df)
    assert r["converged"]
    assert abs(r["energy"] - float(g["e_scf"])) < 1e-9
    for k in ("P", "F", "J", "K"):
        assert np.max(np.abs(r[k] - g[k])) < 1e-9, k


def test_df_pair_screening_changes_little():
    atoms = water_cluster(4)
    ctx = Context(CartesianBasis.build(atoms, "cc-pvdz"))
    aux = CartesianBasis.build(atoms, "def2-universal-jkfit")
    C = occ_coeffs(ctx.n, 20, 4)
    J0, K0 = DFTensor(ctx, aux).jk(C)
    J1, K1 = DFTensor(ctx, aux, pair_threshold=1e-10).jk(C)
    assert np.max(np.abs(J1 - J0)) < 1e-7 and np.max(np.abs(K1 - K0)) < 1e-7


def test_df_chunked_build_matches_single_chunk(monkeypatch):
    # B built over many narrow column chunks equals the one-chunk build
    atoms = water_cluster(2)
    ctx = Context(CartesianBasis.build(atoms, "cc-pvdz"))
    aux = CartesianBasis.build(atoms, "def2-universal-jkfit")
    C = occ_coeffs(ctx.n, 10, 5)
    for storage, tol in [(HFG_DF_FP64, 1e-11), (HFG_DF_FP32, 1e-5), (HFG_DF_BF16, 2e-2)]:
        monkeypatch.delenv("HFG_DF_CHUNK_COLS", raising=False)
        J1, K1 = DFTensor(ctx, aux, storage=storage).jk(C, mma=storage)
        monkeypatch.setenv("HFG_DF_CHUNK_COLS", "64")
        d = DFTensor(ctx, aux, storage=storage)
        assert d.sizes()[2] > 10 * 64  # about 20 chunks
        J2, K2 = d.jk(C, mma=storage)
        assert np.max(np.abs(J2 - J1)) < tol and np.max(np.abs(K2 - K1)) < tol, storage


@pytest.mark.parametrize("storage,mma,tol", [(HFG_DF_FP32, HFG_DF_FP32, 1e-5), (HFG_DF_FP32, HFG_DF_BF16, 1e-5),
                                              (HFG_DF_BF16, HFG_DF_BF16, 0.2)])
def test_df_rhf_tensor_core_phase_then_fp64_refinement(storage, mma, tol):
    # TF32 / BF16 J/K until loosely converged, then FP64 arithmetic on the
    # stored factor: converges, and differs from FP64 DF only by the storage
    # rounding of B (FP32 storage: ~2e-6 Eh of 152 Eh, about 1e-8 relative;
    # BF16 storage: ~0.11 Eh, 7e-4 relative)
    atoms = water_cluster(2)
    ctx = Context(CartesianBasis.build(atoms, "cc-pvdz"))
    aux = CartesianBasis.build(atoms, "def2-universal-jkfit")
    e64 = ctx.scf_df(DFTensor(ctx, aux), spherical=True)
    r = ctx.scf_df(DFTensor(ctx, aux, storage=storage), mma=mma, spherical=True)
    assert e64["converged"] and r["converged"]
    assert r["fock_builds_mixed"] > 0 and r["fock_builds_fp64"] >= 2
    assert abs(r["energy"] - e64["energy"]) < tol


def test_df_rhf_sad_start_reaches_the_same_energy():
    # the SAD start (an option; hf-rs's DF driver starts from the core
    # Hamiltonian) converges to the same DF-RHF solution in fewer iterations
    atoms = water_cluster(3)
    ctx = Context(CartesianBasis.build(atoms, "cc-pvdz"))
    aux = CartesianBasis.build(atoms, "def2-universal-jkfit")
    df = DFTensor(ctx, aux)
    rc = ctx.scf_df(df, spherical=True)
    rs = ctx.scf_df(df, spherical=True, guess="sad")
    assert rc["converged"] and rs["converged"]
    assert abs(rc["energy"] - rs["energy"]) < 1e-9
    assert rs["iterations"] < rc["iterations"]


@pytest.mark.parametrize("mma", [HFG_DF_FP64, HFG_DF_BF16])
def test_df_shards_over_the_auxiliary_index_sum_to_the_full_build(mma):
    # the multi-GPU DF decomposition run shard after shard on one GPU
    atoms = water_cluster(2)
    ctx = Context(CartesianBasis.build(atoms, "cc-pvdz"))
    aux = CartesianBasis.build(atoms, "def2-universal-jkfit")
    d = DFTensor(ctx, aux, storage=HFG_DF_FP64 if mma == HFG_DF_FP64 else HFG_DF_FP32)
    C = occ_coeffs(ctx.n, 10, 6)
    J0, K0 = d.jk(C, mma=mma)
    for nshards in (2, 3):
        Js, Ks = np.zeros_like(J0), np.zeros_like(K0)
        for s in range(nshards):
            J, K = d.jk_shard(C, s, nshards, mma=mma)
            Js += J
            Ks += K
        tol = 1e-11 if mma == HFG_DF_FP64 else 1e-5 * np.max(np.abs(K0))
        assert np.max(np.abs(Js - J0)) < 1e-11 and np.max(np.abs(Ks - K0)) < tol, (mma, nshards)
    ctx.close()


@pytest.mark.parametrize("mma", [HFG_DF_FP64, HFG_DF_BF16])
def test_shard_factors_sum_to_the_full_build(mma):
    # each rank of a multi-GPU DF build holds only its rows of the factor
    # (hfg_df_build_shard); their J and K sum to the whole factor's
    from hfgpu import HfgError
    atoms = water_cluster(2)
    ctx = Context(CartesianBasis.build(atoms, "cc-pvdz"))
    aux = CartesianBasis.build(atoms, "def2-universal-jkfit")
    storage = HFG_DF_FP64 if mma == HFG_DF_FP64 else HFG_DF_FP32
    full = DFTensor(ctx, aux, storage=storage)
    C = occ_coeffs(ctx.n, 10, 6)
    J0, K0 = full.jk(C, mma=mma)
    rank = full.sizes()[1]
    full.close()
    for nshards in (2, 3):
        Js, Ks, rows = np.zeros_like(J0), np.zeros_like(K0), 0
        for s in range(nshards):
            d = DFTensor(ctx, aux, storage=storage, shard=s, nshards=nshards)
            rows += d.sizes()[1]
            J, K = d.jk(C, mma=mma)
            Js += J
            Ks += K
            if s == 0:
                with pytest.raises(HfgError, match="whole factor"):
                    d.mp2_energy(np.eye(ctx.n), np.arange(ctx.n, dtype=float), 5)
                with pytest.raises(HfgError, match="whole factor"):
                    ctx.scf_df(d)
            d.close()
        assert rows == rank
        tol = 1e-11 if mma == HFG_DF_FP64 else 1e-5 * np.max(np.abs(K0))
        assert np.max(np.abs(Js - J0)) < 1e-11 and np.max(np.abs(Ks - K0)) < tol, (mma, nshards)
    ctx.close()


def test_df_transform_matches_the_oracle_factor_in_the_mo_basis():
    # DfTensor::transform (src/df.rs:182-210): C^T B_Q C packed over p >= q
    ctx = Context(CartesianBasis.build(ATOMS, "sto-3g"))
    aux = CartesianBasis.build(ATOMS, "def2-svp-ri")
    r = ctx.scf(tol=1e-12, want=("C", "eps"))
    C = r["C"][0]
    Bmo = DFTensor(ctx, aux).transform(C)
    B = O.df_tensor(O.build_basis(ATOMS, O.load_basis("sto-3g")), O.build_basis(ATOMS, O.load_basis("def2-svp-ri")))
    n, m = C.shape
    iu = np.tril_indices(m)
    ref = np.stack([(C.T @ O.unpack_pairs(B[q:q + 1], n)[0] @ C)[iu] for q in range(B.shape[0])])
    assert Bmo.shape == ref.shape
    # the rows depend on the metric's eigenvector basis (signs, order,
    # degenerate rotations); the fitted MO integrals (pq|rs) = B^T B do not
    assert np.max(np.abs(Bmo.T @ Bmo - ref.T @ ref)) < 1e-10
    ctx.close()


def test_ri_mp2_matches_golden(golden_dir):
    # hf-rs tests/df_test.rs:22-71: RHF (tol 1e-13), DF factor with metric
    # cutoff 1e-10, RI-MP2 in the canonical MO basis within 1e-9 Eh of PySCF
    g = np.load(os.path.join(golden_dir, "df.npz"))
    ctx = Context(CartesianBasis.build(ATOMS, "sto-3g"))
    r = ctx.scf(tol=1e-13, max_iter=150, want=("C", "eps"))
    assert r["converged"]
    df = DFTensor(ctx, CartesianBasis.build(ATOMS, "def2-svp-ri"))
    e = df.mp2_energy(r["C"][0], r["eps"][0], n_occ=5)
    assert abs(e - float(g["ri_mp2"])) < 1e-9, (e, float(g["ri_mp2"]))
    # a frozen core changes the energy; an invalid partition is rejected
    assert df.mp2_energy(r["C"][0], r["eps"][0], n_occ=5, n_frozen=1) > e
    with pytest.raises(Exception):
        df.mp2_energy(r["C"][0], r["eps"][0], n_occ=5, n_frozen=6)
    ctx.close()


def test_cholesky_factor_and_cd_hf_match_golden(golden_dir):
    # hf-rs tests/cd_hf_test.rs:42-70: the pivot sequence, vector count and
    # largest residual of pivoted_cholesky_eri, and the CD-HF energy (run_cd_hf,
    # tol 1e-12: residual 1e-8, density 1e-10) within 1e-9 Eh
    d = json.load(open(os.path.join(golden_dir, "cd_hf.json")))
    for c in d["cases"]:
        atoms = [(a[0], tuple(a[1])) for a in c["atoms"]]
        ctx = Context(CartesianBasis.build(atoms, c["basis"]))
        for t in c["thresholds"]:
            f, piv, mres = DFTensor.cholesky(ctx, t["threshold"])
            assert piv == t["pivots"], (c["name"], t["threshold"])
            assert f.sizes()[1] == t["n_vectors"]
            assert mres <= t["threshold"] and abs(mres - t["max_residual"]) < 1e-12
            r = ctx.scf_df(f, tol=(1e-12, 1e-8, 1e-10), max_iter=300)
            assert r["converged"]
            assert abs(r["energy"] - t["e_cd_hf"]) < 1e-9, (c["name"], t["threshold"], r["energy"], t["e_cd_hf"])
            f.close()
        ctx.close()


def test_cholesky_reconstruction_obeys_the_residual_bound(golden_dir):
    # |(pq|rs) - sum_K L_K(pq) L_K(rs)| <= max residual diagonal
    # (hf-rs tests/cd_hf_test.rs:72-100), the vectors seen through the fitted
    # integrals of their own J/K: exact ERIs from the packed tensor
    d = json.load(open(os.path.join(golden_dir, "cd_hf.json")))
    c = [x for x in d["cases"] if x["name"] == "water"][0]
    atoms = [(a[0], tuple(a[1])) for a in c["atoms"]]
    ctx = Context(CartesianBasis.build(atoms, c["basis"]))
    n = ctx.n
    np_ = n * (n + 1) // 2
    eri = ctx.eri_packed(threshold=0.0)
    ii, jj = np.tril_indices(np_)
    V = np.zeros((np_, np_))
    V[ii, jj] = eri
    V[jj, ii] = eri
    for delta in (1e-2, 1e-4, 1e-7):
        f, _, mres = DFTensor.cholesky(ctx, delta)
        # the factor's own DF J/K with unit-vector densities reproduce columns
        # of L^T L; compare the whole reconstruction through MO transform with C = I
        Bmo = f.transform(np.eye(n))
        assert np.max(np.abs(Bmo.T @ Bmo - V)) <= mres + 1e-12, delta
        f.close()
    with pytest.raises(Exception):
        DFTensor.cholesky(ctx, 1e-7, budget=1024)
    ctx.close()
