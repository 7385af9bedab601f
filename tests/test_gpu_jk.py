"""GPU parity of the direct J/K build against the CPU oracle (the hf-rs
restatement), through the C ABI."""
import numpy as np
import pytest

import oracle as O
from hfgpu import CartesianBasis, Context, JKOptions
from hfgpu.clusters import water_cluster

pytestmark = pytest.mark.gpu


def rand_sym(n, seed):
    rng = np.random.default_rng(seed)
    a = rng.standard_normal((n, n)) * 0.3
    return a + a.T


def oracle_basis(atoms, name):
    return O.build_basis(atoms, O.load_basis(name))


@pytest.mark.parametrize("name", ["sto-3g", "6-31g*", "cc-pvdz"])
def test_schwarz_bounds_match_oracle(name):
    atoms = water_cluster(2)
    ctx = Context(CartesianBasis.build(atoms, name))
    q = ctx.schwarz()
    ref = O.schwarz(oracle_basis(atoms, name))
    assert q.shape == ref.shape
    assert np.max(np.abs(q - ref) / np.maximum(ref, 1e-300)) < 1e-11


def test_spdf_shell_quartets_match_pyscf_for_spd(golden_dir):
    # the hf-rs SPDF problem without its f shells: every (s,p,d)^4 class
    import os
    g = np.load(os.path.join(golden_dir, "spdf_eri.npz"))
    text = str(g["basis"])
    blocks, keep = text.split("****"), []
    for blk in blocks:
        lines = [ln for ln in blk.strip().splitlines()]
        if not lines:
            continue
        out, i = [lines[0]], 1
        while i < len(lines):
            head = lines[i].split()
            n = int(head[1])
            if head[0].upper() != "F":
                out.extend(lines[i:i + 1 + n])
            i += 1 + n
        keep.append("\n".join(out))
    spd = "\n****\n".join(keep) + "\n****\n"
    atoms = [(str(s), tuple(p)) for s, p in zip(g["symbols"], g["geometry"])]
    from hfgpu.basis import read_gaussian94
    basis = CartesianBasis(atoms, read_gaussian94(spd))
    assert basis.n == 40
    ctx = Context(basis)
    lookup = {tuple(x): v for x, v in zip(g["ijkl"].tolist(), g["eri"])}
    ranges = [(0, 1), (1, 4), (4, 10)]
    worst, checked = 0.0, 0
    for blk in range(81):
        ang = [blk // 27, blk // 9 % 3, blk // 3 % 3, blk % 3]
        dims = [ranges[x][1] - ranges[x][0] for x in ang]
        q = ctx.shell_quartet(3 * 0 + ang[0], 3 * 1 + ang[1], 3 * 2 + ang[2], 3 * 3 + ang[3], dims)
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
    assert checked > 1000
    assert worst < 2e-10, worst


@pytest.mark.parametrize("name,nw", [("sto-3g", 1), ("6-31g*", 2), ("cc-pvdz", 1), ("cc-pvdz", 3)])
def test_jk_matches_oracle_rhf_and_uhf(name, nw):
    atoms = water_cluster(nw)
    ours = CartesianBasis.build(atoms, name)
    ref = oracle_basis(atoms, name)
    n = ours.n
    Pa, Pb = rand_sym(n, 1), rand_sym(n, 2)
    ctx = Context(ours)
    J, K = ctx.jk(Pa)
    Jr, Kr = O.direct_jk(ref, Pa, [Pa])
    assert np.max(np.abs(J - Jr)) < 1e-11
    assert np.max(np.abs(K[0] - Kr[0])) < 1e-11
    Ju, Ku = ctx.jk(Pa + Pb, [Pa, Pb])
    Jur, Kur = O.direct_jk(ref, Pa + Pb, [Pa, Pb])
    assert np.max(np.abs(Ju - Jur)) < 1e-11
    assert np.max(np.abs(Ku - Kur)) < 1e-11


def test_fock_rhf_matches_reference_digestion():
    atoms = water_cluster(2)
    ours = CartesianBasis.build(atoms, "cc-pvdz")
    ref = oracle_basis(atoms, "cc-pvdz")
    S, T, V = O.one_electron(ref, atoms)
    H = T + V
    P = rand_sym(ours.n, 3)
    ctx = Context(ours)
    F = ctx.fock_rhf(H, P)
    eri = O.eri_packed(ref)
    J, K = O.contract_jk(eri, P, [P])
    assert np.max(np.abs(F - (H + J - 0.5 * K[0]))) < 1e-11
    Pb = rand_sym(ours.n, 4)
    Fa, Fb = ctx.fock_uhf(H, P, Pb)
    J, K = O.contract_jk(eri, P + Pb, [P, Pb])
    assert np.max(np.abs(Fa - (H + J - K[0]))) < 1e-11
    assert np.max(np.abs(Fb - (H + J - K[1]))) < 1e-11


def test_primitive_screening_error_is_bounded():
    atoms = water_cluster(4)
    ours = CartesianBasis.build(atoms, "cc-pvdz")
    ctx = Context(ours)
    P = rand_sym(ours.n, 5)
    J0, K0 = ctx.jk(P)
    J1, K1 = ctx.jk(P, opts=JKOptions.make(prim=1e-15))
    assert np.max(np.abs(J1 - J0)) < 1e-11
    assert np.max(np.abs(K1 - K0)) < 1e-11


@pytest.mark.parametrize("nw,name", [(1, "cc-pvdz"), (2, "6-31g*")])
def test_eri_packed_matches_oracle(nw, name):
    # compute_eri_tensor: every slot of the packed 8-fold tensor, screened
    # quartets zero in both
    atoms = water_cluster(nw)
    ctx = Context(CartesianBasis.build(atoms, name))
    got = ctx.eri_packed(1e-12)
    ref = O.eri_packed(oracle_basis(atoms, name))
    assert got.shape == ref.shape
    assert np.max(np.abs(got - ref)) < 1e-12
    # same screened slots (symmetry-zero integrals are 1e-17 noise in one
    # engine and exact zeros in the other, so compare above 1e-13)
    assert np.all(got[np.abs(ref) > 1e-13] != 0.0)
    # contract_jk over the device tensor reproduces the direct J/K build
    P = rand_sym(ctx.n, 3)
    Jr, Kr = O.contract_jk(got, P, [P])
    J, K = ctx.jk(P)
    assert np.max(np.abs(J - Jr)) < 1e-11
    assert np.max(np.abs(K[0] - Kr[0])) < 1e-11


def test_eri_packed_rejects_wrong_length():
    from hfgpu import HfgError
    ctx = Context(CartesianBasis.build(water_cluster(1), "sto-3g"))
    with pytest.raises(HfgError, match="INVALID_INPUT"):
        ctx.eri_packed(1e-12, length=10)


def test_autotune_picks_fastest_within_energy_budget():
    # the autotuner's choice meets its energy budget when checked independently
    import torch
    atoms = water_cluster(4)
    ctx = Context(CartesianBasis.build(atoms, "cc-pvdz"))
    P = ctx.scf(spherical=True, tol=1e-10, max_iter=3, want=("P",))["P"][0]
    dP = torch.from_numpy(np.ascontiguousarray(P)).to(torch.device("cuda", 0))
    torch.cuda.synchronize()  # the context runs on its own stream
    best, rep = ctx.autotune(dP.data_ptr(), dP.data_ptr(), max_energy_error=5e-9, repeats=1)
    # 12 threshold pairs, then the library's four extra quartet tiles on the best pair
    assert rep["found"] and len(rep["candidates"]) == 16
    assert [c.get("tile") for c in rep["candidates"][12:]] == [8, 16, 32, 256]
    ok = [c for c in rep["candidates"] if abs(c["energy_error"]) <= 5e-9]
    assert rep["best_ms"] == min(c["ms"] for c in ok)
    assert best.tile in (0, 8, 16, 32, 256)
    J0, K0 = ctx.jk(P, opts=JKOptions.make(prim=0.0))
    J1, K1 = ctx.jk(P, opts=best)
    dE = 0.5 * np.sum(P * (J1 - J0)) - 0.25 * np.sum(P * (K1[0] - K0[0]))
    assert abs(dE - rep["best_energy_error"]) < 1e-10
    assert abs(dE) <= 5e-9


@pytest.mark.parametrize("tile", [1, 16, 256, 4096])
def test_quartet_tile_changes_scheduling_not_results(tile):
    atoms = water_cluster(3)
    ctx = Context(CartesianBasis.build(atoms, "cc-pvdz"))
    P = rand_sym(ctx.n, 9)
    J0, K0 = ctx.jk(P)
    J1, K1 = ctx.jk(P, opts=JKOptions.make(tile=tile))
    assert np.max(np.abs(J1 - J0)) < 1e-11
    assert np.max(np.abs(K1 - K0)) < 1e-11
    ctx.close()


@pytest.mark.parametrize("nshards", [2, 3, 5])
def test_shards_sum_to_the_full_build(nshards):
    # the multi-GPU decomposition, run shard after shard on one GPU: the
    # partial J/K of all shards sum to the single build (FP64 and mixed)
    import torch
    dev = torch.device("cuda", 0)
    atoms = water_cluster(4)
    ctx = Context(CartesianBasis.build(atoms, "cc-pvdz"))
    n = ctx.n
    P = torch.from_numpy(rand_sym(n, 9)).to(dev)
    J = torch.empty((n, n), dtype=torch.float64, device=dev)
    K = torch.empty((n, n), dtype=torch.float64, device=dev)
    for opts in [JKOptions.make(), JKOptions.make(prim=1e-15, mixed=1e-7)]:
        torch.cuda.synchronize()
        ctx.jk_device(P.data_ptr(), P.data_ptr(), J.data_ptr(), K.data_ptr(), 1, opts)
        ctx.jk_device(P.data_ptr(), P.data_ptr(), J.data_ptr(), K.data_ptr(), 1, opts)  # plan made
        torch.cuda.synchronize()
        J0, K0 = J.cpu().numpy().copy(), K.cpu().numpy().copy()
        Js, Ks = np.zeros_like(J0), np.zeros_like(K0)
        for s in range(nshards):
            ctx.jk_device_shard(P.data_ptr(), P.data_ptr(), J.data_ptr(), K.data_ptr(), s, nshards, opts=opts)
            torch.cuda.synchronize()
            Js += J.cpu().numpy()
            Ks += K.cpu().numpy()
        assert np.max(np.abs(Js - J0)) < 1e-11
        assert np.max(np.abs(Ks - K0)) < 1e-11


def test_graph_replayed_builds_match_eager(monkeypatch):
    # the same buffers, new densities each call: build 1 eager, build 2
    # captured, builds 3-4 replayed; each equals an eager-only context
    import torch
    dev = torch.device("cuda", 0)
    atoms = water_cluster(3)
    basis = CartesianBasis.build(atoms, "cc-pvdz")
    monkeypatch.delenv("HFG_NO_GRAPHS", raising=False)
    ctx = Context(basis)
    monkeypatch.setenv("HFG_NO_GRAPHS", "1")
    eager = Context(basis)
    n = ctx.n
    P = torch.empty((n, n), dtype=torch.float64, device=dev)
    J = torch.empty((n, n), dtype=torch.float64, device=dev)
    K = torch.empty((n, n), dtype=torch.float64, device=dev)
    for opts in [JKOptions.make(), JKOptions.make(prim=1e-15, mixed=1e-7)]:
        for call in range(4):
            Ph = rand_sym(n, 20 + call)
            P.copy_(torch.from_numpy(Ph))
            torch.cuda.synchronize()
            ctx.jk_device(P.data_ptr(), P.data_ptr(), J.data_ptr(), K.data_ptr(), 1, opts)
            torch.cuda.synchronize()
            Jg, Kg = J.cpu().numpy().copy(), K.cpu().numpy().copy()
            Je, Ke = eager.jk(Ph, opts=opts)
            assert np.max(np.abs(Jg - Je)) < 1e-12 and np.max(np.abs(Kg - Ke[0])) < 1e-12, call


@pytest.mark.parametrize("name,nw,mixed", [("cc-pvdz", 1, None), ("sto-3g", 2, None), ("cc-pvdz", 1, 1e-6)])
def test_deterministic_mode_is_bitwise_reproducible(name, nw, mixed):
    # the debugging mode: one warp takes the work queue in order and its lanes
    # add into J'/K' one at a time, so repeated builds agree to the bit; the
    # atomic mode agrees with it to FP64 summation order
    ctx = Context(CartesianBasis.build(water_cluster(nw), name))
    n = ctx.n
    rng = np.random.default_rng(3)
    Pa, Pb = (lambda a: a + a.T)(rng.standard_normal((n, n)) * 0.2), (lambda a: a + a.T)(rng.standard_normal((n, n)) * 0.2)
    det = JKOptions.make(mixed=mixed, deterministic=True)
    fast = JKOptions.make(mixed=mixed)
    for spins in ([Pa], [Pa, Pb]):
        total = sum(spins)
        J1, K1 = ctx.jk(total, spins, opts=det)
        J2, K2 = ctx.jk(total, spins, opts=det)
        assert np.array_equal(J1, J2) and np.array_equal(K1, K2)
        J3, K3 = ctx.jk(total, spins, opts=fast)
        scale = max(1.0, np.abs(J3).max())
        assert np.max(np.abs(J1 - J3)) < 1e-12 * scale
        assert np.max(np.abs(K1 - K3)) < 1e-12 * scale
    ctx.close()
