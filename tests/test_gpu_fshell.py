"""f shells (l = 3): the generic McMurchie-Davidson engine, through the C ABI.

hf-rs's SPDF problem (four centres, each with an s, p, d and f shell of two
primitives; spdf_eri.npz) pins every one of its 256 angular classes against
PySCF.  Classes with an f shell run on the generic engine, the others on the
generated kernels; Schwarz bounds, the packed tensor, RHF/UHF J/K (also in
deterministic mode and sharded) and the SCF are checked against the oracle
and the golden energies of make_spdf_scf.py.
"""
import json
import os

import numpy as np
import pytest

import oracle as O
from hfgpu import CartesianBasis, Context, HfgError, JKOptions
from hfgpu.basis import read_gaussian94

pytestmark = pytest.mark.gpu

RANGES = [(0, 1), (1, 4), (4, 10), (10, 20)]  # s, p, d, f functions of one centre


@pytest.fixture(scope="module")
def spdf(golden_dir):
    g = np.load(os.path.join(golden_dir, "spdf_eri.npz"))
    atoms = [(str(s), tuple(float(x) for x in p)) for s, p in zip(g["symbols"], g["geometry"])]
    text = str(g["basis"])
    ours = CartesianBasis(atoms, read_gaussian94(text))
    ref = O.build_basis(atoms, O.parse_gaussian94(text))
    return {"g": g, "atoms": atoms, "ours": ours, "ref": ref}


def rand_sym(n, seed):
    a = np.random.default_rng(seed).standard_normal((n, n)) * 0.3
    return a + a.T


def test_all_256_spdf_classes_match_pyscf(spdf):
    g = spdf["g"]
    ctx = Context(spdf["ours"])
    assert ctx.n == 80
    lookup = {tuple(x): v for x, v in zip(g["ijkl"].tolist(), g["eri"])}
    worst, checked, classes = 0.0, 0, 0
    for blk in range(256):
        ang = [blk // 64, blk // 16 % 4, blk // 4 % 4, blk % 4]
        dims = [RANGES[x][1] - RANGES[x][0] for x in ang]
        q = ctx.shell_quartet(4 * 0 + ang[0], 4 * 1 + ang[1], 4 * 2 + ang[2], 4 * 3 + ang[3], dims)
        cnt, hit = 0, 0
        for i in range(*RANGES[ang[0]]):
            for j in range(*RANGES[ang[1]]):
                for k in range(*RANGES[ang[2]]):
                    for l in range(*RANGES[ang[3]]):
                        v = lookup.get((i, j, k, l))
                        if v is not None:
                            worst = max(worst, abs(q[cnt] - v))
                            hit += 1
                        cnt += 1
        checked += hit
        classes += hit > 0
    ctx.close()
    # all 256 blocks are computed; the fixture keeps every 7th of the 160,000
    # integrals, which leaves entries in 250 classes (the six without any are
    # (ss|sp)-type s/p classes) and in every class with an f shell
    assert classes == 250 and checked == len(g["eri"])
    assert worst < 2e-10, worst


def test_schwarz_and_packed_tensor_match_oracle(spdf):
    ctx = Context(spdf["ours"])
    q = ctx.schwarz()
    ref = O.schwarz(spdf["ref"])
    assert np.max(np.abs(q - ref) / np.maximum(ref, 1e-300)) < 1e-11
    got = ctx.eri_packed(1e-12)
    eref = O.eri_packed(spdf["ref"])
    assert np.max(np.abs(got - eref)) < 1e-12
    assert np.all(got[np.abs(eref) > 1e-13] != 0.0)
    ctx.close()


def test_jk_rhf_uhf_match_oracle(spdf):
    ctx = Context(spdf["ours"])
    n = ctx.n
    Pa, Pb = rand_sym(n, 1), rand_sym(n, 2)
    J, K = ctx.jk(Pa)
    Jr, Kr = O.direct_jk(spdf["ref"], Pa, [Pa])
    assert np.max(np.abs(J - Jr)) < 1e-11
    assert np.max(np.abs(K[0] - Kr[0])) < 1e-11
    Ju, Ku = ctx.jk(Pa + Pb, [Pa, Pb])
    Jur, Kur = O.direct_jk(spdf["ref"], Pa + Pb, [Pa, Pb])
    assert np.max(np.abs(Ju - Jur)) < 1e-11
    assert np.max(np.abs(Ku - Kur)) < 1e-11
    # mixed precision keeps the f classes in FP64; deterministic mode is
    # bitwise reproducible; shards sum to the full build
    Jm, Km = ctx.jk(Pa, opts=JKOptions.make(mixed=1e-7))
    assert np.max(np.abs(Jm - Jr)) < 1e-8 and np.max(np.abs(Km[0] - Kr[0])) < 1e-8
    det = JKOptions.make(deterministic=True)
    J1, K1 = ctx.jk(Pa, opts=det)
    J2, K2 = ctx.jk(Pa, opts=det)
    assert np.array_equal(J1, J2) and np.array_equal(K1, K2)
    assert np.max(np.abs(J1 - Jr)) < 1e-11
    import torch
    dev = torch.device("cuda", 0)
    P = torch.from_numpy(Pa).to(dev)
    Js = torch.zeros((n, n), dtype=torch.float64, device=dev)
    Ks = torch.zeros((n, n), dtype=torch.float64, device=dev)
    for s in range(3):
        Jt, Kt = torch.empty_like(Js), torch.empty_like(Ks)
        torch.cuda.synchronize()
        ctx.jk_device_shard(P.data_ptr(), P.data_ptr(), Jt.data_ptr(), Kt.data_ptr(), s, 3)
        torch.cuda.synchronize()
        Js += Jt
        Ks += Kt
    assert np.max(np.abs(Js.cpu().numpy() - Jr)) < 1e-11
    assert np.max(np.abs(Ks.cpu().numpy() - Kr[0])) < 1e-11
    ctx.close()


@pytest.mark.parametrize("space", ["cartesian", "spherical"])
def test_scf_matches_oracle_energy(spdf, golden_dir, space):
    ref = json.load(open(os.path.join(golden_dir, "spdf_scf.json")))[space]
    ctx = Context(spdf["ours"])
    r = ctx.scf(spherical=(space == "spherical"), tol=1e-10, max_iter=150)
    ctx.close()
    assert r["converged"]
    assert abs(r["energy"] - ref["energy"]) <= 1e-9, (r["energy"], ref["energy"])


def test_f_shells_outside_the_generic_engine_are_rejected(spdf):
    # density fitting covers orbital s, p and d shells
    ctx = Context(spdf["ours"])
    aux = CartesianBasis(spdf["atoms"], read_gaussian94(str(spdf["g"]["basis"])))
    from hfgpu.lib import DFTensor, HFG_DF_FP64
    with pytest.raises(HfgError, match="s, p and d"):
        DFTensor(ctx, aux, storage=HFG_DF_FP64)
    # ERI derivatives raise a shell by one: f is beyond them
    with pytest.raises(HfgError, match="s, p and d"):
        ctx.eri_gradient(np.eye(ctx.n))
    ctx.close()
