"""CPU-side checks of the product: the C-ABI library loads and exports every
entry point of include/hfg.h, its option defaults are the documented ones,
and the host-side basis and cluster builders agree with the oracle's
restatement of hf-rs's build_basis."""
import os
import subprocess

import numpy as np
import pytest

import oracle as O
from hfgpu import lib as hl
from hfgpu.basis import CartesianBasis
from hfgpu.clusters import water_cluster


def test_library_exports_every_declared_symbol():
    path = hl.library_path()
    if not os.path.exists(path):
        pytest.skip("libhfg.so not built")
    declared = hl.exported_functions()
    assert len(declared) >= 10
    out = subprocess.run(["nm", "-D", "--defined-only", path], capture_output=True, text=True).stdout
    exported = {ln.split()[-1] for ln in out.splitlines() if ln.strip()}
    missing = [f for f in declared if f not in exported]
    assert not missing, missing
    L = hl.load_library()
    for f in declared:
        assert hasattr(L, f)


@pytest.mark.parametrize("name", ["sto-3g", "6-31g*", "cc-pvdz", "def2-universal-jkfit"])
def test_basis_builder_matches_oracle(name):
    atoms = water_cluster(2)
    ours = CartesianBasis.build(atoms, name)
    ref = O.build_basis(atoms, O.load_basis(name))
    assert ours.n == len(ref)
    for i, g in enumerate(ref):
        assert tuple(ours.lxyz[i]) == g["l"]
        assert ours.atom[i] == g["atom"]
        e = ours.exps[ours.prim_off[i]:ours.prim_off[i + 1]]
        c = ours.coefs[ours.prim_off[i]:ours.prim_off[i + 1]]
        assert np.array_equal(e, g["exps"])
        assert np.allclose(c, g["coefs"], rtol=1e-14, atol=0)


def test_water_cluster_is_seeded_and_sane():
    a = water_cluster(16)
    b = water_cluster(16)
    assert a == b and len(a) == 48
    assert water_cluster(1)[0] == ("O", (0.0, 0.0, 0.2217))
    pos = np.array([p for _, p in a])
    d = np.linalg.norm(pos[:, None] - pos[None], axis=-1) + np.eye(len(a)) * 1e9
    assert d.min() > 1.0  # bohr


def test_default_options_are_the_documented_ones():
    # the option defaults of include/hfg.h, read through the C ABI (host
    # code only: no device is touched)
    if not os.path.exists(hl.library_path()):
        pytest.skip("libhfg.so not built")
    import ctypes
    L = hl.load_library()
    j = hl.JKOptions()
    L.hfg_jk_opts_default(ctypes.byref(j))
    assert (j.schwarz_threshold, j.prim_threshold, j.precision, j.deterministic, j.tile) == (1e-12, 0.0, 0, 0, 0)
    a = hl.AutotuneOptions()
    L.hfg_autotune_opts_default(ctypes.byref(a))
    assert list(a.fp32_thresholds[:a.n_fp32]) == [1e-7, 1e-6, 1e-5, 1e-4]
    assert list(a.prim_thresholds[:a.n_prim]) == [1e-15, 1e-14, 1e-13]
    assert list(a.tiles[:a.n_tile]) == [8, 16, 32, 256]
    assert a.max_energy_error == 5e-9 and a.repeats == 2
