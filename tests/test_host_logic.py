"""Host-side logic that needs no GPU: the seeded job stream's mix, and the
convergence tolerances derived from an energy tolerance."""
import ctypes

import numpy as np

from hfgpu import lib as L
from hfgpu.serve import BASES, make_stream


def test_job_stream_mix_and_determinism():
    jobs = make_stream(2000, rate=50.0, max_waters=48, seed=4242)
    assert jobs == make_stream(2000, rate=50.0, max_waters=48, seed=4242)
    t = np.array([j["arrival_s"] for j in jobs])
    assert np.all(np.diff(t) > 0) and abs(len(jobs) / t[-1] - 50.0) < 5.0  # Poisson arrivals at the rate
    w = np.array([j["waters"] for j in jobs])
    assert w.min() == 1 and w.max() == 48
    counts = {b: sum(j["basis"] == b for j in jobs) for b in BASES}
    assert all(550 < c < 790 for c in counts.values())  # uniform over the three bases
    uhf = [j for j in jobs if j["uhf"]]
    assert 150 < len(uhf) < 250  # 10 % UHF
    assert all(j["multiplicity"] == 2 and j["charge"] in (-1, 1) for j in uhf)
    assert all(j["charge"] == 0 and j["multiplicity"] == 1 for j in jobs if not j["uhf"])
    assert all(j["spherical"] == (j["basis"] == "cc-pvdz") for j in jobs)


def test_convergence_from_tol_matches_the_c_defaults():
    # hfg_scf_opts_default derives its criteria from 1e-10 as hf-rs does
    # (src/scf.rs:393-399); the Python helper must give the same numbers
    o = L.SCFOptions()
    L.load_library().hfg_scf_opts_default(ctypes.byref(o))
    assert L.convergence_from_tol(1e-10) == (o.energy_tol, o.residual_tol, o.density_tol)
    assert o.incremental_tol == 1e-12 and o.rebuild_every == 8 and o.refine_iters == 2 and o.diis_size == 8


def test_generated_recursions_match_the_generator():
    # eri_gen.cuh is the output of gen_eri.py for s, p, d (the Makefile
    # regenerates it when the generator changes); the committed file must be
    # exactly what the generator produces
    import importlib.util
    import os
    csrc = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "hf-rs_b200", "csrc")
    spec = importlib.util.spec_from_file_location("gen_eri", os.path.join(csrc, "gen_eri.py"))
    gen = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(gen)
    text, stats = gen.render(2)
    assert text == open(os.path.join(csrc, "eri_gen.cuh")).read()
    # every four-centre class the J/K kernels are built for is generated
    classes = {s[:4] for s in stats}
    for la in range(3):
        for lb in range(la + 1):
            for lc in range(3):
                for ld in range(lc + 1):
                    assert (la, lb, lc, ld) in classes
