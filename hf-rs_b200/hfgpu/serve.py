"""Seeded SCF job streams and a driver that feeds them to hfg_server.

The stream restates the served workload: jobs arrive as a Poisson process of
rate `rate` (jobs/s); each is a water cluster (H2O)_n built like the bench
clusters with n uniform in {1..max_waters}, in a basis drawn uniformly from
STO-3G, 6-31G* and cc-pVDZ (cc-pVDZ in its real spherical AO space, the
others Cartesian, as hf-rs's BasisKind::default_for_name picks), and 10% of
the jobs are UHF doublets with charge +1 or -1.
"""
import time

import numpy as np

from .basis import CartesianBasis
from .clusters import water_cluster
from .lib import JKOptions, Server

BASES = ["sto-3g", "6-31g*", "cc-pvdz"]


def make_stream(njobs, rate, max_waters=48, seed=4242):
    rng = np.random.default_rng(seed)
    t = np.cumsum(rng.exponential(1.0 / rate, size=njobs))
    jobs = []
    for i in range(njobs):
        nw = int(rng.integers(1, max_waters + 1))
        basis = BASES[int(rng.integers(0, 3))]
        uhf = bool(rng.random() < 0.1)
        charge = int(rng.choice([-1, 1])) if uhf else 0
        jobs.append({"tag": i, "arrival_s": float(t[i]), "waters": nw, "basis": basis, "uhf": uhf,
                     "charge": charge, "multiplicity": 2 if uhf else 1, "spherical": basis == "cc-pvdz",
                     "seed": 1000 + i})
    return jobs


def build_inputs(jobs):
    return {j["tag"]: CartesianBasis.build(water_cluster(j["waters"], seed=j["seed"]), j["basis"]) for j in jobs}


def run_stream(jobs, slots, budget_bytes, jk=None, tol=1e-10, honour_arrivals=True, inputs=None, device=0,
               mixed_min_ao=None, batch_max_ao=None, batch_window_us=300.0, stats_out=None):
    """Submit jobs at their arrival times; return per-job results (latency =
    end - arrival) and the makespan.  batch_max_ao: the server's cross-job
    Fock-build batching bound (0: off; None: the server default); stats_out,
    when a dict, receives the server's batch statistics."""
    inputs = inputs or build_inputs(jobs)
    srv = Server(device=device, slots=slots, hbm_budget_bytes=budget_bytes, mixed_min_ao=mixed_min_ao,
                 batch_max_ao=batch_max_ao, batch_window_us=batch_window_us)
    t0 = time.time()
    submit_wall = {}
    results = []
    for j in jobs:
        if honour_arrivals:
            dt = j["arrival_s"] - (time.time() - t0)
            if dt > 0:
                time.sleep(dt)
        submit_wall[j["tag"]] = time.time() - t0
        srv.submit(inputs[j["tag"]], charge=j["charge"], multiplicity=j["multiplicity"], uhf=j["uhf"],
                   spherical=j["spherical"], tol=tol, jk=jk, tag=j["tag"])
        results.extend(srv.poll(wait=False))
    while len(results) < len(jobs):
        got = srv.poll(wait=True)
        if not got:
            break
        results.extend(got)
    makespan = time.time() - t0
    if stats_out is not None:
        stats_out.update(srv.batch_stats())
    srv.close()
    by_tag = {r["tag"]: r for r in results}
    out = []
    for j in jobs:
        r = dict(by_tag[j["tag"]])
        r.update(j)
        # server clock: submit_ms is when the job entered the queue (its arrival)
        r["latency_s"] = (r["end_ms"] - r["submit_ms"]) / 1000.0
        out.append(r)
    return out, makespan


def summarize(results, makespan):
    lat = np.array([r["latency_s"] for r in results])
    return {"jobs": len(results), "jobs_per_s": len(results) / makespan, "makespan_s": makespan,
            "p50_s": float(np.percentile(lat, 50)), "p99_s": float(np.percentile(lat, 99)),
            "converged": int(sum(r["converged"] for r in results)),
            "failed": int(sum(r["status"] not in (0,) for r in results))}


# the mixed form for whole SCFs (served jobs, the SCF bench leg): FP32
# below Q_ab Q_cd < 3e-5, primitive screening 1e-13.  Swept on (H2O)32 and
# (H2O)48 cc-pVDZ SCFs it keeps the FP64 iteration count and is fastest;
# larger FP32 thresholds win single builds but cost SCF iterations (1e-4:
# 21-33 iterations instead of 18).  Build energy error ~2e-9 Eh at (H2O)64;
# the FP64 refinement removes it.
MIXED = JKOptions.make(prim=1e-13, mixed=3e-5)
