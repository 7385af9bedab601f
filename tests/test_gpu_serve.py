"""Serving loop: every job's result is the same alone and in a mix, and
admission respects the device-memory budget."""
import pytest

from hfgpu.serve import build_inputs, make_stream, run_stream, summarize

pytestmark = pytest.mark.gpu


def test_results_same_alone_and_in_the_mix():
    jobs = make_stream(12, rate=1000.0, max_waters=4, seed=7)
    inputs = build_inputs(jobs)
    alone, _ = run_stream(jobs, slots=1, budget_bytes=8 << 30, honour_arrivals=False, inputs=inputs)
    mixed, span = run_stream(jobs, slots=6, budget_bytes=8 << 30, honour_arrivals=False, inputs=inputs)
    assert all(r["status"] == 0 and r["converged"] for r in alone + mixed)
    for a, m in zip(alone, mixed):
        assert abs(a["energy"] - m["energy"]) < 1e-10, (a["tag"], a["energy"], m["energy"])
    s = summarize(mixed, span)
    assert s["jobs"] == 12 and s["failed"] == 0


def test_admission_by_footprint_limits_concurrency():
    jobs = make_stream(6, rate=1000.0, max_waters=3, seed=9)
    inputs = build_inputs(jobs)
    res, _ = run_stream(jobs, slots=6, budget_bytes=24 << 20, honour_arrivals=False, inputs=inputs)
    # with a 24 MiB budget the jobs (each several MiB) cannot all run at once:
    # some job must start only after another ended
    assert any(b["start_ms"] >= a["end_ms"] for a in res for b in res if a is not b)
    assert all(r["status"] == 0 for r in res)


def test_mixed_jobs_same_alone_and_in_the_mix_with_arrivals():
    # the served precision policy (mixed J/K with FP64 refinement, here for
    # every job) and arrivals honoured: jobs enter while others are running,
    # and each converged energy equals the job's energy run alone
    from hfgpu.serve import MIXED
    jobs = make_stream(10, rate=25.0, max_waters=6, seed=11)
    inputs = build_inputs(jobs)
    alone, _ = run_stream(jobs, slots=1, budget_bytes=8 << 30, honour_arrivals=False, inputs=inputs, jk=MIXED,
                          mixed_min_ao=0)
    mixed, span = run_stream(jobs, slots=4, budget_bytes=8 << 30, honour_arrivals=True, inputs=inputs, jk=MIXED,
                             mixed_min_ao=0)
    assert all(r["status"] == 0 and r["converged"] for r in alone + mixed)
    for a, m in zip(alone, mixed):
        assert abs(a["energy"] - m["energy"]) < 1e-9, (a["tag"], a["energy"], m["energy"])
    # some job was submitted while another was already running
    assert any(o["start_ms"] < m["submit_ms"] < o["end_ms"] for m in mixed for o in mixed if o is not m)


def test_batched_fock_builds_match_unbatched_jobs():
    # RHF jobs below the size bound hand their Fock builds to the server's
    # batcher, which runs the builds of the running jobs as one batched
    # build; every converged energy equals the job run alone, unbatched
    jobs = make_stream(12, rate=1000.0, max_waters=5, seed=23)
    inputs = build_inputs(jobs)
    alone, _ = run_stream(jobs, slots=1, budget_bytes=8 << 30, honour_arrivals=False, inputs=inputs, batch_max_ao=0)
    stats = {}
    batched, _ = run_stream(jobs, slots=8, budget_bytes=8 << 30, honour_arrivals=False, inputs=inputs,
                            batch_max_ao=1 << 20, batch_window_us=2000.0, stats_out=stats)
    assert all(r["status"] == 0 and r["converged"] for r in alone + batched)
    for a, m in zip(alone, batched):
        assert abs(a["energy"] - m["energy"]) < 1e-9, (a["tag"], a["energy"], m["energy"])
    # builds of different jobs shared batches
    assert stats["batches"] > 0 and stats["batched_builds"] > stats["batches"], stats
