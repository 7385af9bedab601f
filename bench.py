"""Benchmark: direct Fock builds per second, (H2O)_64 cc-pVDZ, on B200.

A step is one Fock build: the direct J and K of a closed-shell density
(hfg_jk_device: Schwarz-screened four-centre ERIs digested into J/K, plus
the symmetrisation epilogue) for the synthetic water cluster (H2O)_64 in
cc-pVDZ (1600 Cartesian functions).  `value` is the mixed-precision build
(FP32 for shell quartets with Q_ab Q_cd below the FP32 threshold, FP64
accumulation) with the density resident in HBM; the same builds in plain
FP64 are reported beside it.  `e2e` is the same build through the C ABI
with host buffers (hfg_jk): density host->device, J and K device->host.

Under torchrun the N ranks share one Fock build (strong scaling): each rank
runs a cost-balanced shard of every launch's work queue and one NCCL
all-reduce sums J and K; the step time is the maximum over ranks.

--impl reference times the CPU restatement of hf-rs's path (the oracle:
the same screened shell quartets, McMurchie-Davidson integrals, contract_jk
digestion) on this host's cores on a bounded sample of the same build and
scales it to whole builds by the share of McMurchie-Davidson work sampled.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "hf-rs_b200"))

METRIC = "fock_builds_per_s"
UNIT = "Fock builds/s"


def workload(waters, n_ao):
    return "(H2O)%d cc-pVDZ direct RHF Fock build (J+K), %d Cartesian AOs, Schwarz 1e-12" % (waters, n_ao)
SCHWARZ = 1e-12
PRIM = 1e-15
TUNE_BUDGET = 5e-9


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--waters", type=int, default=64)
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-serve", action="store_true")
    ap.add_argument("--serve-jobs", type=int, default=16)
    ap.add_argument("--serve-max-waters", type=int, default=48)
    ap.add_argument("--df-waters", type=int, default=128,
                    help="also time DF J/K on (H2O)_n (0: skip; default the DF-RHF workload, (H2O)128)")
    ap.add_argument("--scf-waters", type=int, default=-1,
                    help="full SCF in FP64 and in the mixed form on (H2O)_n (-1: --waters, 0: skip)")
    ap.add_argument("--jk-only", action="store_true",
                    help="only the mixed builds (fixed thresholds, no autotuning, no other legs): for profilers")
    return ap.parse_args()


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


class Clocks:
    """nvidia-smi sampling during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), "--query-gpu=" + self.Q,
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            out, _ = self.proc.communicate(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
            out, _ = self.proc.communicate()
        rows = [r.split(",") for r in out.strip().splitlines() if r.count(",") >= 8]
        if not rows:
            return None
        sm = [float(r[1]) for r in rows if r[1].strip().replace(".", "").isdigit()]
        mx = max(float(r[2]) for r in rows)
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4) if r[5 + k].strip() == "Active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": reasons,
                "samples": len(rows)}


def timed(torch, stream, fn, steps, flush=None):
    """Per-step device time (ms) with CUDA events on `stream`."""
    times = []
    for _ in range(steps):
        if flush is not None:
            flush()
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record(stream)
        fn()
        b.record(stream)
        b.synchronize()
        times.append(a.elapsed_time(b))
    return times


class CpuWorkload:
    """The oracle (CPU restatement of hf-rs) on the same build: the screened
    shell quartets, their McMurchie-Davidson work, and timed samples of bra
    shell-pair rows."""

    W = {(0, 0, 0, 0): 61, (1, 0, 0, 0): 126, (1, 0, 1, 0): 333, (1, 1, 0, 0): 327, (1, 1, 1, 0): 1072,
         (1, 1, 1, 1): 3916, (2, 0, 0, 0): 256, (2, 0, 1, 0): 771, (2, 0, 1, 1): 2683, (2, 0, 2, 0): 1872,
         (2, 1, 0, 0): 747, (2, 1, 1, 0): 2647, (2, 1, 1, 1): 9994, (2, 1, 2, 0): 6751, (2, 1, 2, 1): 25570,
         (2, 2, 0, 0): 1776, (2, 2, 1, 0): 6607, (2, 2, 1, 1): 25354, (2, 2, 2, 0): 16978, (2, 2, 2, 1): 64681,
         (2, 2, 2, 2): 162643}

    def __init__(self, atoms, threads):
        import numpy as np
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import oracle as O
        self.np, self.O = np, O
        os.environ["ORACLE_THREADS"] = str(threads)
        self.threads = threads
        self.basis = O.build_basis(atoms, O.load_basis("cc-pvdz"))
        self.fb = O.FlatBasis(self.basis)
        shells = O.shell_ranges(self.basis)
        L = np.array([sum(self.basis[s]["l"]) for s, _ in shells])
        K = np.array([len(self.basis[s]["exps"]) for s, _ in shells])
        self.Q = O.schwarz(self.basis)
        a_idx, b_idx = [], []
        for a in range(len(shells)):
            for b in range(a + 1):
                a_idx.append(a)
                b_idx.append(b)
        pa, pb = np.array(a_idx), np.array(b_idx)
        self.code = np.maximum(L[pa], L[pb]) * 3 + np.minimum(L[pa], L[pb])
        self.npp = (K[pa] * K[pb]).astype(np.float64)
        self.wtab = np.zeros((9, 9))
        for (a, b, c, d), v in self.W.items():
            self.wtab[a * 3 + b, c * 3 + d] = v
            self.wtab[c * 3 + d, a * 3 + b] = v
        self.total = self._total_work()
        n = len(self.basis)
        rng = np.random.default_rng(7)
        P = rng.standard_normal((n, n)) * 0.1
        self.P = P + P.T
        self.rng = rng
        self.rate = None

    def _total_work(self):
        # sum over unique quartets ij >= kl with Q_ij Q_kl > thr of
        # npp_ij npp_kl W(class): half the ordered double sum plus half the
        # diagonal, the double sum by sorted prefixes per angular class.
        np = self.np
        tot = 0.0
        for c in range(9):
            sel = np.nonzero(self.code == c)[0]
            if len(sel) == 0:
                continue
            o = sel[np.argsort(-self.Q[sel], kind="stable")]
            qs, cum = self.Q[o], np.concatenate([[0.0], np.cumsum(self.npp[o])])
            # count of kets with Q_ij * q > thr
            cnt = np.searchsorted(-qs, -(SCHWARZ / np.maximum(self.Q, 1e-300)), side="left")
            # exact predicate fix-up at the boundary
            for _ in range(2):
                over = (cnt < len(qs))
                nxt = np.where(over, qs[np.minimum(cnt, len(qs) - 1)] * self.Q > SCHWARZ, False)
                cnt = cnt + nxt
                under = cnt > 0
                prv = np.where(under, qs[np.maximum(cnt - 1, 0)] * self.Q <= SCHWARZ, False)
                cnt = cnt - prv
            tot += float(np.sum(self.npp * cum[cnt] * self.wtab[self.code, c]))
        diag = self.Q * self.Q > SCHWARZ
        tot += float(np.sum((self.npp ** 2 * self.wtab[self.code, self.code])[diag]))
        return 0.5 * tot

    def row_work(self, ij):
        np = self.np
        ks = np.nonzero(self.Q[ij] * self.Q[:ij + 1] > SCHWARZ)[0]
        return float(np.sum(self.npp[ij] * self.npp[ks] * self.wtab[self.code[ij], self.code[ks]]))

    def sample(self, target_s):
        """Time the oracle on random rows worth ~target_s seconds; returns
        (seconds, sampled work, rows)."""
        np = self.np
        if self.rate is None:
            probe = self.rng.permutation(len(self.Q))[:8]
            t0 = time.time()
            self.O.direct_jk(self.basis, self.P, [self.P], SCHWARZ, rows=probe, fb=self.fb)
            self.rate = max(sum(self.row_work(r) for r in probe) / max(time.time() - t0, 1e-3), 1.0)
        rows, w = [], 0.0
        for r in self.rng.permutation(len(self.Q)):
            rows.append(int(r))
            w += self.row_work(r)
            if w / self.rate >= target_s or len(rows) >= 200000:
                break
        t0 = time.time()
        self.O.direct_jk(self.basis, self.P, [self.P], SCHWARZ, rows=np.array(rows), fb=self.fb)
        dt = time.time() - t0
        self.rate = w / dt
        return dt, w, len(rows)

    def builds_per_s(self, target_s):
        dt, w, nrows = self.sample(target_s)
        return (w / self.total) / dt, dt, nrows


def run_reference(args):
    rank, world, local = dist_env()
    if rank != 0:
        return
    from hfgpu.clusters import water_cluster
    threads = os.cpu_count() or 1
    cw = CpuWorkload(water_cluster(args.waters), threads)
    per_step = min(15.0, 150.0 / max(1, args.steps + args.warmup))
    vals, rows = [], 0
    for s in range(args.warmup + args.steps):
        v, dt, nrows = cw.builds_per_s(per_step)
        if s >= args.warmup:
            vals.append(v)
            rows = nrows
    v = statistics.median(vals)
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1000.0 / v, "higher_is_better": True, "scaling": "strong",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": workload(args.waters, 25 * args.waters) + ", CPU restatement of hf-rs (McMurchie-Davidson, contract_jk)",
                       "parallelism": "openmp-%d" % threads},
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": threads, "kind": "port",
                             "sample": "%d random bra shell-pair rows per step (~%.0f s of CPU work), scaled by "
                                       "sampled / total McMurchie-Davidson flops (%.3e per build)"
                                       % (rows, per_step, cw.total)},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def run_ours(args):
    import numpy as np
    import torch

    from hfgpu import CartesianBasis, Context, JKOptions
    from hfgpu.clusters import water_cluster
    from hfgpu.lib import fma_peak_tflops
    from hfgpu.parallel import ShardedJK

    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=600))
    dev = torch.device("cuda", local)
    # one non-default stream shared by torch and the library, so the CUDA
    # events below bracket the library's kernels
    stream = torch.cuda.Stream(device=dev)
    torch.cuda.set_stream(stream)
    atoms = water_cluster(args.waters)
    basis = CartesianBasis.build(atoms, "cc-pvdz")
    n = basis.n
    ctx = Context(basis, device=local, stream=stream.cuda_stream)
    # a physical density: three SCF iterations from the SAD guess (FP64 J/K)
    scf = ctx.scf(spherical=True, tol=1e-10, max_iter=3, jk=JKOptions.make(schwarz=SCHWARZ, prim=1e-15),
                  want=("P",))
    Ph = np.ascontiguousarray(scf["P"][0])
    P = torch.from_numpy(Ph).to(dev)
    J = torch.empty((n, n), dtype=torch.float64, device=dev)
    K = torch.empty((n, n), dtype=torch.float64, device=dev)
    flush_buf = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)

    def flush():
        flush_buf.zero_()

    def barrier():
        torch.cuda.synchronize()
        if world > 1:
            torch.distributed.barrier()
        torch.cuda.synchronize()

    torch.cuda.synchronize()
    if args.jk_only:
        # profiler runs: the mixed builds alone, with the options the
        # autotuner picks on (H2O)64
        opt = JKOptions.make(schwarz=SCHWARZ, prim=1e-13, mixed=1e-4, tile=16)
        last = args.warmup + args.steps - 1
        for i in range(last + 1):
            if i == last:
                # the last build is an NVTX range "jk_build" (ncu --nvtx-include "jk_build/")
                torch.cuda.synchronize()
                torch.cuda.nvtx.range_push("jk_build")
            ctx.jk_device(P.data_ptr(), P.data_ptr(), J.data_ptr(), K.data_ptr(), 1, opt)
            if i == last:
                torch.cuda.synchronize()
                torch.cuda.nvtx.range_pop()
        torch.cuda.synchronize()
        if rank == 0:
            print(json.dumps({"jk_only": True, "waters": args.waters, "builds": args.warmup + args.steps}))
        return
    # mixed form chosen by the autotuner (FP32 threshold 1e-7..1e-4, primitive
    # threshold 1e-15..1e-13, build energy error within 5e-9 Eh of the plain
    # FP64 build); untimed
    opt_mixed, tune = ctx.autotune(P.data_ptr(), P.data_ptr(), base=JKOptions.make(schwarz=SCHWARZ),
                                   max_energy_error=TUNE_BUDGET, repeats=1)
    if world > 1:
        # every rank must run the same plan: rank 0's choice
        ch = torch.tensor([opt_mixed.mixed_threshold, opt_mixed.prim_threshold, opt_mixed.tile],
                          dtype=torch.float64, device=dev)
        torch.distributed.broadcast(ch, 0)
        opt_mixed = JKOptions.make(schwarz=SCHWARZ, prim=float(ch[1]), mixed=float(ch[0]), tile=int(ch[2]))
    opt_plain = JKOptions.make(schwarz=SCHWARZ)            # the reference's arithmetic in FP64
    opt_fp64 = JKOptions.make(schwarz=SCHWARZ, prim=PRIM)  # FP64 with primitive screening

    def build(opt):
        if world == 1:
            return lambda: ctx.jk_device(P.data_ptr(), P.data_ptr(), J.data_ptr(), K.data_ptr(), 1, opt)
        # N GPUs: each rank builds its cost-balanced shard, then one NCCL
        # all-reduce of J and K (strong scaling of one Fock build)
        sharded = ShardedJK(rank, world, ctx=ctx, opts=opt)
        return lambda: sharded(P, P, J, K)

    # warm-up (plans are built on first use)
    for _ in range(args.warmup):
        build(opt_mixed)()
    build(opt_fp64)()
    torch.cuda.synchronize()
    build(opt_mixed)()
    stats_mixed = ctx.last_stats()
    Jm, Km = J.cpu().numpy().copy(), K.cpu().numpy().copy()
    build(opt_fp64)()
    stats_fp64 = ctx.last_stats()
    build(opt_plain)()
    stats_plain = ctx.last_stats()
    Jf, Kf = J.cpu().numpy().copy(), K.cpu().numpy().copy()
    jk_diff = float(max(np.max(np.abs(Jm - Jf)), np.max(np.abs(Km - Kf))))
    dE_build = float(0.5 * np.sum(Ph * (Jm - Jf)) - 0.25 * np.sum(Ph * (Km - Kf)))

    clocks = Clocks(local)
    barrier()
    clocks.start()
    t_mixed = timed(torch, stream, build(opt_mixed), args.steps, flush)
    barrier()
    t_fp64 = timed(torch, stream, build(opt_fp64), args.steps, flush)
    barrier()
    t_plain = timed(torch, stream, build(opt_plain), args.steps, flush)
    barrier()
    ck = clocks.stop()

    def max_over_ranks(x):
        if world == 1:
            return x
        t = torch.tensor([x], dtype=torch.float64, device=dev)
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        return float(t.item())

    tot_mixed = max_over_ranks(sum(t_mixed))
    tot_fp64 = max_over_ranks(sum(t_fp64))
    tot_plain = max_over_ranks(sum(t_plain))
    # one Fock build per step, shared by all ranks
    value = args.steps / (tot_mixed / 1000.0)
    value_fp64 = args.steps / (tot_fp64 / 1000.0)
    value_plain = args.steps / (tot_plain / 1000.0)

    e2e = None
    if not args.no_e2e:
        Phost = torch.from_numpy(Ph).pin_memory()
        Jh = torch.empty((n, n), dtype=torch.float64).pin_memory()
        Kh = torch.empty((n, n), dtype=torch.float64).pin_memory()
        import ctypes
        lib = ctx.lib
        DP = ctypes.POINTER(ctypes.c_double)

        sharded_e2e = build(opt_mixed)

        def e2e_step():
            if world == 1:
                # the C-ABI host entry point: copies in, build, copies out
                rc = lib.hfg_jk(ctx.h, ctypes.byref(opt_mixed), 1, ctypes.cast(Phost.data_ptr(), DP),
                                ctypes.cast(Phost.data_ptr(), DP), ctypes.cast(Jh.data_ptr(), DP),
                                ctypes.cast(Kh.data_ptr(), DP))
                if rc != 0:
                    raise RuntimeError(lib.hfg_last_error(ctx.h).decode())
            else:
                P.copy_(Phost, non_blocking=True)
                sharded_e2e()
                Jh.copy_(J, non_blocking=True)
                Kh.copy_(K, non_blocking=True)

        e2e_step()
        barrier()
        t_e2e = timed(torch, stream, e2e_step, args.steps, flush)
        barrier()
        tot_e2e = max_over_ranks(sum(t_e2e))
        e2e = {"value": args.steps / (tot_e2e / 1000.0), "unit": UNIT, "h2d_bytes_per_step": n * n * 8,
               "d2h_bytes_per_step": 2 * n * n * 8, "ms_per_step": tot_e2e / args.steps}

    if rank != 0:
        if world > 1:
            torch.distributed.destroy_process_group()
        return

    p64 = fma_peak_tflops(local, False)
    p32 = fma_peak_tflops(local, True)
    t_step = tot_mixed / args.steps / 1000.0
    pipe_frac = (stats_mixed["wmd_flops_fp64"] / (p64 * 1e12) + stats_mixed["wmd_flops_fp32"] / (p32 * 1e12)) / t_step
    pipe_frac /= world  # against the pipes of all N GPUs
    # DRAM bytes of one mixed build of (H2O)64 from the committed ncu summary
    # (dominated by register spills of the L >= 5 classes); other sizes
    # have no capture
    traffic = None
    prof = os.path.join(ROOT, "profiles", "jk_dram_h2o64_mixed.md")
    if os.path.exists(prof) and args.waters == 64:
        for ln in open(prof):
            if ln.startswith("traffic_bytes_per_mixed_build_h2o64:"):
                traffic = float(ln.split(":")[1])
    roofline = {"bound": "fp64", "achieved": pipe_frac * p64, "peak": p64, "unit": "TFLOP/s", "frac": pipe_frac,
                "traffic": traffic,
                "traffic_source": "ncu dram__bytes_read+write summed over the 42 launches of one mixed build "
                                  "of (H2O)64 (profiles/jk_dram_h2o64_mixed.md); mostly register spills of the "
                                  "L>=5 classes",
                "peak_source": "measured FMA chains on this device (hfg_fma_peak); FP32 work weighted by the "
                               "measured FP32 peak %.1f TFLOP/s" % p32,
                "work_unit": "McMurchie-Davidson flops per evaluated primitive quartet (hf-rs loops), "
                             "%.3e FP64 + %.3e FP32 per build" % (stats_mixed["wmd_flops_fp64"],
                                                                   stats_mixed["wmd_flops_fp32"])}
    cpu = None
    if world == 1 and not args.no_cpu:
        try:
            cw = CpuWorkload(atoms, os.cpu_count() or 1)
            v, dt, nrows = cw.builds_per_s(15.0)
            cpu = {"value": v, "unit": UNIT, "cores": os.cpu_count() or 1, "kind": "port",
                   "sample": "%d random bra shell-pair rows of the same build (%.1f s), scaled by sampled / "
                             "total McMurchie-Davidson flops (%.3e per build)" % (nrows, dt, cw.total)}
        except Exception as exc:  # the CPU leg must not hide the GPU result
            cpu = {"unavailable": str(exc)[:200]}
    serving = None
    if world == 1 and not args.no_serve:
        serving = measure_serving(args)
    dfres = None
    if world == 1 and args.df_waters > 0:
        dfres = measure_df(args, torch)
    scfres = None
    scf_waters = args.waters if args.scf_waters < 0 else args.scf_waters
    if world == 1 and scf_waters > 0:
        from hfgpu.serve import MIXED
        scfres = measure_scf(scf_waters, ctx if scf_waters == args.waters else None, MIXED)
    mt, pt, tl = opt_mixed.mixed_threshold, opt_mixed.prim_threshold, opt_mixed.tile or 64
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": tot_mixed / args.steps, "higher_is_better": True,
            "scaling": "strong", "vs_baseline": None, "dtype": "f64/f32-mixed", "data": "synthetic",
            "config": {"workload": workload(args.waters, n) + ", mixed precision (FP32 below Q_ab*Q_cd < %g, "
                                   "primitive screening %g, quartet tile %d; autotuned)" % (mt, pt, tl),
                       "n_ao": n, "waters": args.waters, "parallelism": ("%d shards + NCCL all-reduce of J, K" % world) if world > 1 else "single",
                       "density": "SCF density after 3 iterations from the SAD guess",
                       "l2": "flushed (256 MB write) before every timed step"},
            "mixed_energy_error_per_build": dE_build,
            "jk_max_abs_diff_mixed_vs_plain_fp64": jk_diff,
            "fp64_plain": {"value": value_plain, "unit": UNIT, "ms_per_step": tot_plain / args.steps,
                           "form": "FP64, Schwarz screening only (the reference's arithmetic)",
                           "wmd_flops": stats_plain["wmd_flops_fp64"]},
            "fp64": {"value": value_fp64, "unit": UNIT, "ms_per_step": tot_fp64 / args.steps,
                     "form": "FP64 with primitive screening %g" % PRIM, "wmd_flops": stats_fp64["wmd_flops_fp64"]},
            "mixed_over_fp64_plain": value / value_plain, "mixed_over_fp64": value / value_fp64,
            "autotune": {"chosen": {"fp32_threshold": mt, "prim_threshold": pt, "tile": tl}, "budget_eh": TUNE_BUDGET,
                         "candidates": tune["candidates"]},
            "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e, "clocks": ck, "serving": serving, "df": dfres,
            "scf": scfres,
            # per build: the plan's J/K launches plus two symmetrisation kernels;
            # timed: K mixed, K FP64, K plain FP64 and K end-to-end mixed builds
            "gpu_launches": args.steps * (stats_mixed["launches"] + 2) * (1 if e2e is None else 2)
            + args.steps * (stats_fp64["launches"] + 2) + args.steps * (stats_plain["launches"] + 2)}
    # the figures a reader needs first, last on the line (a log tail keeps them)
    line["summary"] = {
        "mixed_ms": round(tot_mixed / args.steps, 2), "fp64_ms": round(tot_fp64 / args.steps, 2),
        "fp64_plain_ms": round(tot_plain / args.steps, 2),
        "mixed_over_fp64_plain": round(value / value_plain, 3), "mixed_over_fp64": round(value / value_fp64, 3),
        "roofline_frac": round(pipe_frac, 4), "e2e_builds_per_s": None if e2e is None else round(e2e["value"], 4),
        "serving_jobs_per_s_ratio": None if serving is None else round(serving["jobs_per_s_ratio"], 3),
        "serving_p50_p99_s": None if serving is None else [round(serving["served_mixed_8_slots"]["p50_s"], 3),
                                                           round(serving["served_mixed_8_slots"]["p99_s"], 3)],
        "scf_mixed_minus_fp64_eh": None if scfres is None else scfres["mixed_minus_fp64_eh"],
        "scf_before_refinement_minus_fp64_eh": None if scfres is None else scfres["before_refinement_minus_fp64_eh"],
        "df_k_tflops": None if dfres is None else dfres.get("k_tflops_best"),
        "df_waters": None if dfres is None else dfres.get("waters"),
        "df_bf16_tensor_frac": None if dfres is None else dfres.get("bf16", {}).get("tensor_peak_frac")}
    print(json.dumps(line), flush=True)
    if world > 1:
        torch.distributed.destroy_process_group()


def measure_serving(args):
    """Served SCF stream vs sequential plain solves on a bounded sample of the
    seeded job stream (first `serve_jobs` jobs, waters uniform in
    {1..serve_max_waters}, bases uniform over STO-3G / 6-31G* / cc-pVDZ, 10%
    UHF doublets).  Sequential: one FP64 solve at a time, each with its own
    builds.  Served: 8 slots, mixed precision with FP64 refinement, all jobs
    submitted at once (an arrival rate above capacity); jobs under 256 basis
    functions run FP64, and their RHF Fock builds are batched across the
    running jobs."""
    from hfgpu.serve import MIXED, build_inputs, make_stream, run_stream, summarize
    jobs = make_stream(args.serve_jobs, rate=1000.0, max_waters=args.serve_max_waters, seed=4242)
    inputs = build_inputs(jobs)
    seq, span_seq = run_stream(jobs, slots=1, budget_bytes=120 << 30, honour_arrivals=False, inputs=inputs,
                               batch_max_ao=0)
    batch = {}
    srv, span_srv = run_stream(jobs, slots=8, budget_bytes=120 << 30, honour_arrivals=False, inputs=inputs,
                               jk=MIXED, mixed_min_ao=256, batch_max_ao=256, stats_out=batch)
    a, b = summarize(seq, span_seq), summarize(srv, span_srv)
    de = max(abs(x["energy"] - y["energy"]) for x, y in zip(seq, srv) if x["status"] == 0 and y["status"] == 0)
    return {"sample": "%d jobs, waters 1..%d, STO-3G/6-31G*/cc-pVDZ, 10%% UHF" % (len(jobs), args.serve_max_waters),
            "sequential_fp64": a, "served_mixed_8_slots": b, "jobs_per_s_ratio": b["jobs_per_s"] / a["jobs_per_s"],
            "batched_fock_builds": batch, "max_abs_dE_served_vs_sequential": de}


def measure_scf(waters, ctx, opt_mixed):
    """Full SCF of (H2O)_n cc-pVDZ (spherical AO space, tol 1e-10, SAD start,
    CDIIS): FP64 builds with primitive screening 1e-15, and the mixed form
    tuned for whole SCFs (hfgpu.serve.MIXED; incremental builds, FP64
    refinement of at least two builds).  Reports both energies, the mixed
    energy's error and the error before refinement, iterations and wall
    times (basis to converged energy)."""
    from hfgpu import CartesianBasis, Context, JKOptions
    from hfgpu.clusters import water_cluster
    own = ctx is None
    if own:
        ctx = Context(CartesianBasis.build(water_cluster(waters), "cc-pvdz"))
    out = {"waters": waters, "n_ao": ctx.n, "tol": 1e-10}
    t0 = time.time()
    r64 = ctx.scf(spherical=True, tol=1e-10, jk=JKOptions.make(schwarz=SCHWARZ, prim=PRIM), want=())
    t64 = time.time() - t0
    t0 = time.time()
    rmx = ctx.scf(spherical=True, tol=1e-10, jk=opt_mixed, want=())
    tmx = time.time() - t0
    out["fp64"] = {"energy": r64["energy"], "iterations": r64["iterations"], "converged": bool(r64["converged"]),
                   "wall_s": t64, "builds": r64["fock_builds_fp64"]}
    out["mixed"] = {"energy": rmx["energy"], "energy_before_refinement": rmx["energy_before_refinement"],
                    "iterations": rmx["iterations"], "converged": bool(rmx["converged"]), "wall_s": tmx,
                    "builds_mixed": rmx["fock_builds_mixed"], "builds_fp64": rmx["fock_builds_fp64"],
                    "builds_incremental": rmx["fock_builds_incremental"],
                    "fp32_threshold": opt_mixed.mixed_threshold, "prim_threshold": opt_mixed.prim_threshold}
    out["mixed_minus_fp64_eh"] = rmx["energy"] - r64["energy"]
    out["before_refinement_minus_fp64_eh"] = rmx["energy_before_refinement"] - r64["energy"]
    out["speedup_wall"] = t64 / tmx
    if own:
        ctx.close()
    return out


def measure_df(args, torch):
    """DF J/K (hfg_df_jk) on (H2O)_n cc-pVDZ with def2-universal-JKFIT.

    The FP64-stored factor with FP64 arithmetic is the reference; the
    FP32-stored factor runs the exchange on the tensor cores (this library's
    tcgen05 kernels) with TF32 and with BF16 operands.  Per form: factor
    build time, J/K wall time, the exchange's device time and executed
    tensor-core TFLOP/s (both GEMMs, zero tiles skipped, lower triangle of K),
    the reference's algorithmic rate (4 n^2 nocc naux flops), the fraction
    of the measured BF16 tensor peak (TF32 runs at half of it), the error of
    K against the FP64 form, and the same J/K through cuBLAS GEMMs on the
    same factor (HFG_DF_K_CUBLAS=1) for comparison."""
    import numpy as np
    from hfgpu import CartesianBasis, Context
    from hfgpu.clusters import water_cluster
    from hfgpu.lib import HFG_DF_BF16, HFG_DF_FP32, HFG_DF_FP64, DFTensor
    peaks = {}
    pk = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(pk):
        peaks = json.load(open(pk))
    bf16_peak = peaks.get("bf16_tflops_sustained") or 1356.3
    atoms = water_cluster(args.df_waters)
    ctx = Context(CartesianBasis.build(atoms, "cc-pvdz"))
    aux = CartesianBasis.build(atoms, "def2-universal-jkfit")
    n, nocc = ctx.n, 5 * args.df_waters
    q, _ = np.linalg.qr(np.random.default_rng(5).standard_normal((n, nocc)))
    out = {"waters": args.df_waters, "n_ao": n, "naux": aux.n, "nocc": nocc,
           "peak_tflops_bf16_sustained": bf16_peak, "peak_source": "MEASURED_PEAKS.json" if peaks else "fallback"}

    def wall(fn, reps=3):
        fn()
        ts = []
        for _ in range(reps):
            t0 = time.time()
            r = fn()
            ts.append(time.time() - t0)
        return min(ts), r

    # the reference: FP64 arithmetic on an FP64 factor; above (H2O)64 an FP64
    # factor does not fit next to the FP32 one, and FP64 arithmetic on the
    # FP32 factor stands in (its K differs from the FP64 factor's by the
    # storage rounding only)
    big = args.df_waters > 64
    d32 = None
    if not big:
        t0 = time.time()
        d64 = DFTensor(ctx, aux, pair_threshold=1e-12, storage=HFG_DF_FP64)
        out["fp64"] = {"build_s": time.time() - t0, "factor": "FP64"}
    t0 = time.time()
    if big:
        d32 = DFTensor(ctx, aux, pair_threshold=1e-12, storage=HFG_DF_FP32)
        d64 = d32
        out["fp64"] = {"factor": "FP32 (an FP64 factor does not fit at this size)"}
    build32 = time.time() - t0
    t64, (J64, K64) = wall(lambda: d64.jk(q, mma=HFG_DF_FP64), reps=1)
    naux, rank, ncol = d64.sizes()
    out["fp64"].update({"jk_s": t64, "rank": rank, "pairs": ncol, "arith": "FP64 (cuBLAS DGEMM)"})
    if not big:
        d64.close()
        t0 = time.time()
        d32 = DFTensor(ctx, aux, pair_threshold=1e-12, storage=HFG_DF_FP32)
        build32 = time.time() - t0
    alg = 4.0 * n * n * nocc * rank
    best = 0.0
    for name, mma, scale in (("tf32", HFG_DF_FP32, 0.5), ("bf16", HFG_DF_BF16, 1.0)):
        tj, (J, K) = wall(lambda: d32.jk(q, mma=mma))
        st = d32.last_stats()
        ex = st["k_flops"] / (st["k_ms"] * 1e-3) / 1e12
        os.environ["HFG_DF_K_CUBLAS"] = "1"
        tc, (Jc, Kc) = wall(lambda: d32.jk(q, mma=mma))
        del os.environ["HFG_DF_K_CUBLAS"]
        out[name] = {"factor": "FP32", "build_s": build32, "jk_s": tj, "k_ms": st["k_ms"],
                     "k_tflops_executed": ex, "k_tflops_algorithmic": alg / (st["k_ms"] * 1e-3) / 1e12,
                     "tensor_peak_frac": ex / (bf16_peak * scale), "nonzero_tile_share": st["tiles_fraction"],
                     "rel_err_K_vs_fp64": float(np.linalg.norm(K - K64) / np.linalg.norm(K64)),
                     "max_abs_dJ_vs_fp64": float(np.max(np.abs(J - J64))),
                     "cublas_jk_s": tc, "speedup_vs_cublas": tc / tj,
                     "cublas_rel_err_K_vs_fp64": float(np.linalg.norm(Kc - K64) / np.linalg.norm(K64))}
        best = max(best, ex)
    d32.close()
    out["k_tflops_best"] = best
    ctx.close()
    return out


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
