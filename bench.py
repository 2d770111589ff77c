#!/usr/bin/env python
"""Throughput of the batched projection time step on B200.

Workload (default): the 256-case batched sweep -- seeded draws N in {65,129,193,257},
skew U[0,0.2], Re logU[50,1000], Ri logU[0.1,10], Pr in {0.71,7} -- in its O-grid twin
form (the reference's own geometry, boundary conditions, flow angle and dt = 1e-4), the
form the compiled reference can run; `--form cavity` runs the lid-driven cavity form.
One bench step = one outer time step of every case of the sweep (PSolver.cpp:1058-1983:
RHS, five u/v/T/up/vp solves, continuity source, pressure correction, correction, BCs,
diagnostics). value = grid points advanced per second over all ranks (cell-updates/s).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Multi-GPU: one process per GPU (torchrun); every rank runs its own seeded sweep
(weak scaling, no collective in the data path); time = max over ranks.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time
from concurrent.futures import ProcessPoolExecutor
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "cell-updates/s"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--form", choices=["twin", "cavity"], default="twin")
    ap.add_argument("--ncases", type=int, default=256)
    ap.add_argument("--precision", choices=["fp64", "mixed"], default="fp64",
                    help="plain FP64 path or the precision form (FP32 corrections in FP64 defect correction)")
    ap.add_argument("--e2e-steps", type=int, default=8)
    ap.add_argument("--e2e-split", type=int, default=4, help="sub-batches (host threads) of the e2e pass")
    ap.add_argument("--cpu-budget", type=float, default=15.0, help="seconds of CPU-baseline work")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--config", choices=["c1", "c2", "c3"], default="c3",
                    help="single-case configuration of the precision workload")
    ap.add_argument("--workload", choices=["step", "converged", "serve", "precision"], default="step",
                    help="step: outer-step throughput of the sweep (default); converged: every case of "
                         "the sweep to its steady tolerance or the step cap, batched vs the plain "
                         "single-case FP64 path; serve: Poisson request stream through cfd_serve")
    ap.add_argument("--tol", type=float, default=1e-8, help="steady-residual tolerance (converged/serve)")
    ap.add_argument("--no-converged", action="store_true",
                    help="leave the converged-cases block out of the default line")
    ap.add_argument("--conv-cap", type=int, default=20000, help="step cap per case of the converged block")
    ap.add_argument("--cap", type=int, default=30000, help="step cap per case (converged)")
    ap.add_argument("--chunk", type=int, default=100, help="steps between retirement checks")
    ap.add_argument("--requests", type=int, default=48, help="requests of the serve workload")
    ap.add_argument("--rate", type=float, default=4.0, help="Poisson arrival rate (requests/s)")
    ap.add_argument("--max-steps", type=int, default=30000, help="step cap per request (serve)")
    ap.add_argument("--serve-sizes", default="129,257",
                    help="request classes (N) of the serve workload, a subset of 129,257,513,1025")
    ap.add_argument("--serve-gb", type=float, default=24.0, help="device memory budget of the served pool (GB)")
    ap.add_argument("--plain-sample", type=int, default=8, help="requests the plain server runs for real")
    ap.add_argument("--no-serve", action="store_true", help="leave the serve block out of the default line")
    ap.add_argument("--mg", default=None,
                    help="multigrid schedule pre,post,coarse,fused (default: the library's)")
    return ap.parse_args()


# ------------------------------------------------------------------ reference (CPU) runs
def _ref_case_worker(task):
    """Run the compiled reference on one twin case at two step counts; per-step wall time
    from the difference (cancels set-up and the loop-0 file writes)."""
    from cfd_solver_b200.grid import write_inp
    from cfd_solver_b200.workloads import make_case
    d, s1, s2, binary = task
    g, prm = make_case(d, "twin")
    env = dict(os.environ)
    env.update({"CFD_RE": repr(prm["Re"]), "CFD_RI": repr(prm["Ri"]), "CFD_PR": repr(prm["Pr"]),
                "CFD_DT": repr(prm["dt"]), "CFD_ALPHA": repr(prm["alpha"])})
    with tempfile.TemporaryDirectory(prefix="cfdbench_") as td:
        write_inp(g, Path(td) / "INP.DAT")
        times = []
        for s in (s1, s2):
            env["CFD_MAXSTEP"] = str(s)
            t0 = time.perf_counter()
            subprocess.run([binary], cwd=td, env=env, stdout=subprocess.DEVNULL, check=True)
            times.append(time.perf_counter() - t0)
    return g.n0 * g.n1 * (s2 - s1), max(times[1] - times[0], 1e-9)


def host_cores() -> int:
    try:
        return len(os.sched_getaffinity(0))
    except Exception:
        return os.cpu_count() or 1


def reference_sample(draws, budget_s: float, cores: int, offset: int = 0):
    """cell-updates/s of the reference on a bounded sample of the sweep, all cores busy."""
    binary = str(ROOT / "oracle" / "_ref" / "cfd_ref")
    if not Path(binary).exists():
        return None, "oracle/_ref/cfd_ref not built"
    # the reference's step time per size on one core (0.84 s at 257^2, measured on this
    # image's host); the sample is sized to the budget from these
    per_step = {65: 0.02, 129: 0.1, 193: 0.35, 257: 0.84}
    tasks, est = [], 0.0
    k = offset
    while est < budget_s * cores and len(tasks) < 4 * cores:
        d = draws[k % len(draws)]
        k += 1
        s1, s2 = 1, 3
        tasks.append((d, s1, s2, binary))
        est += per_step[d["N"]] * (s1 + s2) + 0.5
    t0 = time.perf_counter()
    import multiprocessing as mp
    with ProcessPoolExecutor(max_workers=cores, mp_context=mp.get_context("spawn")) as ex:
        res = list(ex.map(_ref_case_worker, tasks))
    wall = time.perf_counter() - t0
    cells = sum(r[0] for r in res)
    busy = sum(r[1] for r in res)
    value = cells / (busy / cores)
    sizes = sorted({t[0]["N"] for t in tasks})
    sample = (f"{len(tasks)} twin cases of the sweep (N in {sizes}), 2 reference steps each "
              f"(difference of 1- and 3-step runs), {cores} processes, {wall:.1f} s wall")
    return value, sample


def run_reference_arm(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from cfd_solver_b200.workloads import sweep_draws
    draws = sweep_draws(args.ncases)
    cores = host_cores()
    vals = []
    sample = None
    for s in range(args.warmup + args.steps):
        v, sample = reference_sample(draws, budget_s=2.0, cores=cores, offset=s * cores)
        if v is None:
            print(json.dumps({"impl": "reference", "unavailable": sample}))
            return
        if s >= args.warmup:
            vals.append(v)
    value = statistics.mean(vals)
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": "cell-updates/s",
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded sweep draws)",
            "config": workload_config(args),
            "cpu_baseline": {"value": value, "unit": "cell-updates/s", "cores": cores,
                             "kind": "reference", "sample": "per step: " + sample},
            "e2e": {"value": value, "unit": "cell-updates/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


def workload_config(args):
    return {"workload": f"256-case batched sweep ({args.form} form)" if args.ncases == 256
            else f"{args.ncases}-case batched sweep ({args.form} form)",
            "cases": args.ncases, "sizes": "N x N, N in {65,129,193,257}",
            "params": "skew U[0,0.2], Re logU[50,1000], Ri logU[0.1,10], Pr {0.71,7}, seed 1234+rank",
            "dt": "1e-4 (reference)" if args.form == "twin" else "CFL 0.4 / max(1, sqrt(Ri))",
            "inner_tolerances": "reference: relative L1 0.75e-2 (momentum and pressure)",
            "precision": args.precision,
            "mg_schedule": args.mg or "library default (1,3,12,2)",
            "l2_flush": "inputs larger than L2 (>= 2.4 GB resident per step)",
            "parallelism": f"case-sharded, dp{args.gpus}"}


# ------------------------------------------------------------------ clocks
class NvmlClockSampler:
    """SM clock and clock-event reasons read through NVML every 10 ms on a thread (reads only);
    only the samples inside [mark_start, mark_end] count."""

    HW, HW_THERMAL, SW_THERMAL, SW_POWER = 0x8, 0x40, 0x20, 0x4

    def __init__(self, index: int):
        import threading
        import pynvml
        self.nv = pynvml
        pynvml.nvmlInit()
        self.h = None
        try:  # the CUDA device's own NVML handle (CUDA and NVML orders can differ)
            import torch
            pr = torch.cuda.get_device_properties(index)
            bus = "%08X:%02X:%02X.0" % (pr.pci_domain_id, pr.pci_bus_id, pr.pci_device_id)
            self.h = pynvml.nvmlDeviceGetHandleByPciBusId(bus)
        except Exception:
            self.h = pynvml.nvmlDeviceGetHandleByIndex(index)
        self.max_mhz = pynvml.nvmlDeviceGetMaxClockInfo(self.h, pynvml.NVML_CLOCK_SM)
        self.samples = []
        self.t0 = self.t1 = None
        self.run = True

        def poll():
            while self.run:
                try:
                    mhz = pynvml.nvmlDeviceGetClockInfo(self.h, pynvml.NVML_CLOCK_SM)
                    rs = pynvml.nvmlDeviceGetCurrentClocksEventReasons(self.h)
                    self.samples.append((time.time(), mhz, rs))
                except Exception:
                    pass
                time.sleep(0.01)

        self.th = threading.Thread(target=poll, daemon=True)
        self.th.start()

    def mark_start(self):
        self.t0 = time.time()

    def mark_end(self):
        self.t1 = time.time()

    def stop(self):
        self.run = False
        self.th.join(timeout=5)
        names = {self.HW: "hw_slowdown", self.HW_THERMAL: "hw_thermal_slowdown",
                 self.SW_THERMAL: "sw_thermal_slowdown", self.SW_POWER: "sw_power_cap"}

        def collect(lo, hi):
            sm, reasons = [], set()
            for ts, mhz, rs in self.samples:
                if lo is not None and not (lo <= ts <= (hi if hi is not None else ts)):
                    continue
                sm.append(float(mhz))
                for bit, n in names.items():
                    if rs & bit:
                        reasons.add(n)
            return sm, reasons

        sm, reasons = collect(self.t0, self.t1)
        window = "timed region"
        if not sm and self.t0 is not None:
            # a timed region of a few tens of ms can fall between two polls: take the samples
            # within 50 ms of it, and say so
            sm, reasons = collect(self.t0 - 0.05, (self.t1 or self.t0) + 0.05)
            window = "timed region +- 50 ms"
        try:
            self.nv.nvmlShutdown()
        except Exception:
            pass
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": float(self.max_mhz), "reasons": sorted(reasons),
                "samples": len(sm), "source": "nvml, 10 ms", "window": window}


def clock_sampler(index: int):
    try:
        return NvmlClockSampler(index)
    except Exception:
        return ClockSampler(index)


class ClockSampler:
    """nvidia-smi samples stamped on arrival; only those inside [mark_start, mark_end] count."""

    def __init__(self, index: int):
        import threading
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        self.lines = []
        self.t0 = self.t1 = None
        try:
            self.p = subprocess.Popen(["nvidia-smi", f"--query-gpu={q}", "--format=csv,noheader,nounits",
                                       "-lms", "100", "-i", str(index)], stdout=subprocess.PIPE,
                                      stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.p = None
            return

        def reader():
            for line in self.p.stdout:
                self.lines.append((time.time(), line))

        self.th = threading.Thread(target=reader, daemon=True)
        self.th.start()

    def mark_start(self):
        self.t0 = time.time()

    def mark_end(self):
        self.t1 = time.time()

    def stop(self):
        if not self.p:
            return None
        self.p.terminate()
        try:
            self.p.wait(timeout=5)
        except Exception:
            self.p.kill()
        self.th.join(timeout=5)
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ts, line in self.lines:
            if self.t0 is not None and not (self.t0 <= ts <= (self.t1 or ts)):
                continue
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx.append(float(f[2]))
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "reasons": sorted(reasons),
                "samples": len(sm)}


# ------------------------------------------------------------------ ranks
def rank_draws(ncases: int, rank: int):
    """Rank r runs its own seeded sweep (seed 1234 + r): whole cases per rank, no data
    exchange between ranks (weak scaling)."""
    from cfd_solver_b200.workloads import SWEEP_SEED, sweep_draws
    return sweep_draws(ncases, seed=SWEEP_SEED + rank)


def job_totals(dist, device, cells: float, ms: float, world: int):
    """Whole-job figures: cells summed over ranks, time the max over ranks."""
    if world == 1:
        return float(cells), float(ms)
    import torch
    c = torch.tensor([float(cells)], dtype=torch.float64, device=device)
    t = torch.tensor([float(ms)], dtype=torch.float64, device=device)
    dist.all_reduce(c, op=dist.ReduceOp.SUM)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(c.item()), float(t.item())


# ------------------------------------------------------------------ plain single-case path
def plain_step_ms(grid, prm, warm: int, timed: int) -> float:
    """Device time per step of one case alone on the plain FP64 path (a batch of one), after
    `warm` untimed steps past the start-up transient."""
    import torch
    from cfd_solver_b200.solver import Batch, case_params
    with Batch([grid], [case_params(grid, precision=0, **prm)]) as b:
        b.step(warm)
        b.sync()
        stream = torch.cuda.ExternalStream(b.stream())
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        b.step(timed)
        e1.record(stream)
        e1.synchronize()
        return e0.elapsed_time(e1) / timed


def plain_times_by_size(cases, warm=1500, timed=500):
    """Per-step time of the plain path for each grid size, on the first case of that size."""
    out = {}
    for g, prm in cases:
        if g.n0 not in out:
            out[g.n0] = plain_step_ms(g, prm, warm, timed)
    return out


def plain_solve(grid, prm, tol: float, cap: int, chunk: int):
    """One case alone on the plain FP64 path (a batch of one) until steady_res_rel <= tol or
    `cap` steps, checked every `chunk` steps as the batched arm checks. Returns (seconds of
    host wall clock around the run, steps, stats, fields)."""
    import torch
    from cfd_solver_b200.solver import Batch, case_params
    with Batch([grid], [case_params(grid, precision=0, **prm)]) as b:
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        steps = 0
        while True:
            b.step(chunk)
            steps += chunk
            s = b.stats(0)
            if (s["status"] & 4) or s["steady_res_rel"] <= tol or steps >= cap:
                break
        wall = time.perf_counter() - t0
        f = _case_fields(b, 0)
    return wall, steps, s, f


def _case_fields(b, i):
    f = {k: b.plane(i, k) for k in ("u", "v", "T", "p")}
    f["p"] = f["p"] - f["p"].mean()  # the closed cavity fixes p up to a constant
    return f


def converged_block(args, ncases: int, cap: int, tol: float, chunk: int):
    """Converged cases/s on the batched sweep (the benchmark's headline), both arms run.

    Batched arm: the `ncases` seeded sweep draws in cavity form, precision form, one batch;
    each case retires when its steady residual reaches `tol` (checked every `chunk` steps),
    diverges, or hits `cap` steps; its slot then drops out of every launch. Time = host wall
    clock around the whole run. Plain arm: every case the batched arm converged, run alone
    on the plain FP64 path to the same rule (measured, host wall clock); a case the batched
    arm capped costs the plain path `cap` steps at that size's measured plain step time.
    Each converged case's precision-form result is compared with its plain FP64 result."""
    import numpy as np
    import torch
    from cfd_solver_b200.solver import Batch, case_params
    from cfd_solver_b200.workloads import SWEEP_SEED, make_case, sweep_draws
    draws = sweep_draws(ncases, seed=SWEEP_SEED)
    cases = [make_case(d, "cavity") for d in draws]
    b = Batch([g for g, _ in cases], [case_params(g, precision=1, **p) for g, p in cases])
    n = len(cases)
    active = [True] * n
    steps_at, outcome, nu, fields = [0] * n, [""] * n, [0.0] * n, [None] * n
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    while any(active):
        b.step(chunk)
        st = b.all_stats()
        for i in range(n):
            if not active[i]:
                continue
            s = st[i]
            bad = bool(s["status"] & 4) or s["steady_res_rel"] != s["steady_res_rel"]
            conv = s["steps"] >= 2 and s["steady_res_rel"] <= tol
            if bad or conv or s["steps"] >= cap:
                active[i] = False
                b.set_active(i, False)
                steps_at[i], nu[i] = s["steps"], s["nu"]
                outcome[i] = "diverged" if bad else ("converged" if conv else "capped")
                if conv:
                    fields[i] = _case_fields(b, i)
    b.sync()
    makespan = time.perf_counter() - t0
    b.close()
    conv_ids = [i for i in range(n) if outcome[i] == "converged"]
    # plain arm, run for real on every converged case
    plain_wall, plain_conv, errs = 0.0, 0, []
    for i in conv_ids:
        g, prm = cases[i]
        wall, steps, s, f = plain_solve(g, prm, tol, cap, chunk)
        plain_wall += wall
        ok = not (s["status"] & 4) and s["steady_res_rel"] <= tol
        plain_conv += ok
        rel = {k: float(np.linalg.norm(fields[i][k] - f[k]) / max(np.linalg.norm(f[k]), 1e-300)) for k in f}
        errs.append({"case": i, "N": g.n0, "steps_batched": steps_at[i], "steps_plain": steps,
                     "rel_l2_max": max(rel.values()), "nu_rel": abs(nu[i] - s["nu"]) / max(abs(s["nu"]), 1e-300)})
    # capped or diverged cases: their steps at the plain path's measured step time per size
    rest = [i for i in range(n) if outcome[i] != "converged"]
    pt = plain_times_by_size([cases[i] for i in rest], warm=200, timed=200) if rest else {}
    plain_rest = sum(steps_at[i] * pt[cases[i][0].n0] for i in rest) / 1e3
    plain_total = plain_wall + plain_rest
    nconv = len(conv_ids)
    return {"metric": "converged cases/s", "value": nconv / makespan, "unit": "cases/s",
            "workload": f"{n} sweep draws (seed {SWEEP_SEED}), cavity form, precision form, batched "
                        f"with retirement", "tol": tol, "step_cap": cap, "retire_check_every": chunk,
            "cases": n, "converged": nconv, "capped": outcome.count("capped"),
            "diverged": outcome.count("diverged"), "makespan_s": makespan,
            "plain": {"path": "single case alone, FP64", "value": nconv / plain_total if plain_total else None,
                      "seconds_total": plain_total, "seconds_measured_converged": plain_wall,
                      "converged_measured": plain_conv,
                      "seconds_capped_at_measured_step_time": plain_rest, "ms_per_step_by_N": pt},
            "batched_over_plain": plain_total / makespan if makespan else None,
            "precision_vs_fp64": {"max_rel_l2": max((e["rel_l2_max"] for e in errs), default=None),
                                  "max_nu_rel": max((e["nu_rel"] for e in errs), default=None),
                                  "per_case": errs},
            "timing": "host wall clock on both arms (retirement checks included)",
            "per_case": [[cases[i][0].n0, round(draws[i]["Re"], 1), round(draws[i]["Ri"], 3), draws[i]["Pr"],
                          steps_at[i], outcome[i]] for i in range(n)]}


def run_converged(args):
    """The converged block alone, printed as its own line (--workload converged)."""
    blk = converged_block(args, args.ncases, args.cap, args.tol, args.chunk)
    line = dict(blk, n_gpus=1, higher_is_better=True, vs_baseline=None, dtype="f64+f32",
                data="synthetic (seeded sweep draws)")
    print(json.dumps(line))


def serve_block(nreq: int, rate: float, tol: float, cap: int, tick: int, budget_gb: float, plain_sample: int,
                sizes=None):
    """The served form: a Poisson stream of the benchmark's request mix through cfd_serve's
    admission by free device memory, against a plain FP64 single-case server run for real on
    the stream's first `plain_sample` requests.

    Stream: `nreq` requests at `rate`/s, N in {129, 257, 513, 1025} w.p. {.4, .3, .2, .1}
    (or the `sizes` subset of those classes, renormalised), physics as the sweep, cavity
    form, precision form; each is retired at steady_res_rel <= `tol` or after `cap` steps. Plain server: the sampled requests, FIFO, each run alone on the
    FP64 path to the same rule (service times measured, host wall clock); their latencies
    follow from those service times and the arrival times."""
    from cfd_solver_b200.solver import case_params, serve
    from cfd_solver_b200.workloads import SERVE_PROBS, SERVE_SIZES, make_case, serve_stream
    sizes = tuple(sizes or SERVE_SIZES)
    reqs, cases = [], []
    for t, d in serve_stream(nreq, rate, sizes=sizes):
        g, prm = make_case(d, "cavity")
        cases.append((g, prm))
        reqs.append((t, g, case_params(g, precision=1, **prm), tol, cap))
    budget = int(budget_gb * (1 << 30))
    results, st = serve(reqs, [], steps_per_tick=tick, slots=None, hbm_budget=budget, precision=1)
    lat = sorted(r["latency_s"] for r in results)
    conv = sorted(r["latency_s"] for r in results if r["status"] == 0)

    def pct(v, q):
        return v[min(len(v) - 1, max(0, math.ceil(q * len(v)) - 1))] if v else None

    # plain FP64 server, run for real on the first requests of the stream (FIFO)
    free, plain_lat, plain_conv, served_lat = 0.0, [], 0, []
    for i in range(min(plain_sample, len(reqs))):
        g, prm = cases[i]
        wall, steps, s1, _ = plain_solve(g, prm, tol, cap, tick)
        start = max(free, reqs[i][0])
        free = start + wall
        plain_lat.append(free - reqs[i][0])
        plain_conv += (s1["steady_res_rel"] <= tol) and not (s1["status"] & 4)
        served_lat.append(results[i]["latency_s"])
    return {"metric": "served cases/s", "value": len(results) / max(st["makespan_s"], 1e-9), "unit": "cases/s",
            "value_counts": "finished requests (converged or at the step cap) per second",
            "workload": f"{nreq} requests, Poisson {rate}/s, N in {list(sizes)} (the classes of N in "
                        f"{list(SERVE_SIZES)} w.p. {list(SERVE_PROBS)} kept, renormalised), cavity form, "
                        f"precision form, admission by free device memory ({budget_gb} GB)",
            "sub_sample": None if sizes == tuple(SERVE_SIZES) else
                ("the 513 and 1025 classes need 1e5 steps or more to converge (dt falls with N), "
                 "beyond a bench run; the block keeps the classes whose requests can converge "
                 "within its step cap"),
            "tol": tol, "step_cap": cap, "steps_per_tick": tick,
            "p50_latency_s": pct(lat, 0.5), "p99_latency_s": pct(lat, 0.99),
            "converged": len(conv), "p50_latency_converged_s": pct(conv, 0.5),
            "p99_latency_converged_s": pct(conv, 0.99), "makespan_s": st["makespan_s"],
            "peak_cases_resident": max_resident(results),
            "cell_updates_per_s": st["cell_updates"] / max(st["makespan_s"], 1e-9),
            "plain_sample": {"requests": len(plain_lat), "path": "single case alone, FP64, FIFO, run for real",
                             "p50_latency_s": pct(sorted(plain_lat), 0.5), "max_latency_s": max(plain_lat, default=None),
                             "converged": plain_conv, "served_p50_latency_same_requests_s":
                                 pct(sorted(served_lat), 0.5),
                             "served_max_latency_same_requests_s": max(served_lat, default=None)}}


def max_resident(results):
    ev = sorted([(r["admit_s"], 1) for r in results] + [(r["done_s"], -1) for r in results])
    cur = peak = 0
    for _, d in ev:
        cur += d
        peak = max(peak, cur)
    return peak


def run_serve(args):
    """The serve block alone, printed as its own line (--workload serve)."""
    blk = serve_block(args.requests, args.rate, args.tol, args.max_steps, args.chunk, args.serve_gb, args.plain_sample,
                      [int(x) for x in args.serve_sizes.split(",")])
    print(json.dumps(dict(blk, n_gpus=1, higher_is_better=True, dtype="f64+f32", data="synthetic (seeded Poisson stream)")))


def run_precision(args):
    """One single-case configuration (cavity form) in the plain FP64 path and in the
    precision form for the same number of steps: time per step of each and the relative
    L2 difference of u, v, p (mean removed), T and Nu of the precision form."""
    import numpy as np
    import torch
    from cfd_solver_b200.grid import cavity
    from cfd_solver_b200.solver import Batch, case_params
    from cfd_solver_b200.workloads import CONFIGS, cavity_dt
    c = CONFIGS[args.config]
    g = cavity(c["N"], c["N"], skew=c["skew"])
    dt = cavity_dt(c["N"], c["Ri"], c["Re"], c["Pr"])
    out = {}
    for prec in (0, 1):
        with Batch([g], [case_params(g, Re=c["Re"], Ri=c["Ri"], Pr=c["Pr"], dt=dt, precision=prec)]) as b:
            b.step(args.warmup)
            b.sync()
            stream = torch.cuda.ExternalStream(b.stream())
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            b.step(args.steps)
            e1.record(stream)
            e1.synchronize()
            st = b.stats(0)
            f = {k: b.plane(0, k) for k in ("u", "v", "p", "T")}
            f["p"] = f["p"] - f["p"][1:-1, 1:-1].mean()
            out[prec] = (e0.elapsed_time(e1) / args.steps, f, st)
    rel = {k: float(np.linalg.norm(out[1][1][k] - out[0][1][k]) / max(np.linalg.norm(out[0][1][k]), 1e-300))
           for k in ("u", "v", "p", "T")}
    nu0, nu1 = out[0][2]["nu"], out[1][2]["nu"]
    line = {"metric": "precision form vs FP64", "config": {"workload": f"{args.config}: {c['N']}x{c['N']} cavity, "
            f"skew {c['skew']}, Re {c['Re']}, Ri {c['Ri']}, Pr {c['Pr']}", "dt": dt,
            "steps": args.steps + args.warmup},
            "ms_per_step_fp64": out[0][0], "ms_per_step_mixed": out[1][0],
            "speedup": out[0][0] / out[1][0], "rel_l2": rel, "nu_fp64": nu0, "nu_mixed": nu1,
            "nu_rel": abs(nu1 - nu0) / max(abs(nu0), 1e-300),
            "steady_res_rel_fp64": out[0][2]["steady_res_rel"], "steady_res_rel_mixed": out[1][2]["steady_res_rel"],
            "status": [out[0][2]["status"], out[1][2]["status"]]}
    print(json.dumps(line))


# ------------------------------------------------------------------ our arm
def main():
    args = parse()
    if args.impl == "reference":
        run_reference_arm(args)
        return
    if args.workload == "converged":
        if args.form == "twin" and "--form" not in sys.argv:
            args.form = "cavity"
        if "--precision" not in sys.argv:
            args.precision = "mixed"
        run_converged(args)
        return
    if args.workload == "precision":
        run_precision(args)
        return
    if args.workload == "serve":
        if "--precision" not in sys.argv:
            args.precision = "mixed"
        run_serve(args)
        return
    import torch
    import torch.distributed as dist
    from cfd_solver_b200 import _lib
    from cfd_solver_b200.solver import Batch, case_params
    from cfd_solver_b200.workloads import SWEEP_SEED, make_case, sweep_draws

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    _lib.check(_lib.lib().cfd_set_device(local), "cfd_set_device")
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))

    def barrier():
        if world > 1:
            dist.barrier(device_ids=[local])

    draws = rank_draws(args.ncases, rank)
    grids, params = [], []
    for d in draws:
        g, prm = make_case(d, args.form)
        grids.append(g)
        params.append(case_params(g, precision=1 if args.precision == "mixed" else 0, **prm))
    cells = sum(g.n0 * g.n1 for g in grids)
    b = Batch(grids, params)
    mg = tuple(int(x) for x in args.mg.split(",")) if args.mg else None
    if mg:
        b.set_mg(*mg)
    stream = torch.cuda.ExternalStream(b.stream())

    clocks = clock_sampler(local)
    for _ in range(args.warmup):
        b.step(1)
    b.sync()
    barrier()
    torch.cuda.synchronize()
    clocks.mark_start()
    launches0 = b.launches()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        b.step(1)
    e1.record(stream)
    e1.synchronize()
    b.sync()
    torch.cuda.synchronize()
    clocks.mark_end()
    barrier()
    clk = clocks.stop()
    ms = e0.elapsed_time(e1)
    launches = b.launches() - launches0

    # roofline pass: the same steps again with a CUDA event pair around every launch on the
    # library's stream (host-driven loops instead of the step graph)
    prof_steps = max(3, min(args.steps, 10))
    b.profile(True)
    work0 = b.work()
    for _ in range(prof_steps):
        b.step(1)
    b.sync()
    work1 = b.work()
    kt = b.kernel_times()
    b.profile(False)
    job_cells, ms_max = job_totals(dist, "cuda", cells, ms, world)
    value = job_cells * args.steps / (ms_max / 1e3)

    # roofline of the dominant kernel (the u/v/T sweeps): algorithmic bytes per launch from
    # the traffic counters (field-cells of all sweeps, of sweep 0, of sweep 1; cells).
    # FP64: per field-cell read x_k, rhs, x_{k-1}, write x_{k+1} (32 B; sweep 0 has no x_{k-1}).
    # Precision form: sweep 0 reads x0 and rhs (FP64), writes r and d_1 (FP32): 24 B; later
    # sweeps read d_k, r, d_{k-1}, write d_{k+1} in FP32: 16 B (12 B at sweep 1, d_0 = 0).
    # Every sweep reads alpha, beta, gamma (24 B per cell).
    dom = max(kt.items(), key=lambda kv: kv[1][0])
    jac_ms, jac_n = kt.get("k_sweep", (0.0, 0))
    fc = work1[0] - work0[0]
    cc = work1[1] - work0[1]
    f0 = work1[2] - work0[2]
    f1 = work1[3] - work0[3]
    if args.precision == "mixed":
        jac_bytes = 24 * f0 + 12 * f1 + 16 * (fc - f0 - f1) + 24 * cc
    else:
        jac_bytes = 32 * fc - 8 * f0 + 24 * cc
    peaks = {}
    try:
        peaks = json.loads((ROOT / "MEASURED_PEAKS.json").read_text())
        peak, peak_src = float(peaks["hbm_gbs"]), "measured"
    except Exception:
        peak, peak_src = 6650.0, "fallback"
    achieved = (jac_bytes / 1e9) / (jac_ms / 1e3) if jac_ms > 0 else 0.0
    traffic = None
    tf = ROOT / "profiles" / "k_sweep_traffic.json"
    if tf.exists() and jac_n:
        try:
            tj = json.loads(tf.read_text())
            # ncu-measured DRAM bytes per algorithmic byte of this kernel (captured on the
            # 64-case sweep), scaled to this run's per-launch algorithmic bytes
            traffic = tj["dram_over_algorithmic"] * jac_bytes / jac_n
        except Exception:
            traffic = None
    roofline = {"kernel": "k_sweep", "bound": "hbm", "achieved": achieved, "peak": peak,
                "peak_source": peak_src, "unit": "GB/s", "frac": achieved / peak,
                "traffic": traffic, "algorithmic_bytes_per_launch": jac_bytes / max(jac_n, 1),
                "avg_launch_us": jac_ms / max(jac_n, 1) * 1e3, "launches": jac_n,
                "share_of_kernel_time": jac_ms / max(sum(v[0] for v in kt.values()), 1e-12)}
    kernels = {k: {"ms": round(v[0], 3), "launches": v[1]} for k, v in kt.items() if v[1]}
    kernels["_steps"] = prof_steps

    # end to end through the C ABI with host-owned state: every step uploads the state of
    # every case from pinned host memory, steps, and reads the new state and stats back. The
    # sweep is split into sub-batches, each driven by its own host thread on its own stream,
    # so the uploads of one, the step of another and the downloads of a third overlap (the
    # copy engines move both directions at once); the threads release the interpreter lock
    # inside every library call.
    import threading
    nsub = max(1, min(args.e2e_split, len(grids)))
    parts = [list(range(k, len(grids), nsub)) for k in range(nsub)]
    subs = [Batch([grids[i] for i in p], [params[i] for i in p]) for p in parts]
    hosts = []
    for sb in subs:
        if mg:
            sb.set_mg(*mg)
        sb.step(1)  # builds the step graphs
        h = torch.empty(sb.state_bytes(), dtype=torch.uint8, pin_memory=True)
        sb.get_state(h)
        hosts.append(h)
    nbytes = sum(int(h.numel()) for h in hosts)
    errs = []

    def drive(k):
        try:
            _lib.check(_lib.lib().cfd_set_device(local), "cfd_set_device")
            sb, h = subs[k], hosts[k]
            for _ in range(args.e2e_steps):
                sb.set_state(h)
                sb.step(1)
                sb.get_state(h)
                sb.stats(0)
        except Exception as e:  # reported after the join
            errs.append(e)

    barrier()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    threads = [threading.Thread(target=drive, args=(k,)) for k in range(nsub)]
    for th in threads:
        th.start()
    for th in threads:
        th.join()
    e2e_s = time.perf_counter() - t0
    if errs:
        raise errs[0]
    for sb in subs:
        sb.close()
    _, e2e_max = job_totals(dist, "cuda", cells, e2e_s, world)
    e2e_value = job_cells * args.e2e_steps / e2e_max

    cpu = None
    if rank == 0 and not args.no_cpu_baseline and args.form == "twin":
        v, sample = reference_sample(draws, budget_s=args.cpu_budget, cores=host_cores())
        if v is not None:
            cpu = {"value": v, "unit": "cell-updates/s", "cores": host_cores(), "kind": "reference",
                   "sample": sample}
        else:
            cpu = {"value": None, "unavailable": sample}
    st0 = b.stats(0)
    b.close()
    conv = srv = None
    if rank == 0 and world == 1 and not args.no_converged:
        # the headline metric (converged cases/s, batched vs plain), both arms run on this GPU
        conv = converged_block(args, args.ncases, args.conv_cap, args.tol, args.chunk)
    if rank == 0 and world == 1 and not args.no_serve:
        srv = serve_block(args.requests, args.rate, args.tol, args.max_steps, args.chunk, args.serve_gb,
                          args.plain_sample, [int(x) for x in args.serve_sizes.split(",")])
    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": "cell-updates/s", "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_max / args.steps,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                "dtype": "f64" if args.precision == "fp64" else "f64+f32",
                "data": "synthetic (seeded sweep draws; grids generated in INP.DAT format)",
                "config": workload_config(args),
                "cells_per_step": job_cells,
                "roofline": roofline, "cpu_baseline": cpu,
                "e2e": {"value": e2e_value, "unit": "cell-updates/s",
                        "h2d_bytes_per_step": nbytes, "d2h_bytes_per_step": nbytes + 200 * nsub,
                        "sub_batches": nsub},
                "clocks": clk, "gpu_launches": launches, "kernels": kernels,
                "dominant_kernel": dom[0],
                "converged": conv,
                "serve": srv,
                "baseline_metric_note": ("the headline metric is converged cases/s (the `converged` "
                                         "block: batched precision form vs the plain FP64 single-case "
                                         "path, both run); a case needs 1e3-1e5 steps to its steady "
                                         "state, so a bench step is one outer step of the whole sweep"),
                "case0": {"it_mom": st0["it_mom"], "it_p": st0["it_p"], "status": st0["status"]}}
        print(json.dumps(line))
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
