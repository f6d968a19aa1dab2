"""Throughput benchmark of the B200 BGK1D1V implicit time step.

python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
               [--workload NAME] [--no-cpu-baseline] [--no-e2e]

Metric: cell-velocity updates/s = sum over instances of nx*nv*steps / seconds
(one update = one (x_i, v_k) entry advanced one full time step, whatever the
number of Picard iterations).  Default workload: the large plain FP64 case,
4096 x 512 cells, v in [-10, 10], dt = 1e-5, tau_tilde = 5e-5, Sod initial
state, Picard tolerance 1e-10 (cap 64), Anderson depth m = 5 (200 steps =
the case's T_total).

ours:      K time steps, each ONE launch of the persistent step kernel, timed
           with CUDA events on the launching stream; L2 is flushed (256 MiB
           write) before every step outside the timed window.  e2e repeats the
           measurement through the C ABI with host buffers: pinned f^n -> device,
           step, f^{n+1} -> pinned host, all inside the timed window.
reference: the CPU oracle (C restatement of the reference's cpu_kernel path,
           all host threads) on the same workload, a bounded number of steps.
Multi-GPU (torchrun): every rank steps its own replica (independent
instances, no collective on the data path); value = all ranks' updates /
max-over-ranks time.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

WORKLOADS = {
    # name: (nx, nv, dt, tau_tilde, implicit params, steps of the case)
    "implicit-4096x512-aa5-tau5e-5": (4096, 512, 1e-5, 5e-5,
                                      dict(picard_iter=64, picard_tol=1e-10, abs_tol=1e-16,
                                           aa_enable=True, aa_m=5), 200),
    "implicit-4096x512-tau5e-5": (4096, 512, 1e-5, 5e-5,
                                  dict(picard_iter=64, picard_tol=1e-10, abs_tol=1e-16), 200),
    "implicit-4096x512-aa5-tau5e-3": (4096, 512, 1e-5, 5e-3,
                                      dict(picard_iter=64, picard_tol=1e-10, abs_tol=1e-16,
                                           aa_enable=True, aa_m=5), 200),
    "implicit-256x128-tau5e-5": (256, 128, 5e-6, 5e-5,
                                 dict(picard_iter=64, picard_tol=1e-10, abs_tol=1e-16), 100),
    "implicit-8192x1024-aa5-tau1e-4": (8192, 1024, 1e-5, 1e-4,
                                       dict(picard_iter=64, picard_tol=1e-10, abs_tol=1e-16,
                                            aa_enable=True, aa_m=5), 200),
    "implicit-8192x1024-tau1e-4": (8192, 1024, 1e-5, 1e-4,
                                   dict(picard_iter=64, picard_tol=1e-10, abs_tol=1e-16), 200),
    # the precision form: FP32 sweeps then FP64 sweeps; the bench line adds the
    # error in rho, u, T against the FP64 method over the same steps
    "implicit-8192x1024-tau1e-4-mixed": (8192, 1024, 1e-5, 1e-4,
                                         dict(picard_iter=64, picard_tol=1e-10, abs_tol=1e-16,
                                              precision="mixed"), 200),
    "holo-4096x512-tau5e-5": (4096, 512, 1e-5, 5e-5,
                              dict(scheme="holo", ho_iter=64, ho_tol=1e-10, lo_iter=64,
                                   lo_tol=1e-10), 200),
    "holo-4096x512-tau5e-3": (4096, 512, 1e-5, 5e-3,
                              dict(scheme="holo", ho_iter=64, ho_tol=1e-10, lo_iter=64,
                                   lo_tol=1e-10), 200),
    "holo-256x128-tau5e-5": (256, 128, 5e-6, 5e-5,
                             dict(scheme="holo", ho_iter=64, ho_tol=1e-10, lo_iter=64,
                                  lo_tol=1e-10), 100),
    "holo-8192x1024-tau1e-4": (8192, 1024, 1e-5, 1e-4,
                               dict(scheme="holo", ho_iter=64, ho_tol=1e-10, lo_iter=64,
                                    lo_tol=1e-10), 200),
}


def is_holo(name: str) -> bool:
    return WORKLOADS[name][4].get("scheme") == "holo"


def scheme_params(name: str) -> dict:
    return {k: v for k, v in WORKLOADS[name][4].items() if k != "scheme"}
DEFAULT_WORKLOAD = "implicit-4096x512-aa5-tau5e-5"
# Sod initial state (the InitialCondition1D defaults of the reference)
SOD_REGIONS = ({"x_range": (0.0, 0.5), "n": 1.0, "u": 0.0, "T": 1.0},
               {"x_range": (0.5, 1.0), "n": 0.125, "u": 0.0, "T": 0.8})
METRIC = "cell-velocity updates/s"
BYTES_PER_CELL_ITER = 24  # read f^n, read f^(m), write f^(m+1) (FP64)


def _peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def _traffic_from_profiles(workload: str):
    """DRAM bytes per cell and iteration that a committed ncu summary measured
    for this workload (profiles/*.md lines
    'traffic_bytes_per_cell_iter[<workload>]: X'); scaled to a launch by the
    caller."""
    key = f"traffic_bytes_per_cell_iter[{workload}]:"
    for p in sorted((ROOT / "profiles").glob("*.md")):
        for line in p.read_text().splitlines():
            if line.startswith(key):
                try:
                    return float(line.split(":", 1)[1].strip().split()[0]), p.name
                except ValueError:
                    pass
    return None, None


class ClockSampler:
    """nvidia-smi clocks/throttle sampling during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.path = Path(f"/tmp/keq_clocks_{os.getpid()}.csv")

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        if not self.path.exists():
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"]}
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.path.read_text().splitlines():
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax = float(parts[2])
            except ValueError:
                continue
            for nm, val in zip(names, parts[5:9]):
                if val.lower() in ("active", "1", "yes"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


def _dist():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    if ws > 1:
        import torch
        import torch.distributed as dist
        from datetime import timedelta

        os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
        dist.init_process_group("nccl", timeout=timedelta(seconds=120))
        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
        return dist, dist.get_rank(), ws
    return None, 0, 1


def _max_over_ranks(dist, x: float) -> float:
    if dist is None:
        return x
    import torch

    t = torch.tensor([x], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def _barrier(dist):
    if dist is not None:
        dist.barrier()


def make_instance(name: str):
    import torch

    from kineticeq_b200.plan import (HoloPlan, ImplicitPlan, InstanceSpec, holo_params_struct,
                                     implicit_params_struct)
    from kineticeq_b200.schemes.common import maxwellian, region_moments
    from kineticeq_b200.state import allocate_state_1d1v

    nx, nv, dt, tau, _, _ = WORKLOADS[name]
    sp = scheme_params(name)
    st = allocate_state_1d1v(nx, nv, 1.0, 10.0, "cuda", torch.float64)
    st.n, st.u, st.T = region_moments(st.x, SOD_REGIONS)
    maxwellian(st, out=st.f)
    spec = InstanceSpec(v=st.v, dx=st.dx, dv=st.dv, dt=dt, tau_tilde=tau, a=st.f,
                        b=torch.empty_like(st.f))
    if is_holo(name):
        plan = HoloPlan([spec], holo_params_struct(**sp))
    else:
        plan = ImplicitPlan([spec], implicit_params_struct(**sp))
    return plan, st


def run_ours(args, dist, rank, world):
    import torch

    from kineticeq_b200 import _native as N

    name = args.workload
    nx, nv, dt, tau, _, case_steps = WORKLOADS[name]
    sp = scheme_params(name)
    holo = is_holo(name)
    plan, st = make_instance(name)
    f0 = st.f.clone()
    stream = torch.cuda.current_stream()
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")

    for _ in range(args.warmup):
        plan.step(1)
    torch.cuda.synchronize()
    # restart from the initial state so the timed steps are the case's first K
    plan.state(0).copy_(f0)
    iters0 = int(plan.stats.fetch()[0]["total_iters"])
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    launches = 0
    _barrier(dist)
    torch.cuda.synchronize()
    with ClockSampler(torch.cuda.current_device()) as clk:
        for k in range(args.steps):
            flush.fill_(float(k))
            starts[k].record(stream)
            plan.step(1)
            launches += 1
            ends[k].record(stream)
        torch.cuda.synchronize()
    _barrier(dist)
    ms = sum(s.elapsed_time(e) for s, e in zip(starts, ends))
    rec = plan.stats.fetch()[0]
    if int(rec["status"]) != 0:
        raise RuntimeError(f"device status {N.status_text(int(rec['status']))}")
    iters = int(rec["total_iters"]) - iters0
    prec_err = _precision_error(name, plan.state(0), f0, st, args.steps) \
        if sp.get("precision") == "mixed" else None
    # conservation drift over the timed steps (row moments on the device)
    from kineticeq_b200.schemes.common import conservation_totals, drift

    drift_k = drift(conservation_totals(plan.state(0), st.v, st.dx, st.dv),
                    conservation_totals(f0, st.v, st.dx, st.dv))
    ms_max = _max_over_ranks(dist, ms)
    cells = nx * nv
    value = world * cells * args.steps / (ms_max / 1e3)

    # e2e through the C ABI with host buffers (pinned), copies inside the timing
    e2e = None
    if not args.no_e2e:
        host_in = f0.cpu().pin_memory()
        host_out = torch.empty_like(host_in).pin_memory()
        e_s = torch.cuda.Event(enable_timing=True)
        e_e = torch.cuda.Event(enable_timing=True)
        ksteps = args.steps
        _barrier(dist)
        torch.cuda.synchronize()
        e_s.record(stream)
        src = host_in
        for k in range(ksteps):
            plan.state(0).copy_(src, non_blocking=True)
            plan.step(1)
            host_out.copy_(plan.state(0), non_blocking=True)
            src = host_out
        e_e.record(stream)
        torch.cuda.synchronize()
        e2e_ms = _max_over_ranks(dist, e_s.elapsed_time(e_e))
        nb = host_in.numel() * host_in.element_size()
        e2e = {"value": world * cells * ksteps / (e2e_ms / 1e3), "unit": METRIC,
               "h2d_bytes_per_step": nb, "d2h_bytes_per_step": nb}

    # roofline of the step kernel (one launch per step): 24 B per cell and
    # Picard (HO) iteration, plus 16 B per cell and step for HOLO's explicit term
    peak, peak_kind = _peaks()
    bytes_per_launch = BYTES_PER_CELL_ITER * cells * (iters / args.steps) + (16 * cells if holo else 0)
    achieved = bytes_per_launch / (ms / args.steps / 1e3) / 1e9
    tpc, tsrc = _traffic_from_profiles(name)
    roof = {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
            "frac": round(achieved / peak, 4), "peak_kind": peak_kind,
            "traffic": (round(tpc * cells * iters / args.steps) if tpc else None),
            "traffic_source": tsrc, "bytes_per_launch_algorithmic": round(bytes_per_launch),
            "kernel": "keq::holo::holo_step_kernel" if holo else "keq::implicit_step_kernel"}

    cpu = None
    if rank == 0 and not args.no_cpu_baseline:
        cpu = cpu_baseline(name, f0.cpu().numpy(), st, budget_s=args.cpu_seconds)

    if rank == 0:
        out = {
            "metric": METRIC, "value": round(value, 1), "unit": METRIC, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms_max / args.steps, 5),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (Sod initial state, generated on the device)",
            **({"dtype": "f32 sweeps then f64 sweeps (mixed)", "precision_error": prec_err}
               if prec_err is not None else {}),
            "config": {"workload": name, "scheme": "holo" if holo else "implicit", "nx": nx,
                       "nv": nv, "dt": dt, "tau_tilde": tau, **sp,
                       "instances_per_gpu": 1, "parallelism": f"replicas x{world}",
                       "l2": "flushed (256 MiB write) before every timed step",
                       ("mean_ho_iters_per_step" if holo else "mean_picard_iters_per_step"):
                           round(iters / args.steps, 3)},
            "drift": {**{k: float(f"{x:.6e}") for k, x in drift_k.items()},
                      "over_steps": args.steps, "from": "initial state"},
            "e2e": e2e, "roofline": roof, "cpu_baseline": cpu, "gpu_launches": launches,
            "clocks": clk.summary(),
        }
        print(json.dumps(out))


def _precision_error(name, f_mixed, f0, st, steps):
    """Relative max error of the mixed-precision result against the FP64
    method run from the same initial state for the same steps: f normwise and
    the row moments rho, u, T (max |d| / max |ref|)."""
    import torch

    from kineticeq_b200.plan import ImplicitPlan, InstanceSpec, implicit_params_struct

    nx, nv, dt, tau, _, _ = WORKLOADS[name]
    sp = dict(scheme_params(name), precision="fp64")
    a = f0.clone()
    spec = InstanceSpec(v=st.v, dx=st.dx, dv=st.dv, dt=dt, tau_tilde=tau, a=a,
                        b=torch.empty_like(a))
    ref_plan = ImplicitPlan([spec], implicit_params_struct(**sp))
    ref_plan.step(steps)
    ref = ref_plan.state(0)

    def mom(f):
        n = f.sum(1) * st.dv
        u = (f * st.v).sum(1) * st.dv / n
        T = (f * st.v * st.v).sum(1) * st.dv / n - u * u
        return n, u, T

    def rel(x, y):
        return float((x - y).abs().max() / y.abs().max().clamp_min(1e-300))

    (n1, u1, T1), (n0, u0, T0) = mom(f_mixed), mom(ref)
    return {"f": rel(f_mixed, ref), "rho": rel(n1, n0), "u": rel(u1, u0), "T": rel(T1, T0),
            "against": f"FP64 method, same {steps} steps from the same state"}


def cpu_baseline(name, f0, st, budget_s=20.0):
    """The oracle (C restatement of the reference's cpu_kernel path) on the
    host cores: as many time steps of the same workload as fit the budget."""
    threads = os.cpu_count() or 1
    os.environ.setdefault("OMP_NUM_THREADS", str(threads))
    from oracle import oracle as O

    nx, nv, dt, tau, _, _ = WORKLOADS[name]
    sp = scheme_params(name)
    v = st.v.cpu().numpy()
    holo = is_holo(name)
    p = O.holo_params(None, **sp) if holo else O.implicit_params(None, **sp)
    step = O.holo_step if holo else O.implicit_step
    key = "ho_iter" if holo else "picard_iter"
    f = f0.copy()
    O.lib()
    t0 = time.perf_counter()
    steps = iters = 0
    while True:
        bl = step(f, v, st.dx, st.dv, dt, tau, p)
        steps += 1
        iters += bl[key]
        el = time.perf_counter() - t0
        if el >= budget_s or steps >= 200:
            break
    val = nx * nv * steps / el
    return {"value": round(val, 1), "unit": METRIC, "cores": int(os.environ["OMP_NUM_THREADS"]),
            "kind": "port", "sample": f"first {steps} time steps of {name} ({iters} "
                                      f"{'HO' if holo else 'Picard'} iterations) in {el:.1f} s"}


def run_reference(args, dist, rank, world):
    """--impl reference: the reference's CPU implementation of the path (its
    C restatement; the reference itself does not travel) on the host cores."""
    if rank != 0:
        return
    import torch

    threads = os.cpu_count() or 1
    os.environ["OMP_NUM_THREADS"] = str(threads)
    from oracle import oracle as O

    name = args.workload
    nx, nv, dt, tau, _, _ = WORKLOADS[name]
    sp = scheme_params(name)
    holo = is_holo(name)
    g = O.Grid(nx, nv)
    v = g.v()
    f = O.initial_condition(g)
    p = O.holo_params(None, **sp) if holo else O.implicit_params(None, **sp)
    step = O.holo_step if holo else O.implicit_step
    key = "ho_iter" if holo else "picard_iter"
    # bounded sample: at most ~budget seconds of timed steps
    for _ in range(min(args.warmup, 1)):
        step(f.copy(), v, g.dx, g.dv, dt, tau, p)
    t0 = time.perf_counter()
    steps = iters = 0
    while steps < args.steps:
        bl = step(f, v, g.dx, g.dv, dt, tau, p)
        steps += 1
        iters += bl[key]
        if time.perf_counter() - t0 > args.cpu_seconds * 6:
            break
    el = time.perf_counter() - t0
    val = nx * nv * steps / el
    sample = (f"first {steps} time steps of {name} ({iters} {'HO' if holo else 'Picard'} "
              f"iterations), {el:.1f} s")
    out = {"impl": "reference", "metric": METRIC, "value": round(val, 1), "unit": METRIC,
           "n_gpus": world, "steps": steps, "warmup": min(args.warmup, 1),
           "ms_per_step": round(el * 1e3 / steps, 3), "higher_is_better": True,
           "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (Sod)",
           "config": {"workload": name, "nx": nx, "nv": nv, "dt": dt, "tau_tilde": tau},
           "cpu_baseline": {"value": round(val, 1), "unit": METRIC, "cores": threads,
                            "kind": "port", "sample": sample},
           "e2e": {"value": round(val, 1), "unit": METRIC, "h2d_bytes_per_step": 0,
                   "d2h_bytes_per_step": 0},
           "torch_threads": torch.get_num_threads()}
    print(json.dumps(out))


# ---------------------------------------------------------------------------
# Mixed workloads: the batching form (256 seeded uneven instances, 100 steps)
# and the serving form (Poisson request stream with the same size and state
# distribution, 100..2000 steps per request).
# ---------------------------------------------------------------------------
MIX_WORKLOADS = {
    # name: (kind, instances, seed, rate per s, precision of the solves)
    "batch-cfg3-256": ("batch", 256, 0, None, "fp64"),
    "batch-cfg3-256-mixed": ("batch", 256, 0, None, "mixed"),
    "serve-cfg5-r200": ("serve", 64, 0, 200.0, "fp64"),
    "serve-cfg5-r200-mixed": ("serve", 64, 0, 200.0, "mixed"),
    "serve-cfg5-r50": ("serve", 32, 1, 50.0, "fp64"),
}
MIX_PARAMS = dict(picard_iter=64, picard_tol=1e-10, abs_tol=1e-16)


def _plain_rate(descs, steps, params):
    """Plain FP64 path: every instance alone, one launch per step."""
    import torch

    from kineticeq_b200.batch import make_state, spec_of
    from kineticeq_b200.plan import ImplicitPlan, implicit_params_struct

    t = 0.0
    cells = 0
    for d in descs:
        st = make_state(d)
        plan = ImplicitPlan([spec_of(d, st)], implicit_params_struct(None, **params))
        plan.step(1)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        plan.step(steps)
        e1.record()
        e1.synchronize()
        t += e0.elapsed_time(e1) / 1e3
        cells += d.cells * steps
    return cells / t


def _oracle_rate(descs, params, budget_s):
    """The oracle on the host cores over a bounded sample of the instances."""
    from oracle import oracle as O

    p = O.implicit_params(None, **params)
    O.lib()
    t = 0.0
    cells = steps = 0
    for d in descs:
        g = O.Grid(d.nx, d.nv, d.Lx, d.v_max)
        reg = [(r["x_range"][0], r["x_range"][1], r["n"], r["u"], r["T"]) for r in d.regions]
        f = O.initial_condition(g, reg)
        t0 = time.perf_counter()
        O.implicit_step(f, g.v(), g.dx, g.dv, d.dt, d.tau_tilde, p)
        t += time.perf_counter() - t0
        cells += d.cells
        steps += 1
        if t > budget_s:
            break
    return cells / t, f"first time step of the first {steps} instances of the mix ({t:.1f} s)"


def run_mix(args, dist, rank, world):
    import torch

    from kineticeq_b200 import autotune
    from kineticeq_b200.batch import BatchSolver, sample_instances
    from kineticeq_b200.serving import Server, plain_throughput, poisson_stream

    kind, n_inst, seed, rate, prec = MIX_WORKLOADS[args.workload]
    # our solves run in `prec`; the plain comparison and the CPU baseline are
    # always the reference's FP64 method
    params = dict(MIX_PARAMS, precision=prec) if prec != "fp64" else MIX_PARAMS
    table = autotune.load() or {}
    out = {"metric": METRIC, "unit": METRIC, "n_gpus": world, "higher_is_better": True,
           "scaling": "weak", "vs_baseline": None,
           "dtype": "f64" if prec == "fp64" else "f32 sweeps then f64 sweeps (mixed)",
           "data": "synthetic (seeded two-state Riemann instances, sizes and states as the "
                   "batching distribution)"}
    launches = 0
    if kind == "batch":
        descs = sample_instances(n_inst, seed=seed + rank)
        solver = BatchSolver(descs, params, table=table)
        cells = solver.cells
        for _ in range(args.warmup):
            solver.step(1)
        torch.cuda.synchronize()
        solver.reset()
        use_graph = args.steps % 2 == 0
        if use_graph:
            solver.capture(2)
        it0 = solver.plan.stats.fetch()["total_iters"].astype(np.int64)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        _barrier(dist)
        torch.cuda.synchronize()
        with ClockSampler(torch.cuda.current_device()) as clk:
            e0.record()
            if use_graph:
                for _ in range(args.steps // 2):
                    solver.replay()
            else:
                solver.step(args.steps)
            e1.record()
            torch.cuda.synchronize()
        _barrier(dist)
        ms = _max_over_ranks(dist, e0.elapsed_time(e1))
        launches = args.steps
        rec = solver.plan.stats.fetch()
        iters = rec["total_iters"].astype(np.int64) - it0
        cell_iters = float(sum(int(i) * d.cells for i, d in zip(iters, descs)))
        value = world * cells * args.steps / (ms / 1e3)
        plain = _plain_rate(descs[:64], 2, MIX_PARAMS)
        e2e = None
        if not args.no_e2e:
            # per step: every instance's f^n from pinned host memory to the
            # device, one step, f^{n+1} back to pinned host memory
            hosts = [s.a.cpu().pin_memory() for s in solver.specs]
            outs = [torch.empty_like(h).pin_memory() for h in hosts]
            k2 = 2
            solver.reset()
            torch.cuda.synchronize()
            q0, q1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            q0.record()
            for _ in range(k2):
                for i, h in enumerate(hosts):
                    solver.plan.state(i).copy_(h, non_blocking=True)
                solver.step(1)
                for i, o in enumerate(outs):
                    o.copy_(solver.plan.state(i), non_blocking=True)
                hosts = outs
            q1.record()
            torch.cuda.synchronize()
            nb = 8 * cells
            e2e = {"value": round(world * cells * k2 / (q0.elapsed_time(q1) / 1e3), 1),
                   "unit": METRIC, "h2d_bytes_per_step": nb, "d2h_bytes_per_step": nb}
        out["e2e"] = e2e
        peak, peak_kind = _peaks()
        achieved = BYTES_PER_CELL_ITER * cell_iters / (ms / 1e3) / 1e9
        out.update({"value": round(value, 1), "steps": args.steps, "warmup": args.warmup,
                    "ms_per_step": round(ms / args.steps, 4),
                    "plain_value": round(plain, 1), "speedup_vs_plain": round(value / plain, 3),
                    "config": {"workload": args.workload, "instances": n_inst, "seed": seed,
                               "cells_per_step": cells, "dt": 5e-6, **params,
                               "tile_rows_table": bool(table), "cuda_graph": use_graph,
                               "l2": "inputs larger than L2 (535 MB per FP64 field)",
                               "mean_picard_iters_per_step":
                                   round(cell_iters / cells / args.steps, 3),
                               "plain": "first 64 instances, each alone, 2 steps after 1 warm-up"},
                    "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak,
                                 "unit": "GB/s", "frac": round(achieved / peak, 4),
                                 "peak_kind": peak_kind, "traffic": None,
                                 "kernel": "keq::implicit_step_kernel"},
                    "clocks": clk.summary()})
        sample_descs = descs
    else:
        reqs = poisson_stream(n_inst, rate, seed=seed + rank)
        warm = poisson_stream(4, 1e6, seed=99, steps_range=(3, 3))
        Server(params=params, table=table).run(warm, realtime=False)
        _barrier(dist)
        with ClockSampler(torch.cuda.current_device()) as clk:
            res = Server(params=params, table=table).run(reqs)
        _barrier(dist)
        ms = _max_over_ranks(dist, res["makespan_s"] * 1e3)
        launches = res["launches"]
        value = world * res["cell_steps"] / (ms / 1e3)
        e2e = None
        if not args.no_e2e:
            # the same stream with host inputs and outputs: each request's
            # initial state comes from pinned host memory at admission and its
            # final state goes back to pinned host memory at retirement
            from kineticeq_b200.batch import make_state

            reqs2 = poisson_stream(n_inst, rate, seed=seed + rank)
            for r in reqs2:
                r.f0_host = make_state(r.desc).f.cpu().pin_memory()
            torch.cuda.synchronize()
            res2 = Server(params=params, table=table, copy_out=True).run(reqs2)
            nb = sum(8 * r.desc.cells for r in reqs2)
            e2e = {"value": round(world * res2["cell_steps"] / res2["makespan_s"], 1),
                   "unit": METRIC, "h2d_bytes_per_step": round(nb / res2["steps"]),
                   "d2h_bytes_per_step": round(nb / res2["steps"]),
                   "p50_latency_s": round(res2["p50_latency_s"], 4),
                   "p99_latency_s": round(res2["p99_latency_s"], 4)}
        out["e2e"] = e2e
        plain, plain_t, plain_sample = plain_throughput(reqs, MIX_PARAMS, steps_cap=10)
        out.update({"value": round(value, 1), "steps": res["steps"], "warmup": 1,
                    "ms_per_step": round(ms / max(res["steps"], 1), 4),
                    "p50_latency_s": round(res["p50_latency_s"], 4),
                    "p99_latency_s": round(res["p99_latency_s"], 4),
                    "plain_value": round(plain, 1), "speedup_vs_plain": round(value / plain, 3),
                    "config": {"workload": args.workload, "requests": n_inst, "rate_per_s": rate,
                               "seed": seed, "steps_per_request": "uniform 100..2000",
                               **params, "rebuilds": res["rebuilds"],
                               "l2": "inputs larger than L2 in aggregate; not flushed",
                               "plain": plain_sample},
                    "clocks": clk.summary()})
        sample_descs = [r.desc for r in reqs]
    out["gpu_launches"] = launches
    if rank == 0 and not args.no_cpu_baseline:
        v, sample = _oracle_rate(sample_descs, MIX_PARAMS, args.cpu_seconds)
        out["cpu_baseline"] = {"value": round(v, 1), "unit": METRIC,
                               "cores": os.cpu_count() or 1, "kind": "port", "sample": sample}
    if rank == 0:
        print(json.dumps(out))


def run_mix_reference(args, dist, rank, world):
    if rank != 0:
        return
    from kineticeq_b200.batch import sample_instances

    kind, n_inst, seed, rate, _prec = MIX_WORKLOADS[args.workload]
    descs = sample_instances(n_inst, seed=seed,
                             steps_range=None if kind == "batch" else (100, 2000))
    v, sample = _oracle_rate(descs, MIX_PARAMS, args.cpu_seconds * 6)
    print(json.dumps({"impl": "reference", "metric": METRIC, "value": round(v, 1), "unit": METRIC,
                      "n_gpus": world, "steps": 1, "warmup": 0, "higher_is_better": True,
                      "scaling": "weak", "vs_baseline": None, "dtype": "f64",
                      "data": "synthetic", "config": {"workload": args.workload},
                      "cpu_baseline": {"value": round(v, 1), "unit": METRIC,
                                       "cores": os.cpu_count() or 1, "kind": "port",
                                       "sample": sample},
                      "e2e": {"value": round(v, 1), "unit": METRIC, "h2d_bytes_per_step": 0,
                              "d2h_bytes_per_step": 0}}))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", choices=sorted(WORKLOADS) + sorted(MIX_WORKLOADS),
                    default=DEFAULT_WORKLOAD)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    args = ap.parse_args()
    if args.warmup < 3 and args.impl == "ours":
        args.warmup = 3
    dist, rank, world = _dist()
    try:
        mix = args.workload in MIX_WORKLOADS
        if args.impl == "reference":
            (run_mix_reference if mix else run_reference)(args, dist, rank, world)
        else:
            (run_mix if mix else run_ours)(args, dist, rank, world)
    finally:
        if dist is not None:
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
