"""Serving form: a continuous-batching request loop over the implicit step.

Requests (one BGK1D1V implicit solve each: grid, tau_tilde, initial
Riemann state, number of steps) arrive over time.  The loop

- admits pending requests that have arrived, first come first served, while
  the HBM bytes of the live set (two state buffers plus the kernel workspace
  per solve, from the workspace query) stay under the budget;
- keeps every live solve's state and workspace resident on the device;
- steps ALL live solves together, one persistent-kernel launch per step
  (ImplicitPlan over the live set);
- retires a solve after its last step: its slot is switched off in the
  plan's device-side enable mask (no rebuild), its final state is kept, and
  its completion is stamped with a CUDA event on the launch stream;
- rebuilds the plan over the current live set when new requests are admitted
  (at most every ``admit_every`` steps while others are running).

Latency of a request = completion (device event) - arrival (host clock, both
relative to the start of the run).  Each solve's arithmetic depends only on
its own data, so its result in the mix equals its result alone, bitwise.
"""
from __future__ import annotations

import ctypes as C
import math
import time
from collections import deque
from dataclasses import dataclass
from typing import Sequence

import numpy as np
import torch

from . import _native as N
from .batch import InstanceDesc, bucket_of, make_state, sample_instances
from .plan import ImplicitPlan, InstanceSpec, implicit_params_struct, velocity_facts


@dataclass
class Request:
    rid: int
    desc: InstanceDesc
    arrival: float  # seconds after the start of the run
    f0_host: torch.Tensor | None = None  # optional initial state in (pinned) host memory


def poisson_stream(n: int, rate: float, seed: int = 0, steps_range=(100, 2000),
                   dt: float = 5e-6) -> list[Request]:
    """n requests with exponential inter-arrival times (``rate`` per second)
    and sizes/states from the batching distribution; steps uniform in
    ``steps_range``."""
    descs = sample_instances(n, seed=seed, dt=dt, steps_range=steps_range)
    g = torch.Generator("cpu").manual_seed(seed + 7919)
    gaps = torch.empty(n, dtype=torch.float64).exponential_(1.0, generator=g) / rate
    t = torch.cumsum(gaps, 0) - gaps[0]
    return [Request(i, d, float(t[i])) for i, d in enumerate(descs)]


def solve_bytes(desc: InstanceDesc, params) -> int:
    """HBM bytes a live solve holds: two (nx, nv) FP64 state buffers plus the
    step kernel's workspace (keq_implicit_instance_workspace_size)."""
    lib = N.load(require_cuda=False)
    grid = N.Grid(desc.nx, desc.nv, 1.0, 1.0, 0, -1, 0.0)
    nb = C.c_size_t(0)
    N.check(lib.keq_implicit_instance_workspace_size(C.byref(grid), C.byref(params),
                                                     C.byref(nb)), "workspace query")
    return 2 * 8 * desc.nx * desc.nv + int(nb.value)


class _Live:
    __slots__ = ("req", "a", "b", "cur", "steps_done", "slot", "v", "dx", "dv", "kp", "vmax",
                 "bytes")

    def __init__(self, req: Request, bytes_: int):
        d = req.desc
        st = make_state(d) if req.f0_host is None else _grid_only(d)
        self.req = req
        if req.f0_host is not None:
            st.f.copy_(req.f0_host, non_blocking=True)
        self.a, self.b = st.f, torch.empty_like(st.f)
        self.cur = 0  # 0: newest state in a
        self.steps_done = 0
        self.slot = -1
        self.v, self.dx, self.dv = st.v, st.dx, st.dv
        self.kp, self.vmax = velocity_facts(d.nv, d.v_max)
        self.bytes = bytes_

    def state(self) -> torch.Tensor:
        return self.a if self.cur == 0 else self.b

    def other(self) -> torch.Tensor:
        return self.b if self.cur == 0 else self.a


def _grid_only(d: InstanceDesc):
    from .state import allocate_state_1d1v

    return allocate_state_1d1v(d.nx, d.nv, d.Lx, d.v_max, "cuda", torch.float64)


class Server:
    def __init__(self, hbm_budget: int = 16 << 30, params: dict | None = None,
                 table: dict | None = None, admit_every: int = 4, max_live: int = 512,
                 inflight: int = 4, copy_out: bool = False):
        self.params = params or dict(picard_iter=64, picard_tol=1e-10, abs_tol=1e-16)
        self.table = table or {}
        self.budget = int(hbm_budget)
        self.admit_every = int(admit_every)
        self.max_live = int(max_live)
        self.inflight = int(inflight)
        self.copy_out = bool(copy_out)  # final states to pinned host memory at retirement

    def _pstruct(self, d: InstanceDesc):
        R = int(self.table.get(bucket_of(d.nx, d.nv), 0))
        return implicit_params_struct(None, tile_rows=R, **self.params)

    def run(self, requests: Sequence[Request], realtime: bool = True) -> dict:
        """Serve the requests; with realtime=False every request counts as
        arrived at time 0 (admission is then limited by the budget only)."""
        pending = deque(sorted(requests, key=lambda r: r.arrival))
        live: list[_Live] = []
        done: dict[int, dict] = {}
        used = 0
        plan = mask = None
        stream = torch.cuda.current_stream()
        start_ev = torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        start_ev.record(stream)
        step_events: deque = deque()
        steps_since_admit = 10 ** 9
        n_steps_total = rebuilds = launches = 0
        cell_steps = 0
        while pending or live:
            now = time.perf_counter() - t0 if realtime else math.inf
            admitted = []
            if pending and (not live or steps_since_admit >= self.admit_every):
                while (pending and pending[0].arrival <= now and
                       len(live) + len(admitted) < self.max_live):
                    r = pending[0]
                    need = solve_bytes(r.desc, self._pstruct(r.desc))
                    if used + need > self.budget and (live or admitted):
                        break
                    pending.popleft()
                    admitted.append(_Live(r, need))
                    used += need
            if admitted:
                live.extend(admitted)
                specs = []
                for k, s in enumerate(live):
                    s.slot = k
                    cur, oth = s.state(), s.other()
                    s.a, s.b, s.cur = cur, oth, 0
                    specs.append(InstanceSpec(v=s.v, dx=s.dx, dv=s.dv, dt=s.req.desc.dt,
                                              tau_tilde=s.req.desc.tau_tilde, a=s.a, b=s.b,
                                              kp=s.kp, v_max=s.vmax))
                plan = ImplicitPlan(specs, [self._pstruct(s.req.desc) for s in live])
                mask = torch.ones(len(live), dtype=torch.int32, device=specs[0].a.device)
                plan.set_enable_mask(mask)
                rebuilds += 1
                steps_since_admit = 0
            if not live:
                if pending and realtime:
                    time.sleep(max(0.0, min(1e-3, pending[0].arrival - now)))
                continue
            plan.step(1)
            launches += 1
            n_steps_total += 1
            steps_since_admit += 1
            ev = torch.cuda.Event(enable_timing=True)
            ev.record(stream)
            step_events.append(ev)
            if len(step_events) > self.inflight:
                step_events.popleft().synchronize()
            retired = []
            for s in live:
                s.cur ^= 1
                s.steps_done += 1
                cell_steps += s.req.desc.cells
                if s.steps_done >= s.req.desc.n_steps:
                    retired.append(s)
            for s in retired:
                mask[s.slot] = 0
                live.remove(s)
                used -= s.bytes
                fin = s.state()
                if self.copy_out:
                    host = torch.empty(fin.shape, dtype=fin.dtype, pin_memory=True)
                    host.copy_(fin, non_blocking=True)
                    ev = torch.cuda.Event(enable_timing=True)
                    ev.record(stream)
                    fin = host
                done[s.req.rid] = {"event": ev, "state": fin, "req": s.req}
        torch.cuda.synchronize()
        wall = time.perf_counter() - t0
        lat = []
        finish = 0.0
        for r in done.values():
            t_done = start_ev.elapsed_time(r["event"]) / 1e3
            finish = max(finish, t_done)
            r["latency_s"] = t_done - (r["req"].arrival if realtime else 0.0)
            lat.append(r["latency_s"])
        lat = np.array(lat)
        return {"results": done, "makespan_s": finish, "wall_s": wall,
                "cell_steps": cell_steps, "updates_per_s": cell_steps / finish,
                "p50_latency_s": float(np.percentile(lat, 50)),
                "p99_latency_s": float(np.percentile(lat, 99)),
                "launches": launches, "rebuilds": rebuilds, "steps": n_steps_total,
                "requests": len(done)}


def solve_alone(req: Request, params: dict, table: dict | None = None) -> torch.Tensor:
    """The request's final state from a plan of its own (reference for the
    'same alone and in the mix' check)."""
    d = req.desc
    st = make_state(d)
    kp, vmax = velocity_facts(d.nv, d.v_max)
    spec = InstanceSpec(v=st.v, dx=st.dx, dv=st.dv, dt=d.dt, tau_tilde=d.tau_tilde, a=st.f,
                        b=torch.empty_like(st.f), kp=kp, v_max=vmax)
    R = int((table or {}).get(bucket_of(d.nx, d.nv), 0))
    plan = ImplicitPlan([spec], implicit_params_struct(None, tile_rows=R, **params))
    plan.step(d.n_steps)
    return plan.state(0)


def plain_throughput(requests: Sequence[Request], params: dict, steps_cap: int | None = None):
    """The plain FP64 path on the same requests: one request at a time, each
    stepped alone (one launch per step).  With steps_cap, each request is
    timed over min(n_steps, steps_cap) steps and its time scaled to n_steps
    (per-step cost is near constant over a solve).  Returns (updates/s,
    total seconds, sample description)."""
    total_t = 0.0
    cells = 0
    for r in requests:
        d = r.desc
        st = make_state(d)
        kp, vmax = velocity_facts(d.nv, d.v_max)
        spec = InstanceSpec(v=st.v, dx=st.dx, dv=st.dv, dt=d.dt, tau_tilde=d.tau_tilde, a=st.f,
                            b=torch.empty_like(st.f), kp=kp, v_max=vmax)
        plan = ImplicitPlan([spec], implicit_params_struct(None, **params))
        k = d.n_steps if steps_cap is None else min(d.n_steps, steps_cap)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        plan.step(k)
        e1.record()
        e1.synchronize()
        total_t += e0.elapsed_time(e1) / 1e3 * (d.n_steps / k)
        cells += d.cells * d.n_steps
    sample = ("every request stepped alone, one launch per step" +
              (f"; timed over its first min(n_steps, {steps_cap}) steps and scaled to n_steps"
               if steps_cap else ""))
    return cells / total_t, total_t, sample
