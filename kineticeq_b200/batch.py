"""Batching form: many independent implicit solves of uneven sizes stepped
together, one persistent-kernel launch per time step for the whole list.

- ``sample_instances``: the seeded two-state Riemann mix of the batching
  workload (nx uniform in [128, 2048], nv in {64, 128, 256, 512}, tau_tilde
  log-uniform in [1e-5, 1e-1], left/right Maxwellian states, discontinuity
  in [0.3, 0.7]), drawn per instance in a fixed order.
- ``BatchSolver``: the instances' states on the device, one plan over all of
  them with per-(nx, nv)-bucket tile heights from the autotuner table, and
  an optional CUDA graph of the per-step launch sequence.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field
from typing import Sequence

import torch

from .plan import HoloPlan, ImplicitPlan, InstanceSpec, holo_params_struct, \
    implicit_params_struct, velocity_facts
from .schemes.common import maxwellian, region_moments
from .state import allocate_state_1d1v

NV_CHOICES = (64, 128, 256, 512)


@dataclass
class InstanceDesc:
    nx: int
    nv: int
    tau_tilde: float
    regions: tuple
    n_steps: int = 100
    dt: float = 5e-6
    Lx: float = 1.0
    v_max: float = 10.0

    @property
    def cells(self) -> int:
        return self.nx * self.nv


def sample_instances(n: int = 256, seed: int = 0, dt: float = 5e-6, n_steps: int = 100,
                     steps_range: tuple | None = None) -> list[InstanceDesc]:
    """Seeded instances; per instance the draws are, in order: nx, nv,
    log10 tau_tilde, rho_L, rho_R, u_L, u_R, T_L, T_R, x_d (and the step count
    when ``steps_range`` = (lo, hi) is given)."""
    g = torch.Generator("cpu").manual_seed(seed)

    def u(a, b):
        return float(a + (b - a) * torch.rand((), generator=g, dtype=torch.float64))

    out = []
    for _ in range(n):
        nx = int(torch.randint(128, 2049, (), generator=g))
        nv = NV_CHOICES[int(torch.randint(0, 4, (), generator=g))]
        tau = 10.0 ** u(-5.0, -1.0)
        rl, rr = u(0.5, 2.0), u(0.05, 0.5)
        ul, ur = u(-0.5, 0.5), u(-0.5, 0.5)
        tl, tr = u(0.5, 2.0), u(0.5, 2.0)
        xd = u(0.3, 0.7)
        steps = n_steps
        if steps_range is not None:
            steps = int(torch.randint(steps_range[0], steps_range[1] + 1, (), generator=g))
        regions = ({"x_range": (0.0, xd), "n": rl, "u": ul, "T": tl},
                   {"x_range": (xd, 1.0), "n": rr, "u": ur, "T": tr})
        out.append(InstanceDesc(nx, nv, tau, regions, steps, dt))
    return out


def make_state(desc: InstanceDesc, device="cuda"):
    """Initial state of one instance (set_initial_condition semantics)."""
    st = allocate_state_1d1v(desc.nx, desc.nv, desc.Lx, desc.v_max, device, torch.float64)
    st.n, st.u, st.T = region_moments(st.x, desc.regions)
    maxwellian(st, out=st.f)
    return st


def bucket_of(nx: int, nv: int) -> str:
    """Autotuner bucket: nx by powers of two, nv exact."""
    return f"nx{1 << max(0, int(math.log2(max(nx, 1))))}-nv{nv}"


def spec_of(desc: InstanceDesc, st) -> InstanceSpec:
    kp, vmax = velocity_facts(desc.nv, desc.v_max)
    return InstanceSpec(v=st.v, dx=st.dx, dv=st.dv, dt=desc.dt, tau_tilde=desc.tau_tilde,
                        a=st.f, b=torch.empty_like(st.f), kp=kp, v_max=vmax)


@dataclass
class BatchSolver:
    """Steps of a list of instances in one plan (one launch per step)."""
    descs: Sequence[InstanceDesc]
    params: dict = field(default_factory=lambda: dict(picard_iter=64, picard_tol=1e-10,
                                                      abs_tol=1e-16))
    table: dict | None = None   # autotuner table: bucket -> tile_rows
    scheme: str = "implicit"

    def __post_init__(self):
        self.states = [make_state(d) for d in self.descs]
        self.specs = [spec_of(d, s) for d, s in zip(self.descs, self.states)]
        self.f0 = [s.a.clone() for s in self.specs]
        if self.scheme == "holo":
            self.plan = HoloPlan(self.specs, holo_params_struct(None, **self.params))
        else:
            plist = [implicit_params_struct(None, tile_rows=self.tile_rows(d), **self.params)
                     for d in self.descs]
            self.plan = ImplicitPlan(self.specs, plist)
        self.graph = None

    def tile_rows(self, d: InstanceDesc) -> int:
        if not self.table:
            return 0
        return int(self.table.get(bucket_of(d.nx, d.nv), 0))

    @property
    def cells(self) -> int:
        return sum(d.cells for d in self.descs)

    def reset(self) -> None:
        """Back to the initial states (newest state in buffer a)."""
        self.plan.parity = 0
        for s, f0 in zip(self.specs, self.f0):
            s.a.copy_(f0)

    def step(self, n: int = 1) -> None:
        self.plan.step(n)

    def capture(self, steps_per_replay: int = 2) -> None:
        """Capture ``steps_per_replay`` (even) steps of the plan into a CUDA
        graph; ``replay()`` then launches them with one call."""
        if steps_per_replay % 2:
            raise ValueError("steps_per_replay must be even (state ping-pong)")
        parity = self.plan.parity
        s = torch.cuda.Stream()
        s.wait_stream(torch.cuda.current_stream())
        g = torch.cuda.CUDAGraph()
        with torch.cuda.stream(s):
            self.plan._stream = s
            try:
                with torch.cuda.graph(g, stream=s):
                    self.plan.step(steps_per_replay)
            finally:
                self.plan._stream = None
        torch.cuda.current_stream().wait_stream(s)
        self.plan.parity = parity  # capturing does not run the steps
        self.graph = g
        self.graph_steps = steps_per_replay

    def replay(self) -> None:
        self.graph.replay()
        self.plan.parity = (self.plan.parity + self.graph_steps) & 1
