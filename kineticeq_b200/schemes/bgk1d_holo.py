"""HOLO stepper on the B200 library.

Drop-in for core/schemes/BGK1D1V/bgk1d_holo_cuda_kernel.py:598-618
(build_stepper) and :416-595 (step): the builder checks the CFL condition
first (bgk1d_check_CFL), applies the initial condition, and returns a stepper
that advances one dt per call, swaps ``state.f``/``state.f_tmp``, carries
``.benchlog`` with the reference's keys (ho_iter, ho_residual,
std_ho_residual, lo_iter, lo_residual, std_lo_residual, max_YI), leaves
``state.n/u/T`` at the moments of the last LO solve (the reference's side
effect, :513-514) and raises ValueError("NaN/Inf detected in f_tmp") on the
100-step check.

One call = one launch of the persistent HOLO kernel (HO and LO iterations
and both convergence tests run on the device).
"""
from __future__ import annotations

import logging
from typing import Callable

import torch

from .. import _native as N
from ..plan import HoloPlan, InstanceSpec, holo_params_struct
from .bgk1d_implicit import LazyBenchlog
from .common import check_CFL, require_fixed_bc, set_initial_condition

logger = logging.getLogger("kineticEQ")
Stepper = Callable[[int], None]

HOLO_KEYS = {"ho_iter": "iters", "ho_residual": "residual", "std_ho_residual": "std_residual",
             "lo_iter": "lo_iters", "lo_residual": "lo_residual",
             "std_lo_residual": "std_lo_residual", "max_YI": "max_YI"}


def build_stepper(cfg, state) -> Stepper:
    check_CFL(cfg)
    sp = cfg.model_cfg.scheme_params
    params = holo_params_struct(sp)
    require_fixed_bc(cfg.model_cfg.boundary)
    if not state.f.is_cuda:
        raise RuntimeError("the B200 backend needs device='cuda'")
    if state.f.dtype != torch.float64:
        raise RuntimeError("the B200 HOLO backend computes in float64 (dtype='float64')")
    N.load()
    set_initial_condition(state, cfg)
    spec = InstanceSpec(v=state.v, dx=float(state.dx), dv=float(state.dv),
                        dt=float(cfg.model_cfg.time.dt),
                        tau_tilde=float(cfg.model_cfg.params.tau_tilde),
                        a=state.f, b=state.f_tmp)
    plan = HoloPlan([spec], params)
    nx = state.f.shape[0]
    wlo = plan._ws[0][: 3 * nx * 8].view(torch.float64).view(3, nx)

    def _stepper(num_steps: int) -> None:
        if state.f.data_ptr() != plan.state(0).data_ptr():
            plan.state(0).copy_(state.f)
        plan.step(1)
        state.f, state.f_tmp = plan.state(0), plan.other(0)
        state.n, state.u, state.T = wlo[0], wlo[1], wlo[2]
        if num_steps % 100 == 0:
            rec = plan.stats.fetch()[0]
            if int(rec["status"]) == N.KEQ_ERR_NONFINITE:
                raise ValueError("NaN/Inf detected in f_tmp")
            N.check(int(rec["status"]), "HOLO step")
        _stepper.benchlog = LazyBenchlog(plan.snapshot(), 0, HOLO_KEYS)

    _stepper.benchlog = None
    _stepper.plan = plan
    return _stepper
