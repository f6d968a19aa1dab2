"""Implicit (Picard + Anderson) stepper on the B200 library.

Drop-in for core/schemes/BGK1D1V/bgk1d_implicit_cuda_kernel.py:313-405
(build_stepper) and :28-311 (step): same builder signature, the stepper
advances exactly one dt per call, swaps ``state.f``/``state.f_tmp``, carries
``.benchlog`` (picard_iter, picard_residual, std_picard_residual) and ``.ws``,
and raises ValueError("NaN/Inf detected in f_tmp") on the 100-step check.

One call = one launch of the persistent kernel (all Picard iterations and the
convergence test run on the device); the host never synchronises inside a
step.  benchlog values are fetched from the device only when read.
"""
from __future__ import annotations

import logging
from collections.abc import Mapping
from typing import Callable

import torch

from .. import _native as N
from ..plan import ImplicitPlan, InstanceSpec, implicit_params_struct
from .common import require_fixed_bc, set_initial_condition

logger = logging.getLogger("kineticEQ")
Stepper = Callable[[int], None]


class LazyBenchlog(Mapping):
    """benchlog dict of one step: a snapshot of the step's device stats record,
    copied asynchronously when the step is queued and read (with one wait) on
    first access, so reading it later still gives that step's values."""

    def __init__(self, snap, idx: int, keys: dict):
        self._snap, self._idx, self._keys, self._vals = snap, idx, keys, None

    def _load(self):
        if self._vals is None:
            rec = self._snap.fetch()[self._idx]
            self._vals = {k: (int(rec[f]) if f in ("iters", "lo_iters", "aa_applied")
                              else float(rec[f])) for k, f in self._keys.items()}
        return self._vals

    def __getitem__(self, k):
        return self._load()[k]

    def __iter__(self):
        return iter(self._keys)

    def __len__(self):
        return len(self._keys)

    def __repr__(self):
        return repr(dict(self._load()))


IMPLICIT_KEYS = {"picard_iter": "iters", "picard_residual": "residual",
                 "std_picard_residual": "std_residual"}


class ImplicitWorkspace:
    """Workspace handle exposed as ``stepper.ws``: the plan and views of the
    current moments W = (n, nu, T) (first 3*nx doubles of the instance
    workspace)."""

    def __init__(self, plan: ImplicitPlan, nx: int):
        self.plan = plan
        w = plan._ws[0][: 3 * nx * 8].view(torch.float64)
        self.n, self.nu, self.T = w[:nx], w[nx:2 * nx], w[2 * nx:3 * nx]
        self._init_W = None
        self._warm_prev_W = None


def _check_warm_start(sp) -> None:
    path = getattr(sp, "moments_cnn_modelpath", None)
    warm = getattr(sp, "warm_enable", None)
    if path and warm is not False:
        raise NotImplementedError("CNN warm start (moments_cnn_modelpath) is not provided by "
                                  "the B200 backend")


def build_stepper(cfg, state) -> Stepper:
    sp = cfg.model_cfg.scheme_params
    params = implicit_params_struct(sp)
    _check_warm_start(sp)
    require_fixed_bc(cfg.model_cfg.boundary)
    if state.f.dtype != torch.float64:
        raise RuntimeError("the B200 implicit backend computes in float64 (dtype='float64')")
    if not state.f.is_cuda:
        raise RuntimeError("the B200 backend needs device='cuda'")
    N.load()
    set_initial_condition(state, cfg)
    spec = InstanceSpec(v=state.v, dx=float(state.dx), dv=float(state.dv),
                        dt=float(cfg.model_cfg.time.dt),
                        tau_tilde=float(cfg.model_cfg.params.tau_tilde),
                        a=state.f, b=state.f_tmp)
    plan = ImplicitPlan([spec], params)
    ws = ImplicitWorkspace(plan, state.f.shape[0])

    def _stepper(num_steps: int) -> None:
        if ws._init_W is not None:
            raise NotImplementedError("W injection (ws._init_W) is not provided by the B200 backend")
        # the plan ping-pongs between its two buffers; rebind if the caller
        # replaced state.f since the last call
        if state.f.data_ptr() != plan.state(0).data_ptr():
            plan.state(0).copy_(state.f)
        plan.step(1)
        state.f, state.f_tmp = plan.state(0), plan.other(0)
        if num_steps % 100 == 0:
            rec = plan.stats.fetch()[0]
            if int(rec["status"]) == N.KEQ_ERR_NONFINITE:
                raise ValueError("NaN/Inf detected in f_tmp")
            N.check(int(rec["status"]), "implicit step")
        _stepper.benchlog = LazyBenchlog(plan.snapshot(), 0, IMPLICIT_KEYS)

    _stepper.benchlog = None
    _stepper.ws = ws
    return _stepper
