"""Initial condition, Maxwellian and boundary rows of the BGK1D1V model.

set_initial_condition   core/schemes/BGK1D1V/bgk1d_utils/general/bgk1d_set_initial_condition.py:9-44
maxwellian              bgk1d_utils/general/bgk1d_maxwellian.py:7-33
boundary_rows/apply_bc  bgk1d_utils/general/bgk1d_apply_BC.py:51-152 (fixed_maxwellian)
check_CFL               bgk1d_utils/general/bgk1d_check_CFL.py:7-19
These run once per build (or once per step for two rows) with torch ops on
the state's device; the time step itself runs in the CUDA library.
"""
from __future__ import annotations

import logging

import torch

logger = logging.getLogger("kineticEQ")

FIXED_BC = ("fixed_maxwellian", "fixed", "dirichlet")


@torch.no_grad()
def maxwellian(state) -> torch.Tensor:
    coeff = (state.n * state.inv_sqrt_2pi) / torch.sqrt(state.T)
    invT = 0.5 / state.T
    diff = state.v_col - state.u[:, None]
    e = diff.mul(diff)
    e.mul_(-invT[:, None])
    torch.exp(e, out=e)
    e.mul_(coeff[:, None])
    return e


@torch.no_grad()
def set_initial_condition(state, cfg) -> None:
    x = state.x
    nx = x.numel()
    n = torch.full((nx,), 1.0, device=state.f.device, dtype=state.f.dtype)
    u = torch.full((nx,), 0.0, device=state.f.device, dtype=state.f.dtype)
    T = torch.full((nx,), 1.0, device=state.f.device, dtype=state.f.dtype)
    regions = getattr(cfg.model_cfg.initial, "initial_regions", ())
    for idx, r in enumerate(regions):
        if isinstance(r, dict):
            a, b = r["x_range"]
            rn, ru, rT = r["n"], r["u"], r["T"]
        else:
            a, b = r.x_range
            rn, ru, rT = r.n, r.u, r.T
        last = idx == len(regions) - 1
        mask = (x >= a) & (x <= b) if last else (x >= a) & (x < b)
        n[mask] = float(rn)
        u[mask] = float(ru)
        T[mask] = float(rT)
    state.n, state.u, state.T = n, u, T
    state.f.copy_(maxwellian(state))


def bc_type_of(boundary) -> str:
    bc = getattr(boundary, "bc_type", boundary)
    return str(bc).strip().lower()


def require_fixed_bc(boundary) -> None:
    """The fused kernels hold rows 0 and nx-1 at their step-start values
    (fixed_maxwellian, the default of BoundaryCondition1D)."""
    bc = bc_type_of(boundary)
    if bc not in FIXED_BC:
        if bc in ("reflective", "specular", "specular_reflective", "diffuse",
                  "diffuse_reflective", "diffuse_reflection"):
            raise NotImplementedError(
                f"boundary condition {bc!r} is not provided by the B200 backend "
                "(fixed_maxwellian only)")
        raise ValueError(f"Unknown boundary condition type: {bc}")


def check_CFL(cfg) -> None:
    if cfg.model_cfg.time.dt <= 0:
        raise ValueError("dt must be positive")
    dx = cfg.model_cfg.grid.Lx / (cfg.model_cfg.grid.nx - 1)
    cfl = cfg.model_cfg.grid.v_max * cfg.model_cfg.time.dt / dx
    logger.info(f"CFL: {cfl:.3g}")
    if cfl > 0.9:
        raise ValueError(f"CFL violated: vmax*dt/dx = {cfl:.3g} > 0.9. "
                         f"(vmax={cfg.model_cfg.grid.v_max}, dt={cfg.model_cfg.time.dt}, dx={dx})")
