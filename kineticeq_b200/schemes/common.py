"""Initial condition, Maxwellian and boundary rows of the BGK1D1V model.

set_initial_condition   core/schemes/BGK1D1V/bgk1d_utils/general/bgk1d_set_initial_condition.py:9-44
maxwellian              bgk1d_utils/general/bgk1d_maxwellian.py:7-33
boundary_rows/apply_bc  bgk1d_utils/general/bgk1d_apply_BC.py:51-152 (fixed_maxwellian)
check_CFL               bgk1d_utils/general/bgk1d_check_CFL.py:7-19
The per-row region masks are set up with torch on the state's device (O(nx));
the Maxwellian itself and the time steps run in the CUDA library.
"""
from __future__ import annotations

import logging

import torch

from .. import _native as N

logger = logging.getLogger("kineticEQ")

FIXED_BC = ("fixed_maxwellian", "fixed", "dirichlet")


def _f64_cuda(t: torch.Tensor, name: str) -> torch.Tensor:
    if not t.is_cuda or t.dtype != torch.float64:
        raise RuntimeError(f"{name} must be a float64 CUDA tensor")
    return t.contiguous()


@torch.no_grad()
def maxwellian(state, out: torch.Tensor | None = None) -> torch.Tensor:
    """f_M(n, u, T) of the state's per-row moments (bgk1d_maxwellian.py:7-33),
    computed by keq_maxwellian."""
    lib = N.load()
    n, u, T = (_f64_cuda(t, k) for t, k in ((state.n, "n"), (state.u, "u"), (state.T, "T")))
    v = _f64_cuda(state.v, "v")
    nx, nv = n.numel(), v.numel()
    if out is None:
        out = torch.empty((nx, nv), dtype=torch.float64, device=n.device)
    N.check(lib.keq_maxwellian(n.data_ptr(), u.data_ptr(), T.data_ptr(), v.data_ptr(), nx, nv,
                               out.data_ptr(), N.stream_handle()), "maxwellian")
    return out


def region_moments(x: torch.Tensor, regions):
    """Piecewise-constant (n, u, T) over the region masks of
    bgk1d_set_initial_condition.py:9-44: defaults (1, 0, 1), half-open
    intervals, the region equal to the last one closed on the right."""
    nx = x.numel()
    n = torch.full((nx,), 1.0, device=x.device, dtype=torch.float64)
    u = torch.full((nx,), 0.0, device=x.device, dtype=torch.float64)
    T = torch.full((nx,), 1.0, device=x.device, dtype=torch.float64)
    regions = tuple(regions)
    for r in regions:
        if isinstance(r, dict):
            a, b = r["x_range"]
            rn, ru, rT = r["n"], r["u"], r["T"]
        else:
            a, b = r.x_range
            rn, ru, rT = r.n, r.u, r.T
        mask = (x >= a) & (x <= b) if r == regions[-1] else (x >= a) & (x < b)
        n[mask] = float(rn)
        u[mask] = float(ru)
        T[mask] = float(rT)
    return n, u, T


@torch.no_grad()
def set_initial_condition(state, cfg) -> None:
    regions = getattr(cfg.model_cfg.initial, "initial_regions", ())
    state.n, state.u, state.T = region_moments(state.x, regions)
    maxwellian(state, out=state.f)


@torch.no_grad()
def conservation_totals(f: torch.Tensor, v: torch.Tensor, dx: float, dv: float) -> torch.Tensor:
    """(mass, momentum, energy) of a state: the row moments of keq_row_moments
    summed over x times dx (a float64 device tensor of 3)."""
    lib = N.load()
    f = _f64_cuda(f, "f")
    nx, nv = f.shape
    rows = torch.empty((nx, 3), dtype=torch.float64, device=f.device)
    N.check(lib.keq_row_moments(f.data_ptr(), _f64_cuda(v, "v").data_ptr(), nx, nv, float(dv),
                                rows.data_ptr(), N.stream_handle()), "row moments")
    return rows.sum(0) * float(dx)


def drift(tot: torch.Tensor, tot0: torch.Tensor) -> dict:
    """Conservation drift relative to a reference state: mass and energy
    relative to their reference totals, momentum relative to the reference
    mass (momentum per unit mass, since the total momentum can be zero)."""
    t, t0 = [float(x) for x in tot.cpu()], [float(x) for x in tot0.cpu()]
    return {"mass": (t[0] - t0[0]) / abs(t0[0]), "momentum": (t[1] - t0[1]) / abs(t0[0]),
            "energy": (t[2] - t0[2]) / abs(t0[2])}


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
