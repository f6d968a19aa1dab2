"""BGK1D1V state (core/states/state_1d.py:8-66).

f is (nx, nv) row-major, v contiguous.  The velocity and space grids are
``torch.linspace`` on the host in float64 and copied to the device, so every
device sees the same grid values bit for bit.
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import torch

from .api.config import Config, DType


@dataclass
class State1D1V:
    f: torch.Tensor
    f_tmp: torch.Tensor
    f_m: torch.Tensor
    x: torch.Tensor
    v: torch.Tensor
    n: torch.Tensor
    u: torch.Tensor
    T: torch.Tensor
    dv: float
    dx: float
    v_col: torch.Tensor
    inv_sqrt_2pi: torch.Tensor
    pos_mask: torch.Tensor
    neg_mask: torch.Tensor
    v_coeff: torch.Tensor
    k0: int


def allocate_state_1d1v(nx, nv, Lx, v_max, device, dtype) -> State1D1V:
    if nx < 3 or nv < 2:
        raise ValueError(f"grid too small: nx={nx} (>=3), nv={nv} (>=2)")
    f = torch.zeros((nx, nv), device=device, dtype=dtype)
    n = torch.ones(nx, device=device, dtype=dtype)
    u = torch.zeros(nx, device=device, dtype=dtype)
    T = torch.ones(nx, device=device, dtype=dtype)
    x = torch.linspace(0, Lx, nx, dtype=torch.float64).to(device=device, dtype=dtype)
    v = torch.linspace(-v_max, v_max, nv, dtype=torch.float64).to(device=device, dtype=dtype)
    dx = float(Lx / (nx - 1))
    dv = float((2.0 * v_max) / (nv - 1))
    pos = v > 0
    k0 = int(torch.searchsorted(v.cpu(), torch.tensor(0.0, dtype=v.dtype)))
    return State1D1V(
        f=f, f_tmp=torch.zeros_like(f), f_m=torch.zeros_like(f), x=x, v=v, n=n, u=u, T=T,
        dv=dv, dx=dx, v_col=v[None, :],
        inv_sqrt_2pi=torch.tensor(1.0 / math.sqrt(2.0 * math.pi), device=device, dtype=dtype),
        pos_mask=pos, neg_mask=~pos, v_coeff=(-v / dx), k0=k0)


def build_state(cfg: Config) -> State1D1V:
    g = cfg.model_cfg.grid
    dtype = torch.float64 if cfg.dtype == DType.FLOAT64 else torch.float32
    return allocate_state_1d1v(g.nx, g.nv, g.Lx, g.v_max, cfg.device, dtype)
