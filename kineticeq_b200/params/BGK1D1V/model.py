"""BGK1D1V model configuration (params/BGK1D1V/BGK1D1V_params.py:6-61)."""
from __future__ import annotations

import math
from dataclasses import dataclass, field
from typing import Any


@dataclass(frozen=True)
class Grid1D1V:
    nx: int = 124
    nv: int = 64
    Lx: float = 1.0
    v_max: float = 10.0


@dataclass(frozen=True)
class TimeConfig:
    dt: float = 5e-4
    T_total: float = 0.05

    @property
    def n_steps(self) -> int:
        """ceil(T_total/dt), at least 1."""
        return int(max(1, math.ceil(self.T_total / self.dt)))


@dataclass(frozen=True)
class BGK1D1VParams:
    tau_tilde: float = 5e-1


@dataclass(frozen=True)
class InitialCondition1D:
    initial_regions: tuple = (
        {"x_range": (0.0, 0.5), "n": 1.0, "u": 0.0, "T": 1.0},
        {"x_range": (0.5, 1.0), "n": 0.125, "u": 0.0, "T": 0.8},
    )


@dataclass(frozen=True)
class BoundaryCondition1D:
    bc_type: str = "fixed_maxwellian"
    Lwall_temperature: float = 1.0
    Rwall_temperature: float = 1.0


@dataclass(frozen=True)
class ModelConfig:
    grid: Grid1D1V = field(default_factory=Grid1D1V)
    time: TimeConfig = field(default_factory=TimeConfig)
    params: BGK1D1VParams = field(default_factory=BGK1D1VParams)
    initial: InitialCondition1D = field(default_factory=InitialCondition1D)
    boundary: BoundaryCondition1D = field(default_factory=BoundaryCondition1D)
    scheme_params: Any = None
