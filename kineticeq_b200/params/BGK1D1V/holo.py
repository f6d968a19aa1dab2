"""holo.Params (params/BGK1D1V/holo.py:4-13)."""
from __future__ import annotations

from dataclasses import dataclass


@dataclass(frozen=True)
class Params:
    ho_iter: int = 8
    ho_tol: float = 1e-4
    ho_abs_tol: float = 1e-12
    lo_iter: int = 16
    lo_tol: float = 1e-4
    lo_abs_tol: float = 1e-12
    Con_Terms_do: bool = True
    flux_consistency_do: bool = True
