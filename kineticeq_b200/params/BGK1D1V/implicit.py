"""implicit.Params (params/BGK1D1V/implicit.py:4-37)."""
from __future__ import annotations

from dataclasses import dataclass


@dataclass(frozen=True)
class Params:
    # Picard iteration
    picard_iter: int = 16
    picard_tol: float = 1e-4
    abs_tol: float = 1e-16
    # convergence type: "f" (distribution) or "w" (moments)
    conv_type: str = "f"
    # Anderson acceleration on W = (n, nu, T)
    aa_enable: bool = False
    aa_m: int = 6
    aa_beta: float = 1.0
    aa_stride: int = 1
    aa_start_iter: int = 2
    aa_reg: float = 1e-10
    aa_alpha_max: float = 50.0
    # CNN warm start (not provided by this backend; a model path raises)
    warm_enable: bool | None = None
    moments_cnn_modelpath: str | None = None
    warm_delta_weight_mode: str = "none"
    warm_delta_weight_floor: float = 0.2
    warm_delta_weight_center: float = 0.5
    warm_delta_weight_sharpness: float = 10.0
    warm_delta_weight_sigma: float = 3.0
    warm_delta_exclude_cells: int = 0
