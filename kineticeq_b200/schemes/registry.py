"""(Model, Scheme, Backend) -> stepper builder (core/schemes/registry.py:7-35).

This backend registers the two entries it replaces,
(BGK1D1V, IMPLICIT, CUDA_KERNEL) and (BGK1D1V, HOLO, CUDA_KERNEL); any other
key raises NotImplementedError exactly as the reference does.
"""
from __future__ import annotations

from typing import Any, Callable

from ..api.config import Backend, Config, Model, Scheme
from . import bgk1d_holo, bgk1d_implicit

_FACTORIES: dict = {
    (Model.BGK1D1V, Scheme.IMPLICIT, Backend.CUDA_KERNEL): bgk1d_implicit.build_stepper,
    (Model.BGK1D1V, Scheme.HOLO, Backend.CUDA_KERNEL): bgk1d_holo.build_stepper,
}


def build_stepper(cfg: Config, state: Any) -> Stepper:
    key = (cfg.model, cfg.scheme, cfg.backend)
    try:
        builder = _FACTORIES[key]
    except KeyError as e:
        raise NotImplementedError(f"scheme not registered: {key}") from e
    return builder(cfg, state)
