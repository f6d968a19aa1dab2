"""Default model / scheme parameters (params/registry.py:9-37)."""
from __future__ import annotations

from typing import Any

from ..api.config import Model, Scheme
from .BGK1D1V import holo, implicit
from .BGK1D1V.model import ModelConfig

_FACTORIES = {Model.BGK1D1V: ModelConfig}
_SCHEME_PARAMS = {(Model.BGK1D1V, Scheme.IMPLICIT): implicit.Params,
                  (Model.BGK1D1V, Scheme.HOLO): holo.Params}


def default_model_cfg(model: Model) -> Any:
    try:
        return _FACTORIES[model]()
    except KeyError as e:
        raise NotImplementedError(f"model not provided by this backend: {model}") from e


def expected_model_cfg_type(model: Model) -> type:
    try:
        return _FACTORIES[model]
    except KeyError as e:
        raise NotImplementedError(f"model not provided by this backend: {model}") from e


def default_scheme_params(model: Model, scheme: Scheme) -> Any:
    f = _SCHEME_PARAMS.get((model, scheme))
    return None if f is None else f()
