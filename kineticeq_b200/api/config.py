"""Config mirror of kineticEQ's api/config.py:9-149.

Same field names, enum values, aliases and validation errors, so scripts that
build a ``kineticEQ.Config`` run unchanged against this package.
"""
from __future__ import annotations

from dataclasses import dataclass
from enum import Enum
from typing import Any, Mapping, Type, TypeVar

E = TypeVar("E", bound=Enum)


def parse_enum(enum_cls: Type[E], x, *, aliases: Mapping[str, E] | None = None) -> E:
    """Normalise a string/enum to ``enum_cls`` (api/config.py:9-32): enum
    members pass through; strings are stripped, lower-cased, looked up in the
    aliases, then matched against the member values.  Unknown -> ValueError."""
    if isinstance(x, enum_cls):
        return x
    key = str(x).strip().lower()
    if aliases and key in aliases:
        return aliases[key]
    for member in enum_cls:
        if key == str(member.value).lower():
            return member
    allowed = [str(m.value) for m in enum_cls]
    if aliases:
        allowed += [f"{k}->{v.value}" for k, v in aliases.items()]
    raise ValueError(f"unknown {enum_cls.__name__}: {x!r}. allowed: {allowed}")


class Model(str, Enum):
    BGK1D1V = "BGK1D1V"
    BGK2D2V = "BGK2D2V"


class Scheme(str, Enum):
    EXPLICIT = "explicit"
    IMPLICIT = "implicit"
    HOLO = "holo"


class Backend(str, Enum):
    TORCH = "torch"
    CUDA_KERNEL = "cuda_kernel"
    CPU_KERNEL = "cpu_kernel"


class DType(str, Enum):
    FLOAT32 = "float32"
    FLOAT64 = "float64"


class LogLevel(str, Enum):
    DEBUG = "debug"
    INFO = "info"
    WARNING = "warning"
    ERROR = "error"


class UseTqdm(str, Enum):
    TRUE = "true"
    FALSE = "false"


_MODEL_ALIASES = {"bgk1d": Model.BGK1D1V, "bgk1d1v": Model.BGK1D1V, "bgk2d2v": Model.BGK2D2V}
_SCHEME_ALIASES = {"exp": Scheme.EXPLICIT, "imp": Scheme.IMPLICIT, "hl": Scheme.HOLO}
_BACKEND_ALIASES = {"pytorch": Backend.TORCH, "cuda_backend": Backend.CUDA_KERNEL,
                    "cpu_backend": Backend.CPU_KERNEL}
_DTYPE_ALIASES = {"fp32": DType.FLOAT32, "fp64": DType.FLOAT64}
_TQDM_ALIASES = {"true": UseTqdm.TRUE, "false": UseTqdm.FALSE}
_LOG_ALIASES = {"debug": LogLevel.DEBUG, "info": LogLevel.INFO, "warning": LogLevel.WARNING,
                "err": LogLevel.ERROR}


@dataclass(frozen=True)
class Config:
    model: Any = Model.BGK1D1V
    scheme: Any = Scheme.EXPLICIT
    backend: Any = Backend.TORCH
    device: str = "cuda"
    dtype: Any = DType.FLOAT64
    log_level: Any = LogLevel.INFO
    model_cfg: Any | None = None
    use_tqdm: Any = UseTqdm.TRUE

    def __post_init__(self):
        put = lambda k, v: object.__setattr__(self, k, v)  # noqa: E731
        put("model", parse_enum(Model, self.model, aliases=_MODEL_ALIASES))
        put("scheme", parse_enum(Scheme, self.scheme, aliases=_SCHEME_ALIASES))
        put("backend", parse_enum(Backend, self.backend, aliases=_BACKEND_ALIASES))
        put("dtype", parse_enum(DType, self.dtype, aliases=_DTYPE_ALIASES))
        put("device", str(self.device).strip())
        put("use_tqdm", parse_enum(UseTqdm, self.use_tqdm, aliases=_TQDM_ALIASES))
        put("log_level", parse_enum(LogLevel, self.log_level, aliases=_LOG_ALIASES))

    @property
    def model_name(self) -> str:
        return self.model.value

    @property
    def scheme_name(self) -> str:
        return self.scheme.value

    @property
    def backend_name(self) -> str:
        return self.backend.value

    @property
    def dtype_name(self) -> str:
        return self.dtype.value

    @property
    def log_level_name(self) -> str:
        return self.log_level.value

    @property
    def use_tqdm_name(self) -> str:
        return self.use_tqdm.value

    @property
    def use_tqdm_bool(self) -> bool:
        return self.use_tqdm == UseTqdm.TRUE

    @property
    def as_dict(self) -> dict:
        return {"model": self.model.value, "scheme": self.scheme.value,
                "backend": self.backend.value, "device": self.device,
                "dtype": self.dtype.value, "log_level": self.log_level.value,
                "model_cfg": self.model_cfg, "use_tqdm": self.use_tqdm.value}
