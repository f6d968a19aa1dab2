from .config import Backend, Config, DType, Model, Scheme  # noqa: F401
from .engine import Engine, Result, run  # noqa: F401
