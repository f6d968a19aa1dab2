from .model import (  # noqa: F401
    BGK1D1VParams,
    BoundaryCondition1D,
    Grid1D1V,
    InitialCondition1D,
    ModelConfig,
    TimeConfig,
)
from . import holo, implicit  # noqa: F401
