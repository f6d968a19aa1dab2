"""Parameter dataclasses mirroring kineticEQ's params/ package
(params/BGK1D1V/BGK1D1V_params.py:6-61, implicit.py:4-37, holo.py:4-13,
params/registry.py:9-37).  ``BGK1D`` is the namespace the reference exports."""
from . import BGK1D1V as BGK1D  # noqa: F401
from .registry import default_model_cfg, default_scheme_params, expected_model_cfg_type  # noqa: F401
