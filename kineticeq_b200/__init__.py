"""kineticeq_b200 -- B200-native (sm_100a) backend for kineticEQ's BGK1D1V
implicit (Picard + Anderson) and HOLO time steps.

Public surface mirrors the reference's: ``Config``, ``Engine``, ``run``,
``BGK1D`` (parameter dataclasses); ``plugin.install()`` routes an unmodified
kineticEQ installation's ``backend="cuda_kernel"`` implicit/HOLO entries to
this backend.  All compute runs in ``lib/libkeq_b200.so`` (C ABI in
``include/keq_b200.h``).
"""
from .api import Config, Engine, Result, run  # noqa: F401
from .params import BGK1D  # noqa: F401

__version__ = "0.1.0"
__all__ = ["Config", "Engine", "run", "Result", "BGK1D", "__version__"]
