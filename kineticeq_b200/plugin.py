"""Drop-in registration into an installed kineticEQ.

kineticEQ routes ``Engine(Config(...))`` through the scheme registry
``kineticEQ.core.schemes.registry._FACTORIES`` (core/schemes/registry.py:15-27),
keyed by (Model, Scheme, Backend); ``Backend`` is a closed enum
(api/config.py:46-49), so this backend does not add a new backend name but
rebinds the two ``cuda_kernel`` entries it replaces:

    (BGK1D1V, IMPLICIT, CUDA_KERNEL)  bgk1d_implicit_cuda_kernel.build_stepper
    (BGK1D1V, HOLO,     CUDA_KERNEL)  bgk1d_holo_cuda_kernel.build_stepper

After ``install()`` an unmodified ``Config(backend="cuda_kernel")`` steps on
the B200 kernels of this package.  The builders take kineticEQ's own Config
and State1D1V objects (same fields as this package's mirror of them) and
keep the reference's stepper contract: ``stepper(step_index)`` advances one
dt, swaps ``state.f``/``state.f_tmp`` and carries ``.benchlog``.
"""
from __future__ import annotations

from typing import Any

_INSTALLED: dict = {}


def _implicit_builder(cfg, state):
    from .schemes import bgk1d_implicit

    return bgk1d_implicit.build_stepper(cfg, state)


def _holo_builder(cfg, state):
    from .schemes import bgk1d_holo

    return bgk1d_holo.build_stepper(cfg, state)


def install(registry: Any = None) -> dict:
    """Rebind kineticEQ's (BGK1D1V, IMPLICIT|HOLO, CUDA_KERNEL) builders to
    this backend.  ``registry`` defaults to the imported
    ``kineticEQ.core.schemes.registry`` module.  Returns the builders that
    were replaced (pass them to ``uninstall``)."""
    if registry is None:
        import kineticEQ.core.schemes.registry as registry  # noqa: PLW0621
    from kineticEQ.api.config import Backend, Model, Scheme

    prev = {}
    for scheme, builder in ((Scheme.IMPLICIT, _implicit_builder), (Scheme.HOLO, _holo_builder)):
        key = (Model.BGK1D1V, scheme, Backend.CUDA_KERNEL)
        prev[key] = registry._FACTORIES.get(key)
        registry._FACTORIES[key] = builder
    _INSTALLED.update(prev)
    return prev


def uninstall(prev: dict | None = None, registry: Any = None) -> None:
    """Restore the builders that ``install`` replaced."""
    if registry is None:
        import kineticEQ.core.schemes.registry as registry  # noqa: PLW0621
    prev = dict(_INSTALLED) if prev is None else prev
    for key, builder in prev.items():
        if builder is None:
            registry._FACTORIES.pop(key, None)
        else:
            registry._FACTORIES[key] = builder
    _INSTALLED.clear()


def installed(registry: Any = None) -> bool:
    if registry is None:
        import kineticEQ.core.schemes.registry as registry  # noqa: PLW0621
    from kineticEQ.api.config import Backend, Model, Scheme

    key = (Model.BGK1D1V, Scheme.IMPLICIT, Backend.CUDA_KERNEL)
    return registry._FACTORIES.get(key) is _implicit_builder
