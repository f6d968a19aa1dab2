"""install() rebinds the real kineticEQ registry (imported from a scratch
copy of the reference checkout, the recipe of tests/golden/make_golden.py).
Runs on the CPU: the dispatch is shown by reaching this backend's builder,
which refuses a CPU state with its own error message.  Skipped where the
reference checkout is absent."""
import importlib.metadata as md
import os
import shutil
import sys
import tempfile
from pathlib import Path

import pytest

REF = Path(os.environ.get("KEQ_REFERENCE", "/root/reference"))


@pytest.fixture(scope="module")
def kineticEQ():
    if not (REF / "src" / "kineticEQ").exists():
        pytest.skip("reference checkout not available")
    scratch = Path(tempfile.gettempdir()) / "keq_plugin_ref"
    if scratch.exists():
        shutil.rmtree(scratch)
    shutil.copytree(REF / "src", scratch / "src")
    orig = md.version
    md.version = lambda n: "2.2.0" if n == "kineticEQ" else orig(n)
    sys.path.insert(0, str(scratch / "src"))
    try:
        import kineticEQ as K
    finally:
        md.version = orig
    return K


def test_install_rebinds_cuda_kernel_entries(kineticEQ):
    from kineticEQ.api.config import Backend, Model, Scheme
    import kineticEQ.core.schemes.registry as R

    from kineticeq_b200 import plugin

    orig_imp = R._FACTORIES[(Model.BGK1D1V, Scheme.IMPLICIT, Backend.CUDA_KERNEL)]
    prev = plugin.install()
    try:
        assert plugin.installed()
        for sch in (Scheme.IMPLICIT, Scheme.HOLO):
            assert R._FACTORIES[(Model.BGK1D1V, sch, Backend.CUDA_KERNEL)].__module__ == \
                "kineticeq_b200.plugin"
        # other entries untouched; unknown keys still raise NotImplementedError
        assert R._FACTORIES[(Model.BGK1D1V, Scheme.IMPLICIT, Backend.CPU_KERNEL)].__module__.startswith(
            "kineticEQ.")
        # an unmodified Config(backend="cuda_kernel") now reaches this backend
        cfg = kineticEQ.Config(model="BGK1D1V", scheme="implicit", backend="cuda_kernel",
                               device="cpu", dtype="float64", log_level="warning")
        from kineticEQ.params.registry import default_model_cfg, default_scheme_params
        from dataclasses import replace

        mc = default_model_cfg(cfg.model)
        mc = replace(mc, scheme_params=default_scheme_params(cfg.model, cfg.scheme))
        cfg = replace(cfg, model_cfg=mc)
        from kineticEQ.core.states.registry import build_state

        state = build_state(cfg)
        with pytest.raises(RuntimeError, match="B200 backend needs device='cuda'"):
            R.build_stepper(cfg, state)
        cfg_h = replace(cfg, scheme=Scheme.HOLO,
                        model_cfg=replace(mc, scheme_params=default_scheme_params(cfg.model,
                                                                                  Scheme.HOLO)))
        with pytest.raises(RuntimeError, match="B200 backend needs device='cuda'"):
            R.build_stepper(cfg_h, state)
    finally:
        plugin.uninstall(prev)
    assert R._FACTORIES[(Model.BGK1D1V, Scheme.IMPLICIT, Backend.CUDA_KERNEL)] is orig_imp
    assert not plugin.installed()
