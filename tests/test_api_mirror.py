"""Host-side mirror of the reference interface (no GPU)."""
import pytest

from kineticeq_b200 import BGK1D, Config
from kineticeq_b200.api.config import Backend, Model, Scheme
from kineticeq_b200.params.registry import default_scheme_params
from kineticeq_b200.schemes import registry


def test_config_aliases_and_errors():
    c = Config(model="bgk1d", scheme="imp", backend="cuda_backend", dtype="fp64", log_level="err",
               use_tqdm="false")
    assert c.model is Model.BGK1D1V and c.scheme is Scheme.IMPLICIT
    assert c.backend is Backend.CUDA_KERNEL and c.dtype_name == "float64"
    assert c.as_dict["backend"] == "cuda_kernel" and not c.use_tqdm_bool
    with pytest.raises(ValueError, match="unknown Scheme"):
        Config(scheme="holo_nn")


def test_params_defaults_match_reference():
    sp = BGK1D.implicit.Params()
    assert (sp.picard_iter, sp.picard_tol, sp.abs_tol, sp.conv_type) == (16, 1e-4, 1e-16, "f")
    assert (sp.aa_m, sp.aa_beta, sp.aa_start_iter, sp.aa_reg, sp.aa_alpha_max) == (6, 1.0, 2, 1e-10, 50.0)
    hp = BGK1D.holo.Params()
    assert (hp.ho_iter, hp.ho_tol, hp.lo_iter, hp.lo_abs_tol) == (8, 1e-4, 16, 1e-12)
    assert BGK1D.TimeConfig(dt=5e-6, T_total=5e-4).n_steps == 100
    assert isinstance(default_scheme_params(Model.BGK1D1V, Scheme.IMPLICIT), BGK1D.implicit.Params)


def test_registry_rejects_unregistered_keys():
    cfg = Config(model="BGK1D1V", scheme="explicit", backend="cuda_kernel")
    with pytest.raises(NotImplementedError, match="scheme not registered"):
        registry.build_stepper(cfg, None)
    cfg = Config(model="BGK1D1V", scheme="implicit", backend="torch")
    with pytest.raises(NotImplementedError):
        registry.build_stepper(cfg, None)
