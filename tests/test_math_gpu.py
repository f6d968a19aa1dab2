"""Device math helpers against CUDA's own exp and IEEE division."""
import numpy as np
import pytest
import torch

from kineticeq_b200 import _native as N

pytestmark = pytest.mark.gpu


def _run(kind, x):
    lib = N.load()
    xd = torch.from_numpy(x).cuda()
    yd = torch.empty_like(xd)
    N.check(lib.keq_math_selftest(kind, xd.data_ptr(), yd.data_ptr(), xd.numel(), N.stream_handle()),
            "selftest")
    return yd


def ulp_err(a, b):
    a = a.cpu().numpy() if hasattr(a, "cpu") else a
    b = b.cpu().numpy() if hasattr(b, "cpu") else b
    return np.abs(a - b) / np.spacing(np.maximum(np.abs(b), np.finfo(np.float64).tiny))


def test_exp_nonpos_matches_cuda_exp():
    rng = np.random.default_rng(11)
    x = np.concatenate([-rng.uniform(0, 1, 200000), -rng.uniform(0, 40, 200000),
                        -rng.uniform(0, 745, 200000), -np.logspace(-300, 2.8, 20000),
                        np.array([0.0, -0.0, -1e-320, -708.39, -708.4, -744.0, -745.1, -746.0, -1e300])])
    y = _run(0, x)
    ref = torch.exp(torch.from_numpy(x).cuda())
    normal = ref.cpu().numpy() >= np.finfo(np.float64).tiny
    assert ulp_err(y, ref)[normal].max() <= 2.0
    # subnormal results: absolute agreement within one subnormal step
    assert np.abs((y - ref).cpu().numpy()[~normal]).max() <= 2 * 4.9407e-324
    assert torch.isnan(_run(0, np.array([np.nan])))[0]
    assert _run(0, np.array([-np.inf]))[0].item() == 0.0


def test_recip_ge1_matches_division():
    rng = np.random.default_rng(12)
    x = np.concatenate([1.0 + rng.uniform(0, 1, 200000), 10 ** rng.uniform(0, 30, 200000),
                        np.array([1.0, 2.0, 3.0, 1e38, 3e38])])
    y = _run(1, x)
    assert ulp_err(y, 1.0 / x).max() <= 1.0
