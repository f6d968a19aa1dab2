"""Parity of the CUDA HOLO step with the reference (golden fixtures made by
tests/golden/make_golden.py from the reference's own HOLO step) and with the
CPU oracle, through the public API and the batched plan.  Tolerance:
normwise relative max|d| / max|ref| <= 1e-12 in f and in the row moments;
HO and LO iteration counts equal; max_YI within 1e-6 relative (it is a
maximum of consistency terms that are differences of nearly equal sums)."""
import json

import numpy as np
import pytest
import torch

from kineticeq_b200 import BGK1D, Config, Engine
from kineticeq_b200 import _native as N
from kineticeq_b200.plan import HoloPlan, InstanceSpec, holo_params_struct
from kineticeq_b200.schemes.common import maxwellian, region_moments
from kineticeq_b200.state import allocate_state_1d1v
from oracle import oracle as O

pytestmark = pytest.mark.gpu
TOL = 1e-12
_SKIP = ("nx", "nv", "dt", "T_total", "tau_tilde", "steps")


def rel(a, b):
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


def moments(f, v, dv):
    n = f.sum(1) * dv
    nu = (f * v).sum(1) * dv
    s2 = (f * v * v).sum(1) * dv
    return n, nu, s2 / n - (nu / n) ** 2


def engine_for(nx, nv, dt, tau, sp, regions=None):
    kw = {}
    if regions is not None:
        kw["initial"] = BGK1D.InitialCondition1D(initial_regions=regions)
    mc = BGK1D.ModelConfig(grid=BGK1D.Grid1D1V(nx=nx, nv=nv, Lx=1.0, v_max=10.0),
                           time=BGK1D.TimeConfig(dt=dt, T_total=dt),
                           params=BGK1D.BGK1D1VParams(tau_tilde=tau), scheme_params=sp, **kw)
    cfg = Config(model="BGK1D1V", scheme="holo", backend="cuda_kernel", device="cuda",
                 dtype="float64", use_tqdm="false", log_level="warning", model_cfg=mc)
    return Engine(cfg, apply_logging_flag=False)


@pytest.mark.parametrize("tag", ["holo64", "holo_nocons"])
def test_holo_matches_reference_golden(golden_dir, tag):
    d = np.load(golden_dir / "holo.npz")
    meta = json.loads(str(d[f"{tag}_meta"]))
    sp = BGK1D.holo.Params(**{k: v for k, v in meta.items() if k not in _SKIP})
    eng = engine_for(meta["nx"], meta["nv"], meta["dt"], meta["tau_tilde"], sp)
    eng.state.f.copy_(torch.from_numpy(d[f"{tag}_f0"]))
    logs = []
    for s in range(meta["steps"]):
        eng.stepper(s)
        bl = eng.stepper.benchlog
        logs.append([bl["ho_iter"], bl["lo_iter"], bl["std_ho_residual"], bl["max_YI"]])
    logs = np.array(logs)
    ref = d[f"{tag}_log"]
    assert (logs[:, :2] == ref[:, :2]).all(), (logs, ref)
    np.testing.assert_allclose(logs[:, 3], ref[:, 3], rtol=1e-6, atol=1e-300)
    f = eng.state.f.cpu().numpy()
    assert rel(f, d[f"{tag}_f"]) <= TOL, rel(f, d[f"{tag}_f"])


def _sod(nx, nv):
    st = allocate_state_1d1v(nx, nv, 1.0, 10.0, "cuda", torch.float64)
    st.n, st.u, st.T = region_moments(st.x, ({"x_range": (0.0, 0.5), "n": 1.0, "u": 0.0, "T": 1.0},
                                             {"x_range": (0.5, 1.0), "n": 0.125, "u": 0.0,
                                              "T": 0.8}))
    maxwellian(st, out=st.f)
    return st


def _run_vs_oracle(st, dt, tau, steps, replay=False, **sp):
    f_o = st.f.cpu().numpy().copy()
    v = st.v.cpu().numpy()
    p_o = O.holo_params(None, **sp)
    spec = InstanceSpec(v=st.v, dx=st.dx, dv=st.dv, dt=dt, tau_tilde=tau, a=st.f,
                        b=torch.empty_like(st.f))
    plan = HoloPlan([spec], holo_params_struct(None, **sp))
    for s in range(steps):
        bl = O.holo_step(f_o, v, st.dx, st.dv, dt, tau, p_o)
        if replay:
            cur = plan.state(0)
            spec2 = InstanceSpec(v=st.v, dx=st.dx, dv=st.dv, dt=dt, tau_tilde=tau, a=cur,
                                 b=torch.empty_like(cur))
            plan = HoloPlan([spec2], holo_params_struct(None, fixed_ho_iters=bl["ho_iter"], **sp))
        plan.step(1)
        rec = plan.stats.fetch()[0]
        assert int(rec["status"]) == N.KEQ_OK
        assert int(rec["iters"]) == bl["ho_iter"], (s, int(rec["iters"]), bl)
        if not replay:
            assert int(rec["lo_iters"]) == bl["lo_iter"], (s, int(rec["lo_iters"]), bl)
        f = plan.state(0).cpu().numpy()
        assert rel(f, f_o) <= TOL, (s, rel(f, f_o))
    for a, b in zip(moments(f, v, st.dv), moments(f_o, v, st.dv)):
        assert rel(a, b) <= TOL
    return plan


def test_holo_sod_256x128_vs_oracle():
    _run_vs_oracle(_sod(256, 128), 5e-6, 5e-5, 5, ho_iter=64, ho_tol=1e-10, lo_iter=64,
                   lo_tol=1e-10)


def test_holo_4096x512_vs_oracle():
    _run_vs_oracle(_sod(4096, 512), 1e-5, 5e-5, 2, ho_iter=64, ho_tol=1e-10, lo_iter=64,
                   lo_tol=1e-10)


@pytest.mark.parametrize("seed", [0, 1, 2])
def test_holo_random_riemann_vs_oracle(seed):
    rng = np.random.default_rng(100 + seed)
    nx = int(rng.integers(20, 300))
    nv = int(rng.choice([16, 33, 48, 64, 70]))
    xd = float(rng.uniform(0.3, 0.7))
    regions = ({"x_range": (0.0, xd), "n": float(rng.uniform(0.5, 2)), "u": float(rng.uniform(-0.5, 0.5)),
                "T": float(rng.uniform(0.5, 2))},
               {"x_range": (xd, 1.0), "n": float(rng.uniform(0.05, 0.5)), "u": float(rng.uniform(-0.5, 0.5)),
                "T": float(rng.uniform(0.5, 2))})
    st = allocate_state_1d1v(nx, nv, 1.0, 10.0, "cuda", torch.float64)
    st.n, st.u, st.T = region_moments(st.x, regions)
    maxwellian(st, out=st.f)
    tau = float(10 ** rng.uniform(-4, -1))
    dt = 0.5 / (10.0 * (nx - 1))  # CFL 0.5
    flags = dict(Con_Terms_do=bool(seed != 1), flux_consistency_do=bool(seed != 2))
    _run_vs_oracle(st, dt, tau, 4, ho_iter=40, ho_tol=1e-10, lo_iter=40, lo_tol=1e-10, **flags)


def test_holo_replay_fixed_iterations():
    _run_vs_oracle(_sod(300, 64), 5e-6, 5e-4, 3, replay=True, ho_iter=64, ho_tol=1e-10,
                   lo_iter=64, lo_tol=1e-10)


def test_holo_batch_equals_alone():
    sizes = [(40, 16, 1e-3), (200, 64, 5e-5), (129, 33, 2e-2), (520, 128, 1e-4)]
    sp = dict(ho_iter=32, ho_tol=1e-10, lo_iter=32, lo_tol=1e-10)
    dt = 5e-6
    specs, alone = [], []
    for nx, nv, tau in sizes:
        st = _sod(nx, nv)
        f0 = st.f.clone()
        spec = InstanceSpec(v=st.v, dx=st.dx, dv=st.dv, dt=dt, tau_tilde=tau, a=st.f,
                            b=torch.empty_like(st.f))
        p = HoloPlan([spec], holo_params_struct(None, **sp))
        p.step(2)
        alone.append(p.state(0).cpu().numpy())
        specs.append(InstanceSpec(v=st.v, dx=st.dx, dv=st.dv, dt=dt, tau_tilde=tau, a=f0,
                                  b=torch.empty_like(f0)))
    plan = HoloPlan(specs, holo_params_struct(None, **sp))
    plan.step(2)
    for i in range(len(sizes)):
        assert np.array_equal(plan.state(i).cpu().numpy(), alone[i]), i


def test_holo_cfl_violation_raises():
    sp = BGK1D.holo.Params()
    with pytest.raises(ValueError, match="CFL violated"):
        engine_for(256, 64, 1e-3, 5e-3, sp)


def test_holo_state_moments_side_effect():
    """state.n/u/T hold the last LO moments (bgk1d_holo_cuda_kernel.py:513-514):
    finite, one value per cell, and close to the moments of the new f."""
    sp = BGK1D.holo.Params(ho_iter=32, ho_tol=1e-10, lo_iter=32, lo_tol=1e-10)
    eng = engine_for(100, 48, 5e-6, 5e-4, sp)
    eng.stepper(0)
    n, u, T = (t.cpu().numpy() for t in (eng.state.n, eng.state.u, eng.state.T))
    f = eng.state.f.cpu().numpy()
    v = eng.state.v.cpu().numpy()
    assert n.shape == (100,) and np.isfinite(n).all() and np.isfinite(u).all() and np.isfinite(T).all()
    nf, nuf, Tf = moments(f, v, eng.state.dv)
    assert rel(n, nf) < 1e-3 and rel(T, Tf) < 1e-3
