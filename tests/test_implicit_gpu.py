"""Parity of the CUDA implicit step with the reference (golden fixtures) and
with the CPU oracle, through the public API (Engine / stepper) and the
batched plan.  Tolerance: normwise relative max|d| / max|ref| <= 1e-12 for f
and for the moments (n, nu, T); Picard iteration counts must match."""
import json

import numpy as np
import pytest
import torch

from kineticeq_b200 import BGK1D, Config, Engine
from kineticeq_b200.plan import ImplicitPlan, InstanceSpec, implicit_params_struct
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


def engine_for(nx, nv, dt, tau, sp, steps=1, regions=None):
    mc = BGK1D.ModelConfig(grid=BGK1D.Grid1D1V(nx=nx, nv=nv, Lx=1.0, v_max=10.0),
                           time=BGK1D.TimeConfig(dt=dt, T_total=dt * steps),
                           params=BGK1D.BGK1D1VParams(tau_tilde=tau), scheme_params=sp)
    if regions is not None:
        mc = BGK1D.ModelConfig(grid=mc.grid, time=mc.time, params=mc.params,
                               initial=BGK1D.InitialCondition1D(initial_regions=regions),
                               scheme_params=sp)
    cfg = Config(model="BGK1D1V", scheme="implicit", backend="cuda_kernel", device="cuda",
                 dtype="float64", use_tqdm="false", log_level="warning", model_cfg=mc)
    return Engine(cfg, apply_logging_flag=False)


@pytest.fixture(scope="module")
def gold(golden_dir):
    return np.load(golden_dir / "implicit.npz")


@pytest.mark.parametrize("tag", ["smoke", "sod256", "aa96", "convw", "odd"])
def test_matches_reference_golden(gold, tag):
    meta = json.loads(str(gold[f"{tag}_meta"]))
    sp = BGK1D.implicit.Params(**{k: v for k, v in meta.items() if k not in _SKIP})
    eng = engine_for(meta["nx"], meta["nv"], meta["dt"], meta["tau_tilde"], sp)
    eng.state.f.copy_(torch.from_numpy(gold[f"{tag}_f0"]))
    its = []
    for s in range(meta["steps"]):
        eng.stepper(s)
        its.append(eng.stepper.benchlog["picard_iter"])
    torch.cuda.synchronize()
    assert its == list(gold[f"{tag}_iters"]), (its, list(gold[f"{tag}_iters"]))
    f = eng.state.f.cpu().numpy()
    v = eng.state.v.cpu().numpy()
    if f"{tag}_f" in gold:
        fr = gold[f"{tag}_f"]
        assert rel(f, fr) <= TOL
        for a, b in zip(moments(f, v, eng.state.dv), moments(fr, v, eng.state.dv)):
            assert rel(a, b) <= TOL
    else:
        assert rel(f.sum(1) * eng.state.dv, gold[f"{tag}_n"]) <= TOL


@pytest.mark.parametrize("seed", [0, 1, 2])
def test_matches_oracle_random_riemann(seed):
    rng = np.random.default_rng(seed)
    nx = int(rng.integers(20, 140))
    nv = int(rng.choice([16, 33, 48, 64, 70]))
    xd = float(rng.uniform(0.3, 0.7))
    regions = ({"x_range": (0.0, xd), "n": float(rng.uniform(0.5, 2)), "u": float(rng.uniform(-0.5, 0.5)),
                "T": float(rng.uniform(0.5, 2))},
               {"x_range": (xd, 1.0), "n": float(rng.uniform(0.05, 0.5)), "u": float(rng.uniform(-0.5, 0.5)),
                "T": float(rng.uniform(0.5, 2))})
    tau = float(10 ** rng.uniform(-5, -1))
    aa = bool(seed % 2)
    sp = BGK1D.implicit.Params(picard_iter=60, picard_tol=1e-10, abs_tol=1e-16, aa_enable=aa, aa_m=5)
    dt = 5e-5
    eng = engine_for(nx, nv, dt, tau, sp, regions=regions)
    f_o = eng.state.f.cpu().numpy().copy()
    v = eng.state.v.cpu().numpy()
    p = O.implicit_params(sp)
    for s in range(6):
        eng.stepper(s)
        bl = O.implicit_step(f_o, v, eng.state.dx, eng.state.dv, dt, tau, p)
        assert eng.stepper.benchlog["picard_iter"] == bl["picard_iter"]
        f = eng.state.f.cpu().numpy()
        assert rel(f, f_o) <= TOL, (s, rel(f, f_o))


def test_fixed_iteration_replay_and_residuals():
    sp = BGK1D.implicit.Params(picard_iter=40, picard_tol=1e-10, abs_tol=1e-16)
    eng = engine_for(130, 64, 5e-6, 5e-5, sp)
    f_o = eng.state.f.cpu().numpy().copy()
    v = eng.state.v.cpu().numpy()
    p = O.implicit_params(sp, fixed_iters=3)
    spec = InstanceSpec(v=eng.state.v, dx=eng.state.dx, dv=eng.state.dv, dt=5e-6, tau_tilde=5e-5,
                        a=eng.state.f.clone(), b=torch.empty_like(eng.state.f))
    plan = ImplicitPlan([spec], implicit_params_struct(sp, fixed_iters=3))
    plan.step(1)
    bl = O.implicit_step(f_o, v, eng.state.dx, eng.state.dv, 5e-6, 5e-5, p)
    rec = plan.stats.fetch()[0]
    assert int(rec["iters"]) == 3 == bl["picard_iter"]
    assert rel(plan.state(0).cpu().numpy(), f_o) <= TOL
    np.testing.assert_allclose(float(rec["std_residual"]), bl["std_picard_residual"], rtol=1e-6)


def test_deterministic_bitwise():
    sp = BGK1D.implicit.Params(picard_iter=64, picard_tol=1e-10, abs_tol=1e-16, aa_enable=True, aa_m=5)
    outs = []
    for _ in range(2):
        eng = engine_for(300, 96, 5e-6, 5e-5, sp)
        for s in range(3):
            eng.stepper(s)
        outs.append(eng.state.f.cpu().numpy())
    assert np.array_equal(outs[0], outs[1])


def test_batch_equals_alone():
    sizes = [(40, 16, 1e-3), (200, 64, 5e-5), (129, 33, 2e-2), (520, 128, 1e-4)]
    sp = BGK1D.implicit.Params(picard_iter=64, picard_tol=1e-10, abs_tol=1e-16)
    dt = 5e-6
    specs, alone = [], []
    for nx, nv, tau in sizes:
        eng = engine_for(nx, nv, dt, tau, sp)
        f0 = eng.state.f.clone()
        for s in range(2):
            eng.stepper(s)
        alone.append(eng.state.f.cpu().numpy())
        specs.append(InstanceSpec(v=eng.state.v, dx=eng.state.dx, dv=eng.state.dv, dt=dt,
                                  tau_tilde=tau, a=f0, b=torch.empty_like(f0)))
    plan = ImplicitPlan(specs, sp)
    plan.step(2)
    for i in range(len(sizes)):
        assert np.array_equal(plan.state(i).cpu().numpy(), alone[i]), i


def test_nonfinite_raises_value_error():
    sp = BGK1D.implicit.Params(picard_iter=8, picard_tol=1e-6)
    eng = engine_for(50, 32, 5e-6, 5e-3, sp)
    eng.state.f[10, 5] = float("nan")
    with pytest.raises(ValueError, match="NaN/Inf detected in f_tmp"):
        eng.stepper(0)


def test_kernel_dropins_match_reference(golden_dir):
    from kineticeq_b200.cuda_kernel import load_gtsv, load_implicit_fused, load_lo_blocktridiag

    d = np.load(golden_dir / "kernels.npz")
    cu = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()  # noqa: E731
    mod = load_implicit_fused()
    f = cu(d["kat_mom_f"])
    v = cu(d["kat_mom_v"])
    nx = f.shape[0]
    n, nu, T = (torch.zeros(nx, dtype=torch.float64, device="cuda") for _ in range(3))
    mod.moments_n_nu_T(f, v, float(d["kat_mom_dv"]), n, nu, T)
    for a, b in ((n, "n"), (nu, "nu"), (T, "T")):
        assert rel(a.cpu().numpy(), d[f"kat_mom_{b}"]) <= 1e-14
    dt, dx, tau = (float(x) for x in d["kat_sys_scal"])
    B0 = cu(d["kat_sys_B0"])
    dl, dd, du, B = (torch.zeros_like(B0) for _ in range(4))
    mod.build_system_from_moments(B0, v, dt, dx, tau, 1.0 / np.sqrt(2 * np.pi), cu(d["kat_sys_n"]),
                                  cu(d["kat_sys_nu"]), cu(d["kat_sys_T"]), cu(d["kat_sys_fl"]),
                                  cu(d["kat_sys_fr"]), dl, dd, du, B)
    for a, b in ((dl, "dl"), (dd, "dd"), (du, "du"), (B, "B")):
        assert rel(a.cpu().numpy(), d[f"kat_sys_{b}"]) <= 1e-14, b
    gt = load_gtsv()
    X = gt.gtsv_strided(dl, dd, du, B)
    assert rel(X.cpu().numpy(), d["kat_gtsv_X"]) <= 1e-14
    Xg = gt.gtsv_strided(cu(d["kat_gen_dl"]), cu(d["kat_gen_d"]), cu(d["kat_gen_du"]), cu(d["kat_gen_B"]))
    assert rel(Xg.cpu().numpy(), d["kat_gen_X"]) <= 1e-13
    rng = np.random.default_rng(3)
    nb = 40
    A = rng.normal(size=(nb, 3, 3)) * 0.1
    C = rng.normal(size=(nb, 3, 3)) * 0.1
    Bm = np.eye(3)[None] * 2.0 + rng.normal(size=(nb, 3, 3)) * 0.1
    D = rng.normal(size=(nb, 3))
    Xb = load_lo_blocktridiag().block_tridiag_solve(cu(A), cu(Bm), cu(C), cu(D))
    assert rel(Xb.cpu().numpy(), O.block_tridiag_solve(A, Bm, C, D)) <= 1e-13
