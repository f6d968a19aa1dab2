"""Parity of the CUDA implicit step with the CPU oracle at the benchmarked
sizes: 4096 x 512 (Anderson m=5 on and off, tau_tilde 5e-5 and 5e-3, three
steps each) and 8192 x 1024 (Anderson m=5, tau_tilde 1e-4: one free-running
step, then three steps replayed with the oracle's per-step iteration counts).
Tolerance: normwise relative max|d| / max|ref| <= 1e-12 in f and in the row
moments (n, nu, T); per-step Picard iteration counts equal; conservation
drift (mass, momentum, energy) equal to the oracle's within 1e-12.
Also the initial condition (Sod and seeded two-state Riemann regions)
against the oracle's."""
import numpy as np
import pytest
import torch

from kineticeq_b200.plan import ImplicitPlan, InstanceSpec, implicit_params_struct
from kineticeq_b200.schemes.common import conservation_totals, drift, maxwellian, region_moments
from kineticeq_b200.state import allocate_state_1d1v
from oracle import oracle as O

pytestmark = pytest.mark.gpu
TOL = 1e-12


def rel(a, b):
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


def row_moments(f, v, dv):
    n = f.sum(1) * dv
    nu = (f * v).sum(1) * dv
    s2 = (f * v * v).sum(1) * dv
    return n, nu, s2 / n - (nu / n) ** 2


def totals_np(f, v, dx, dv):
    return np.array([f.sum() * dv * dx, (f * v).sum() * dv * dx, 0.5 * (f * v * v).sum() * dv * dx])


def drift_np(t, t0):
    return {"mass": (t[0] - t0[0]) / abs(t0[0]), "momentum": (t[1] - t0[1]) / abs(t0[0]),
            "energy": (t[2] - t0[2]) / abs(t0[2])}


def sod_state(nx, nv):
    st = allocate_state_1d1v(nx, nv, 1.0, 10.0, "cuda", torch.float64)
    regions = ({"x_range": (0.0, 0.5), "n": 1.0, "u": 0.0, "T": 1.0},
               {"x_range": (0.5, 1.0), "n": 0.125, "u": 0.0, "T": 0.8})
    st.n, st.u, st.T = region_moments(st.x, regions)
    maxwellian(st, out=st.f)
    return st


def run_case(nx, nv, dt, tau, steps, replay_after=None, **sp):
    st = sod_state(nx, nv)
    f_o = st.f.cpu().numpy().copy()
    f0 = f_o.copy()
    v = st.v.cpu().numpy()
    p_o = O.implicit_params(None, **sp)
    tot0 = conservation_totals(st.f, st.v, st.dx, st.dv)
    spec = InstanceSpec(v=st.v, dx=st.dx, dv=st.dv, dt=dt, tau_tilde=tau, a=st.f,
                        b=torch.empty_like(st.f))
    plan = ImplicitPlan([spec], implicit_params_struct(None, **sp))
    for s in range(steps):
        bl = O.implicit_step(f_o, v, st.dx, st.dv, dt, tau, p_o)
        if replay_after is not None and s >= replay_after:
            # replay: a fresh plan forced to the oracle's iteration count
            cur = plan.state(0)
            spec2 = InstanceSpec(v=st.v, dx=st.dx, dv=st.dv, dt=dt, tau_tilde=tau, a=cur,
                                 b=torch.empty_like(cur))
            plan = ImplicitPlan([spec2], implicit_params_struct(None, fixed_iters=bl["picard_iter"],
                                                                **sp))
        plan.step(1)
        rec = plan.stats.fetch()[0]
        assert int(rec["status"]) == 0
        assert int(rec["iters"]) == bl["picard_iter"], (s, int(rec["iters"]), bl["picard_iter"])
        f = plan.state(0).cpu().numpy()
        assert rel(f, f_o) <= TOL, (s, rel(f, f_o))
    for a, b in zip(row_moments(f, v, st.dv), row_moments(f_o, v, st.dv)):
        assert rel(a, b) <= TOL
    dg = drift(conservation_totals(plan.state(0), st.v, st.dx, st.dv), tot0)
    do = drift_np(totals_np(f_o, v, st.dx, st.dv), totals_np(f0, v, st.dx, st.dv))
    for k in dg:
        assert abs(dg[k] - do[k]) <= TOL, (k, dg[k], do[k])


@pytest.mark.parametrize("aa", [True, False])
@pytest.mark.parametrize("tau", [5e-5, 5e-3])
def test_parity_4096x512(aa, tau):
    run_case(4096, 512, 1e-5, tau, 3, picard_iter=64, picard_tol=1e-10, abs_tol=1e-16,
             aa_enable=aa, aa_m=5)


def test_parity_8192x1024_free_then_replay():
    run_case(8192, 1024, 1e-5, 1e-4, 4, replay_after=1, picard_iter=64, picard_tol=1e-10,
             abs_tol=1e-16, aa_enable=True, aa_m=5)


@pytest.mark.parametrize("seed", [None, 0, 1, 2])
def test_initial_condition_matches_oracle(seed):
    if seed is None:
        nx, nv = 256, 128
        regions = ({"x_range": (0.0, 0.5), "n": 1.0, "u": 0.0, "T": 1.0},
                   {"x_range": (0.5, 1.0), "n": 0.125, "u": 0.0, "T": 0.8})
    else:
        g = torch.Generator("cpu").manual_seed(seed)
        u01 = lambda a, b: float(a + (b - a) * torch.rand((), generator=g, dtype=torch.float64))  # noqa: E731
        nx = int(torch.randint(128, 2049, (), generator=g))
        nv = int([64, 128, 256, 512][int(torch.randint(0, 4, (), generator=g))])
        xd = u01(0.3, 0.7)
        regions = ({"x_range": (0.0, xd), "n": u01(0.5, 2), "u": u01(-0.5, 0.5), "T": u01(0.5, 2)},
                   {"x_range": (xd, 1.0), "n": u01(0.05, 0.5), "u": u01(-0.5, 0.5), "T": u01(0.5, 2)})
    st = allocate_state_1d1v(nx, nv, 1.0, 10.0, "cuda", torch.float64)
    st.n, st.u, st.T = region_moments(st.x, regions)
    maxwellian(st, out=st.f)
    reg = [(r["x_range"][0], r["x_range"][1], r["n"], r["u"], r["T"]) for r in regions]
    f_o = O.initial_condition(O.Grid(nx, nv), reg)
    assert rel(st.f.cpu().numpy(), f_o) <= 1e-14
