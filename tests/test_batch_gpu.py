"""Batching form: uneven instances in one plan.  Each of 16 seeded mixed
instances (sizes, tau_tilde and Riemann states drawn as in the batching
workload, Anderson on every other one) equals its solo run bitwise; every
tile height R gives the oracle's result within 1e-12; a CUDA-graph replay of
the per-step launches equals direct stepping bitwise; a disabled instance
(enable mask 0) is left untouched."""
import numpy as np
import pytest
import torch

from kineticeq_b200.batch import BatchSolver, make_state, sample_instances, spec_of
from kineticeq_b200.plan import ImplicitPlan, implicit_params_struct
from oracle import oracle as O

pytestmark = pytest.mark.gpu
SP = dict(picard_iter=64, picard_tol=1e-10, abs_tol=1e-16)


def _small(descs, cap=512):
    for d in descs:
        d.nx = min(d.nx, cap)
    return descs


def test_sixteen_mixed_instances_equal_their_solo_runs():
    descs = _small(sample_instances(16, seed=3))
    params = [implicit_params_struct(None, aa_enable=bool(i % 2), aa_m=5, **SP)
              for i in range(16)]
    states = [make_state(d) for d in descs]
    f0 = [s.f.clone() for s in states]
    solo = []
    for i, (d, s) in enumerate(zip(descs, states)):
        sp = spec_of(d, s)
        sp.a.copy_(f0[i])
        p = ImplicitPlan([sp], params[i])
        p.step(3)
        solo.append(p.state(0).cpu().numpy())
    specs = []
    for d, s, f in zip(descs, states, f0):
        sp = spec_of(d, s)
        sp.a.copy_(f)
        specs.append(sp)
    plan = ImplicitPlan(specs, params)
    plan.step(3)
    for i in range(16):
        assert np.array_equal(plan.state(i).cpu().numpy(), solo[i]), i


@pytest.mark.parametrize("R", [8, 16, 24, 32])
def test_tile_rows_match_oracle(R):
    d = sample_instances(1, seed=11)[0]
    d.nx = 700
    st = make_state(d)
    f_o = st.f.cpu().numpy().copy()
    v = st.v.cpu().numpy()
    plan = ImplicitPlan([spec_of(d, st)], implicit_params_struct(None, tile_rows=R, **SP))
    p_o = O.implicit_params(None, **SP)
    for _ in range(3):
        plan.step(1)
        bl = O.implicit_step(f_o, v, st.dx, st.dv, d.dt, d.tau_tilde, p_o)
        assert int(plan.stats.fetch()[0]["iters"]) == bl["picard_iter"]
        f = plan.state(0).cpu().numpy()
        assert np.abs(f - f_o).max() / np.abs(f_o).max() <= 1e-12


def test_graph_replay_equals_direct_steps():
    descs = _small(sample_instances(8, seed=5), cap=400)
    a = BatchSolver(descs, SP)
    a.step(4)
    ref = [a.plan.state(i).cpu().numpy() for i in range(len(descs))]
    b = BatchSolver(descs, SP)
    b.capture(2)
    b.replay()
    b.replay()
    torch.cuda.synchronize()
    for i in range(len(descs)):
        assert np.array_equal(b.plan.state(i).cpu().numpy(), ref[i]), i


def test_enable_mask_leaves_instance_untouched():
    descs = _small(sample_instances(3, seed=9), cap=300)
    s = BatchSolver(descs, SP)
    mask = torch.tensor([1, 0, 1], dtype=torch.int32, device="cuda")
    s.plan.set_enable_mask(mask)
    before = s.plan.state(1).clone()
    s.step(1)
    torch.cuda.synchronize()
    # the disabled instance's newest state is still in the buffer it was in
    assert torch.equal(s.plan.other(1), before)
