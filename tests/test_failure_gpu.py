"""Device-side failure handling of the persistent step kernel, exercised
without faulting or hanging the GPU: the plan's spin limit is set to 0, so
every grid-barrier wait that is not already satisfied gives up at once and
the launch returns early.  The step must then report KEQ_ERR_TIMEOUT (in the
instance's stats record and in the plan's error bits), and after the error
bits are reset and the limit restored the plan must step correctly again."""
import numpy as np
import pytest
import torch

from kineticeq_b200 import _native as N
from kineticeq_b200.plan import ImplicitPlan, InstanceSpec, grid_of, implicit_params_struct
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _sod_plan(nx=200, nv=64, dt=5e-6, tau=5e-5, **sp):
    v, dx, dv = grid_of(nx, nv)
    g = O.Grid(nx, nv)
    f0 = O.initial_condition(g)
    a = torch.from_numpy(f0).cuda()
    spec = InstanceSpec(v=v, dx=dx, dv=dv, dt=dt, tau_tilde=tau, a=a, b=torch.empty_like(a))
    p = implicit_params_struct(None, picard_iter=40, picard_tol=1e-10, abs_tol=1e-16, **sp)
    return ImplicitPlan([spec], p), f0, g, dict(picard_iter=40, picard_tol=1e-10, abs_tol=1e-16, **sp)


@pytest.mark.parametrize("aa", [False, True])
def test_timeout_reported_and_plan_recovers(aa):
    plan, f0, g, sp = _sod_plan(aa_enable=aa, aa_m=5)
    assert plan.device_error_bits() == 0
    plan.set_spin_limit(0)
    plan.step(1)
    torch.cuda.synchronize()
    rec = plan.stats.fetch()[0]
    assert int(rec["status"]) == N.KEQ_ERR_TIMEOUT
    assert plan.device_error_bits() & (1 << N.KEQ_ERR_TIMEOUT)
    # a second timed-out launch must not poison anything either
    plan.step(1)
    torch.cuda.synchronize()
    # recover: restore the limit, clear the sticky bits, restart from f0
    plan.set_spin_limit(1 << 25)
    plan.reset_errors()
    plan.state(0).copy_(torch.from_numpy(f0))
    plan.step(1)
    torch.cuda.synchronize()
    rec = plan.stats.fetch()[0]
    assert int(rec["status"]) == N.KEQ_OK
    assert plan.device_error_bits() == 0
    f_o = f0.copy()
    bl = O.implicit_step(f_o, g.v(), g.dx, g.dv, 5e-6, 5e-5, O.implicit_params(None, **sp))
    assert int(rec["iters"]) == bl["picard_iter"]
    got = plan.state(0).cpu().numpy()
    assert np.abs(got - f_o).max() / np.abs(f_o).max() <= 1e-12
