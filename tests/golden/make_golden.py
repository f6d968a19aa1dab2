"""Generate the golden fixtures in this directory from the reference itself.

Runs kineticEQ (the reference project, read-only) from a scratch copy of its
``src`` tree, on the CPU, and records inputs/outputs of the path the CUDA
backend replaces:

* kernel known-answer vectors from the reference CPU extensions
  (moments_n_nu_T, build_system_from_moments, gtsv_strided_inplace);
* whole implicit steps through ``Engine`` with ``backend="cpu_kernel"``
  (plain, Anderson, conv_type="w", and the 256x128 Sod case);
* HOLO steps through the reference's device-agnostic torch ``step()`` on CPU
  tensors, fed with the reference CPU gtsv module and the block-Thomas
  stand-in below for the 3x3 block-tridiagonal LO solve (the registered
  builder only loads CUDA modules).

Usage:  python tests/golden/make_golden.py [--ref /path/to/kineticEQ]
Needs the reference checkout (not present on GPU machines); the committed
``.npz`` fixtures are what the tests read.
"""
from __future__ import annotations

import argparse
import importlib.metadata as md
import json
import math
import os
import shutil
import sys
import tempfile
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent


def _import_reference(ref_root: str):
    scratch = Path(tempfile.gettempdir()) / "keq_golden_ref"
    if scratch.exists():
        shutil.rmtree(scratch)
    shutil.copytree(Path(ref_root) / "src", scratch / "src")
    orig = md.version
    md.version = lambda n: "2.2.0" if n == "kineticEQ" else orig(n)
    sys.path.insert(0, str(scratch / "src"))
    import kineticEQ  # noqa: F401

    return scratch


class BlockThomasStandIn:
    """CPU stand-in for the reference's CUDA ``block_tridiag_solve`` (harness
    code, written from the block-tridiagonal system's definition): block
    Thomas sweep; a 3x3 block with |det| < 1e-30 contributes a zero inverse,
    the convention of cuda_kernel/BGK1D1V/lo_blocktridiag/block_tridiag_kernel.cu.
    """

    @staticmethod
    def _inv(M):
        import torch

        det = torch.linalg.det(M)
        if abs(float(det)) < 1e-30:
            return torch.zeros_like(M)
        return torch.linalg.inv(M)

    def block_tridiag_solve(self, A, B, C, D):
        import torch

        n = D.shape[0]
        Cp = torch.zeros_like(C)
        Dp = torch.zeros_like(D)
        for i in range(n):
            if i == 0:
                M, r = B[0], D[0]
            else:
                M = B[i] - A[i] @ Cp[i - 1]
                r = D[i] - A[i] @ Dp[i - 1]
            Mi = self._inv(M)
            if i < n - 1:
                Cp[i] = Mi @ C[i]
            Dp[i] = Mi @ r
        X = torch.zeros_like(D)
        X[n - 1] = Dp[n - 1]
        for i in range(n - 2, -1, -1):
            X[i] = Dp[i] - Cp[i] @ X[i + 1]
        return X


def kernel_kats(out):
    import torch
    from kineticEQ.cpu_kernel.compile import load_gtsv_cpu, load_implicit_fused_cpu

    mod = load_implicit_fused_cpu()
    gt = load_gtsv_cpu()
    g = torch.Generator().manual_seed(1234)
    nx, nv = 37, 24
    v = torch.linspace(-10.0, 10.0, nv, dtype=torch.float64)
    dv = float(20.0 / (nv - 1))
    f = torch.rand((nx, nv), generator=g, dtype=torch.float64) * 0.3
    f[5] = 0.0  # zero row -> clamps n and T
    n, nu, T = (torch.zeros(nx, dtype=torch.float64) for _ in range(3))
    mod.moments_n_nu_T(f, v, dv, n, nu, T)
    out["kat_mom_f"], out["kat_mom_v"] = f.numpy(), v.numpy()
    out["kat_mom_dv"] = np.array(dv)
    out["kat_mom_n"], out["kat_mom_nu"], out["kat_mom_T"] = n.numpy(), nu.numpy(), T.numpy()

    ni = nx - 2
    B0 = f[1:-1, :].T.contiguous()
    dl, dd, du, B = (torch.zeros((nv, ni), dtype=torch.float64) for _ in range(4))
    n2 = n.clone()
    n2[1:-1] += 0.5
    T2 = T.clone() + 0.3
    fl, fr = f[0].contiguous(), f[-1].contiguous()
    dt, dx, tau = 2e-3, 1.0 / (nx - 1), 3e-2
    mod.build_system_from_moments(B0, v, dt, dx, tau, 1.0 / math.sqrt(2.0 * math.pi), n2, nu, T2,
                                  fl, fr, dl, dd, du, B)
    out["kat_sys_B0"], out["kat_sys_n"], out["kat_sys_nu"], out["kat_sys_T"] = (
        B0.numpy(), n2.numpy(), nu.numpy(), T2.numpy())
    out["kat_sys_fl"], out["kat_sys_fr"] = fl.numpy(), fr.numpy()
    out["kat_sys_scal"] = np.array([dt, dx, tau])
    out["kat_sys_dl"], out["kat_sys_dd"], out["kat_sys_du"], out["kat_sys_B"] = (
        dl.numpy().copy(), dd.numpy().copy(), du.numpy().copy(), B.numpy().copy())
    ws = torch.empty((max(int(gt.gtsv_ws_bytes(dl, dd, du, B)), 1),), dtype=torch.uint8)
    gt.gtsv_strided_inplace(dl, dd, du, B, ws)
    out["kat_gtsv_X"] = B.numpy().copy()

    # general (non-bidiagonal) tridiagonal systems
    bt, nn = 9, 50
    dl = torch.rand((bt, nn), generator=g, dtype=torch.float64) - 0.5
    du = torch.rand((bt, nn), generator=g, dtype=torch.float64) - 0.5
    d = 2.5 + torch.rand((bt, nn), generator=g, dtype=torch.float64)
    rhs = torch.rand((bt, nn), generator=g, dtype=torch.float64)
    out["kat_gen_dl"], out["kat_gen_d"], out["kat_gen_du"], out["kat_gen_B"] = (
        dl.numpy().copy(), d.numpy().copy(), du.numpy().copy(), rhs.numpy().copy())
    gt.gtsv_strided_inplace(dl, d, du, rhs, ws)
    out["kat_gen_X"] = rhs.numpy().copy()


def implicit_case(out, tag, nx, nv, dt, T_total, tau, sp_kwargs, n_steps=None, keep_f=True):
    import torch
    from kineticEQ import BGK1D, Config, Engine

    cfg = Config(model="BGK1D1V", scheme="implicit", backend="cpu_kernel", device="cpu",
                 dtype="float64", use_tqdm="false", log_level="warning",
                 model_cfg=BGK1D.ModelConfig(
                     grid=BGK1D.Grid1D1V(nx=nx, nv=nv, Lx=1.0, v_max=10.0),
                     time=BGK1D.TimeConfig(dt=dt, T_total=T_total),
                     params=BGK1D.BGK1D1VParams(tau_tilde=tau),
                     scheme_params=BGK1D.implicit.Params(**sp_kwargs)))
    torch.set_num_threads(os.cpu_count() or 1)
    eng = Engine(cfg, apply_logging_flag=False)
    steps = cfg.model_cfg.time.n_steps if n_steps is None else n_steps
    f0 = eng.state.f.clone().numpy()
    iters, res = [], []
    for s in range(steps):
        eng.stepper(s)
        iters.append(eng.stepper.benchlog["picard_iter"])
        res.append(eng.stepper.benchlog["std_picard_residual"])
    f = eng.state.f.numpy()
    v = eng.state.v.numpy()
    n = f.sum(1) * eng.state.dv
    out[f"{tag}_f0"] = f0
    if keep_f:
        out[f"{tag}_f"] = f.copy()
    out[f"{tag}_n"] = n
    out[f"{tag}_nu"] = (f * v[None, :]).sum(1) * eng.state.dv
    out[f"{tag}_iters"] = np.array(iters, dtype=np.int32)
    out[f"{tag}_std_res"] = np.array(res)
    out[f"{tag}_meta"] = np.array(json.dumps(dict(nx=nx, nv=nv, dt=dt, T_total=T_total,
                                                  tau_tilde=tau, steps=steps, **sp_kwargs)))


def holo_case(out, tag, nx, nv, dt, tau, steps, sp_kwargs):
    import torch
    from kineticEQ import BGK1D, Config
    from kineticEQ.core.schemes.BGK1D1V import bgk1d_holo_cuda_kernel as H
    from kineticEQ.core.schemes.BGK1D1V.bgk1d_utils.general.bgk1d_set_initial_condition import (
        set_initial_condition)
    from kineticEQ.core.schemes.BGK1D1V.bgk1d_utils.implicit.bgk1d_holo_ws import (
        allocate_holo_workspace)
    from kineticEQ.core.states.registry import build_state
    from kineticEQ.cpu_kernel.compile import load_gtsv_cpu

    cfg = Config(model="BGK1D1V", scheme="holo", backend="cuda_kernel", device="cpu",
                 dtype="float64", use_tqdm="false", log_level="warning",
                 model_cfg=BGK1D.ModelConfig(
                     grid=BGK1D.Grid1D1V(nx=nx, nv=nv, Lx=1.0, v_max=10.0),
                     time=BGK1D.TimeConfig(dt=dt, T_total=dt * steps),
                     params=BGK1D.BGK1D1VParams(tau_tilde=tau),
                     scheme_params=BGK1D.holo.Params(**sp_kwargs)))
    state = build_state(cfg)
    set_initial_condition(state, cfg)
    ws = allocate_holo_workspace(nx, nv, state.f.device, state.f.dtype)
    gt = load_gtsv_cpu()
    lo = BlockThomasStandIn()
    f0 = state.f.clone().numpy()
    logs = []
    for s in range(steps):
        _, bl = H.step(state, cfg, ws, gt, lo, s)
        logs.append([bl["ho_iter"], bl["lo_iter"], bl["std_ho_residual"], bl["max_YI"]])
    out[f"{tag}_f0"] = f0
    out[f"{tag}_f"] = state.f.numpy().copy()
    out[f"{tag}_log"] = np.array(logs)
    out[f"{tag}_meta"] = np.array(json.dumps(dict(nx=nx, nv=nv, dt=dt, tau_tilde=tau,
                                                  steps=steps, **sp_kwargs)))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default="/root/reference")
    args = ap.parse_args()
    _import_reference(args.ref)

    out: dict = {}
    kernel_kats(out)
    np.savez_compressed(HERE / "kernels.npz", **out)

    out = {}
    # reference smoke configuration (tests/smoke/test_cpu.py)
    implicit_case(out, "smoke", 65, 33, 5e-5, 1e-4, 5e-2,
                  dict(picard_iter=32, picard_tol=1e-3, abs_tol=1e-13))
    # plain, small, FP64: 256x128 Sod, dt=5e-6, 100 steps, tau=5e-5, tol 1e-10 (cap 64)
    implicit_case(out, "sod256", 256, 128, 5e-6, 5e-4, 5e-5,
                  dict(picard_iter=64, picard_tol=1e-10, abs_tol=1e-16))
    # Anderson m=5 on a 96x48 grid, 20 steps
    implicit_case(out, "aa96", 96, 48, 2e-5, 4e-4, 5e-4,
                  dict(picard_iter=64, picard_tol=1e-10, abs_tol=1e-16, aa_enable=True, aa_m=5))
    # conv_type="w"
    implicit_case(out, "convw", 80, 40, 2e-5, 2e-4, 1e-3,
                  dict(picard_iter=40, picard_tol=1e-9, abs_tol=1e-14, conv_type="w"))
    # odd nv (v = 0 node), slow relaxation
    implicit_case(out, "odd", 41, 31, 1e-4, 5e-4, 5e-2,
                  dict(picard_iter=30, picard_tol=1e-8, abs_tol=1e-14))
    np.savez_compressed(HERE / "implicit.npz", **out)

    out = {}
    holo_case(out, "holo64", 64, 32, 5e-5, 5e-3, 4,
              dict(ho_iter=32, ho_tol=1e-10, lo_iter=32, lo_tol=1e-10))
    holo_case(out, "holo_nocons", 48, 24, 5e-5, 5e-2, 3,
              dict(ho_iter=16, ho_tol=1e-8, lo_iter=16, lo_tol=1e-8, Con_Terms_do=False))
    np.savez_compressed(HERE / "holo.npz", **out)
    for p in sorted(HERE.glob("*.npz")):
        print(p.name, p.stat().st_size)


if __name__ == "__main__":
    main()
