"""The CPU oracle against the reference's own outputs (golden fixtures made by
tests/golden/make_golden.py from the reference's CPU path)."""
import json

import numpy as np
import pytest

from oracle import oracle as O

IMPLICIT_CASES = ["smoke", "sod256", "aa96", "convw", "odd"]
_SKIP = ("nx", "nv", "dt", "T_total", "tau_tilde", "steps")


def _rel(a, b):
    return float(np.abs(a - b).max() / np.abs(b).max())


@pytest.fixture(scope="module")
def implicit_gold(golden_dir):
    return np.load(golden_dir / "implicit.npz")


@pytest.mark.parametrize("tag", IMPLICIT_CASES)
def test_oracle_implicit_matches_reference(implicit_gold, tag):
    d = implicit_gold
    meta = json.loads(str(d[f"{tag}_meta"]))
    g = O.Grid(meta["nx"], meta["nv"])
    p = O.implicit_params(None, **{k: v for k, v in meta.items() if k not in _SKIP})
    f = d[f"{tag}_f0"].copy()
    its = []
    for _ in range(meta["steps"]):
        its.append(O.implicit_step(f, g.v(), g.dx, g.dv, meta["dt"], meta["tau_tilde"], p)["picard_iter"])
    assert its == list(d[f"{tag}_iters"])
    if f"{tag}_f" in d:
        tol = 0.0 if not meta.get("aa_enable") else 1e-14
        assert _rel(f, d[f"{tag}_f"]) <= tol


@pytest.mark.parametrize("tag", ["holo64", "holo_nocons"])
def test_oracle_holo_matches_reference(golden_dir, tag):
    d = np.load(golden_dir / "holo.npz")
    meta = json.loads(str(d[f"{tag}_meta"]))
    g = O.Grid(meta["nx"], meta["nv"])
    p = O.holo_params(None, **{k: v for k, v in meta.items() if k not in _SKIP})
    f = d[f"{tag}_f0"].copy()
    logs = []
    for _ in range(meta["steps"]):
        bl = O.holo_step(f, g.v(), g.dx, g.dv, meta["dt"], meta["tau_tilde"], p)
        logs.append([bl["ho_iter"], bl["lo_iter"], bl["std_ho_residual"], bl["max_YI"]])
    logs = np.array(logs)
    ref = d[f"{tag}_log"]
    assert (logs[:, :2] == ref[:, :2]).all()
    np.testing.assert_allclose(logs[:, 3], ref[:, 3], rtol=1e-10, atol=1e-300)
    assert _rel(f, d[f"{tag}_f"]) < 1e-14


def test_oracle_kernels_match_reference(golden_dir):
    d = np.load(golden_dir / "kernels.npz")
    n, nu, T = O.moments_n_nu_T(d["kat_mom_f"], d["kat_mom_v"], float(d["kat_mom_dv"]))
    assert np.array_equal(n, d["kat_mom_n"]) and np.array_equal(nu, d["kat_mom_nu"])
    assert np.array_equal(T, d["kat_mom_T"])
    dt, dx, tau = d["kat_sys_scal"]
    dl, dd, du, B = O.build_system(d["kat_sys_B0"], d["kat_mom_v"], dt, dx, tau, d["kat_sys_n"],
                                   d["kat_sys_nu"], d["kat_sys_T"], d["kat_sys_fl"], d["kat_sys_fr"])
    for a, b in ((dl, "dl"), (dd, "dd"), (du, "du"), (B, "B")):
        assert np.array_equal(a, d[f"kat_sys_{b}"]), b
    X = O.gtsv(dl, dd, du, B)
    assert np.array_equal(X, d["kat_gtsv_X"])
    Xg = O.gtsv(d["kat_gen_dl"], d["kat_gen_d"], d["kat_gen_du"], d["kat_gen_B"])
    assert np.array_equal(Xg, d["kat_gen_X"])


def test_block_solver_matches_dense():
    rng = np.random.default_rng(7)
    n = 17
    A = rng.normal(size=(n, 3, 3)) * 0.1
    C = rng.normal(size=(n, 3, 3)) * 0.1
    B = np.eye(3)[None] * 2.0 + rng.normal(size=(n, 3, 3)) * 0.1
    D = rng.normal(size=(n, 3))
    X = O.block_tridiag_solve(A, B, C, D)
    M = np.zeros((3 * n, 3 * n))
    for i in range(n):
        M[3 * i:3 * i + 3, 3 * i:3 * i + 3] = B[i]
        if i > 0:
            M[3 * i:3 * i + 3, 3 * (i - 1):3 * i] = A[i]
        if i < n - 1:
            M[3 * i:3 * i + 3, 3 * (i + 1):3 * (i + 2)] = C[i]
    ref = np.linalg.solve(M, D.reshape(-1)).reshape(n, 3)
    assert np.abs(X - ref).max() < 1e-13


def test_uniform_maxwellian_stays_uniform():
    g = O.Grid(24, 16)
    f = O.initial_condition(g, regions=((0.0, 1.0, 0.7, 0.2, 1.3),))
    f0 = f.copy()
    p = O.implicit_params(None, picard_iter=30, picard_tol=1e-12, abs_tol=1e-16)
    O.implicit_step(f, g.v(), g.dx, g.dv, 1e-4, 1e-2, p)
    # a discrete Maxwellian is not an exact discrete equilibrium, but every
    # interior row stays identical to every other one
    assert np.abs(f[1:-1] - f[1:-1].mean(axis=0)).max() < 1e-12 * np.abs(f0).max() * 1e3
