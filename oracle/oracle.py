"""ctypes front end of the CPU oracle (test infrastructure only).

The oracle restates kineticEQ's BGK1D1V implicit and HOLO time steps on the
host (see ``keq_oracle.c``).  Only ``tests/``, ``__graft_entry__.smoke()`` and
the CPU legs of ``bench.py`` import this module; the product package never
does.

All arrays are numpy float64, C-contiguous.  ``f`` has shape (nx, nv).
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass

import numpy as np

from . import build as _build

_dp = C.POINTER(C.c_double)
_lib = None


class ImplicitParams(C.Structure):
    _fields_ = [
        ("picard_iter", C.c_int), ("picard_tol", C.c_double), ("abs_tol", C.c_double),
        ("conv_type", C.c_int), ("aa_enable", C.c_int), ("aa_m", C.c_int),
        ("aa_beta", C.c_double), ("aa_stride", C.c_int), ("aa_start_iter", C.c_int),
        ("aa_reg", C.c_double), ("aa_alpha_max", C.c_double), ("fixed_iters", C.c_int),
    ]


class ImplicitLog(C.Structure):
    _fields_ = [
        ("picard_iter", C.c_int), ("picard_residual", C.c_double),
        ("std_picard_residual", C.c_double), ("aa_applied", C.c_int),
    ]


class HoloParams(C.Structure):
    _fields_ = [
        ("ho_iter", C.c_int), ("ho_tol", C.c_double), ("ho_abs_tol", C.c_double),
        ("lo_iter", C.c_int), ("lo_tol", C.c_double), ("lo_abs_tol", C.c_double),
        ("con_terms_do", C.c_int), ("flux_consistency_do", C.c_int), ("sv_down", C.c_int),
        ("fixed_ho_iters", C.c_int), ("fixed_lo_iters", C.c_int),
    ]


class HoloLog(C.Structure):
    _fields_ = [
        ("ho_iter", C.c_int), ("ho_residual", C.c_double), ("std_ho_residual", C.c_double),
        ("lo_iter", C.c_int), ("lo_residual", C.c_double), ("std_lo_residual", C.c_double),
        ("max_YI", C.c_double),
    ]


def lib():
    global _lib
    if _lib is None:
        path = _build.build()
        L = C.CDLL(str(path))
        L.keqo_moments_n_nu_T.argtypes = [_dp, _dp, C.c_int, C.c_int, C.c_double, _dp, _dp, _dp]
        L.keqo_build_system.argtypes = [_dp, _dp, C.c_int, C.c_int, C.c_double, C.c_double,
                                        C.c_double, C.c_double, _dp, _dp, _dp, _dp, _dp,
                                        _dp, _dp, _dp, _dp]
        L.keqo_gtsv.argtypes = [_dp, _dp, _dp, _dp, C.c_int, C.c_int]
        L.keqo_implicit_step.argtypes = [C.c_int, C.c_int, _dp, C.c_double, C.c_double,
                                         C.c_double, C.c_double, C.POINTER(ImplicitParams), _dp,
                                         C.POINTER(ImplicitLog)]
        L.keqo_implicit_step.restype = C.c_int
        L.keqo_holo_step.argtypes = [C.c_int, C.c_int, _dp, C.c_double, C.c_double, C.c_double,
                                     C.c_double, C.POINTER(HoloParams), _dp, C.POINTER(HoloLog)]
        L.keqo_holo_step.restype = C.c_int
        L.keqo_block_tridiag_solve.argtypes = [_dp, _dp, _dp, _dp, _dp, C.c_int]
        L.keqo_initial_condition.argtypes = [_dp, C.c_int, _dp, C.c_int, _dp, C.c_int, _dp]
        _lib = L
    return _lib


def _p(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags["C_CONTIGUOUS"], "oracle arrays must be C float64"
    return a.ctypes.data_as(_dp)


def _c(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.float64)


# ---------------------------------------------------------------------------
# Grid (core/states/state_1d.py:30-58).  v and x follow torch.linspace exactly,
# so callers normally pass the product's own v; these helpers build them with
# the same two-sided formula for stand-alone use.
# ---------------------------------------------------------------------------
def linspace(a: float, b: float, n: int) -> np.ndarray:
    import torch

    return torch.linspace(a, b, n, dtype=torch.float64).numpy().copy()


@dataclass
class Grid:
    nx: int
    nv: int
    Lx: float = 1.0
    v_max: float = 10.0

    @property
    def dx(self) -> float:
        return float(self.Lx / (self.nx - 1))

    @property
    def dv(self) -> float:
        return float((2.0 * self.v_max) / (self.nv - 1))

    def v(self) -> np.ndarray:
        return linspace(-self.v_max, self.v_max, self.nv)

    def x(self) -> np.ndarray:
        return linspace(0.0, self.Lx, self.nx)


SOD = ((0.0, 0.5, 1.0, 0.0, 1.0), (0.5, 1.0, 0.125, 0.0, 0.8))


def initial_condition(grid: Grid, regions=SOD) -> np.ndarray:
    reg = _c(np.asarray(regions, dtype=np.float64).reshape(-1, 5))
    f = np.zeros((grid.nx, grid.nv))
    x, v = _c(grid.x()), _c(grid.v())
    lib().keqo_initial_condition(_p(x), grid.nx, _p(v), grid.nv, _p(reg), reg.shape[0], _p(f))
    return f


# ---------------------------------------------------------------------------
# Kernel-level restatements (C1 moments / assembly, C2 Thomas, K5 semantics).
# ---------------------------------------------------------------------------
def moments_n_nu_T(f, v, dv):
    f, v = _c(f), _c(v)
    nx, nv = f.shape
    n, nu, T = np.zeros(nx), np.zeros(nx), np.zeros(nx)
    lib().keqo_moments_n_nu_T(_p(f), _p(v), nx, nv, float(dv), _p(n), _p(nu), _p(T))
    return n, nu, T


def build_system(B0, v, dt, dx, tau_tilde, n, nu, T, f_bc_l, f_bc_r,
                 inv_sqrt_2pi=1.0 / math.sqrt(2.0 * math.pi)):
    B0, v, n, nu, T = _c(B0), _c(v), _c(n), _c(nu), _c(T)
    fl, fr = _c(f_bc_l), _c(f_bc_r)
    nv, n_inner = B0.shape
    nx = n_inner + 2
    dl, dd, du, B = (np.zeros_like(B0) for _ in range(4))
    lib().keqo_build_system(_p(B0), _p(v), nx, nv, float(dt), float(dx), float(tau_tilde),
                            float(inv_sqrt_2pi), _p(n), _p(nu), _p(T), _p(fl), _p(fr), _p(dl),
                            _p(dd), _p(du), _p(B))
    return dl, dd, du, B


def gtsv(dl, d, du, B):
    dl, d, du, B = _c(dl).copy(), _c(d).copy(), _c(du).copy(), _c(B).copy()
    batch, n = d.shape
    lib().keqo_gtsv(_p(dl), _p(d), _p(du), _p(B), batch, n)
    return B


def block_tridiag_solve(A, B, C_, D):
    A, B, C_, D = _c(A), _c(B), _c(C_), _c(D)
    n = D.shape[0]
    X = np.zeros_like(D)
    lib().keqo_block_tridiag_solve(_p(A), _p(B), _p(C_), _p(D), _p(X), n)
    return X


# ---------------------------------------------------------------------------
# Whole time steps.
# ---------------------------------------------------------------------------
def implicit_params(sp=None, fixed_iters: int = 0, **kw) -> ImplicitParams:
    """Map an ``implicit.Params``-like object (or keywords) to the C struct."""
    g = (lambda k, d: kw.get(k, getattr(sp, k, d)))
    conv = str(g("conv_type", "f")).lower()
    if conv not in ("f", "w"):
        raise ValueError(f"invalid conv_type={conv!r}, expected 'f' or 'w'")
    return ImplicitParams(
        int(g("picard_iter", 16)), float(g("picard_tol", 1e-4)), float(g("abs_tol", 1e-16)),
        1 if conv == "w" else 0, int(bool(g("aa_enable", False))), int(g("aa_m", 6)),
        float(g("aa_beta", 1.0)), int(g("aa_stride", 1)), int(g("aa_start_iter", 2)),
        float(g("aa_reg", 1e-10)), float(g("aa_alpha_max", 50.0)), int(fixed_iters))


def holo_params(sp=None, fixed_ho_iters: int = 0, fixed_lo_iters: int = 0, **kw) -> HoloParams:
    g = (lambda k, d: kw.get(k, getattr(sp, k, d)))
    return HoloParams(
        int(g("ho_iter", 8)), float(g("ho_tol", 1e-4)), float(g("ho_abs_tol", 1e-12)),
        int(g("lo_iter", 16)), float(g("lo_tol", 1e-4)), float(g("lo_abs_tol", 1e-12)),
        int(bool(g("Con_Terms_do", True))), int(bool(g("flux_consistency_do", True))),
        int(bool(g("SVdown", False))), int(fixed_ho_iters), int(fixed_lo_iters))


def implicit_step(f: np.ndarray, v, dx, dv, dt, tau_tilde, params: ImplicitParams) -> dict:
    """Advance f (nx, nv) one implicit step in place; returns the benchlog."""
    assert f.dtype == np.float64 and f.flags["C_CONTIGUOUS"]
    v = _c(v)
    nx, nv = f.shape
    log = ImplicitLog()
    rc = lib().keqo_implicit_step(nx, nv, _p(v), float(dx), float(dv), float(dt),
                                  float(tau_tilde), C.byref(params), _p(f), C.byref(log))
    if rc != 0:
        raise ValueError("oracle implicit step rejected its inputs")
    return {"picard_iter": log.picard_iter, "picard_residual": log.picard_residual,
            "std_picard_residual": log.std_picard_residual, "aa_applied": log.aa_applied}


def holo_step(f: np.ndarray, v, dx, dv, dt, tau_tilde, params: HoloParams) -> dict:
    assert f.dtype == np.float64 and f.flags["C_CONTIGUOUS"]
    v = _c(v)
    nx, nv = f.shape
    log = HoloLog()
    rc = lib().keqo_holo_step(nx, nv, _p(v), float(dx), float(dv), float(dt), float(tau_tilde),
                              C.byref(params), _p(f), C.byref(log))
    if rc != 0:
        raise ValueError("oracle HOLO step rejected its inputs")
    return {"ho_iter": log.ho_iter, "ho_residual": log.ho_residual,
            "std_ho_residual": log.std_ho_residual, "lo_iter": log.lo_iter,
            "lo_residual": log.lo_residual, "std_lo_residual": log.std_lo_residual,
            "max_YI": log.max_YI}
