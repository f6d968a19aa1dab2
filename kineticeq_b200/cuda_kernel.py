"""Module-level drop-ins for kineticEQ's cuda_kernel/compile.py loaders.

``load_implicit_fused()``, ``load_gtsv()`` and ``load_lo_blocktridiag()``
return objects with the same method names and tensor arguments as the
reference's pybind modules (implicit_fused/implicit_binding.cpp:38-142,
gtsv/gtsv_binding.cpp:48-117, lo_blocktridiag/block_tridiag_binding.cpp:25-108),
backed by the C ABI of libkeq_b200.so.  Input validation mirrors the
reference's TORCH_CHECKs and raises RuntimeError.
"""
from __future__ import annotations

import ctypes as C
import functools
import math

import torch

from . import _native as N


def _chk(t: torch.Tensor, name: str) -> None:
    if not isinstance(t, torch.Tensor) or not t.is_cuda:
        raise RuntimeError(f"{name} must be CUDA tensor")
    if t.dtype != torch.float64:
        raise RuntimeError(f"{name} must be float64")
    if not t.is_contiguous():
        raise RuntimeError(f"{name} must be contiguous")


def _s() -> int:
    return N.stream_handle()


class ImplicitFused:
    """implicit_fused module: moments_n_nu_T, build_system_from_moments."""

    def moments_n_nu_T(self, fz, v, dv, n, nu, T) -> None:
        for t, nm in ((fz, "fz"), (v, "v"), (n, "n"), (nu, "nu"), (T, "T")):
            _chk(t, nm)
        if fz.dim() != 2 or v.dim() != 1:
            raise RuntimeError("fz must be (nx, nv) and v must be (nv,)")
        nx, nv = fz.shape
        if v.numel() != nv or n.numel() != nx or nu.numel() != nx or T.numel() != nx:
            raise RuntimeError("n/nu/T size must match fz.nx and v size must match fz.nv")
        N.check(N.load().keq_moments_n_nu_T(fz.data_ptr(), v.data_ptr(), nx, nv, float(dv),
                                            n.data_ptr(), nu.data_ptr(), T.data_ptr(), _s()),
                "moments_n_nu_T")

    def build_system_from_moments(self, B0, v, dt, dx, tau_tilde, inv_sqrt_2pi, n, nu, T,
                                  f_bc_l, f_bc_r, dl, dd, du, B) -> None:
        for t, nm in ((B0, "B0"), (v, "v"), (n, "n"), (nu, "nu"), (T, "T"), (f_bc_l, "f_bc_l"),
                      (f_bc_r, "f_bc_r"), (dl, "dl"), (dd, "dd"), (du, "du"), (B, "B")):
            _chk(t, nm)
        nx, nv = n.numel(), v.numel()
        if nx < 3:
            raise RuntimeError("n must have nx >= 3")
        shp = (nv, nx - 2)
        for t, nm in ((B0, "B0"), (dl, "dl"), (dd, "dd"), (du, "du"), (B, "B")):
            if tuple(t.shape) != shp:
                raise RuntimeError(f"{nm} must be (nv, nx-2)")
        N.check(N.load().keq_build_system_from_moments(
            B0.data_ptr(), v.data_ptr(), nx, nv, float(dt), float(dx), float(tau_tilde),
            float(inv_sqrt_2pi), n.data_ptr(), nu.data_ptr(), T.data_ptr(), f_bc_l.data_ptr(),
            f_bc_r.data_ptr(), dl.data_ptr(), dd.data_ptr(), du.data_ptr(), B.data_ptr(), _s()),
            "build_system_from_moments")


class Gtsv:
    """gtsv module: gtsv_ws_bytes, gtsv_strided_inplace, gtsv_strided."""

    @staticmethod
    def _core(dl, d, du, B):
        for t, nm in ((dl, "dl"), (d, "d"), (du, "du"), (B, "B")):
            _chk(t, nm)
        if d.dim() != 2:
            raise RuntimeError("d must be 2D: (batch, n)")
        if dl.shape != d.shape or du.shape != d.shape or B.shape != d.shape:
            raise RuntimeError("dl, d, du, B must have the same shape: (batch, n)")
        return int(d.shape[0]), int(d.shape[1])

    def gtsv_ws_bytes(self, dl, d, du, B) -> int:
        batch, n = self._core(dl, d, du, B)
        nb = C.c_size_t(0)
        N.check(N.load().keq_gtsv_workspace_size(n, batch, C.byref(nb)), "gtsv_ws_bytes")
        return int(nb.value)

    def gtsv_strided_inplace(self, dl, d, du, B, workspace):
        batch, n = self._core(dl, d, du, B)
        if not workspace.is_cuda or workspace.dtype != torch.uint8 or not workspace.is_contiguous():
            raise RuntimeError("workspace must be a contiguous uint8 CUDA tensor")
        if workspace.numel() <= 0:
            raise RuntimeError("workspace must be preallocated with positive size")
        N.check(N.load().keq_gtsv_strided_inplace(dl.data_ptr(), d.data_ptr(), du.data_ptr(),
                                                  B.data_ptr(), n, batch, workspace.data_ptr(),
                                                  workspace.numel(), _s()), "gtsv_strided_inplace")
        return B

    def gtsv_strided(self, dl, d, du, B):
        ws = torch.empty((max(self.gtsv_ws_bytes(dl, d, du, B), 1),), dtype=torch.uint8,
                         device=d.device)
        return self.gtsv_strided_inplace(dl, d, du, B, ws)


class LoBlockTridiag:
    """lo_blocktridiag module: block_tridiag_solve(A, B, C, D) -> X."""

    def block_tridiag_solve(self, A, B, Cm, D):
        for t, nm in ((A, "A"), (B, "B"), (Cm, "C"), (D, "D")):
            if not isinstance(t, torch.Tensor) or not t.is_cuda:
                raise RuntimeError(f"{nm} must be CUDA tensor")
        if not (A.dtype == B.dtype == Cm.dtype == D.dtype):
            raise RuntimeError("dtype mismatch")
        if A.dtype != torch.float64:
            raise RuntimeError("block_tridiag_solve: float64 only on this backend")
        was3 = A.dim() == 3
        if was3:
            A, B, Cm, D = A.unsqueeze(0), B.unsqueeze(0), Cm.unsqueeze(0), D.unsqueeze(0)
        if A.dim() != 4 or A.shape[2:] != (3, 3):
            raise RuntimeError("A must be (batch, n, 3, 3)")
        if B.shape != A.shape:
            raise RuntimeError("B shape mismatch")
        if Cm.shape != A.shape:
            raise RuntimeError("C shape mismatch")
        if D.dim() != 3 or D.shape[0] != A.shape[0] or D.shape[1] != A.shape[1] or D.shape[2] != 3:
            raise RuntimeError("D shape mismatch")
        A, B, Cm, D = (t.contiguous() for t in (A, B, Cm, D))
        batch, n = int(A.shape[0]), int(A.shape[1])
        X = torch.empty_like(D)
        nb = C.c_size_t(0)
        lib = N.load()
        N.check(lib.keq_block_tridiag_workspace_size(n, batch, C.byref(nb)), "block_tridiag")
        ws = torch.empty((max(int(nb.value), 8),), dtype=torch.uint8, device=D.device)
        N.check(lib.keq_block_tridiag_solve(A.data_ptr(), B.data_ptr(), Cm.data_ptr(),
                                            D.data_ptr(), X.data_ptr(), n, batch, ws.data_ptr(),
                                            ws.numel(), _s()), "block_tridiag_solve")
        return X.squeeze(0) if was3 else X


@functools.lru_cache(maxsize=1)
def load_implicit_fused() -> ImplicitFused:
    N.load()
    return ImplicitFused()


@functools.lru_cache(maxsize=1)
def load_gtsv() -> Gtsv:
    N.load()
    return Gtsv()


@functools.lru_cache(maxsize=1)
def load_lo_blocktridiag() -> LoBlockTridiag:
    N.load()
    return LoBlockTridiag()


INV_SQRT_2PI = 1.0 / math.sqrt(2.0 * math.pi)
