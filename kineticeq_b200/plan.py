"""Host-side plans over the C ABI: a list of independent BGK1D1V instances
stepped together by the persistent kernel (one launch per time step for the
whole list).

Each instance owns two state buffers ``a`` and ``b`` (nx, nv) FP64 on the
device; the state ping-pongs between them without copies and
``ImplicitPlan.state(i)`` returns the buffer that holds the newest state.
All device memory is torch-allocated; the library only receives pointers.
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass
from typing import Sequence

import numpy as np
import torch

from . import _native as N

_STATS_DTYPE = np.dtype([
    ("status", "<i4"), ("iters", "<i4"), ("aa_applied", "<i4"), ("lo_iters", "<i4"),
    ("residual", "<f8"), ("std_residual", "<f8"), ("lo_residual", "<f8"),
    ("std_lo_residual", "<f8"), ("max_YI", "<f8"), ("total_iters", "<i8"),
    ("total_steps", "<i8")])
assert _STATS_DTYPE.itemsize == N.STATS_BYTES


def implicit_params_struct(sp=None, fixed_iters: int = 0, tile_rows: int = 0,
                           precision: str = "fp64", mixed_tol: float = 0.0,
                           **kw) -> N.ImplicitParams:
    """implicit.Params (or keywords) -> keq_implicit_params; the clamps of
    bgk1d_implicit_cuda_kernel.py:49-65 are applied inside the library.
    tile_rows (8/16/24/32, 0 = default) is this backend's tile height;
    precision "fp64" (the reference's method) or "mixed" (FP32 sweeps, then
    FP64 sweeps to picard_tol)."""
    if precision not in ("fp64", "mixed"):
        raise ValueError(f"precision must be 'fp64' or 'mixed', not {precision!r}")
    g = (lambda k, d: kw[k] if k in kw else getattr(sp, k, d))
    conv = str(g("conv_type", "f")).lower()
    if conv not in ("f", "w"):
        raise ValueError(f"invalid conv_type={conv!r}, expected 'f' or 'w'")
    return N.ImplicitParams(
        int(g("picard_iter", 16)), float(g("picard_tol", 1e-4)), float(g("abs_tol", 1e-16)),
        1 if conv == "w" else 0, int(bool(g("aa_enable", False))), int(g("aa_m", 6)),
        float(g("aa_beta", 1.0)), int(g("aa_stride", 1)), int(g("aa_start_iter", 2)),
        float(g("aa_reg", 1e-10)), float(g("aa_alpha_max", 50.0)), int(fixed_iters),
        int(tile_rows), 1 if precision == "mixed" else 0, float(mixed_tol))


@dataclass
class InstanceSpec:
    """One solve: grid (nx, nv, dx, dv, v on the device), dt, tau_tilde and
    the two (nx, nv) FP64 device buffers; ``a`` holds f^n on entry.  ``kp``
    (number of velocities <= 0) and ``v_max`` (max |v|) may be given when the
    host knows v, which spares plan creation a device read."""
    v: torch.Tensor
    dx: float
    dv: float
    dt: float
    tau_tilde: float
    a: torch.Tensor
    b: torch.Tensor
    kp: int = -1
    v_max: float = 0.0

    @property
    def nx(self) -> int:
        return int(self.a.shape[0])

    @property
    def nv(self) -> int:
        return int(self.a.shape[1])


def _check_buf(t: torch.Tensor, name: str) -> None:
    if not t.is_cuda:
        raise RuntimeError(f"{name} must be a CUDA tensor")
    if t.dtype != torch.float64:
        raise RuntimeError(f"{name} must be float64")
    if not t.is_contiguous():
        raise RuntimeError(f"{name} must be contiguous")


class LazyStats:
    """Device-resident keq_step_stats records, copied to the host only when
    read (one synchronisation per read, none per step)."""

    def __init__(self, dev: torch.Tensor, n: int):
        self._dev = dev
        self._n = n

    def fetch(self) -> np.ndarray:
        raw = np.ascontiguousarray(self._dev.cpu().numpy()).reshape(-1)
        return raw.view(_STATS_DTYPE)[: self._n].copy()


class StatsRing:
    """Per-step snapshots of the stats records without a host synchronisation
    per step: ``capture()`` queues an asynchronous copy of the device records
    into the next slot of a pinned host ring and returns a ``StatsSnapshot``
    that waits for that copy only when it is read.  A snapshot read after the
    ring has wrapped around (``slots`` later captures) raises instead of
    returning another step's values."""

    def __init__(self, dev: torch.Tensor, n: int, slots: int = 256):
        self._dev = dev
        self._n = n
        self._slots = slots
        self._host = torch.empty((slots,) + tuple(dev.shape), dtype=dev.dtype, pin_memory=True)
        self._events = [None] * slots
        self._gen = [0] * slots
        self._next = 0
        self._count = 0

    def capture(self, stream=None) -> "StatsSnapshot":
        k = self._next
        self._next = (k + 1) % self._slots
        self._count += 1
        s = stream if stream is not None else torch.cuda.current_stream(self._dev.device)
        with torch.cuda.stream(s):
            self._host[k].copy_(self._dev, non_blocking=True)
            ev = torch.cuda.Event()
            ev.record(s)
        self._events[k] = ev
        self._gen[k] = self._count
        return StatsSnapshot(self, k, self._count)

    def read(self, k: int, gen: int) -> np.ndarray:
        if self._gen[k] != gen:
            raise RuntimeError("stats snapshot expired: the ring was reused by later steps")
        self._events[k].synchronize()
        raw = np.ascontiguousarray(self._host[k].numpy()).reshape(-1)
        return raw.view(_STATS_DTYPE)[: self._n].copy()


class StatsSnapshot:
    def __init__(self, ring: StatsRing, k: int, gen: int):
        self._ring, self._k, self._gen = ring, k, gen
        self._vals = None

    def fetch(self) -> np.ndarray:
        if self._vals is None:
            self._vals = self._ring.read(self._k, self._gen)
        return self._vals


def holo_params_struct(sp=None, fixed_ho_iters: int = 0, fixed_lo_iters: int = 0,
                       **kw) -> N.HoloParams:
    """holo.Params (or keywords) -> keq_holo_params (holo.py:5-13 plus the
    hidden SVdown flag read at bgk1d_holo_cuda_kernel.py:443)."""
    g = (lambda k, d: kw[k] if k in kw else getattr(sp, k, d))
    return N.HoloParams(
        int(g("ho_iter", 8)), float(g("ho_tol", 1e-4)), float(g("ho_abs_tol", 1e-12)),
        int(g("lo_iter", 16)), float(g("lo_tol", 1e-4)), float(g("lo_abs_tol", 1e-12)),
        int(bool(g("Con_Terms_do", True))), int(bool(g("flux_consistency_do", True))),
        int(bool(g("SVdown", False))), int(fixed_ho_iters), int(fixed_lo_iters))


class _StepPlan:
    """A list of independent instances stepped together by one persistent
    kernel launch per time step (keq_plan of the C ABI)."""

    _kind = "step"
    _ptype = None

    def _to_struct(self, p):
        raise NotImplementedError

    def _ws_query(self, lib, grid, p, nbytes):
        raise NotImplementedError

    def _plan_ws_query(self, lib, inst, n, parr, per, nbytes):
        raise NotImplementedError

    def _create(self, lib, inst, n, parr, per, ws, nws, sh, handle):
        raise NotImplementedError

    def __init__(self, specs: Sequence[InstanceSpec], params, stream=None):
        lib = N.load()
        if len(specs) == 0:
            raise ValueError("empty instance list")
        plist = list(params) if isinstance(params, (list, tuple)) else [params]
        if len(plist) not in (1, len(specs)):
            raise ValueError("params: one record or one per instance")
        pstructs = [p if isinstance(p, self._ptype) else self._to_struct(p) for p in plist]
        self.device = specs[0].a.device
        self.specs = list(specs)
        self.n = len(specs)
        self._stream = stream
        sh = N.stream_handle(stream)
        self.stats_dev = torch.zeros((self.n, N.STATS_BYTES), dtype=torch.uint8,
                                     device=self.device)
        self._ws = []
        inst = (N.Instance * self.n)()
        for i, s in enumerate(self.specs):
            _check_buf(s.a, "f")
            _check_buf(s.b, "f_tmp")
            _check_buf(s.v, "v")
            if s.a.shape != s.b.shape or s.a.dim() != 2 or s.v.numel() != s.a.shape[1]:
                raise RuntimeError("f / f_tmp must be (nx, nv) and v must be (nv,)")
            p = pstructs[i if len(pstructs) > 1 else 0]
            grid = N.Grid(s.nx, s.nv, float(s.dx), float(s.dv), s.v.data_ptr(), int(s.kp),
                          float(s.v_max))
            nbytes = C.c_size_t(0)
            N.check(self._ws_query(lib, grid, p, nbytes), "workspace query")
            ws = torch.empty((max(int(nbytes.value), 256),), dtype=torch.uint8,
                             device=self.device)
            self._ws.append(ws)
            inst[i] = N.Instance(grid, float(s.dt), float(s.tau_tilde), s.a.data_ptr(),
                                 s.b.data_ptr(), self.stats_dev[i].data_ptr(), ws.data_ptr())
        parr = (self._ptype * len(pstructs))(*pstructs)
        per = 1 if len(pstructs) > 1 else 0
        nbytes = C.c_size_t(0)
        N.check(self._plan_ws_query(lib, inst, self.n, parr, per, nbytes), "plan workspace query")
        self._plan_ws = torch.empty((max(int(nbytes.value), 256),), dtype=torch.uint8,
                                    device=self.device)
        handle = C.c_void_p(0)
        N.check(self._create(lib, inst, self.n, parr, per, self._plan_ws.data_ptr(),
                             self._plan_ws.numel(), sh, handle), "plan creation")
        self._h = handle
        self._lib = lib
        self.parity = 0  # 0: newest state in `a`, 1: in `b`
        self.stats = LazyStats(self.stats_dev, self.n)
        self._ring = None

    def step(self, n_steps: int = 1) -> None:
        N.check(self._lib.keq_plan_step(self._h, int(n_steps), int(self.parity),
                                        N.stream_handle(self._stream)), f"{self._kind} step")
        self.parity = (self.parity + int(n_steps)) & 1

    def snapshot(self) -> StatsSnapshot:
        """Snapshot of the stats records after the steps queued so far."""
        if self._ring is None:
            self._ring = StatsRing(self.stats_dev, self.n)
        return self._ring.capture(self._stream)

    def set_enable_mask(self, mask) -> None:
        """Attach a device int32 mask (one entry per instance; 0 = skip) or None."""
        ptr = 0 if mask is None else mask.data_ptr()
        N.check(self._lib.keq_plan_set_enable_mask(self._h, ptr, N.stream_handle(self._stream)),
                "enable mask")
        self._mask = mask

    def reset_errors(self) -> None:
        """Clear the accumulated device error bits (keq_plan_reset)."""
        N.check(self._lib.keq_plan_reset(self._h, N.stream_handle(self._stream)), "plan reset")

    def set_spin_limit(self, limit: int) -> None:
        """Polls a device-side wait makes before giving up (keq_plan_set_spin_limit)."""
        N.check(self._lib.keq_plan_set_spin_limit(self._h, int(limit),
                                                  N.stream_handle(self._stream)),
                "spin limit")

    def state(self, i: int) -> torch.Tensor:
        s = self.specs[i]
        return s.a if self.parity == 0 else s.b

    def other(self, i: int) -> torch.Tensor:
        s = self.specs[i]
        return s.b if self.parity == 0 else s.a

    def enable_trace(self, iters: int = 256) -> torch.Tensor:
        """Attach a phase trace buffer (see keq_plan_set_trace); returns it."""
        buf = torch.zeros((iters, 4), dtype=torch.int64, device=self.device)
        buf[:, 0] = -1  # all ones = UINT64_MAX
        buf[:, 2] = -1
        N.check(self._lib.keq_plan_set_trace(self._h, buf.data_ptr(), iters,
                                             N.stream_handle(self._stream)), "trace")
        self._trace = buf
        return buf

    def trace_phases(self):
        """Per-iteration (pass_us, gap_to_next_pass_us) of the last step."""
        import numpy as np

        t = self._trace.cpu().numpy().view(np.uint64).astype(np.float64)
        out = []
        for m, row in enumerate(t):
            if row[1] == 0:
                break
            nxt = t[m + 1][0] if m + 1 < len(t) and t[m + 1][1] != 0 else row[1]
            out.append(((row[1] - row[0]) / 1e3, (nxt - row[1]) / 1e3))
        return out

    def reset_trace(self) -> None:
        self._trace.zero_()
        self._trace[:, 0] = -1
        self._trace[:, 2] = -1

    def device_error_bits(self) -> int:
        v = C.c_int32(0)
        N.check(self._lib.keq_plan_error(self._h, N.stream_handle(self._stream), C.byref(v)),
                "plan error query")
        return int(v.value)

    def close(self) -> None:
        if getattr(self, "_h", None) is not None and self._h.value:
            self._lib.keq_plan_destroy(self._h)
            self._h = C.c_void_p(0)

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class ImplicitPlan(_StepPlan):
    """Batched implicit Picard stepping of independent instances."""

    _kind = "implicit"
    _ptype = N.ImplicitParams

    def _to_struct(self, p):
        return implicit_params_struct(p)

    def _ws_query(self, lib, grid, p, nbytes):
        return lib.keq_implicit_instance_workspace_size(C.byref(grid), C.byref(p), C.byref(nbytes))

    def _plan_ws_query(self, lib, inst, n, parr, per, nbytes):
        return lib.keq_implicit_plan_workspace_size(inst, n, parr, per, C.byref(nbytes))

    def _create(self, lib, inst, n, parr, per, ws, nws, sh, handle):
        return lib.keq_implicit_plan_create(inst, n, parr, per, ws, nws, sh, C.byref(handle))

    def moments(self, i: int) -> torch.Tensor:
        """(3, nx) view of instance i's current W = (n, nu, T) (workspace head)."""
        nx = self.specs[i].nx
        return self._ws[i][: 3 * nx * 8].view(torch.float64).view(3, nx)


class HoloPlan(_StepPlan):
    """Batched HOLO stepping of independent instances."""

    _kind = "holo"
    _ptype = N.HoloParams

    def _to_struct(self, p):
        return holo_params_struct(p)

    def _ws_query(self, lib, grid, p, nbytes):
        return lib.keq_holo_instance_workspace_size(C.byref(grid), C.byref(p), C.byref(nbytes))

    def _plan_ws_query(self, lib, inst, n, parr, per, nbytes):
        return lib.keq_holo_plan_workspace_size(inst, n, parr, per, C.byref(nbytes))

    def _create(self, lib, inst, n, parr, per, ws, nws, sh, handle):
        return lib.keq_holo_plan_create(inst, n, parr, per, ws, nws, sh, C.byref(handle))


def grid_of(nx: int, nv: int, Lx: float = 1.0, v_max: float = 10.0, device="cuda"):
    """(v on device, dx, dv) exactly as core/states/state_1d.py:30-58."""
    v = torch.linspace(-v_max, v_max, nv, dtype=torch.float64).to(device)
    return v, float(Lx / (nx - 1)), float((2.0 * v_max) / (nv - 1))


def velocity_facts(nv: int, v_max: float = 10.0):
    """(kp, max |v|) of the velocity grid linspace(-v_max, v_max, nv), computed
    on the host from the same float64 linspace."""
    vh = torch.linspace(-v_max, v_max, nv, dtype=torch.float64)
    kp = int((vh <= 0.0).sum())
    return kp, float(vh.abs().max())


def _inv_sqrt_2pi() -> float:
    return 1.0 / math.sqrt(2.0 * math.pi)
