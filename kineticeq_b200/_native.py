"""ctypes binding of ``lib/libkeq_b200.so`` (C ABI: include/keq_b200.h).

The library is the only compute path of this package: when it is missing,
cannot be loaded, or no CUDA device is present, every entry point raises
``RuntimeError`` -- there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import threading
from pathlib import Path

_LIB_PATH = Path(__file__).resolve().parent / "lib" / "libkeq_b200.so"
_lock = threading.Lock()
_lib = None

KEQ_OK = 0
KEQ_ERR_INVALID = 1
KEQ_ERR_WORKSPACE = 2
KEQ_ERR_CUDA = 3
KEQ_ERR_TIMEOUT = 4
KEQ_ERR_NONFINITE = 5
KEQ_ERR_NOCONV = 6
KEQ_ERR_UNSUPPORTED = 7
KEQ_ERR_CAPACITY = 8

_vp = C.c_void_p
_dp = C.c_void_p  # device pointers travel as integers
_i32 = C.c_int32
_f64 = C.c_double
_sz = C.c_size_t


class Grid(C.Structure):
    _fields_ = [("nx", _i32), ("nv", _i32), ("dx", _f64), ("dv", _f64), ("v", _dp),
                ("kp", _i32), ("v_max", _f64)]


class ImplicitParams(C.Structure):
    _fields_ = [
        ("picard_iter", _i32), ("picard_tol", _f64), ("abs_tol", _f64), ("conv_type", _i32),
        ("aa_enable", _i32), ("aa_m", _i32), ("aa_beta", _f64), ("aa_stride", _i32),
        ("aa_start_iter", _i32), ("aa_reg", _f64), ("aa_alpha_max", _f64),
        ("fixed_iters", _i32), ("tile_rows", _i32), ("precision", _i32), ("mixed_tol", _f64),
    ]


class HoloParams(C.Structure):
    _fields_ = [
        ("ho_iter", _i32), ("ho_tol", _f64), ("ho_abs_tol", _f64), ("lo_iter", _i32),
        ("lo_tol", _f64), ("lo_abs_tol", _f64), ("con_terms_do", _i32),
        ("flux_consistency_do", _i32), ("sv_down", _i32), ("fixed_ho_iters", _i32),
        ("fixed_lo_iters", _i32),
    ]


class StepStats(C.Structure):
    _fields_ = [
        ("status", _i32), ("iters", _i32), ("aa_applied", _i32), ("lo_iters", _i32),
        ("residual", _f64), ("std_residual", _f64), ("lo_residual", _f64),
        ("std_lo_residual", _f64), ("max_YI", _f64), ("total_iters", C.c_int64),
        ("total_steps", C.c_int64),
    ]


class Instance(C.Structure):
    _fields_ = [
        ("grid", Grid), ("dt", _f64), ("tau_tilde", _f64), ("f_in", _dp), ("f_out", _dp),
        ("stats", _dp), ("workspace", _dp),
    ]


STATS_BYTES = C.sizeof(StepStats)

# name -> (restype, argtypes)
_PROTOS = {
    "keq_abi_version": (_i32, []),
    "keq_status_string": (C.c_char_p, [_i32]),
    "keq_last_cuda_error": (C.c_char_p, []),
    "keq_implicit_instance_workspace_size": (_i32, [C.POINTER(Grid), C.POINTER(ImplicitParams),
                                                    C.POINTER(_sz)]),
    "keq_implicit_plan_workspace_size": (_i32, [C.POINTER(Instance), _i32,
                                                C.POINTER(ImplicitParams), _i32,
                                                C.POINTER(_sz)]),
    "keq_implicit_plan_create": (_i32, [C.POINTER(Instance), _i32, C.POINTER(ImplicitParams),
                                        _i32, _vp, _sz, _vp, C.POINTER(_vp)]),
    "keq_plan_set_buffers": (_i32, [_vp, C.POINTER(_vp), C.POINTER(_vp), _vp]),
    "keq_plan_step": (_i32, [_vp, _i32, _i32, _vp]),
    "keq_plan_error": (_i32, [_vp, _vp, C.POINTER(_i32)]),
    "keq_plan_reset": (_i32, [_vp, _vp]),
    "keq_plan_set_enable_mask": (_i32, [_vp, _dp, _vp]),
    "keq_plan_set_spin_limit": (_i32, [_vp, C.c_uint64, _vp]),
    "keq_plan_set_trace": (_i32, [_vp, _vp, _i32, _vp]),
    "keq_plan_destroy": (None, [_vp]),
    "keq_holo_instance_workspace_size": (_i32, [C.POINTER(Grid), C.POINTER(HoloParams),
                                                C.POINTER(_sz)]),
    "keq_holo_plan_workspace_size": (_i32, [C.POINTER(Instance), _i32, C.POINTER(HoloParams),
                                            _i32, C.POINTER(_sz)]),
    "keq_holo_plan_create": (_i32, [C.POINTER(Instance), _i32, C.POINTER(HoloParams), _i32, _vp,
                                    _sz, _vp, C.POINTER(_vp)]),
    "keq_implicit_workspace_size": (_i32, [C.POINTER(Grid), C.POINTER(ImplicitParams),
                                           C.POINTER(_sz)]),
    "keq_implicit_step": (_i32, [C.POINTER(Grid), _f64, _f64, C.POINTER(ImplicitParams), _dp,
                                 _dp, _dp, _vp, _sz, _vp]),
    "keq_moments_n_nu_T": (_i32, [_dp, _dp, _i32, _i32, _f64, _dp, _dp, _dp, _vp]),
    "keq_build_system_from_moments": (_i32, [_dp, _dp, _i32, _i32, _f64, _f64, _f64, _f64,
                                             _dp, _dp, _dp, _dp, _dp, _dp, _dp, _dp, _dp, _vp]),
    "keq_gtsv_workspace_size": (_i32, [_i32, _i32, C.POINTER(_sz)]),
    "keq_gtsv_strided_inplace": (_i32, [_dp, _dp, _dp, _dp, _i32, _i32, _vp, _sz, _vp]),
    "keq_gtsv_strided_inplace_noalloc": (_i32, [_dp, _dp, _dp, _dp, _i32, _i32, _vp]),
    "keq_block_tridiag_workspace_size": (_i32, [_i32, _i32, C.POINTER(_sz)]),
    "keq_block_tridiag_solve": (_i32, [_dp, _dp, _dp, _dp, _dp, _i32, _i32, _vp, _sz, _vp]),
    "keq_math_selftest": (_i32, [_i32, _dp, _dp, _i32, _vp]),
    "keq_maxwellian": (_i32, [_dp, _dp, _dp, _dp, _i32, _i32, _dp, _vp]),
    "keq_row_moments": (_i32, [_dp, _dp, _i32, _i32, _f64, _dp, _vp]),
}

# Entry points that are declared in the header but may be added by later
# library versions are looked up lazily (see ``fn``).
_OPTIONAL: dict = {}


def declared_symbols() -> list[str]:
    """Every function name declared in include/keq_b200.h."""
    import re

    hdr = Path(__file__).resolve().parent.parent / "include" / "keq_b200.h"
    txt = hdr.read_text()
    return sorted(set(re.findall(r"\b(keq_[A-Za-z0-9_]+)\s*\(", txt)))


def lib_path() -> Path:
    return _LIB_PATH


def load(require_cuda: bool = True):
    """Load the CUDA library (building it in-tree first if the sources are
    newer).  Raises RuntimeError when it cannot be loaded or, with
    require_cuda, when no CUDA device is visible."""
    global _lib
    with _lock:
        if _lib is None:
            if not _LIB_PATH.exists():
                try:
                    from . import _build

                    _build.build()
                except Exception as e:  # pragma: no cover - build errors are fatal
                    raise RuntimeError(f"kineticeq_b200: CUDA library missing and build failed: {e}")
            lib = C.CDLL(str(_LIB_PATH))
            for name, (res, args) in _PROTOS.items():
                f = getattr(lib, name)
                f.restype = res
                f.argtypes = args
            _lib = lib
    if require_cuda:
        import torch

        if not torch.cuda.is_available():
            raise RuntimeError("kineticeq_b200 needs a CUDA device (sm_100a); none is visible")
    return _lib


def fn(name: str, restype=None, argtypes=None):
    lib = load(require_cuda=False)
    f = getattr(lib, name)
    if argtypes is not None:
        f.restype = restype
        f.argtypes = argtypes
    return f


def status_text(code: int) -> str:
    lib = load(require_cuda=False)
    s = lib.keq_status_string(int(code)).decode()
    if code == KEQ_ERR_CUDA:
        s += ": " + lib.keq_last_cuda_error().decode()
    return s


def check(code: int, what: str) -> None:
    """Map a keq_status to the reference's exception types: invalid inputs and
    CUDA failures raise RuntimeError (TORCH_CHECK in the reference bindings),
    a non-finite state raises ValueError."""
    if code == KEQ_OK:
        return
    if code == KEQ_ERR_NONFINITE:
        raise ValueError("NaN/Inf detected in f_tmp")
    raise RuntimeError(f"{what} failed: {status_text(code)}")


def stream_handle(stream=None) -> int:
    import torch

    s = stream if stream is not None else torch.cuda.current_stream()
    return int(s.cuda_stream)
