"""C ABI: the library loads, exports every declared symbol, and validates
arguments on the host (no GPU work here)."""
import ctypes as C

import pytest

from kineticeq_b200 import _build
from kineticeq_b200 import _native as N


@pytest.fixture(scope="module")
def lib():
    _build.build()
    return N.load(require_cuda=False)


def test_every_declared_symbol_is_exported(lib):
    names = N.declared_symbols()
    assert len(names) >= 15
    for name in names:
        assert hasattr(lib, name), name


def test_status_strings(lib):
    assert lib.keq_abi_version() == 1
    assert N.status_text(N.KEQ_ERR_NONFINITE) == "NaN/Inf detected in f_tmp"
    with pytest.raises(ValueError, match="NaN/Inf"):
        N.check(N.KEQ_ERR_NONFINITE, "x")
    with pytest.raises(RuntimeError, match="invalid"):
        N.check(N.KEQ_ERR_INVALID, "x")


def test_workspace_queries_validate(lib):
    g = N.Grid(256, 128, 1 / 255, 20 / 127, 0, -1, 0.0)
    p = N.ImplicitParams(64, 1e-10, 1e-16, 0, 0, 5, 1.0, 1, 2, 1e-10, 50.0, 0, 0, 0, 0.0)
    nb = C.c_size_t(0)
    assert lib.keq_implicit_instance_workspace_size(C.byref(g), C.byref(p), C.byref(nb)) == 0
    assert nb.value > 256 * 4 * 8
    bad = N.Grid(2, 128, 1.0, 1.0, 0, -1, 0.0)
    assert lib.keq_implicit_instance_workspace_size(C.byref(bad), C.byref(p), C.byref(nb)) == 1
    p.picard_iter = 0
    assert lib.keq_implicit_instance_workspace_size(C.byref(g), C.byref(p), C.byref(nb)) == 1
    p.picard_iter = 8
    p.aa_enable, p.aa_m = 1, 12  # ring wider than the kernel's capacity
    assert lib.keq_implicit_instance_workspace_size(C.byref(g), C.byref(p), C.byref(nb)) == 1
    assert lib.keq_gtsv_workspace_size(10, 4, C.byref(nb)) == 0 and nb.value == 320
    assert lib.keq_gtsv_strided_inplace(0, 0, 0, 0, 5, 3, 0, 0, 0) == 1
    assert lib.keq_block_tridiag_workspace_size(10, 2, C.byref(nb)) == 0
    assert lib.keq_moments_n_nu_T(0, 0, 4, 4, 1.0, 0, 0, 0, 0) == 1



def test_noalloc_gtsv_rejects_oversize_on_host(lib):
    # n * batch above the fixed scratch (2^21 doubles) is refused before any
    # CUDA call; the pointers are never dereferenced on this path
    assert lib.keq_gtsv_strided_inplace_noalloc(8, 16, 24, 32, 2098, 1000, 0) == N.KEQ_ERR_CAPACITY
    assert lib.keq_gtsv_strided_inplace_noalloc(8, 16, 24, 32, 1 << 21, 2, 0) == N.KEQ_ERR_CAPACITY
    assert lib.keq_gtsv_strided_inplace_noalloc(0, 16, 24, 32, 10, 10, 0) == N.KEQ_ERR_INVALID
    assert lib.keq_gtsv_strided_inplace_noalloc(8, 16, 24, 32, 0, 10, 0) == N.KEQ_OK
