"""The allocation-free tridiagonal solve keq_gtsv_strided_inplace_noalloc.

Some callers cannot allocate device memory (a binding that forwards only the
operation's own tensors, or a host that must not call cudaMalloc), so they
cannot hand keq_gtsv_strided_inplace its workspace.  The noalloc entry point
keeps that scratch in a fixed array inside the library.  This test calls it
through the C ABI twice in a row, on different systems, and checks each
result against keq_gtsv_strided_inplace with a caller workspace (same
kernel, so the tolerance of the other parity tests, 1e-12 normwise, is met
with room).  The rejection of requests above the fixed capacity is a host
check, tested without a GPU in test_abi.py.

The file name sorts last so that a run stopping at the first failure has
already run every other test."""
import ctypes as C

import numpy as np
import pytest
import torch

from kineticeq_b200 import _native as N

pytestmark = pytest.mark.gpu
TOL = 1e-12


def _systems(n, batch, seed):
    g = torch.Generator("cpu").manual_seed(seed)
    dl = torch.rand((batch, n), generator=g, dtype=torch.float64) - 0.5
    du = torch.rand((batch, n), generator=g, dtype=torch.float64) - 0.5
    d = 2.0 + torch.rand((batch, n), generator=g, dtype=torch.float64)
    B = torch.rand((batch, n), generator=g, dtype=torch.float64) * 2 - 1
    return [t.cuda() for t in (dl, d, du, B)]


def _with_workspace(lib, dl, d, du, B, n, batch, sh):
    X = B.clone()
    need = C.c_size_t(0)
    N.check(lib.keq_gtsv_workspace_size(n, batch, C.byref(need)), "gtsv workspace")
    ws = torch.empty((max(int(need.value), 8),), dtype=torch.uint8, device="cuda")
    N.check(lib.keq_gtsv_strided_inplace(dl.data_ptr(), d.data_ptr(), du.data_ptr(), X.data_ptr(),
                                         n, batch, ws.data_ptr(), ws.numel(), sh), "gtsv")
    return X


def test_noalloc_matches_workspace_solve_twice():
    lib = N.load()
    sh = N.stream_handle()
    for call, (n, batch, seed) in enumerate([(4094, 512, 11), (1000, 77, 12)]):
        dl, d, du, B = _systems(n, batch, seed)
        ref = _with_workspace(lib, dl, d, du, B, n, batch, sh)
        X = B.clone()
        rc = lib.keq_gtsv_strided_inplace_noalloc(dl.data_ptr(), d.data_ptr(), du.data_ptr(),
                                                  X.data_ptr(), n, batch, sh)
        assert rc == N.KEQ_OK, N.status_text(rc)
        torch.cuda.synchronize()
        a, b = X.cpu().numpy(), ref.cpu().numpy()
        err = float(np.abs(a - b).max() / np.abs(b).max())
        assert err <= TOL, (call, err)
