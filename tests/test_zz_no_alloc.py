"""fvm_csr_residual_device_noalloc: the residual entry point for callers
that cannot allocate device memory (a stream capture that must not
allocate, a fixed-budget real-time loop, an application whose allocator
owns all device memory). They pass device buffers they already own; the
entry point allocates nothing and keeps its reduction scratch in a fixed
device array inside the library.

Checked against the allocating entry point fvm_csr_residual on the same
system, on two calls in a row (the second with a different x, so stale
scratch contents would show), with the tolerance of the other residual
tests: r exact, L1 norm to 1e-13 relative. This file is collected last so
that a failure here leaves every other test already run.
"""
import ctypes

import numpy as np
import pytest

from fvm_b200 import _lib, fvmbaseExt
from helpers import load_fixture

pytestmark = pytest.mark.gpu


def _system():
    z = load_fixture("mm226.npz")
    return z["row"], z["col"], z["diag"], z["off"], z["b"]


def test_no_alloc_residual_matches_allocating_entry_point():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    lib = _lib.load()
    row, col, diag, off, b = _system()
    n = len(diag)
    dev = torch.device("cuda:0")
    d_row = torch.as_tensor(np.ascontiguousarray(row, np.int32), device=dev)
    d_col = torch.as_tensor(np.ascontiguousarray(col, np.int32), device=dev)
    d_diag = torch.as_tensor(diag, dtype=torch.float64, device=dev)
    d_off = torch.as_tensor(off, dtype=torch.float64, device=dev)
    d_b = torch.as_tensor(b, dtype=torch.float64, device=dev)
    d_r = torch.empty(n, dtype=torch.float64, device=dev)
    d_norm = torch.empty(1, dtype=torch.float64, device=dev)
    rng = np.random.default_rng(11)
    for call in range(2):
        x = rng.standard_normal(n) * (10.0 ** call)
        d_x = torch.as_tensor(x, dtype=torch.float64, device=dev)
        d_r.fill_(np.nan)
        d_norm.fill_(np.nan)
        torch.cuda.synchronize()
        rc = lib.fvm_csr_residual_device_noalloc(
            n, ctypes.c_void_p(d_row.data_ptr()), ctypes.c_void_p(d_col.data_ptr()),
            ctypes.c_void_p(d_diag.data_ptr()), ctypes.c_void_p(d_off.data_ptr()), ctypes.c_void_p(d_x.data_ptr()),
            ctypes.c_void_p(d_b.data_ptr()), ctypes.c_void_p(d_r.data_ptr()), ctypes.c_void_p(d_norm.data_ptr()),
            None)
        assert rc == 0, lib.fvm_last_error().decode()
        torch.cuda.synchronize()
        r_ref, norm_ref = fvmbaseExt.csr_residual(row, col, diag, off, x, b)
        np.testing.assert_array_equal(d_r.cpu().numpy(), r_ref, err_msg="call %d" % call)
        assert abs(float(d_norm.cpu()[0]) - norm_ref) <= 1e-13 * norm_ref, "call %d" % call


def test_no_alloc_rejects_oversized_systems():
    lib = _lib.load()
    one = ctypes.c_void_p(1)  # never dereferenced: the size check comes first
    rc = lib.fvm_csr_residual_device_noalloc(16777216 + 1, one, one, one, one, one, one, None, one, None)
    assert rc == 8
    assert b"16777216" in lib.fvm_last_error()
