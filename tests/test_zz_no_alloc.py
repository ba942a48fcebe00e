"""fvm_csr_residual_device_noalloc: the residual entry point for callers
that cannot allocate device memory (a stream capture that must not
allocate, a fixed-budget real-time loop, an application whose allocator
owns all device memory). They pass device buffers they already own; the
entry point allocates nothing and keeps its reduction scratch in a fixed
device array inside the library.

Checked against the allocating entry point fvm_csr_residual on the same
system, on two calls in a row (the second with a different x, so stale
scratch contents would show), with the tolerance of the other residual
tests: r exact, L1 norm to 1e-13 relative. Two systems: the reference's
226-row MatrixMarket system (one 256-row block) and a 150,000-row
diagonally dominant system (586 block sums in the fixed array, reduced by a
second kernel). This file is collected last so that a failure here leaves
every other test already run.
"""
import ctypes

import numpy as np
import pytest

from fvm_b200 import _lib, fvmbaseExt
from helpers import load_fixture

pytestmark = pytest.mark.gpu


def _mm226():
    z = load_fixture("mm226.npz")
    return z["row"], z["col"], z["diag"], z["off"], z["b"]


def _large(n=150_000, width=7, seed=5):
    """Random pattern with `width` off-diagonals per row, negative diagonal
    dominating the row (the reference's sign convention)."""
    rng = np.random.default_rng(seed)
    col = rng.integers(0, n, size=(n, width)).astype(np.int32)
    row = np.arange(0, n * width + 1, width, dtype=np.int32)
    off = rng.uniform(0.1, 1.0, size=(n, width))
    diag = -(off.sum(axis=1) + rng.uniform(0.0, 1.0, size=n))
    b = rng.standard_normal(n)
    return row, col.ravel(), diag, off.ravel(), b


@pytest.mark.parametrize("system", ["mm226", "large150k"])
def test_no_alloc_residual_matches_allocating_entry_point(system):
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    lib = _lib.load()
    row, col, diag, off, b = _mm226() if system == "mm226" else _large()
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


_RESET_CHILD = r"""
import ctypes, sys
import numpy as np
sys.path.insert(0, sys.argv[1])
sys.path.insert(0, sys.argv[2])
from fvm_b200 import _lib, fvmbaseExt
from test_zz_no_alloc import _large
lib = _lib.load()
rt = ctypes.CDLL("libcudart.so.12")  # the runtime the library itself uses
row, col, diag, off, b = _large(n=120_000, seed=9)
n = len(diag)

def dev(a):
    a = np.ascontiguousarray(a)
    p = ctypes.c_void_p()
    assert rt.cudaMalloc(ctypes.byref(p), ctypes.c_size_t(max(a.nbytes, 8))) == 0
    assert rt.cudaMemcpy(p, a.ctypes.data_as(ctypes.c_void_p), ctypes.c_size_t(a.nbytes), 1) == 0
    return p

for call in range(2):
    x = np.random.default_rng(call).standard_normal(n)
    bufs = [dev(row.astype(np.int32)), dev(col.astype(np.int32)), dev(diag), dev(off), dev(x), dev(b),
            dev(np.full(n, np.nan)), dev(np.full(1, np.nan))]
    rc = lib.fvm_csr_residual_device_noalloc(n, *bufs, None)
    assert rc == 0, lib.fvm_last_error().decode()
    assert rt.cudaDeviceSynchronize() == 0
    r = np.empty(n); nrm = np.empty(1)
    assert rt.cudaMemcpy(r.ctypes.data_as(ctypes.c_void_p), bufs[6], ctypes.c_size_t(r.nbytes), 2) == 0
    assert rt.cudaMemcpy(nrm.ctypes.data_as(ctypes.c_void_p), bufs[7], ctypes.c_size_t(8), 2) == 0
    r_ref, norm_ref = fvmbaseExt.csr_residual(row, col, diag, off, x, b)
    np.testing.assert_array_equal(r, r_ref)
    assert abs(nrm[0] - norm_ref) <= 1e-13 * norm_ref
    for p in bufs:
        assert rt.cudaFree(p) == 0
    if call == 0:
        # ends this process's context; the next call runs in a new one
        assert rt.cudaDeviceReset() == 0
print("reset ok")
"""


def test_no_alloc_after_device_reset():
    """Two calls separated by cudaDeviceReset, in a child process of their
    own (the reset ends every allocation of the process's context): the
    second call looks the scratch array's address up again in the new
    context and matches the allocating entry point again."""
    import os
    import subprocess
    import sys

    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    here = os.path.dirname(os.path.abspath(__file__))
    root = os.path.dirname(here)
    out = subprocess.run([sys.executable, "-c", _RESET_CHILD, root, here], capture_output=True, text=True,
                         timeout=300)
    assert out.returncode == 0 and "reset ok" in out.stdout, out.stdout + out.stderr
