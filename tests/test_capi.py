"""The C-ABI library loads on the CPU and exports every entry point that
include/fvm_b200.h declares; defaults mirror the reference's."""
import os
import re

from fvm_b200 import _lib

HEADER = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include", "fvm_b200.h")


def declared_functions():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(fvm_[a-z0-9_]+)\s*\(", src)))


def test_header_symbols_exported(fvm_lib):
    names = declared_functions()
    assert len(names) >= 20
    for n in names:
        assert hasattr(fvm_lib, n), n
    # and the binding covers exactly the header
    assert sorted(_lib.EXPORTED) == names


def test_reference_defaults():
    o = _lib.default_linear_options()
    # AMG::AMG() (fvmbase/AMG.cpp:15-22)
    assert (o.maxCoarseLevels, o.nPreSweeps, o.nPostSweeps, o.coarseGroupSize) == (30, 0, 1, 2)
    assert o.weightRatioThreshold == 0.65 and o.cycleType == 0 and o.smootherType == 0
    t = _lib.default_thermal_options()
    # ThermalModelOptions (fvmbase/ThermalBC.h:33-67)
    assert t.relativeTolerance == 1e-8 and t.absoluteTolerance == 1e-16
    assert t.initialTemperature == 300.0 and t.timeStep == 1e-7 and t.transient == 0
    assert t.linear.relativeTolerance == 1e-1 and t.linear.nMaxIterations == 20
    # added knobs: the outer loop as one CUDA graph (bitwise the host loop) on
    # by default, its Anderson acceleration off (the reference's plain loop)
    assert o.outerOnDevice == 1 and o.outerAcceleration == 0


def test_outer_acceleration_depth_is_checked():
    """The acceleration depth is checked where the options cross the C ABI
    (no GPU needed: the host-only hierarchy entry point converts them)."""
    import numpy as np
    import pytest

    from fvm_b200 import fvmbaseExt

    row = np.array([0, 1, 3, 4], dtype=np.int32)
    col = np.array([1, 0, 2, 1], dtype=np.int32)
    diag = np.full(3, 2.0)
    off = np.full(4, -1.0)
    a = fvmbaseExt.AMG()
    for depth in (-1, 6):
        a.outerAcceleration = depth
        with pytest.raises(_lib.FvmError) as e:
            a.hierarchy_csr(row, col, diag, off)
        assert "outerAcceleration" in str(e.value)
    a.outerAcceleration = 5
    a.hierarchy_csr(row, col, diag, off)


def test_errors_are_reported(fvm_lib):
    import ctypes

    import numpy as np
    import pytest

    from fvm_b200 import fvmbaseExt

    # a face pointing at a cell that does not exist
    with pytest.raises(_lib.FvmError) as e:
        fvmbaseExt.Mesh(2, 1, np.zeros((3, 3)), [0, 5], [0, 1], [2], [1])
    assert "range" in str(e.value)
    h = ctypes.c_void_p()
    rc = fvm_lib.fvm_mesh_create(4, 1, 1, None, 1, None, None, None, 1, None, ctypes.byref(h))
    assert rc == 1 and b"dimension" in fvm_lib.fvm_last_error()
