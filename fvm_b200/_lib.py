"""ctypes binding of libfvm_b200.so (the C ABI declared in include/fvm_b200.h).

The library is loaded from this package directory only; a missing or stale
build raises instead of falling back to any other implementation.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libfvm_b200.so")

c_int_p = ctypes.POINTER(ctypes.c_int)
c_double_p = ctypes.POINTER(ctypes.c_double)
c_float_p = ctypes.POINTER(ctypes.c_float)


class LinearOptions(ctypes.Structure):
    _fields_ = [
        ("solver", ctypes.c_int),
        ("nMaxIterations", ctypes.c_int),
        ("relativeTolerance", ctypes.c_double),
        ("absoluteTolerance", ctypes.c_double),
        ("verbosity", ctypes.c_int),
        ("maxCoarseLevels", ctypes.c_int),
        ("nPreSweeps", ctypes.c_int),
        ("nPostSweeps", ctypes.c_int),
        ("coarseGroupSize", ctypes.c_int),
        ("weightRatioThreshold", ctypes.c_double),
        ("cycleType", ctypes.c_int),
        ("smootherType", ctypes.c_int),
        ("scaleCorrections", ctypes.c_int),
        ("smootherOrdering", ctypes.c_int),
        ("coarsestSize", ctypes.c_int),
        ("coarseSolver", ctypes.c_int),
        ("precision", ctypes.c_int),
        ("useGraphs", ctypes.c_int),
        ("coarseJacobiRows", ctypes.c_int),
        ("jacobiWeight", ctypes.c_double),
        ("preconditioner", ctypes.c_int),
        ("autotune", ctypes.c_int),
        ("planThreadsPerRow", ctypes.c_int),
        ("planBlock", ctypes.c_int),
        ("setupOnDevice", ctypes.c_int),
        ("matchRounds", ctypes.c_int),
        ("matchBeta", ctypes.c_double),
        ("matchPasses", ctypes.c_int),
        ("coarsePostSweeps", ctypes.c_int),
        ("planEllRows", ctypes.c_int),
        ("chebyshevDegree", ctypes.c_int),
        ("chebyshevFraction", ctypes.c_double),
        ("gsReverse", ctypes.c_int),
        ("patternOnDevice", ctypes.c_int),
        ("fuseProlongation", ctypes.c_int),
        ("outerOnDevice", ctypes.c_int),
        ("outerAcceleration", ctypes.c_int),
    ]


class ThermalOptions(ctypes.Structure):
    _fields_ = [
        ("relativeTolerance", ctypes.c_double),
        ("absoluteTolerance", ctypes.c_double),
        ("transient", ctypes.c_int),
        ("timeDiscretizationOrder", ctypes.c_int),
        ("initialTemperature", ctypes.c_double),
        ("timeStep", ctypes.c_double),
        ("thermalConductivity", ctypes.c_double),
        ("density", ctypes.c_double),
        ("specificHeat", ctypes.c_double),
        ("linear", LinearOptions),
    ]


class Report(ctypes.Structure):
    _fields_ = [
        ("iterations", ctypes.c_int),
        ("linearIterations", ctypes.c_int),
        ("initialNorm", ctypes.c_double),
        ("lastNorm", ctypes.c_double),
        ("converged", ctypes.c_int),
        ("seconds", ctypes.c_double),
        ("setupSeconds", ctypes.c_double),
        ("launches", ctypes.c_longlong),
        ("learnedSteps", ctypes.c_int),
        ("learnedAccepted", ctypes.c_int),
        ("outerOnDevice", ctypes.c_int),
    ]


# name -> (restype, argtypes)
_SIGS = {
    "fvm_last_error": (ctypes.c_char_p, []),
    "fvm_default_linear_options": (None, [ctypes.POINTER(LinearOptions)]),
    "fvm_default_thermal_options": (None, [ctypes.POINTER(ThermalOptions)]),
    "fvm_mesh_create": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_int, c_double_p, ctypes.c_int,
                                       c_int_p, c_int_p, c_int_p, ctypes.c_int, c_int_p,
                                       ctypes.POINTER(ctypes.c_void_p)]),
    "fvm_mesh_set_group": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_char_p]),
    "fvm_mesh_sizes": (ctypes.c_int, [ctypes.c_void_p, c_int_p]),
    "fvm_mesh_connectivity": (ctypes.c_int, [ctypes.c_void_p, c_int_p, c_int_p, c_int_p]),
    "fvm_mesh_geometry": (ctypes.c_int, [ctypes.c_void_p, c_double_p, c_double_p, c_double_p, c_double_p,
                                         c_double_p]),
    "fvm_mesh_destroy": (ctypes.c_int, [ctypes.c_void_p]),
    "fvm_thermal_create": (ctypes.c_int, [ctypes.POINTER(ctypes.c_void_p), ctypes.c_int,
                                          ctypes.POINTER(ctypes.c_void_p)]),
    "fvm_thermal_set_options": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ThermalOptions)]),
    "fvm_thermal_get_options": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ThermalOptions)]),
    "fvm_thermal_set_bc": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                          c_double_p]),
    "fvm_thermal_get_bc": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, c_int_p, c_double_p]),
    "fvm_thermal_init": (ctypes.c_int, [ctypes.c_void_p]),
    "fvm_thermal_set_cell_field": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, c_double_p,
                                                  ctypes.c_int]),
    "fvm_thermal_get_cell_field": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, c_double_p,
                                                  ctypes.c_int]),
    "fvm_thermal_advance": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(Report)]),
    "fvm_thermal_update_time": (ctypes.c_int, [ctypes.c_void_p]),
    "fvm_thermal_heat_flux_integral": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, c_double_p]),
    "fvm_thermal_history": (ctypes.c_int, [ctypes.c_void_p, c_double_p, ctypes.c_int, c_int_p]),
    "fvm_thermal_linear_system": (ctypes.c_int, [ctypes.c_void_p, c_double_p, c_double_p, c_double_p, c_int_p]),
    "fvm_thermal_launch_plans": (ctypes.c_int, [ctypes.c_void_p, c_int_p, c_int_p, c_int_p, ctypes.c_int]),
    "fvm_thermal_level_matrix": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, c_int_p, c_int_p, c_int_p, c_int_p,
                                                 c_double_p, c_double_p, ctypes.c_int]),
    "fvm_thermal_profile_levels": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, c_int_p, c_double_p, ctypes.c_int]),
    "fvm_fluent_read": (ctypes.c_int, [ctypes.c_char_p, ctypes.POINTER(ctypes.c_void_p)]),
    "fvm_fluent_cell_zones": (ctypes.c_int, [ctypes.c_void_p, c_int_p]),
    "fvm_fluent_mesh_sizes": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, c_int_p]),
    "fvm_fluent_mesh_arrays": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, c_double_p, c_int_p, c_int_p, c_int_p,
                                               c_int_p, c_int_p]),
    "fvm_fluent_group_type": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_char_p,
                                              ctypes.c_int]),
    "fvm_fluent_mesh_create": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(ctypes.c_void_p)]),
    "fvm_fluent_destroy": (ctypes.c_int, [ctypes.c_void_p]),
    "fvm_learned_wait_probe": (ctypes.c_int, [ctypes.c_uint, c_int_p]),
    "fvm_learned_set_objective": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int]),
    "fvm_learned_set_useful_factor": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_double]),
    "fvm_learned_residual_factor": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_double)]),
    "fvm_thermal_hierarchy": (ctypes.c_int, [ctypes.c_void_p, c_int_p, c_int_p, ctypes.c_int, c_int_p,
                                             ctypes.c_int]),
    "fvm_thermal_profile": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, c_double_p]),
    "fvm_thermal_destroy": (ctypes.c_int, [ctypes.c_void_p]),
    "fvm_amg_solve_csr": (ctypes.c_int, [ctypes.c_int, c_int_p, c_int_p, c_double_p, c_double_p, c_double_p,
                                         c_double_p, ctypes.POINTER(LinearOptions), ctypes.POINTER(Report),
                                         c_double_p, ctypes.c_int, c_int_p, c_int_p, ctypes.c_int, c_int_p]),
    "fvm_csr_residual": (ctypes.c_int, [ctypes.c_int, c_int_p, c_int_p, c_double_p, c_double_p, c_double_p,
                                        c_double_p, c_double_p, c_double_p]),
    "fvm_csr_residual_device_noalloc": (ctypes.c_int, [ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p,
                                                       ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                                       ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                                       ctypes.c_void_p]),
    "fvm_amg_hierarchy_csr": (ctypes.c_int, [ctypes.c_int, c_int_p, c_int_p, c_double_p, c_double_p,
                                             ctypes.POINTER(LinearOptions), ctypes.c_int, c_int_p, c_int_p,
                                             ctypes.c_int, c_int_p, ctypes.c_int, c_int_p, ctypes.c_int]),
    "fvm_thermal_set_segments": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, c_int_p]),
    "fvm_thermal_segments": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, c_double_p, c_double_p, c_int_p]),
    "fvm_learned_create": (ctypes.c_void_p, [ctypes.c_ulonglong]),
    "fvm_learned_destroy": (ctypes.c_int, [ctypes.c_void_p]),
    "fvm_learned_num_params": (ctypes.c_int, []),
    "fvm_learned_get_params": (ctypes.c_int, [ctypes.c_void_p, c_float_p, ctypes.c_int]),
    "fvm_learned_set_params": (ctypes.c_int, [ctypes.c_void_p, c_float_p, ctypes.c_int]),
    "fvm_learned_harvest": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_int,
                                           ctypes.c_double, ctypes.c_int, c_int_p]),
    "fvm_learned_num_pairs": (ctypes.c_int, [ctypes.c_void_p]),
    "fvm_learned_train": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_float, ctypes.c_ulonglong,
                                         c_double_p]),
    "fvm_learned_evaluate": (ctypes.c_int, [ctypes.c_void_p, c_double_p]),
    "fvm_thermal_set_learned": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p]),
    "fvm_learned_forward_csr": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, c_int_p, c_int_p, c_double_p,
                                               c_double_p, c_double_p, c_double_p]),
    "fvm_learned_gradient_csr": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, c_int_p, c_int_p, c_double_p,
                                                c_double_p, c_double_p, c_double_p, c_float_p, c_double_p]),
    "fvm_learned_set_tensor_cores": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int]),
    "fvm_learned_tensor_cores": (ctypes.c_int, [ctypes.c_void_p, c_int_p]),
}

EXPORTED = tuple(_SIGS)

_lib = None


def load():
    """Loads the in-tree library (building it first when absent and nvcc exists)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        from . import build as _build

        _build.build()
    lib = ctypes.CDLL(LIB_PATH)
    for name, (res, args) in _SIGS.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


class FvmError(RuntimeError):
    """Raised for a non-zero status from the C ABI (the reference raises
    RuntimeError from CException through SWIG)."""

    def __init__(self, status: int, msg: str):
        super().__init__(msg)
        self.status = status


def check(status: int) -> None:
    if status != 0:
        msg = load().fvm_last_error().decode(errors="replace")
        raise FvmError(status, msg)


def dptr(a: np.ndarray):
    return a.ctypes.data_as(c_double_p)


def iptr(a: np.ndarray):
    return a.ctypes.data_as(c_int_p)


def as_f64(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.float64)


def as_i32(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.int32)


def default_linear_options() -> LinearOptions:
    o = LinearOptions()
    load().fvm_default_linear_options(ctypes.byref(o))
    return o


def default_thermal_options() -> ThermalOptions:
    o = ThermalOptions()
    load().fvm_default_thermal_options(ctypes.byref(o))
    return o
