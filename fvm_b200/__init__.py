"""fvm_b200: B200-native FVM thermal diffusion + AMG hot path.

The reference's Python surface for this path is mirrored by the
submodules `fvmbaseExt` (Mesh, AMG, CG, BCGStab) and `models`
(GeomFields, ThermalFields, MeshMetricsCalculatorA, ThermalModelA); the
work runs in libfvm_b200.so (host C++ + sm_100a CUDA) through the C ABI
declared in include/fvm_b200.h.
"""
from . import _lib, fvmbaseExt, meshgen, models  # noqa: F401

atype = "double"


def library_path() -> str:
    return _lib.LIB_PATH
