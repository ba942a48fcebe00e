"""Python mirror of the reference's `models` module for the thermal path:
GeomFields, ThermalFields, MeshMetricsCalculatorA, ThermalModelA.

Usage follows the reference scripts (src/fvm/scripts/testThermalModel.py,
src/fvm/test/THERMAL_MATRIX/testThermalParallel.py):

    geomFields = models.GeomFields('geom')
    metrics = models.MeshMetricsCalculatorA(geomFields, meshes); metrics.init()
    thermalFields = models.ThermalFields('therm')
    tmodel = models.ThermalModelA(geomFields, thermalFields, meshes)
    bc = tmodel.getBCMap()[3]; bc.bcType = 'SpecifiedTemperature'
    bc.setVar('specifiedTemperature', 400)
    tmodel.getOptions().linearSolver = fvmbaseExt.AMG()
    tmodel.init()
    thermalFields.conductivity[mesh.getCells()] = k        # numpy array
    tmodel.advance(100)
    T = thermalFields.temperature[mesh.getCells()]

Settings are held here and pushed through the C ABI at init()/advance().
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib
from ._lib import as_f64, check, dptr, iptr
from .fvmbaseExt import AMG, StorageSite, _KrylovSolver

BC_TYPES = {
    "SpecifiedTemperature": 0,
    "SpecifiedHeatFlux": 1,
    "Symmetry": 2,
    "Convective": 3,
    "Radiative": 4,
    "Mixed": 5,
}
BC_NAMES = {v: k for k, v in BC_TYPES.items()}
BC_VARS = ["specifiedTemperature", "specifiedHeatFlux", "convectiveCoefficient", "farFieldTemperature",
           "surfaceEmissivity"]
FIELD_IDS = {"temperature": 0, "conductivity": 1, "source": 2, "specificHeat": 3, "temperatureN1": 4}


class GeomFields:
    def __init__(self, name: str = "geom"):
        self.name = name


class MeshMetricsCalculatorA:
    """Geometry is computed when the Mesh is built (host FP64, same
    operation order as MeshMetricsCalculator<double>); init() is kept for
    API compatibility and exposes the arrays on geomFields."""

    def __init__(self, geomFields: GeomFields, meshes):
        self._g = geomFields
        self._meshes = list(meshes)

    def init(self) -> None:
        for m in self._meshes:
            setattr(self._g, "mesh%d" % m.getID(), m.getGeometry())


class Field:
    """thermalFields.<name>[cells]: numpy copies in, numpy copies out."""

    def __init__(self, owner: "ThermalFields", name: str):
        self._owner = owner
        self._name = name

    def _model(self):
        m = self._owner._model
        if m is None:
            raise _lib.FvmError(1, "field %s is not attached to a ThermalModel" % self._name)
        return m

    def __getitem__(self, site: StorageSite) -> np.ndarray:
        return self._model()._get_field(self._name, site)

    def __setitem__(self, site: StorageSite, values) -> None:
        self._model()._set_field(self._name, site, values)


class ThermalFields:
    def __init__(self, name: str = "therm"):
        self.name = name
        self._model = None
        for f in FIELD_IDS:
            setattr(self, f, Field(self, f))


class _VarDict(dict):
    """FloatVarDict: defineVar'd names only; setVar/getVar/[]."""

    def setVar(self, name: str, value: float) -> None:
        if name not in self:
            raise KeyError("uknown var " + name)
        self[name] = float(value)

    def getVar(self, name: str) -> float:
        return self[name]


class ThermalBC(_VarDict):
    def __init__(self, bc_type: str):
        super().__init__(specifiedTemperature=300.0, specifiedHeatFlux=0.0, convectiveCoefficient=0.0,
                         farFieldTemperature=300.0, surfaceEmissivity=1.0)
        self.bcType = bc_type


class ThermalVC(_VarDict):
    def __init__(self):
        super().__init__(thermalConductivity=1.0, density=1.0, specificHeat=1.0)
        self.vcType = "flow"


class ThermalModelOptions(_VarDict):
    """ThermalModelOptions (fvmbase/ThermalBC.h:33-67)."""

    def __init__(self):
        super().__init__(initialTemperature=300.0, timeStep=1e-7)
        self.relativeTolerance = 1e-8
        self.absoluteTolerance = 1e-16
        self.linearSolver = None
        self.useCentralDifference = False
        self.transient = False
        self.timeDiscretizationOrder = 1

    def getLinearSolver(self):
        if self.linearSolver is None:
            ls = AMG()
            ls.relativeTolerance = 1e-1
            ls.nMaxIterations = 20
            ls.verbosity = 0
            self.linearSolver = ls
        return self.linearSolver


class ThermalModelA:
    """ThermalModel<double> (fvmbase/ThermalModel.h:28-52) on the GPU."""

    def __init__(self, geomFields: GeomFields, thermalFields: ThermalFields, meshes):
        meshes = list(meshes)
        if len(meshes) != 1:
            raise _lib.FvmError(7, "one mesh per ThermalModelA")
        lib = _lib.load()
        self._mesh = meshes[0]
        arr = (ctypes.c_void_p * 1)(self._mesh.handle())
        h = ctypes.c_void_p()
        check(lib.fvm_thermal_create(arr, 1, ctypes.byref(h)))
        self._h = h
        self._fields = thermalFields
        thermalFields._model = self
        self._bcMap = {}
        for g in self._mesh.getBoundaryFaceGroups():
            t = ctypes.c_int(0)
            vals = np.zeros(5)
            check(lib.fvm_thermal_get_bc(self._h, 0, g.id, ctypes.byref(t), dptr(vals)))
            bc = ThermalBC(BC_NAMES[t.value])
            for name, v in zip(BC_VARS, vals):
                bc[name] = float(v)
            self._bcMap[g.id] = bc
        self._vcMap = {self._mesh.getID(): ThermalVC()}
        self._options = ThermalModelOptions()
        self._lastReport = None

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            try:
                _lib.load().fvm_thermal_destroy(h)
            except Exception:
                pass
            self._h = None

    # --- reference API -----------------------------------------------------
    def getBCMap(self):
        return self._bcMap

    def getVCMap(self):
        return self._vcMap

    def getBC(self, id_: int) -> ThermalBC:
        return self._bcMap[id_]

    def getOptions(self) -> ThermalModelOptions:
        return self._options

    def init(self) -> None:
        self._push()
        check(_lib.load().fvm_thermal_init(self._h))

    def advance(self, niter: int):
        self._push()
        rep = _lib.Report()
        check(_lib.load().fvm_thermal_advance(self._h, int(niter), ctypes.byref(rep)))
        self._lastReport = rep
        ls = self._options.getLinearSolver()
        ls._totalIterations += rep.linearIterations
        return rep

    def updateTime(self) -> None:
        check(_lib.load().fvm_thermal_update_time(self._h))

    def setSegments(self, cellOffsets) -> None:
        """Blocks of self cells (a batch of independent meshes packed into
        this model) that must each meet the outer tolerances on their own
        L1 residual norm; None or [] restores the combined test."""
        if cellOffsets is None or len(cellOffsets) == 0:
            check(_lib.load().fvm_thermal_set_segments(self._h, 0, None))
            self._nseg = 0
            return
        off = np.ascontiguousarray(cellOffsets, dtype=np.int32)
        check(_lib.load().fvm_thermal_set_segments(self._h, len(off) - 1, iptr(off)))
        self._nseg = len(off) - 1

    def getSegmentStatus(self):
        """(first L1 norm, last L1 norm, outer iteration of convergence or -1) per block."""
        n = getattr(self, "_nseg", 0)
        f, l, c = np.zeros(max(n, 1)), np.zeros(max(n, 1)), np.zeros(max(n, 1), np.int32)
        check(_lib.load().fvm_thermal_segments(self._h, max(n, 1), dptr(f), dptr(l), iptr(c)))
        return f[:n], l[:n], c[:n]

    def setLearnedCorrection(self, lc) -> None:
        """Use a trained fvm_b200.learned.LearnedCorrection in the AMG solves
        of advance() (None disables). The model keeps a reference to it."""
        check(_lib.load().fvm_thermal_set_learned(self._h, lc.handle() if lc is not None else None))
        self._learned = lc

    def printBCs(self) -> None:
        for k, bc in self._bcMap.items():
            print("Face Group %d:" % k)
            print("    bc type " + bc.bcType)
            for name, v in bc.items():
                print("   %s %s" % (name, v))

    def getHeatFluxIntegral(self, mesh, faceGroupId: int) -> float:
        """Sum of the boundary heat flux over a face group after the last
        advance() (ThermalModel::getHeatFluxIntegral)."""
        out = ctypes.c_double(0)
        check(_lib.load().fvm_thermal_heat_flux_integral(self._h, 0, int(faceGroupId), ctypes.byref(out)))
        return out.value

    def dumpMatrix(self, fileBase: str) -> None:
        """MatrixMarket dump of the current linearization, in the format of
        ThermalModel::dumpMatrix (fvmbase/ThermalModel_impl.h:499-572)."""
        diag, off, b = self.getLinearSystem()
        row, col = self._interior_pattern()
        n = len(diag)
        with open(fileBase + "_mesh0.mat", "w") as f:
            f.write("%%MatrixMarket matrix coordinate real general\n")
            f.write("%d %d %d\n" % (n, n, n + len(off)))
            for i in range(n):
                f.write("%d %d %f\n" % (i + 1, i + 1, diag[i]))
                for k in range(row[i], row[i + 1]):
                    f.write("%d %d %f\n" % (i + 1, col[k] + 1, off[k]))
        with open(fileBase + ".rhs", "w") as f:
            for i in range(n):
                f.write("%f\n" % (-b[i]))

    # --- additions -------------------------------------------------------------
    def getNormHistory(self) -> np.ndarray:
        lib = _lib.load()
        n = ctypes.c_int(0)
        check(lib.fvm_thermal_history(self._h, None, 0, ctypes.byref(n)))
        out = np.zeros(n.value)
        check(lib.fvm_thermal_history(self._h, dptr(out), n.value, ctypes.byref(n)))
        return out

    def getLinearSystem(self):
        """(diag, off, b) of the system advance() would solve next, in the
        reference's row/column order (self rows, self columns)."""
        self._push()
        n = self._mesh.getCells().getSelfCount()
        row, col = self._interior_pattern()
        diag = np.zeros(n)
        off = np.zeros(len(col))
        b = np.zeros(n)
        nnz = ctypes.c_int(0)
        check(_lib.load().fvm_thermal_linear_system(self._h, dptr(diag), dptr(off), dptr(b), ctypes.byref(nnz)))
        return diag, off, b

    def getHierarchy(self):
        """(sizes, [coarseIndex of each fine level]) of the AMG setup."""
        self._push()
        n = self._mesh.getCells().getSelfCount()
        sizes = np.zeros(64, np.int32)
        nl = ctypes.c_int(0)
        ci = np.zeros(2 * n + 64, np.int32)
        check(_lib.load().fvm_thermal_hierarchy(self._h, ctypes.byref(nl), iptr(sizes), 64, iptr(ci), len(ci)))
        s = [n] + list(sizes[: nl.value])
        out, p = [], 0
        for lvl in range(nl.value):
            out.append(ci[p: p + s[lvl]].copy())
            p += s[lvl]
        return list(sizes[: nl.value]), out

    def getLevelMatrix(self, level: int) -> dict:
        """Level `level` of the AMG hierarchy as CSR {row, col, val, diag},
        numbered as getHierarchy()'s coarseIndex numbers it (level 0 in
        reference cell order); stored zeros left out."""
        self._push()
        lib = _lib.load()
        n = ctypes.c_int(0)
        nnz = ctypes.c_int(0)
        check(lib.fvm_thermal_level_matrix(self._h, int(level), ctypes.byref(n), ctypes.byref(nnz), None, None, None,
                                           None, 0))
        row = np.zeros(n.value + 1, np.int32)
        col = np.zeros(max(nnz.value, 1), np.int32)
        val = np.zeros(max(nnz.value, 1))
        diag = np.zeros(max(n.value, 1))
        cap = max(nnz.value, n.value, 1)
        check(lib.fvm_thermal_level_matrix(self._h, int(level), ctypes.byref(n), ctypes.byref(nnz), iptr(row),
                                           iptr(col), dptr(val), dptr(diag), cap))
        return {"row": row, "col": col[: nnz.value], "val": val[: nnz.value], "diag": diag[: n.value]}

    def getLaunchPlans(self):
        """[(threadsPerRow, threadsPerBlock)] of each level's smoother kernels
        as the autotuner chose them; ELL-32 levels: (-width, 0)."""
        self._push()
        tpr = np.zeros(64, np.int32)
        blk = np.zeros(64, np.int32)
        nl = ctypes.c_int(0)
        check(_lib.load().fvm_thermal_launch_plans(self._h, ctypes.byref(nl), iptr(tpr), iptr(blk), 64))
        return [(int(a), int(b)) for a, b in zip(tpr[: nl.value], blk[: nl.value])]

    def profile(self, reps: int = 5) -> dict:
        """CUDA-event timings of the finest-level kernels (see fvm_thermal_profile)."""
        self._push()
        out = np.zeros(13)
        check(_lib.load().fvm_thermal_profile(self._h, int(reps), dptr(out)))
        keys = ["gs_pass_ms", "gs_pass_bytes", "residual_ms", "residual_bytes", "cycle_ms", "cycle_bytes", "levels",
                "rows", "entries", "kernels_per_cycle", "colors", "face_flux_ms", "face_flux_bytes"]
        return dict(zip(keys, out.tolist()))

    def profileLevels(self, reps: int = 5) -> list:
        """Per AMG level: CUDA-event timings and algorithmic bytes of the
        cycle's kernels (see fvm_thermal_profile_levels)."""
        self._push()
        out = np.zeros(8 * 64)
        nl = ctypes.c_int(0)
        check(_lib.load().fvm_thermal_profile_levels(self._h, int(reps), ctypes.byref(nl), dptr(out), len(out)))
        keys = ["rows", "entries", "smoother_ms", "smoother_bytes", "restrict_ms", "restrict_bytes", "prolong_ms",
                "prolong_bytes"]
        return [dict(zip(keys, out[8 * lvl: 8 * lvl + 8].tolist())) for lvl in range(nl.value)]

    def lastReport(self):
        return self._lastReport

    def _interior_pattern(self):
        n = self._mesh.getCells().getSelfCount()
        row, col = self._mesh.getCellCells()
        r = [0]
        c = []
        for i in range(n):
            cols = col[row[i]: row[i + 1]]
            cols = cols[cols < n]
            c.extend(cols.tolist())
            r.append(len(c))
        return np.asarray(r, np.int32), np.asarray(c, np.int32)

    # --- plumbing ----------------------------------------------------------------
    def _push(self) -> None:
        lib = _lib.load()
        o = _lib.ThermalOptions()
        opts = self._options
        o.relativeTolerance = float(opts.relativeTolerance)
        o.absoluteTolerance = float(opts.absoluteTolerance)
        o.transient = int(bool(opts.transient))
        o.timeDiscretizationOrder = int(opts.timeDiscretizationOrder)
        o.initialTemperature = float(opts["initialTemperature"])
        o.timeStep = float(opts["timeStep"])
        vc = self._vcMap[self._mesh.getID()]
        o.thermalConductivity = float(vc["thermalConductivity"])
        o.density = float(vc["density"])
        o.specificHeat = float(vc["specificHeat"])
        ls = opts.getLinearSolver()
        if isinstance(ls, _KrylovSolver):
            o.linear = ls.options()
        else:
            ls._fill(o.linear, 0)
        prev = _lib.ThermalOptions()
        check(lib.fvm_thermal_get_options(self._h, ctypes.byref(prev)))
        if bytes(prev) != bytes(o):
            check(lib.fvm_thermal_set_options(self._h, ctypes.byref(o)))
        for gid, bc in self._bcMap.items():
            if bc.bcType not in BC_TYPES:
                raise _lib.FvmError(7, bc.bcType + " not implemented for ThermalModel")
            vals = np.array([bc[v] for v in BC_VARS], dtype=np.float64)
            check(lib.fvm_thermal_set_bc(self._h, 0, int(gid), BC_TYPES[bc.bcType], dptr(vals)))

    def _set_field(self, name, site, values) -> None:
        v = as_f64(values).reshape(-1)
        check(_lib.load().fvm_thermal_set_cell_field(self._h, 0, FIELD_IDS[name], dptr(v), len(v)))

    def _get_field(self, name, site) -> np.ndarray:
        n = site.getCount()
        out = np.empty(n)
        check(_lib.load().fvm_thermal_get_cell_field(self._h, 0, FIELD_IDS[name], dptr(out), n))
        return out
