"""Python mirror of the reference's fvmbaseExt module for this path:
Mesh (7-argument constructor), StorageSite, AMG, CG, BCGStab.

Names, fields and defaults follow fvmbase/Mesh.i, AMG.h/AMG.cpp,
LinearSolver.h, CG.h and BCGStab.h of the reference; the solve runs on the
GPU through libfvm_b200.so.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib
from ._lib import as_f64, as_i32, check, dptr, iptr


class StorageSite:
    """Counts of a site: self entries and self + ghost entries."""

    def __init__(self, self_count: int, ghost_count: int = 0):
        self._self = int(self_count)
        self._ghost = int(ghost_count)

    def getSelfCount(self) -> int:
        return self._self

    def getCount(self) -> int:
        return self._self + self._ghost

    def getCountLevel1(self) -> int:
        return self._self + self._ghost


class FaceGroup:
    def __init__(self, id_: int, offset: int, size: int, group_type: str):
        self.id = id_
        self.groupType = group_type
        self.site = StorageSite(size)
        self.offset = offset


class Mesh:
    """Mesh(dimension, nCells, nodes, faceCells, faceNodes, faceNodeCount,
    faceGroupSize) -- fvmbase/Mesh.cpp:132-247. Boundary groups get ids
    1..k and type 'wall'. Connectivity and geometry are computed once, here,
    on the host (bit-identical to the reference)."""

    _lastID = 0

    def __init__(self, dimension, nCells, nodes, faceCells, faceNodes, faceNodeCount, faceGroupSize):
        lib = _lib.load()
        self._nodes = as_f64(np.asarray(nodes).reshape(-1, 3))
        self._faceCells = as_i32(np.asarray(faceCells).reshape(-1))
        self._faceNodes = as_i32(faceNodes)
        self._faceNodeCount = as_i32(faceNodeCount)
        self._groupSize = as_i32(faceGroupSize)
        h = ctypes.c_void_p()
        check(lib.fvm_mesh_create(int(dimension), int(nCells), len(self._nodes), dptr(self._nodes),
                                  len(self._faceNodeCount), iptr(self._faceCells), iptr(self._faceNodes),
                                  iptr(self._faceNodeCount), len(self._groupSize), iptr(self._groupSize),
                                  ctypes.byref(h)))
        self._h = h
        sizes = np.zeros(7, np.int32)
        check(lib.fvm_mesh_sizes(self._h, iptr(sizes)))
        self._dim, self._nCells, self._nGhost, self._nNodes, self._nFaces, self._nnz, ng = map(int, sizes)
        self._id = Mesh._lastID
        Mesh._lastID += 1
        offs = np.concatenate([[0], np.cumsum(self._groupSize)])
        self._groups = [FaceGroup(0, 0, int(self._groupSize[0]), "interior")]
        for g in range(1, ng):
            self._groups.append(FaceGroup(g, int(offs[g]), int(self._groupSize[g]), "wall"))
        self._cells = StorageSite(self._nCells, self._nGhost)
        self._faces = StorageSite(self._nFaces)
        self._nodeSite = StorageSite(self._nNodes)

    @classmethod
    def from_dict(cls, d: dict) -> "Mesh":
        """Builds from the dict the meshgen generators return."""
        return cls(d["dim"], d["nCells"], d["nodes"], d["faceCells"], d["faceNodes"], d["faceNodeCount"],
                   d["faceGroupSize"])

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            try:
                _lib.load().fvm_mesh_destroy(h)
            except Exception:
                pass
            self._h = None

    def handle(self):
        return self._h

    def getID(self) -> int:
        return self._id

    def getDimension(self) -> int:
        return self._dim

    def getCells(self) -> StorageSite:
        return self._cells

    def getFaces(self) -> StorageSite:
        return self._faces

    def getNodes(self) -> StorageSite:
        return self._nodeSite

    def getBoundaryFaceGroups(self):
        return self._groups[1:]

    def getAllFaceGroups(self):
        return list(self._groups)

    def setFaceGroup(self, group: int, id_: int, group_type: str) -> None:
        """Sets id and type of boundary group `group` (1-based position)."""
        check(_lib.load().fvm_mesh_set_group(self._h, int(group), int(id_), group_type.encode()))
        self._groups[group].id = int(id_)
        self._groups[group].groupType = group_type

    def getCellCells(self):
        """(row, col) of Mesh::getCellCells, all rows including ghosts."""
        row = np.zeros(self._nCells + self._nGhost + 1, np.int32)
        col = np.zeros(self._nnz, np.int32)
        check(_lib.load().fvm_mesh_connectivity(self._h, iptr(row), iptr(col), None))
        return row, col

    def getPairToColMapping(self) -> np.ndarray:
        p = np.zeros((self._nFaces, 2), np.int32)
        check(_lib.load().fvm_mesh_connectivity(self._h, None, None, iptr(p)))
        return p

    def getGeometry(self) -> dict:
        nF, nAll = self._nFaces, self._nCells + self._nGhost
        out = {
            "area": np.zeros((nF, 3)),
            "areaMag": np.zeros(nF),
            "faceCentroid": np.zeros((nF, 3)),
            "cellCentroid": np.zeros((nAll, 3)),
            "volume": np.zeros(nAll),
        }
        check(_lib.load().fvm_mesh_geometry(self._h, dptr(out["area"]), dptr(out["areaMag"]),
                                            dptr(out["faceCentroid"]), dptr(out["cellCentroid"]),
                                            dptr(out["volume"])))
        return out


class LinearSolver:
    """Common LinearSolver fields (fvmbase/LinearSolver.h:15-35)."""

    def __init__(self):
        d = _lib.default_linear_options()
        self.nMaxIterations = d.nMaxIterations
        self.verbosity = d.verbosity
        self.relativeTolerance = d.relativeTolerance
        self.absoluteTolerance = d.absoluteTolerance
        self._totalIterations = 0

    def getTotalIterations(self) -> int:
        return self._totalIterations


class AMG(LinearSolver):
    """Algebraic multigrid (fvmbase/AMG.h:27-110, defaults AMG.cpp:15-22)."""

    V_CYCLE, W_CYCLE, F_CYCLE = 0, 1, 2
    GAUSS_SEIDEL, JACOBI = 0, 1
    # additions of this implementation
    MULTICOLOR, SEQUENTIAL = 0, 1
    COARSE_SMOOTH, COARSE_DIRECT = 0, 1
    FP64, MIXED = 0, 1

    def __init__(self):
        super().__init__()
        d = _lib.default_linear_options()
        self.maxCoarseLevels = d.maxCoarseLevels
        self.nPreSweeps = d.nPreSweeps
        self.nPostSweeps = d.nPostSweeps
        self.coarseGroupSize = d.coarseGroupSize
        self.weightRatioThreshold = d.weightRatioThreshold
        self.cycleType = d.cycleType
        self.smootherType = d.smootherType
        self.scaleCorrections = bool(d.scaleCorrections)
        self.smootherOrdering = d.smootherOrdering
        self.coarsestSize = d.coarsestSize
        self.coarseSolver = d.coarseSolver
        self.precision = d.precision
        self.useGraphs = bool(d.useGraphs)
        self.coarseJacobiRows = d.coarseJacobiRows
        self.jacobiWeight = d.jacobiWeight
        # launch plans of the SELL-32 smoother kernels (speed only, never
        # the result): autotuned at setup, or one plan forced everywhere
        self.autotune = bool(d.autotune)
        self.planThreadsPerRow = d.planThreadsPerRow
        self.planBlock = d.planBlock
        self.planEllRows = d.planEllRows  # rows per thread of the ELL-32 Gauss-Seidel pass
        # finest-level Chebyshev smoother (0: multicolour Gauss-Seidel)
        self.chebyshevDegree = d.chebyshevDegree
        self.chebyshevFraction = d.chebyshevFraction
        self.gsReverse = bool(d.gsReverse)  # Gauss-Seidel sweep: forward + reverse (reference) or forward only
        self.patternOnDevice = bool(d.patternOnDevice)  # finest level of a GPU-built hierarchy packed on the GPU
        self.fuseProlongation = bool(d.fuseProlongation)  # prolongation folded into the first smoothing pass
        self.outerOnDevice = bool(d.outerOnDevice)  # a thermal advance() as one CUDA graph when it can be
        self.outerAcceleration = d.outerAcceleration  # Anderson depth of the outer iteration (0: off)
        self.setupOnDevice = bool(d.setupOnDevice)
        self.matchRounds = d.matchRounds
        self.matchBeta = d.matchBeta
        self.matchPasses = d.matchPasses
        self.coarsePostSweeps = d.coarsePostSweeps
        self._printFile = None

    def setMergeLevelSize(self, size: int) -> None:
        # the reference aborts here in serial builds (AMG.h:53-65)
        raise _lib.FvmError(7, "setMergeLevelSize needs the distributed (MPI) build")

    def redirectPrintToFile(self, fname: str) -> None:
        self._printFile = fname

    def redirectPrintToScreen(self) -> None:
        self._printFile = None

    def _fill(self, o: _lib.LinearOptions, solver_kind: int = 0, outer=None) -> None:
        src = outer if outer is not None else self
        o.solver = solver_kind
        o.nMaxIterations = int(src.nMaxIterations)
        o.relativeTolerance = float(src.relativeTolerance)
        o.absoluteTolerance = float(src.absoluteTolerance)
        o.verbosity = int(src.verbosity)
        o.maxCoarseLevels = int(self.maxCoarseLevels)
        o.nPreSweeps = int(self.nPreSweeps)
        o.nPostSweeps = int(self.nPostSweeps)
        o.coarseGroupSize = int(self.coarseGroupSize)
        o.weightRatioThreshold = float(self.weightRatioThreshold)
        o.cycleType = int(self.cycleType)
        o.smootherType = int(self.smootherType)
        o.scaleCorrections = int(bool(self.scaleCorrections))
        o.smootherOrdering = int(self.smootherOrdering)
        o.coarsestSize = int(self.coarsestSize)
        o.coarseSolver = int(self.coarseSolver)
        o.precision = int(self.precision)
        o.useGraphs = int(bool(self.useGraphs))
        o.coarseJacobiRows = int(self.coarseJacobiRows)
        o.jacobiWeight = float(self.jacobiWeight)
        o.autotune = int(bool(self.autotune))
        o.planThreadsPerRow = int(self.planThreadsPerRow)
        o.planBlock = int(self.planBlock)
        o.planEllRows = int(self.planEllRows)
        o.chebyshevDegree = int(self.chebyshevDegree)
        o.chebyshevFraction = float(self.chebyshevFraction)
        o.gsReverse = int(bool(self.gsReverse))
        o.patternOnDevice = int(bool(self.patternOnDevice))
        o.fuseProlongation = int(bool(self.fuseProlongation))
        o.outerOnDevice = int(bool(self.outerOnDevice))
        o.outerAcceleration = int(self.outerAcceleration)
        o.setupOnDevice = int(bool(self.setupOnDevice))
        o.matchRounds = int(self.matchRounds)
        o.matchBeta = float(self.matchBeta)
        o.matchPasses = int(self.matchPasses)
        o.coarsePostSweeps = int(self.coarsePostSweeps)

    def options(self) -> _lib.LinearOptions:
        o = _lib.LinearOptions()
        self._fill(o)
        return o

    def solve_csr(self, row, col, diag, off, b):
        """Solves b + A x = 0 from x = 0 for a matrix with implicit diagonal
        (the reference's MMReader + AMG::solve path). Returns (x, info)."""
        return _solve_csr(self.options(), row, col, diag, off, b, self)

    def hierarchy_csr(self, row, col, diag, off, finestLocalSize: int = 0):
        """Host-only AMG setup: (sizes, [coarseIndex per fine level], colors per level)."""
        return hierarchy_csr(self.options(), row, col, diag, off, finestLocalSize)


class JacobiSolver(LinearSolver):
    """Point Jacobi (fvmbase/JacobiSolver.cpp:27-100): as a solver one
    sweep per iteration; as the preconditioner of CG / BCGStab two sweeps
    from zero (JacobiSolver::smooth)."""

    def _fill(self, o: _lib.LinearOptions, solver_kind: int = 0, outer=None) -> None:
        src = outer if outer is not None else self
        d = _lib.default_linear_options()
        ctypes.memmove(ctypes.byref(o), ctypes.byref(d), ctypes.sizeof(o))
        o.solver = 3 if solver_kind == 0 else solver_kind
        o.preconditioner = 1
        o.maxCoarseLevels = 0
        o.nMaxIterations = int(src.nMaxIterations)
        o.relativeTolerance = float(src.relativeTolerance)
        o.absoluteTolerance = float(src.absoluteTolerance)
        o.verbosity = int(src.verbosity)

    def options(self) -> _lib.LinearOptions:
        o = _lib.LinearOptions()
        self._fill(o)
        return o

    def solve_csr(self, row, col, diag, off, b):
        """Solves b + A x = 0 from x = 0 with Jacobi sweeps."""
        return _solve_csr(self.options(), row, col, diag, off, b, self)


class _KrylovSolver(LinearSolver):
    _kind = 0

    def __init__(self):
        super().__init__()
        self.preconditioner = None

    def options(self) -> _lib.LinearOptions:
        pre = self.preconditioner if self.preconditioner is not None else AMG()
        o = _lib.LinearOptions()
        pre._fill(o, self._kind, outer=self)
        return o

    def smooth(self, ls) -> None:
        raise _lib.FvmError(1, "cannot use %s as preconditioner" % type(self).__name__)

    def solve_csr(self, row, col, diag, off, b):
        return _solve_csr(self.options(), row, col, diag, off, b, self)


class CG(_KrylovSolver):
    """Preconditioned CG in delta form (fvmbase/CG.cpp:26-139)."""

    _kind = 1


class BCGStab(_KrylovSolver):
    """Preconditioned BiCGStab in delta form (fvmbase/BCGStab.cpp:27-170)."""

    _kind = 2


def _solve_csr(opts, row, col, diag, off, b, solver):
    lib = _lib.load()
    row, col = as_i32(row), as_i32(col)
    diag, off, b = as_f64(diag), as_f64(off), as_f64(b)
    n = len(diag)
    x = np.zeros(n)
    rep = _lib.Report()
    cap = max(1, opts.nMaxIterations + 2)
    hist = np.zeros(cap)
    nh = ctypes.c_int(0)
    sizes = np.zeros(64, np.int32)
    nl = ctypes.c_int(0)
    check(lib.fvm_amg_solve_csr(n, iptr(row), iptr(col), dptr(diag), dptr(off), dptr(b), dptr(x),
                                ctypes.byref(opts), ctypes.byref(rep), dptr(hist), cap, ctypes.byref(nh),
                                iptr(sizes), 64, ctypes.byref(nl)))
    solver._totalIterations += rep.iterations
    info = {
        "history": hist[: nh.value].copy(),
        "levelSizes": sizes[: nl.value].copy(),
        "iterations": rep.iterations,
        "converged": bool(rep.converged),
        "seconds": rep.seconds,
        "launches": rep.launches,
    }
    pf = getattr(solver, "_printFile", None)
    if pf:
        with open(pf, "a") as f:
            for i, v in enumerate(info["history"]):
                f.write("%d: %g\n" % (i, v))
    return x, info


def csr_residual(row, col, diag, off, x, b):
    """(r, |r|_1) with r = b + A x for a matrix with implicit diagonal
    (CRMatrix::computeResidual + getOneNorm), computed on the GPU."""
    lib = _lib.load()
    row, col = as_i32(row), as_i32(col)
    diag, off, x, b = as_f64(diag), as_f64(off), as_f64(x), as_f64(b)
    n = len(diag)
    r = np.zeros(n)
    nrm = np.zeros(1)
    check(lib.fvm_csr_residual(n, iptr(row), iptr(col), dptr(diag), dptr(off), dptr(x), dptr(b), dptr(r),
                               dptr(nrm)))
    return r, float(nrm[0])


def hierarchy_csr(opts, row, col, diag, off, finestLocalSize: int = 0):
    lib = _lib.load()
    row, col = as_i32(row), as_i32(col)
    diag, off = as_f64(diag), as_f64(off)
    n = len(diag)
    sizes = np.zeros(64, np.int32)
    nl = ctypes.c_int(0)
    ci = np.zeros(2 * n + 64, np.int32)
    colors = np.zeros(2 * n + 64, np.int32)
    check(lib.fvm_amg_hierarchy_csr(n, iptr(row), iptr(col), dptr(diag), dptr(off), ctypes.byref(opts),
                                    int(finestLocalSize), ctypes.byref(nl), iptr(sizes), 64, iptr(ci), len(ci),
                                    iptr(colors), len(colors)))
    L = nl.value
    s = [n] + list(sizes[:L])
    cis, cols, p, q = [], [], 0, 0
    for lvl in range(L):
        cis.append(ci[p: p + s[lvl]].copy())
        p += s[lvl]
    for lvl in range(L + 1):
        cols.append(colors[q: q + s[lvl]].copy())
        q += s[lvl]
    return list(sizes[:L]), cis, cols
