"""ctypes wrapper of oracle/_ref/libfvmoracle.so: the plain-C restatement of
the reference's thermal linearization + AMG path (oracle/fvm_oracle.c).

TEST INFRASTRUCTURE ONLY -- imported by tests/, by __graft_entry__.smoke()
and by the CPU-baseline leg of bench.py, as the checker. The product
(fvm_b200) never imports it.

The class and function signatures follow oracle/ref.py (the reference
compiled from its own sources), so a test can run the same case through
both and through the GPU product.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_ref", "libfvmoracle.so")
P = ctypes.c_void_p

_lib = None


def available() -> bool:
    return os.path.exists(LIB_PATH)


def load():
    global _lib
    if _lib is None:
        if not available():
            raise FileNotFoundError(LIB_PATH + " (build with: make -C oracle)")
        lib = ctypes.CDLL(LIB_PATH)
        lib.orc_last_error.restype = ctypes.c_char_p
        lib.orc_mesh_create.restype = ctypes.c_void_p
        lib.orc_mesh_create.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, P, ctypes.c_int, P, P, P,
                                        ctypes.c_int, P]
        lib.orc_mesh_destroy.argtypes = [ctypes.c_void_p]
        lib.orc_mesh_set_group.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_char_p]
        lib.orc_mesh_sizes.argtypes = [ctypes.c_void_p, P]
        lib.orc_mesh_connectivity.argtypes = [ctypes.c_void_p, P, P, P]
        lib.orc_mesh_geometry.argtypes = [ctypes.c_void_p, P, P, P, P, P]
        lib.orc_amg_csr.argtypes = [ctypes.c_int, P, P, P, P, P, P, P, P, P, P, P, P, P, ctypes.c_int]
        lib.orc_multicolor.argtypes = [ctypes.c_int, P, P, P]
        lib.orc_thermal_create.restype = ctypes.c_void_p
        lib.orc_thermal_create.argtypes = [ctypes.c_void_p]
        for name in ("orc_thermal_destroy", "orc_thermal_init", "orc_thermal_update_time"):
            getattr(lib, name).argtypes = [ctypes.c_void_p]
        lib.orc_thermal_set_bc.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, P]
        lib.orc_thermal_set_options.argtypes = [ctypes.c_void_p, P, P]
        lib.orc_thermal_set_cell_field.argtypes = [ctypes.c_void_p, ctypes.c_int, P]
        lib.orc_thermal_get_cell_field.argtypes = [ctypes.c_void_p, ctypes.c_int, P]
        lib.orc_thermal_linearize.argtypes = [ctypes.c_void_p, P, P, P, P]
        lib.orc_thermal_advance.argtypes = [ctypes.c_void_p, ctypes.c_int, P, P, P]
        lib.orc_thermal_hierarchy.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_double, ctypes.c_int, P, P, P]
        _lib = lib
    return _lib


def _p(a):
    return a.ctypes.data_as(P) if a is not None else None


def _check(rc):
    if rc != 0:
        raise RuntimeError("oracle: " + load().orc_last_error().decode())


def amg_csr(row, col, diag, off, b, max_iter=41, rel_tol=1e-30, abs_tol=0.0, max_levels=30, n_pre=0, n_post=1,
            group=2, cycle=0, smoother=0, thr=0.65):
    """AMG::solve on an n x n CSR system (no ghosts). Returns (x, coarse
    level sizes, L1 history, coarseIndex per fine level), as ref.amg_csr."""
    lib = load()
    n = len(diag)
    opts = np.array([max_levels, n_pre, n_post, group, cycle, smoother, max_iter], np.int32)
    dopts = np.array([thr, rel_tol, abs_tol])
    x = np.zeros(n)
    nl = ctypes.c_int()
    sizes = np.zeros(64, np.int32)
    hist = np.zeros(max_iter + 2)
    nh = ctypes.c_int()
    cap = 4 * n + 64
    ci = np.zeros(cap, np.int32)
    row, col = np.ascontiguousarray(row, np.int32), np.ascontiguousarray(col, np.int32)
    diag, off, b = (np.ascontiguousarray(a, np.float64) for a in (diag, off, b))
    _check(lib.orc_amg_csr(n, _p(row), _p(col), _p(diag), _p(off), _p(b), _p(opts), _p(dopts), _p(x),
                           ctypes.byref(nl), _p(sizes), _p(hist), ctypes.byref(nh), _p(ci), cap))
    L = nl.value
    s = [n] + list(sizes[:L])
    cis, p = [], 0
    for lvl in range(L):
        cis.append(ci[p: p + s[lvl]].copy())
        p += s[lvl]
    return x, list(sizes[:L]), hist[: nh.value].copy(), cis


def multicolor(row, col) -> tuple[int, np.ndarray]:
    """Colouring of the GPU multicolour smoothers, restated from its
    definition (n-row symmetric pattern, columns < n)."""
    row, col = np.ascontiguousarray(row, np.int32), np.ascontiguousarray(col, np.int32)
    n = len(row) - 1
    color = np.zeros(n, np.int32)
    nc = load().orc_multicolor(n, _p(row), _p(col), _p(color))
    return int(nc), color


class Mesh:
    """Sites, cellCells, pair->col and metrics of a 7-argument mesh."""

    def __init__(self, mesh: dict, group_ids=None, group_types=None):
        lib = load()
        nodes = np.ascontiguousarray(mesh["nodes"], np.float64).reshape(-1)
        fc = np.ascontiguousarray(mesh["faceCells"], np.int32).reshape(-1)
        fn = np.ascontiguousarray(mesh["faceNodes"], np.int32)
        fnc = np.ascontiguousarray(mesh["faceNodeCount"], np.int32)
        gs = np.ascontiguousarray(mesh["faceGroupSize"], np.int32)
        self.nf = len(fnc)
        self.h = lib.orc_mesh_create(int(mesh["dim"]), int(mesh["nCells"]), len(nodes) // 3, _p(nodes), self.nf,
                                     _p(fc), _p(fn), _p(fnc), len(gs), _p(gs))
        s = np.zeros(3, np.int32)
        lib.orc_mesh_sizes(self.h, _p(s))
        self.n, self.nb, self.nnz = (int(v) for v in s)
        if group_ids is not None:
            for g in range(1, len(gs)):
                _check(lib.orc_mesh_set_group(self.h, g, int(group_ids[g]), str(group_types[g]).encode()))

    def __del__(self):
        if getattr(self, "h", None):
            load().orc_mesh_destroy(self.h)
            self.h = None

    def connectivity(self):
        row = np.zeros(self.n + self.nb + 1, np.int32)
        col = np.zeros(self.nnz, np.int32)
        p2c = np.zeros(2 * self.nf, np.int32)
        load().orc_mesh_connectivity(self.h, _p(row), _p(col), _p(p2c))
        return row, col, p2c.reshape(-1, 2)

    def geometry(self):
        na = self.n + self.nb
        fa, fam, fcn = np.zeros(3 * self.nf), np.zeros(self.nf), np.zeros(3 * self.nf)
        ccn, vol = np.zeros(3 * na), np.zeros(na)
        load().orc_mesh_geometry(self.h, _p(fa), _p(fam), _p(fcn), _p(ccn), _p(vol))
        return {"area": fa.reshape(-1, 3), "areaMag": fam, "faceCentroid": fcn.reshape(-1, 3),
                "cellCentroid": ccn.reshape(-1, 3), "volume": vol}


class OracleThermal:
    """ThermalModel<double> restated in C; methods as ref.RefThermal."""

    def __init__(self, mesh: dict, group_ids=None, group_types=None):
        self.mesh = Mesh(mesh, group_ids, group_types)
        self.n, self.nb = self.mesh.n, self.mesh.nb
        self.h = load().orc_thermal_create(self.mesh.h)

    def __del__(self):
        if getattr(self, "h", None):
            load().orc_thermal_destroy(self.h)
            self.h = None

    def set_bc(self, group_id: int, bc_type: int, values):
        v = np.array([300.0, 0.0, 0.0, 300.0, 1.0])
        for i, x in enumerate(values):
            if x is not None:
                v[i] = x
        _check(load().orc_thermal_set_bc(self.h, int(group_id), int(bc_type), _p(v)))

    def set_options(self, solver=0, max_levels=30, n_pre=0, n_post=1, group=2, cycle=0, smoother=0, max_iter=20,
                    transient=False, verbosity=0, rel=1e-8, abs_=1e-16, lin_rel=1e-1, lin_abs=1e-16, thr=0.65,
                    t0=300.0, dt=1e-7, k=1.0, rho=1.0, cp=1.0):
        io = np.array([solver, max_levels, n_pre, n_post, group, cycle, smoother, max_iter, int(transient),
                       verbosity], np.int32)
        do = np.array([rel, abs_, lin_rel, lin_abs, thr, t0, dt, k, rho, cp])
        _check(load().orc_thermal_set_options(self.h, _p(io), _p(do)))

    def init(self):
        _check(load().orc_thermal_init(self.h))

    def set_field(self, field: int, values):
        v = np.ascontiguousarray(values, np.float64)
        assert len(v) == self.n + self.nb
        _check(load().orc_thermal_set_cell_field(self.h, int(field), _p(v)))

    def get_field(self, field: int) -> np.ndarray:
        out = np.zeros(self.n + self.nb)
        _check(load().orc_thermal_get_cell_field(self.h, int(field), _p(out)))
        return out

    def sizes(self):
        return self.n, self.nb, self.mesh.nnz

    def connectivity(self):
        return self.mesh.connectivity()

    def geometry(self):
        return self.mesh.geometry()

    def linearize(self):
        na = self.n + self.nb
        d, o, b = np.zeros(na), np.zeros(self.mesh.nnz), np.zeros(na)
        isb = np.zeros(na, np.int32)
        _check(load().orc_thermal_linearize(self.h, _p(d), _p(o), _p(b), _p(isb)))
        return d, o, b, isb

    def hierarchy(self, group=2, thr=0.65, max_levels=30):
        nl = ctypes.c_int()
        sizes = np.zeros(64, np.int32)
        ci = np.zeros(2 * self.n + 64, np.int32)
        _check(load().orc_thermal_hierarchy(self.h, group, thr, max_levels, ctypes.byref(nl), _p(sizes), _p(ci)))
        L = nl.value
        s = [self.n] + list(sizes[:L])
        cis, p = [], 0
        for lvl in range(L):
            cis.append(ci[p: p + s[lvl]].copy())
            p += s[lvl]
        return list(sizes[:L]), cis

    def advance(self, niter: int):
        """Returns (initial L1 norm of every outer iteration, V-cycles run)."""
        norms = np.zeros(niter)
        nd = ctypes.c_int()
        cyc = ctypes.c_int()
        _check(load().orc_thermal_advance(self.h, int(niter), _p(norms), ctypes.byref(nd), ctypes.byref(cyc)))
        return norms[: nd.value].copy(), cyc.value

    def update_time(self):
        _check(load().orc_thermal_update_time(self.h))
