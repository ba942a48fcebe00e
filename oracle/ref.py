"""ctypes wrapper of oracle/_ref/libfvmref.so: the reference FVM solver
compiled from its own sources by oracle/Makefile.

TEST INFRASTRUCTURE ONLY -- imported by tests/, by __graft_entry__.smoke()
and by the CPU-baseline leg of bench.py, as the checker / baseline. The
product (fvm_b200) never imports it.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_ref", "libfvmref.so")
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
        lib.ref_last_error.restype = ctypes.c_char_p
        lib.ref_thermal_create.restype = ctypes.c_void_p
        lib.ref_thermal_create.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, P, ctypes.c_int, P, P, P,
                                           ctypes.c_int, P, P, P]
        for name in ("ref_thermal_destroy", "ref_thermal_init", "ref_thermal_update_time"):
            getattr(lib, name).argtypes = [ctypes.c_void_p]
        lib.ref_thermal_set_bc.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, P]
        lib.ref_thermal_set_options.argtypes = [ctypes.c_void_p, P, P]
        lib.ref_thermal_set_cell_field.argtypes = [ctypes.c_void_p, ctypes.c_int, P]
        lib.ref_thermal_get_cell_field.argtypes = [ctypes.c_void_p, ctypes.c_int, P]
        lib.ref_thermal_sizes.argtypes = [ctypes.c_void_p, P]
        lib.ref_thermal_connectivity.argtypes = [ctypes.c_void_p, P, P, P]
        lib.ref_thermal_geometry.argtypes = [ctypes.c_void_p, P, P, P, P, P]
        lib.ref_thermal_linearize.argtypes = [ctypes.c_void_p, P, P, P, P]
        lib.ref_thermal_hierarchy.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_double, ctypes.c_int, P, P,
                                              P, P, P, P, P, P]
        lib.ref_thermal_advance.argtypes = [ctypes.c_void_p, ctypes.c_int, P, P, P]
        lib.ref_thermal_heat_flux_integral.argtypes = [ctypes.c_void_p, ctypes.c_int, P]
        lib.ref_mm_read.argtypes = [ctypes.c_char_p, ctypes.c_char_p, P, P, P, P, P, P, P]
        lib.ref_amg_csr.argtypes = [ctypes.c_int, P, P, P, P, P, P, P, P, P, P, P, P, P, ctypes.c_int]
        lib.ref_fluent_read.argtypes = [ctypes.c_char_p, P, P, P, P, P, P, P, P]
        _lib = lib
    return _lib


def _p(a):
    return a.ctypes.data_as(P) if a is not None else None


def _check(rc):
    if rc != 0:
        raise RuntimeError("reference: " + load().ref_last_error().decode())


def mm_read(mat_path: str, rhs_path: str):
    """MMReader::getLS: (row, col, diag, off, b) in the reference's layout."""
    lib = load()
    n = ctypes.c_int()
    z = ctypes.c_int()
    _check(lib.ref_mm_read(mat_path.encode(), rhs_path.encode(), ctypes.byref(n), ctypes.byref(z), None, None,
                           None, None, None))
    row = np.zeros(n.value + 1, np.int32)
    col = np.zeros(z.value, np.int32)
    d = np.zeros(n.value)
    o = np.zeros(z.value)
    b = np.zeros(n.value)
    _check(lib.ref_mm_read(mat_path.encode(), rhs_path.encode(), ctypes.byref(n), ctypes.byref(z), _p(row), _p(col),
                           _p(d), _p(o), _p(b)))
    return row, col, d, o, b


def amg_csr(row, col, diag, off, b, max_iter=41, rel_tol=1e-30, abs_tol=0.0, max_levels=30, n_pre=0, n_post=1,
            group=2, cycle=0, smoother=0, thr=0.65):
    """Reference AMG::solve on a CSR system, cycle by cycle. Returns
    (x, level sizes, L1 history, coarseIndex arrays per fine level)."""
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
    _check(lib.ref_amg_csr(n, _p(row), _p(col), _p(diag), _p(off), _p(b), _p(opts), _p(dopts), _p(x),
                           ctypes.byref(nl), _p(sizes), _p(hist), ctypes.byref(nh), _p(ci), cap))
    L = nl.value
    s = [n] + list(sizes[:L])
    cis, p = [], 0
    for lvl in range(L):
        cis.append(ci[p: p + s[lvl]].copy())
        p += s[lvl]
    return x, list(sizes[:L]), hist[: nh.value].copy(), cis


def fluent_read(path: str) -> dict:
    """FluentReader: the first cell zone as 7-argument Mesh arrays plus group ids/types."""
    lib = load()
    sizes = np.zeros(6, np.int32)
    _check(lib.ref_fluent_read(path.encode(), _p(sizes), None, None, None, None, None, None, None))
    dim, nc, nn, nf, nfn, ng = map(int, sizes)
    xyz = np.zeros(3 * nn)
    fc = np.zeros(2 * nf, np.int32)
    fn = np.zeros(nfn, np.int32)
    fnc = np.zeros(nf, np.int32)
    gs = np.zeros(ng, np.int32)
    gid = np.zeros(ng, np.int32)
    gt = ctypes.create_string_buffer(32 * ng)
    _check(lib.ref_fluent_read(path.encode(), _p(sizes), _p(xyz), _p(fc), _p(fn), _p(fnc), _p(gs), _p(gid),
                               ctypes.cast(gt, P)))
    types = [gt.raw[32 * g: 32 * g + 32].split(b"\0")[0].decode() for g in range(ng)]
    return {"dim": dim, "nCells": nc, "nodes": xyz.reshape(-1, 3), "faceCells": fc.reshape(-1, 2),
            "faceNodes": fn, "faceNodeCount": fnc, "faceGroupSize": gs, "groupId": gid, "groupType": types}


class RefThermal:
    """ThermalModel<double> of the reference on the same mesh arrays."""

    def __init__(self, mesh: dict, group_ids=None, group_types=None):
        lib = load()
        self._keep = []

        def keep(a):
            self._keep.append(a)
            return _p(a)

        nodes = np.ascontiguousarray(mesh["nodes"], np.float64).reshape(-1)
        fc = np.ascontiguousarray(mesh["faceCells"], np.int32).reshape(-1)
        fn = np.ascontiguousarray(mesh["faceNodes"], np.int32)
        fnc = np.ascontiguousarray(mesh["faceNodeCount"], np.int32)
        gs = np.ascontiguousarray(mesh["faceGroupSize"], np.int32)
        gid = np.ascontiguousarray(group_ids, np.int32) if group_ids is not None else None
        gt = None
        if group_types is not None:
            buf = b"".join(t.encode().ljust(32, b"\0")[:32] for t in group_types)
            gt = ctypes.create_string_buffer(buf, len(buf))
            self._keep.append(gt)
        self.n = int(mesh["nCells"])
        self.nb = int(gs[1:].sum())
        self.h = lib.ref_thermal_create(int(mesh["dim"]), self.n, len(nodes) // 3, keep(nodes), len(fnc), keep(fc),
                                        keep(fn), keep(fnc), len(gs), keep(gs),
                                        keep(gid) if gid is not None else None,
                                        ctypes.cast(gt, P) if gt is not None else None)
        if not self.h:
            _check(1)

    def __del__(self):
        if getattr(self, "h", None):
            load().ref_thermal_destroy(self.h)
            self.h = None

    def set_bc(self, group_id: int, bc_type: int, values):
        v = np.zeros(5)
        v[:] = [300.0, 0.0, 0.0, 300.0, 1.0]
        for i, x in enumerate(values):
            if x is not None:
                v[i] = x
        _check(load().ref_thermal_set_bc(self.h, int(group_id), int(bc_type), _p(v)))

    def set_options(self, solver=0, max_levels=30, n_pre=0, n_post=1, group=2, cycle=0, smoother=0, max_iter=20,
                    transient=False, verbosity=0, rel=1e-8, abs_=1e-16, lin_rel=1e-1, lin_abs=1e-16, thr=0.65,
                    t0=300.0, dt=1e-7, k=1.0, rho=1.0, cp=1.0):
        io = np.array([solver, max_levels, n_pre, n_post, group, cycle, smoother, max_iter, int(transient),
                       verbosity], np.int32)
        do = np.array([rel, abs_, lin_rel, lin_abs, thr, t0, dt, k, rho, cp])
        _check(load().ref_thermal_set_options(self.h, _p(io), _p(do)))

    def init(self):
        _check(load().ref_thermal_init(self.h))

    def set_field(self, field: int, values):
        v = np.ascontiguousarray(values, np.float64)
        assert len(v) == self.n + self.nb
        _check(load().ref_thermal_set_cell_field(self.h, int(field), _p(v)))

    def get_field(self, field: int) -> np.ndarray:
        out = np.zeros(self.n + self.nb)
        _check(load().ref_thermal_get_cell_field(self.h, int(field), _p(out)))
        return out

    def sizes(self):
        s = np.zeros(3, np.int32)
        _check(load().ref_thermal_sizes(self.h, _p(s)))
        return tuple(int(x) for x in s)

    def connectivity(self, n_faces: int):
        n, g, z = self.sizes()
        row = np.zeros(n + g + 1, np.int32)
        col = np.zeros(z, np.int32)
        p2c = np.zeros(2 * n_faces, np.int32)
        _check(load().ref_thermal_connectivity(self.h, _p(row), _p(col), _p(p2c)))
        return row, col, p2c.reshape(-1, 2)

    def geometry(self, n_faces: int):
        n, g, _ = self.sizes()
        fa = np.zeros(3 * n_faces)
        fam = np.zeros(n_faces)
        fcn = np.zeros(3 * n_faces)
        ccn = np.zeros(3 * (n + g))
        vol = np.zeros(n + g)
        _check(load().ref_thermal_geometry(self.h, _p(fa), _p(fam), _p(fcn), _p(ccn), _p(vol)))
        return fa.reshape(-1, 3), fam, fcn.reshape(-1, 3), ccn.reshape(-1, 3), vol

    def linearize(self):
        """Matrix over all rows (self + ghost) in cellCells order, b, isBoundary."""
        n, g, z = self.sizes()
        d = np.zeros(n + g)
        o = np.zeros(z)
        b = np.zeros(n + g)
        ib = np.zeros(n + g, np.int32)
        _check(load().ref_thermal_linearize(self.h, _p(d), _p(o), _p(b), _p(ib)))
        return d, o, b, ib

    def hierarchy(self, group=2, thr=0.65, max_levels=30):
        n, g, z = self.sizes()
        nl = ctypes.c_int()
        sizes = np.zeros(64, np.int32)
        ci = np.zeros(2 * n + 64, np.int32)
        cnnz = np.zeros(64, np.int32)
        _check(load().ref_thermal_hierarchy(self.h, int(group), float(thr), int(max_levels), ctypes.byref(nl),
                                            _p(sizes), _p(ci), _p(cnnz), None, None, None, None))
        L = nl.value
        s = [n] + list(sizes[:L])
        out, p = [], 0
        for lvl in range(L):
            out.append(ci[p: p + s[lvl]].copy())
            p += s[lvl]
        return list(sizes[:L]), out

    def advance(self, niter: int):
        norms = np.zeros(max(niter, 1))
        nd = ctypes.c_int()
        sec = ctypes.c_double()
        _check(load().ref_thermal_advance(self.h, int(niter), _p(norms), ctypes.byref(nd), ctypes.byref(sec)))
        return norms[: nd.value].copy(), sec.value

    def update_time(self):
        _check(load().ref_thermal_update_time(self.h))

    def heat_flux_integral(self, group_id: int) -> float:
        out = ctypes.c_double()
        _check(load().ref_thermal_heat_flux_integral(self.h, int(group_id), ctypes.byref(out)))
        return out.value
