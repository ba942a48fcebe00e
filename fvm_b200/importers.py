"""Mirror of the reference's importers module for Fluent case files:

    reader = importers.FluentReader("mesh.cas")
    reader.readMesh()
    meshes = reader.getMeshList()

(src/modules/importers/FluentReader.cpp: readMesh :572-611, getMeshList
:954-1040, createMesh :696-952; SWIG interface importers.i). The file is
parsed by the library's C++ reader (fvm_fluent_* in include/fvm_b200.h);
each cell zone becomes a fvmbaseExt.Mesh built through the 7-argument
constructor, with its boundary groups' Fluent zone ids and types.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib
from ._lib import check, dptr, iptr
from .fvmbaseExt import Mesh


class FluentReader:
    def __init__(self, fileName: str):
        self._path = str(fileName)
        self._h = None

    def readMesh(self) -> None:
        lib = _lib.load()
        h = ctypes.c_void_p()
        check(lib.fvm_fluent_read(self._path.encode(), ctypes.byref(h)))
        self._h = h

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            try:
                _lib.load().fvm_fluent_destroy(h)
            except Exception:
                pass
            self._h = None

    def _need(self):
        if self._h is None:
            raise RuntimeError("FluentReader.readMesh() must be called first")

    def getNumCellZones(self) -> int:
        self._need()
        n = ctypes.c_int(0)
        check(_lib.load().fvm_fluent_cell_zones(self._h, ctypes.byref(n)))
        return n.value

    def getMeshArrays(self, zone: int = 0) -> dict:
        """The 7-argument constructor's arrays of cell zone `zone`, plus the
        boundary groups' Fluent zone ids and types (the dict the mesh
        generators return)."""
        self._need()
        lib = _lib.load()
        sz = np.zeros(6, np.int32)
        check(lib.fvm_fluent_mesh_sizes(self._h, int(zone), iptr(sz)))
        dim, n_cells, n_nodes, n_faces, n_fn, n_groups = map(int, sz)
        xyz = np.zeros((n_nodes, 3))
        fc = np.zeros((n_faces, 2), np.int32)
        fn = np.zeros(max(n_fn, 1), np.int32)
        cnt = np.zeros(max(n_faces, 1), np.int32)
        gs = np.zeros(n_groups, np.int32)
        gid = np.zeros(n_groups, np.int32)
        check(lib.fvm_fluent_mesh_arrays(self._h, int(zone), dptr(xyz), iptr(fc), iptr(fn), iptr(cnt), iptr(gs),
                                         iptr(gid)))
        types = []
        buf = ctypes.create_string_buffer(256)
        for g in range(n_groups):
            check(lib.fvm_fluent_group_type(self._h, int(zone), g, buf, len(buf)))
            types.append(buf.value.decode())
        return {"dim": dim, "nCells": n_cells, "nodes": xyz, "faceCells": fc, "faceNodes": fn[:n_fn],
                "faceNodeCount": cnt[:n_faces], "faceGroupSize": gs, "groupId": gid, "groupType": types}

    def getMeshList(self) -> list:
        meshes = []
        for z in range(self.getNumCellZones()):
            d = self.getMeshArrays(z)
            m = Mesh.from_dict(d)
            for g in range(1, len(d["faceGroupSize"])):
                m.setFaceGroup(g, int(d["groupId"][g]), d["groupType"][g])
            meshes.append(m)
        return meshes
