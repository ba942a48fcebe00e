"""Batches of independent meshes solved as one model (no reference
counterpart: the reference solves each mesh with its own ThermalModel).

The meshes are packed block-diagonally into their disjoint union: cells of
mesh 0, mesh 1, ... (an offset table), interior faces of every mesh, then
boundary group 1 of every mesh, group 2 of every mesh, ... so each boundary
condition stays one face group. On a block-diagonal matrix the greedy
aggregation visits each mesh's rows in their own order and couples no two
meshes, so every mesh gets exactly the AMG levels it would get alone, while
each smoother pass, restriction and prolongation is one launch over all
meshes and each iteration is one CUDA graph. Convergence is tested per mesh
(ThermalModelA.setSegments): the outer loop runs until every mesh meets
the tolerance on its own L1 residual norm.
"""
from __future__ import annotations

import numpy as np

from . import fvmbaseExt, models


def union_mesh(meshes: list[dict]) -> tuple[dict, np.ndarray]:
    """Disjoint union of 7-argument meshes with equal dimension and number
    of face groups; returns (mesh, cell offsets of each input mesh)."""
    dims = {int(m["dim"]) for m in meshes}
    groups = {len(m["faceGroupSize"]) for m in meshes}
    if len(dims) != 1 or len(groups) != 1:
        raise ValueError("union_mesh: meshes need the same dimension and number of face groups")
    G = groups.pop()
    nc = np.array([int(m["nCells"]) for m in meshes], np.int64)
    cell_off = np.concatenate([[0], np.cumsum(nc)])
    n_total = int(cell_off[-1])
    nn = np.array([len(np.asarray(m["nodes"]).reshape(-1, 3)) for m in meshes], np.int64)
    node_off = np.concatenate([[0], np.cumsum(nn)])
    face_start = [np.concatenate([[0], np.cumsum(np.asarray(m["faceGroupSize"], np.int64))]) for m in meshes]
    fn_off = [np.concatenate([[0], np.cumsum(np.asarray(m["faceNodeCount"], np.int64))]) for m in meshes]
    fc_parts, fn_parts, fnc_parts, gsize = [], [], [], []
    ghost = n_total
    for g in range(G):
        size = 0
        for k, m in enumerate(meshes):
            a, b = int(face_start[k][g]), int(face_start[k][g + 1])
            fc = np.asarray(m["faceCells"], np.int64).reshape(-1, 2)[a:b].copy()
            fc[:, 0] += cell_off[k]
            if g == 0:
                fc[:, 1] += cell_off[k]
            else:
                fc[:, 1] = ghost + np.arange(b - a)
                ghost += b - a
            fc_parts.append(fc)
            fn = np.asarray(m["faceNodes"], np.int64)[fn_off[k][a]: fn_off[k][b]] + node_off[k]
            fn_parts.append(fn)
            fnc_parts.append(np.asarray(m["faceNodeCount"], np.int64)[a:b])
            size += b - a
        gsize.append(size)
    out = {
        "dim": dims.pop(),
        "nCells": n_total,
        "nodes": np.concatenate([np.asarray(m["nodes"], np.float64).reshape(-1, 3) for m in meshes]),
        "faceCells": np.concatenate(fc_parts).astype(np.int32),
        "faceNodes": np.concatenate(fn_parts).astype(np.int32),
        "faceNodeCount": np.concatenate(fnc_parts).astype(np.int32),
        "faceGroupSize": np.array(gsize, np.int32),
    }
    return out, cell_off.astype(np.int32)


class BatchedThermal:
    """Steady heat conduction on a batch of meshes with common boundary
    conditions (bcs: {group id: ('T', value) | ('q', value)}), one model."""

    def __init__(self, meshes: list[dict], bcs: dict, linear_solver, relative_tolerance: float = 1e-10):
        self.mesh_dict, self.offsets = union_mesh(meshes)
        self.mesh = fvmbaseExt.Mesh.from_dict(self.mesh_dict)
        self.fields = models.ThermalFields("therm")
        self.model = models.ThermalModelA(models.GeomFields("geom"), self.fields, [self.mesh])
        for gid, (kind, val) in bcs.items():
            bc = self.model.getBCMap()[gid]
            bc.bcType = "SpecifiedTemperature" if kind == "T" else "SpecifiedHeatFlux"
            bc.setVar("specifiedTemperature" if kind == "T" else "specifiedHeatFlux", val)
        o = self.model.getOptions()
        o.linearSolver = linear_solver
        o.relativeTolerance = relative_tolerance
        self.model.setSegments(self.offsets)

    def solve(self, k: list[np.ndarray], s: list[np.ndarray], max_outer: int = 500):
        """Solves every mesh to the tolerance; returns (temperatures per mesh, report)."""
        cells = self.mesh.getCells()
        self.model.init()
        self.fields.conductivity[cells] = np.concatenate(k)
        self.fields.source[cells] = np.concatenate(s)
        rep = self.model.advance(max_outer)
        T = self.fields.temperature[cells]
        return [T[self.offsets[i]: self.offsets[i + 1]] for i in range(len(self.offsets) - 1)], rep

    def status(self):
        return self.model.getSegmentStatus()
