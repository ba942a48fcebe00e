"""Shared helpers for the parity tests (run the GPU path and the reference
oracle on identical inputs)."""
from __future__ import annotations

import os

import numpy as np

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def load_fixture(name: str) -> dict:
    z = np.load(os.path.join(GOLDEN, name), allow_pickle=False)
    d = {k: z[k] for k in z.files}
    for k in ("dim", "nCells"):
        if k in d:
            d[k] = int(d[k])
    if "groupType" in d:
        d["groupType"] = [str(t) for t in d["groupType"]]
    return d


def gpu_model(mesh: dict, bcs: dict, solver=None, fields=None, opts=None, group_ids=None, group_types=None):
    """ThermalModelA on the GPU path. bcs: {groupId: ('T', value) | ('q', value)}."""
    from fvm_b200 import fvmbaseExt, models

    m = fvmbaseExt.Mesh.from_dict(mesh)
    if group_ids is not None:
        for g in range(1, len(group_ids)):
            m.setFaceGroup(g, int(group_ids[g]), group_types[g])
    geom = models.GeomFields("geom")
    models.MeshMetricsCalculatorA(geom, [m]).init()
    tf = models.ThermalFields("therm")
    tm = models.ThermalModelA(geom, tf, [m])
    for gid, (kind, val) in bcs.items():
        bc = tm.getBCMap()[gid]
        if kind == "T":
            bc.bcType = "SpecifiedTemperature"
            bc.setVar("specifiedTemperature", val)
        else:
            bc.bcType = "SpecifiedHeatFlux"
            bc.setVar("specifiedHeatFlux", val)
    o = tm.getOptions()
    if solver is not None:
        o.linearSolver = solver
    for k, v in (opts or {}).items():
        if k in ("initialTemperature", "timeStep"):
            o[k] = v
        else:
            setattr(o, k, v)
    tm.init()
    for name, vals in (fields or {}).items():
        getattr(tf, name)[m.getCells()] = vals
    return tm, tf, m


def ref_model(refo, mesh: dict, bcs: dict, fields=None, group_ids=None, group_types=None, **opts):
    r = refo.RefThermal(mesh, group_ids=group_ids, group_types=group_types)
    r.set_options(**opts)
    for gid, (kind, val) in bcs.items():
        if kind == "T":
            r.set_bc(gid, 0, [val])
        else:
            r.set_bc(gid, 1, [None, val])
    r.init()
    ids = {"temperature": 0, "conductivity": 1, "source": 2, "specificHeat": 3, "temperatureN1": 4}
    n = mesh["nCells"]
    nb = int(np.asarray(mesh["faceGroupSize"])[1:].sum())
    for name, vals in (fields or {}).items():
        vals = np.asarray(vals, dtype=np.float64)
        if len(vals) == n:
            from fvm_b200.meshgen import extend_to_ghosts

            vals = extend_to_ghosts(mesh, vals)
        assert len(vals) == n + nb
        r.set_field(ids[name], vals)
    return r


def rel_l2(a, b) -> float:
    a = np.asarray(a)
    b = np.asarray(b)
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))
