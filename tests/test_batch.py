"""Batched solve of independent meshes (disjoint union, per-mesh
convergence). CPU: the union mesh is block-diagonal, its geometry and its
first AMG aggregation equal each mesh's own (C restatement of the
reference). GPU: every mesh of the batch converges to its own reference
FP64 solution (1e-8 relative L2) and meets the outer tolerance on its own
norm."""
import numpy as np
import pytest

from fvm_b200 import batch, meshgen
from helpers import ref_model, rel_l2


def _batch(n=5, lo=5, hi=14, seed=2):
    return meshgen.config2(n_meshes=n, seed=seed, lo=lo, hi=hi)


def test_union_mesh_layout():
    ms = _batch()
    u, off = batch.union_mesh([m for m, _ in ms])
    assert u["nCells"] == sum(m["nCells"] for m, _ in ms)
    np.testing.assert_array_equal(off, np.concatenate([[0], np.cumsum([m["nCells"] for m, _ in ms])]))
    G = len(ms[0][0]["faceGroupSize"])
    for g in range(G):
        assert u["faceGroupSize"][g] == sum(int(m["faceGroupSize"][g]) for m, _ in ms)
    # ghosts numbered after all self cells, in boundary-face order
    nb = int(u["faceGroupSize"][0])
    np.testing.assert_array_equal(u["faceCells"][nb:, 1], u["nCells"] + np.arange(len(u["faceCells"]) - nb))


def test_union_geometry_and_aggregation_match_each_mesh():
    from oracle import oracle_c as oc

    ms = _batch()
    u, off = batch.union_mesh([m for m, _ in ms])
    ou = oc.OracleThermal(u)
    gu = ou.geometry()
    row, col, _ = ou.connectivity()
    n = u["nCells"]
    seg = np.searchsorted(off, np.arange(n), side="right") - 1
    rid = np.repeat(np.arange(len(row) - 1), np.diff(row))
    inside = (rid < n) & (col < n)
    assert not np.any(seg[rid[inside]] != seg[col[inside]])
    # same linear system per block -> same first-level aggregation
    k = [f["k"] for _, f in ms]
    s = [f["s"] for _, f in ms]
    ou.set_bc(1, 0, [300.0])
    ou.set_bc(2, 0, [400.0])
    ou.init()
    from fvm_b200.meshgen import extend_to_ghosts

    ou.set_field(1, extend_to_ghosts(u, np.concatenate(k)))
    ou.set_field(2, extend_to_ghosts(u, np.concatenate(s)))
    _, cis = ou.hierarchy(max_levels=1)
    base = 0
    for i, (m, f) in enumerate(ms):
        om = oc.OracleThermal(m)
        g = om.geometry()
        a, b = off[i], off[i + 1]
        np.testing.assert_array_equal(gu["cellCentroid"][a:b], g["cellCentroid"][: m["nCells"]])
        np.testing.assert_array_equal(gu["volume"][a:b], g["volume"][: m["nCells"]])
        om.set_bc(1, 0, [300.0])
        om.set_bc(2, 0, [400.0])
        om.init()
        om.set_field(1, extend_to_ghosts(m, f["k"]))
        om.set_field(2, extend_to_ghosts(m, f["s"]))
        _, ci = om.hierarchy(max_levels=1)
        mine = cis[0][a:b]
        # coarse numbering continues across blocks
        np.testing.assert_array_equal(mine, ci[0] + base)
        base += int(ci[0].max()) + 1


@pytest.mark.gpu
@pytest.mark.parametrize("variant", ["plain", "mixed"])
def test_batched_solve_matches_reference_per_mesh(refo, variant):
    from fvm_b200 import fvmbaseExt

    ms = _batch(n=7, lo=6, hi=24, seed=5)
    amg = fvmbaseExt.AMG()
    amg.nPreSweeps = 1
    amg.nPostSweeps = 1
    amg.relativeTolerance = 0.1
    amg.nMaxIterations = 200
    if variant == "mixed":
        amg.precision = fvmbaseExt.AMG.MIXED
        amg.coarseSolver = fvmbaseExt.AMG.COARSE_DIRECT
        amg.coarsestSize = 100
        amg.coarseJacobiRows = 1 << 30
    bt = batch.BatchedThermal([m for m, _ in ms], ms[0][1]["bc"], amg, relative_tolerance=1e-10)
    Ts, rep = bt.solve([f["k"] for _, f in ms], [f["s"] for _, f in ms])
    assert rep.converged
    first, last, at = bt.status()
    assert np.all(at >= 0)
    assert np.all(last / first < 1e-10)
    for (m, f), T in zip(ms, Ts):
        r = ref_model(refo, m, f["bc"], fields={"conductivity": f["k"], "source": f["s"]}, n_pre=1, n_post=1,
                      lin_rel=1e-10, max_iter=500, rel=1e-10)
        r.advance(300)
        assert rel_l2(T, r.get_field(0)[: m["nCells"]]) <= 1e-8


@pytest.mark.gpu
def test_parallel_block_aggregation_equals_sequential():
    """With blocks set, each mesh's aggregation runs on its own thread; the
    hierarchy (every level's coarseIndex) equals the sequential walk's."""
    from fvm_b200 import fvmbaseExt

    ms = _batch(n=9, lo=6, hi=30, seed=7)
    hier = []
    for blocks in (True, False):
        amg = fvmbaseExt.AMG()
        bt = batch.BatchedThermal([m for m, _ in ms], ms[0][1]["bc"], amg)
        if not blocks:
            bt.model.setSegments(None)
        cells = bt.mesh.getCells()
        bt.model.init()
        bt.fields.conductivity[cells] = np.concatenate([f["k"] for _, f in ms])
        bt.fields.source[cells] = np.concatenate([f["s"] for _, f in ms])
        hier.append(bt.model.getHierarchy())
    (s1, c1), (s2, c2) = hier
    assert s1 == s2
    for a, b in zip(c1, c2):
        np.testing.assert_array_equal(a, b)
