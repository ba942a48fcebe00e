"""The mixed-precision path's AMG hierarchy built on the GPU
(AMG.setupOnDevice): parallel pairwise matching, Galerkin products and
SELL-32 packing as kernels.

Bars:
  * aggregation: every fine row in exactly one aggregate, every coarse row
    non-empty, every level smaller than the one above it; aggregates of at
    most 16 rows for one matching per level, 64 for pairs of pairs (rows
    left unpaired join a pair, so a few aggregates grow past 2 or 4);
  * Galerkin: each coarse matrix equals P^T A P of the level above it
    (piecewise-constant P from the aggregation), computed here in numpy from
    the exported levels, to 1e-12 relative (the device sums in another
    order);
  * determinism: two builds of the same system give the same hierarchy
    and bitwise the same converged field;
  * the converged temperature field within 1e-8 relative L2 of the
    reference's FP64 solve.
"""
import numpy as np
import pytest

from fvm_b200 import fvmbaseExt, meshgen
from helpers import gpu_model, ref_model, rel_l2

pytestmark = pytest.mark.gpu


def _mesh(kind):
    if kind == "quad":
        return meshgen.config0(n=48, seed=0)
    if kind == "tet":
        return meshgen.config1(m=14, seed=1)
    return meshgen.config3(n=16, seed=3)


def _amg(device=True, coarsest=100, passes=1):
    a = fvmbaseExt.AMG()
    a.matchPasses = passes
    a.precision = fvmbaseExt.AMG.MIXED
    a.coarseSolver = fvmbaseExt.AMG.COARSE_DIRECT
    a.coarsestSize = coarsest
    a.coarseJacobiRows = 1 << 30
    a.nPreSweeps, a.nPostSweeps = 0, 2
    a.setupOnDevice = device
    return a


def _cg(amg, rel=1e-10):
    cg = fvmbaseExt.CG()
    cg.preconditioner = amg
    cg.relativeTolerance = rel
    cg.nMaxIterations = 500
    return cg


def _model(kind, solver):
    mesh, f = _mesh(kind)
    bcs = {gid: v for gid, v in f["bc"].items()}
    fields = {"conductivity": f["k"], "source": f["s"]}
    tm, tf, m = gpu_model(mesh, bcs, solver=solver, fields=fields, opts={"relativeTolerance": 1e-10})
    return mesh, f, bcs, fields, tm, tf, m


def _galerkin(A, ci, nc):
    """P^T A P as a dict {(I, J): value} plus the coarse diagonal."""
    n = len(A["diag"])
    cd = np.zeros(nc)
    np.add.at(cd, ci, A["diag"])
    rows = np.repeat(np.arange(n), np.diff(A["row"]))
    I, J = ci[rows], ci[A["col"]]
    same = I == J
    np.add.at(cd, I[same], A["val"][same])
    off = {}
    for a, b, v in zip(I[~same], J[~same], A["val"][~same]):
        off[(a, b)] = off.get((a, b), 0.0) + v
    return cd, off


def _as_dict(A):
    n = len(A["diag"])
    rows = np.repeat(np.arange(n), np.diff(A["row"]))
    return {(int(a), int(b)): float(v) for a, b, v in zip(rows, A["col"], A["val"])}


@pytest.mark.parametrize("mode", ["device", "device-pairs-of-pairs", "host"])
@pytest.mark.parametrize("kind", ["quad", "tet", "hex"])
def test_hierarchy_partition_and_galerkin(kind, mode):
    amg = _amg(mode != "host", passes=2 if mode == "device-pairs-of-pairs" else 1)
    _, _, _, _, tm, _, _ = _model(kind, _cg(amg))
    sizes, cis = tm.getHierarchy()
    assert len(sizes) >= 2
    A = tm.getLevelMatrix(0)
    for lvl, ci in enumerate(cis):
        n = len(ci)
        nc = sizes[lvl]
        assert nc < n
        assert ci.min() >= 0 and ci.max() < nc
        counts = np.bincount(ci, minlength=nc)
        assert counts.min() >= 1
        assert counts.max() <= (64 if mode == "device-pairs-of-pairs" else 16)
        Ac = tm.getLevelMatrix(lvl + 1)
        cd, off = _galerkin(A, ci, nc)
        scale = np.abs(cd).max()
        np.testing.assert_allclose(Ac["diag"], cd, rtol=1e-12, atol=1e-12 * scale)
        got = _as_dict(Ac)
        want = {k: v for k, v in off.items() if v != 0.0}
        assert set(got) == set(want), "coarse pattern of level %d" % (lvl + 1)
        g = np.array([got[k] for k in want])
        w = np.array([want[k] for k in want])
        np.testing.assert_allclose(g, w, rtol=1e-12, atol=1e-12 * scale)
        A = Ac


def test_device_hierarchy_is_deterministic():
    solver = _cg(_amg())
    _, f, _, _, tm, tf, m = _model("tet", solver)
    s1, c1 = tm.getHierarchy()
    tm.advance(200)
    T1 = tf.temperature[m.getCells()].copy()
    tm.init()
    tf.conductivity[m.getCells()] = f["k"]
    tf.source[m.getCells()] = f["s"]
    s2, c2 = tm.getHierarchy()
    tm.advance(200)
    T2 = tf.temperature[m.getCells()].copy()
    assert s1 == s2
    for a, b in zip(c1, c2):
        np.testing.assert_array_equal(a, b)
    np.testing.assert_array_equal(T1, T2)


@pytest.mark.parametrize("kind", ["quad", "tet", "hex"])
@pytest.mark.parametrize("variant", ["cg", "amg", "cg-large-coarsest", "cg-pairs-of-pairs"])
def test_device_hierarchy_converged_field_matches_reference(refo, kind, variant):
    amg = _amg(coarsest=4096 if variant == "cg-large-coarsest" else 100,
               passes=2 if variant == "cg-pairs-of-pairs" else 1)
    if variant == "cg-pairs-of-pairs":
        amg.coarsePostSweeps = 1
    amg.relativeTolerance = 1e-10
    amg.nMaxIterations = 500
    solver = amg if variant == "amg" else _cg(amg)
    mesh, f, bcs, fields, tm, tf, m = _model(kind, solver)
    tm.advance(300)
    assert tm.lastReport().converged
    T = tf.temperature[m.getCells()][: mesh["nCells"]]
    r = ref_model(refo, mesh, bcs, fields=fields, n_pre=1, n_post=1, lin_rel=1e-10, max_iter=500, rel=1e-10)
    norms, _ = r.advance(200)
    assert norms[-1] / norms[0] < 1e-10
    assert rel_l2(T, r.get_field(0)[: mesh["nCells"]]) <= 1e-8


@pytest.mark.parametrize("kind", ["quad", "tet", "hex"])
def test_device_pattern_matches_host(kind):
    """A new mesh's finest level coloured and packed on the GPU (row-order
    greedy colouring by fixed-point sweeps, ELL-32 packing) and on the host:
    the same colouring, permutation and slots, so the same hierarchy and
    bitwise the same converged field (meshes of 36-42k cells, ELL-32)."""
    if kind == "quad":
        mesh, f = meshgen.config0(n=192, seed=0)
    elif kind == "tet":
        mesh, f = meshgen.config1(m=20, seed=1)
    else:
        mesh, f = meshgen.config3(n=33, seed=3)
    assert mesh["nCells"] >= 32768
    bcs = {gid: v for gid, v in f["bc"].items()}
    fields = {"conductivity": f["k"], "source": f["s"]}
    out = []
    for on_device in (True, False):
        amg = _amg(passes=2)
        amg.coarsePostSweeps = 1
        amg.patternOnDevice = on_device
        tm, tf, m = gpu_model(mesh, bcs, solver=_cg(amg), fields=fields, opts={"relativeTolerance": 1e-10})
        tm.advance(300)
        rep = tm.lastReport()
        assert rep.converged
        sizes, _ = tm.getHierarchy()
        out.append((tf.temperature[m.getCells()][: mesh["nCells"]].copy(), rep.iterations, rep.linearIterations,
                    list(sizes), tm.getLaunchPlans()[0]))
    (T0, o0, c0, s0, p0), (T1, o1, c1, s1, p1) = out
    assert p0[0] < 0 and p1[0] < 0  # ELL-32 finest level both ways
    assert s0 == s1 and (o0, c0) == (o1, c1)
    np.testing.assert_array_equal(T0, T1)


@pytest.mark.parametrize("kind", ["tet", "hex"])
def test_fused_prolongation_is_bitwise_neutral(kind):
    """The zero-guess cycle folds each prolongation into the level's first
    post-smoothing pass (the finest level's first forward Gauss-Seidel
    sweep, the coarse levels' first damped-Jacobi pass): the same
    iterations and bitwise the same field as separate prolongations
    (finest level ELL-32: 36-42k cells)."""
    if kind == "tet":
        mesh, f = meshgen.config1(m=20, seed=1)
    else:
        mesh, f = meshgen.config3(n=33, seed=3)
    bcs = {gid: v for gid, v in f["bc"].items()}
    fields = {"conductivity": f["k"], "source": f["s"]}
    out = []
    for fuse in (True, False):
        amg = _amg(passes=2)
        amg.coarsePostSweeps = 1
        amg.fuseProlongation = fuse
        tm, tf, m = gpu_model(mesh, bcs, solver=_cg(amg), fields=fields, opts={"relativeTolerance": 1e-10})
        tm.advance(300)
        rep = tm.lastReport()
        assert rep.converged
        out.append((tf.temperature[m.getCells()][: mesh["nCells"]].copy(), rep.iterations, rep.linearIterations))
    (T0, o0, c0), (T1, o1, c1) = out
    assert (o0, c0) == (o1, c1)
    np.testing.assert_array_equal(T0, T1)
