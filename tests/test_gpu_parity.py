"""GPU parity: the CUDA path against the reference oracle on identical
inputs, through the C ABI (Python mirror of the reference API).

Bars (stated per test):
  * integer setup (aggregation) and the FP64 matrix: bit-exact;
  * reference-ordered smoothers (sequential Gauss-Seidel, Jacobi): residual
    histories equal to the reference's to 1e-12 relative (only the L1
    reduction order differs);
  * converged temperature fields: relative L2 error <= 1e-8 against the
    reference's FP64 CPU solve, for every smoother / precision / solver.
"""
import numpy as np
import pytest

from fvm_b200 import fvmbaseExt, meshgen
from helpers import gpu_model, load_fixture, ref_model, rel_l2

pytestmark = pytest.mark.gpu

TOL_FIELD = 1e-8  # relative L2 against the reference FP64 solve


def _amg(**kw):
    a = fvmbaseExt.AMG()
    for k, v in kw.items():
        setattr(a, k, v)
    return a


# ---------------------------------------------------------------------------
# raw AMG on the reference's MatrixMarket known-answer system


def test_mm226_sequential_gs_matches_reference_history():
    z = load_fixture("mm226.npz")
    a = _amg(nMaxIterations=41, relativeTolerance=1e-30, absoluteTolerance=0.0,
             smootherOrdering=fvmbaseExt.AMG.SEQUENTIAL, useGraphs=True)
    x, info = a.solve_csr(z["row"], z["col"], z["diag"], z["off"], z["b"])
    assert list(info["levelSizes"]) == [108, 48, 20, 8]
    h = info["history"]
    assert len(h) == 41
    np.testing.assert_allclose(h, z["ref_hist"], rtol=1e-12, atol=0)
    np.testing.assert_allclose(x, z["ref_x"], rtol=1e-12, atol=1e-12 * np.abs(z["ref_x"]).max())


def test_mm226_jacobi_matches_reference_history(refo):
    z = load_fixture("mm226.npz")
    _, _, rh, _ = refo.amg_csr(z["row"], z["col"], z["diag"], z["off"], z["b"], max_iter=30, rel_tol=1e-30,
                               smoother=1)
    a = _amg(nMaxIterations=30, relativeTolerance=1e-30, absoluteTolerance=0.0, smootherType=fvmbaseExt.AMG.JACOBI)
    _, info = a.solve_csr(z["row"], z["col"], z["diag"], z["off"], z["b"])
    np.testing.assert_allclose(info["history"], rh, rtol=1e-12, atol=0)


@pytest.mark.parametrize("cycle", ["W", "F"])
def test_mm226_w_and_f_cycles_match_reference_history(refo, cycle):
    """W and F cycles (AMG::cycle, fvmbase/AMG.cpp:105-110) with the
    reference-ordered Gauss-Seidel: residual history equal to the reference's
    own W / F cycle history to 1e-12 relative."""
    z = load_fixture("mm226.npz")
    ct = {"W": fvmbaseExt.AMG.W_CYCLE, "F": fvmbaseExt.AMG.F_CYCLE}[cycle]
    _, _, rh, _ = refo.amg_csr(z["row"], z["col"], z["diag"], z["off"], z["b"], max_iter=25, rel_tol=1e-30,
                               n_pre=1, n_post=1, cycle=ct)
    a = _amg(nMaxIterations=25, relativeTolerance=1e-30, absoluteTolerance=0.0, nPreSweeps=1, nPostSweeps=1,
             cycleType=ct, smootherOrdering=fvmbaseExt.AMG.SEQUENTIAL)
    _, info = a.solve_csr(z["row"], z["col"], z["diag"], z["off"], z["b"])
    assert len(info["history"]) == len(rh)
    np.testing.assert_allclose(info["history"], rh, rtol=1e-12, atol=0)


@pytest.mark.parametrize("cycle", ["W", "F"])
@pytest.mark.parametrize("precision", [0, 1])
def test_w_and_f_cycles_converge_to_reference_field(refo, cycle, precision):
    """Multicolour W / F cycles (FP64, and FP32 under FP64 refinement) inside
    the thermal outer loop: converged field within 1e-8 of the reference's
    own W / F cycle solve on the jittered tets."""
    mesh, f = _synthetic("tet")
    bcs = {gid: v for gid, v in f["bc"].items()}
    fields = {"conductivity": f["k"], "source": f["s"]}
    ct = {"W": fvmbaseExt.AMG.W_CYCLE, "F": fvmbaseExt.AMG.F_CYCLE}[cycle]
    amg = _amg(nPreSweeps=1, nPostSweeps=1, relativeTolerance=1e-10, nMaxIterations=500, cycleType=ct,
               precision=precision)
    tm, tf, m = gpu_model(mesh, bcs, solver=amg, fields=fields, opts={"relativeTolerance": 1e-10})
    _converge(tm)
    T = tf.temperature[m.getCells()][: mesh["nCells"]]
    r = ref_model(refo, mesh, bcs, fields=fields, n_pre=1, n_post=1, lin_rel=1e-10, max_iter=500, rel=1e-10,
                  cycle=ct)
    norms, _ = r.advance(200)
    assert norms[-1] / norms[0] < 1e-10
    assert rel_l2(T, r.get_field(0)[: mesh["nCells"]]) <= TOL_FIELD


def test_nan_conductivity_returns_nan_status():
    """A NaN conductivity (a host-made failure) reaches the residual norm of
    the first linear system: advance() raises the NaN status (FVM_ERR_NAN),
    with no GPU fault, and the model stays usable with good data."""
    mesh, f = _synthetic("quad")
    bcs = {gid: v for gid, v in f["bc"].items()}
    k = np.array(f["k"], dtype=np.float64)
    k[len(k) // 2] = np.nan
    amg = _amg(nPreSweeps=1, nPostSweeps=1, relativeTolerance=1e-10, nMaxIterations=100)
    tm, tf, m = gpu_model(mesh, bcs, solver=amg, fields={"conductivity": k, "source": f["s"]},
                          opts={"relativeTolerance": 1e-10})
    from fvm_b200._lib import FvmError

    with pytest.raises(FvmError) as err:
        tm.advance(20)
    assert err.value.status == 4  # FVM_ERR_NAN
    assert "finite" in str(err.value)
    tm.init()
    tf.conductivity[m.getCells()] = f["k"]
    tf.source[m.getCells()] = f["s"]
    _converge(tm)


@pytest.mark.parametrize("precision", [0, 1])
@pytest.mark.parametrize("solver", ["AMG", "CG", "BCGStab"])
def test_mm226_multicolor_converges_to_reference_solution(refo, solver, precision):
    z = load_fixture("mm226.npz")
    xr, _, _, _ = refo.amg_csr(z["row"], z["col"], z["diag"], z["off"], z["b"], max_iter=400, rel_tol=1e-13)
    pre = _amg(precision=precision, coarseSolver=fvmbaseExt.AMG.COARSE_DIRECT)
    if solver == "AMG":
        s = pre
    else:
        s = fvmbaseExt.CG() if solver == "CG" else fvmbaseExt.BCGStab()
        s.preconditioner = pre
    s.nMaxIterations = 400
    s.relativeTolerance = 1e-13
    s.absoluteTolerance = 0.0
    x, info = s.solve_csr(z["row"], z["col"], z["diag"], z["off"], z["b"])
    assert info["converged"]
    assert rel_l2(x, xr) <= 1e-10


# ---------------------------------------------------------------------------
# ThermalModel linearization and AMG setup on the reference's own meshes


def test_cav32_linear_system_bit_exact_and_golden(refo):
    m = load_fixture("cav32_matrix.npz")
    bcs = {3: ("T", 400.0), 4: ("T", 0.0), 5: ("T", 0.0), 6: ("T", 0.0)}
    tm, tf, mesh = gpu_model(m, bcs, solver=_amg(relativeTolerance=1e-9, nMaxIterations=2000, maxCoarseLevels=20),
                             group_ids=m["groupId"], group_types=m["groupType"])
    diag, off, b = tm.getLinearSystem()
    r = ref_model(refo, m, bcs, group_ids=m["groupId"], group_types=m["groupType"], lin_rel=1e-9, max_iter=2000,
                  max_levels=20)
    d_ref, o_ref, b_ref, _ = r.linearize()
    n = m["nCells"]
    row, col = mesh.getCellCells()
    o_ref_int = np.concatenate([o_ref[row[i]:row[i + 1]][col[row[i]:row[i + 1]] < n] for i in range(n)])
    np.testing.assert_array_equal(diag, d_ref[:n])
    np.testing.assert_array_equal(off, o_ref_int)
    np.testing.assert_array_equal(b, b_ref[:n])
    # and the THERMAL_MATRIX golden (printed with %lf: 1e-8 in its ptest.py)
    gold = {(int(i), int(j)): v for i, j, v in zip(m["gold_i"], m["gold_j"], m["gold_v"])}
    rows, cols = tm._interior_pattern()
    for i in range(n):
        assert abs(diag[i] - gold[(i, i)]) <= 1e-8
        for k in range(rows[i], rows[i + 1]):
            assert abs(off[k] - gold[(i, int(cols[k]))]) <= 1e-8
    assert np.abs(-b - m["gold_rhs"]).max() <= 1e-8


@pytest.mark.parametrize("ordering", ["sequential", "multicolor"])
@pytest.mark.parametrize("case", ["quad_1024", "tri_894", "hexa_10k", "tetra_8k"])
def test_parallel_thermal_golden_on_gpu(refo, case, ordering):
    """PARALLEL_TESTS np=1: advance(1) -> within 1e-5 of the golden
    temperatures; the AMG hierarchy (coarseIndex of every level) equals the
    reference's. The golden run stops the inner AMG at relTol 1e-9 with the
    reference's lexicographic Gauss-Seidel: the sequential ordering repeats
    exactly that; the multicolour smoother (different iterates) is run to
    relTol 1e-12 so that its remaining solver error is below the tolerance."""
    m = load_fixture("ptest_%s.npz" % case)
    bcs = {g: ("T", v) for g, v in ((3, 400.0), (4, 0.0), (5, 0.0), (6, 0.0)) if g in m["groupId"]}
    if ordering == "sequential":
        amg = _amg(relativeTolerance=1e-9, nMaxIterations=2000, maxCoarseLevels=20,
                   smootherOrdering=fvmbaseExt.AMG.SEQUENTIAL)
    else:
        amg = _amg(relativeTolerance=1e-12, nMaxIterations=4000, maxCoarseLevels=20)
    tm, tf, mesh = gpu_model(m, bcs, solver=amg, group_ids=m["groupId"], group_types=m["groupType"])
    sizes, cis = tm.getHierarchy()
    r = ref_model(refo, m, bcs, group_ids=m["groupId"], group_types=m["groupType"], lin_rel=1e-9, max_iter=2000,
                  max_levels=20)
    rsizes, rcis = r.hierarchy(max_levels=20)
    assert sizes == rsizes
    for a, b in zip(cis, rcis):
        np.testing.assert_array_equal(a, b)
    tm.advance(1)
    T = tf.temperature[mesh.getCells()][: m["nCells"]]
    assert np.abs(T - m["T_gold"]).max() <= 1e-5


# ---------------------------------------------------------------------------
# converged fields on jittered synthetic meshes (non-orthogonal correction)


def _synthetic(kind):
    if kind == "quad":
        mesh, f = meshgen.config0(n=24, seed=0)
    elif kind == "tet":
        mesh, f = meshgen.config1(m=7, seed=1)
    else:
        mesh, f = meshgen.config3(n=8, seed=3)
    return mesh, f


def _converge(tm, n_outer=200):
    tm.advance(n_outer)
    rep = tm.lastReport()
    assert rep.converged
    return rep


@pytest.mark.parametrize("kind", ["quad", "tet", "hex"])
@pytest.mark.parametrize("variant", ["fp64-gs", "fp64-sequential", "mixed-direct", "mixed-direct-gpu-inverse",
                                     "mixed-coarse-jacobi", "cg-mixed", "bcgstab", "jacobi", "fp64-chebyshev",
                                     "cg-mixed-chebyshev"])
def test_converged_field_matches_reference(refo, kind, variant):
    mesh, f = _synthetic(kind)
    bcs = {gid: v for gid, v in f["bc"].items()}
    fields = {"conductivity": f["k"], "source": f["s"]}
    amg = _amg(nPreSweeps=1, nPostSweeps=1, relativeTolerance=1e-10, nMaxIterations=500)
    solver = amg
    if variant == "fp64-sequential":
        amg.smootherOrdering = fvmbaseExt.AMG.SEQUENTIAL
    elif variant == "mixed-direct":
        amg.precision = fvmbaseExt.AMG.MIXED
        amg.coarseSolver = fvmbaseExt.AMG.COARSE_DIRECT
        amg.coarsestSize = 100
    elif variant == "mixed-direct-gpu-inverse":
        # first coarse level (> 128 rows) inverted by the blocked GPU Gauss-Jordan
        amg.precision = fvmbaseExt.AMG.MIXED
        amg.coarseSolver = fvmbaseExt.AMG.COARSE_DIRECT
        amg.coarsestSize = 4096
    elif variant == "mixed-coarse-jacobi":
        # damped Jacobi on every level below the finest
        amg.precision = fvmbaseExt.AMG.MIXED
        amg.coarseSolver = fvmbaseExt.AMG.COARSE_DIRECT
        amg.coarsestSize = 100
        amg.coarseJacobiRows = 1 << 30
    elif variant == "cg-mixed":
        amg.precision = fvmbaseExt.AMG.MIXED
        amg.coarseSolver = fvmbaseExt.AMG.COARSE_DIRECT
        amg.coarsestSize = 100
        solver = fvmbaseExt.CG()
        solver.preconditioner = amg
        solver.relativeTolerance = 1e-10
        solver.nMaxIterations = 500
    elif variant == "bcgstab":
        solver = fvmbaseExt.BCGStab()
        solver.preconditioner = amg
        solver.relativeTolerance = 1e-10
        solver.nMaxIterations = 500
    elif variant == "jacobi":
        amg.smootherType = fvmbaseExt.AMG.JACOBI
    elif variant == "fp64-chebyshev":
        # finest level: Chebyshev polynomial of degree 3 per sweep
        amg.chebyshevDegree = 3
    elif variant == "cg-mixed-chebyshev":
        amg.precision = fvmbaseExt.AMG.MIXED
        amg.coarseSolver = fvmbaseExt.AMG.COARSE_DIRECT
        amg.coarsestSize = 100
        amg.coarseJacobiRows = 1 << 30
        amg.chebyshevDegree = 2
        amg.nPreSweeps = 0
        amg.nPostSweeps = 2
        solver = fvmbaseExt.CG()
        solver.preconditioner = amg
        solver.relativeTolerance = 1e-10
        solver.nMaxIterations = 500
    tm, tf, m = gpu_model(mesh, bcs, solver=solver, fields=fields, opts={"relativeTolerance": 1e-10})
    _converge(tm)
    T = tf.temperature[m.getCells()][: mesh["nCells"]]
    r = ref_model(refo, mesh, bcs, fields=fields, n_pre=1, n_post=1, lin_rel=1e-10, max_iter=500, rel=1e-10)
    norms, _ = r.advance(200)
    assert norms[-1] / norms[0] < 1e-10
    Tr = r.get_field(0)[: mesh["nCells"]]
    assert rel_l2(T, Tr) <= TOL_FIELD


def test_gpu_inverse_narrow_panels_matches_reference(refo):
    """A coarsest level of more than 3200 rows takes the 4-column panels of
    the blocked GPU Gauss-Jordan inverse (shared-memory bound)."""
    mesh, f = meshgen.config0(n=90, seed=0)
    bcs = {gid: v for gid, v in f["bc"].items()}
    fields = {"conductivity": f["k"], "source": f["s"]}
    amg = _amg(nPreSweeps=1, nPostSweeps=1, relativeTolerance=1e-10, nMaxIterations=500, coarsestSize=4096)
    amg.precision = fvmbaseExt.AMG.MIXED
    amg.coarseSolver = fvmbaseExt.AMG.COARSE_DIRECT
    tm, tf, m = gpu_model(mesh, bcs, solver=amg, fields=fields, opts={"relativeTolerance": 1e-10})
    sizes, _ = tm.getHierarchy()
    assert 3200 < sizes[-1] <= 4096  # 3607 rows
    _converge(tm)
    T = tf.temperature[m.getCells()][: mesh["nCells"]]
    r = ref_model(refo, mesh, bcs, fields=fields, n_pre=1, n_post=1, lin_rel=1e-10, max_iter=500, rel=1e-10)
    r.advance(200)
    assert rel_l2(T, r.get_field(0)[: mesh["nCells"]]) <= TOL_FIELD


@pytest.mark.parametrize("smoother", ["sequential-gs", "jacobi"])
def test_linear_system_bit_exact_on_jittered_tets(refo, smoother):
    """Matrix and right-hand side of the first three outer iterations are
    bit-identical to the reference's. With the reference-ordered smoothers
    the iterates themselves are identical, so the non-zero lagged gradients
    of later linearizations are compared too."""
    mesh, f = meshgen.config1(m=7, seed=1)
    fields = {"conductivity": f["k"], "source": f["s"]}
    if smoother == "jacobi":
        amg = _amg(smootherType=fvmbaseExt.AMG.JACOBI, relativeTolerance=1e-1, nMaxIterations=20)
        sm = 1
    else:
        amg = _amg(smootherOrdering=fvmbaseExt.AMG.SEQUENTIAL, relativeTolerance=1e-1, nMaxIterations=20)
        sm = 0
    tm, tf, m = gpu_model(mesh, f["bc"], solver=amg, fields=fields)
    r = ref_model(refo, mesh, f["bc"], fields=fields, smoother=sm)
    n = mesh["nCells"]
    for it in range(3):  # later linearizations carry a non-zero gradient
        diag, off, b = tm.getLinearSystem()
        d_ref, o_ref, b_ref, _ = r.linearize()
        np.testing.assert_array_equal(diag, d_ref[:n], err_msg="diag, outer iteration %d" % it)
        np.testing.assert_array_equal(b, b_ref[:n], err_msg="b, outer iteration %d" % it)
        tm.advance(1)
        r.advance(1)
    T = tf.temperature[m.getCells()]
    np.testing.assert_array_equal(T[:n], r.get_field(0)[:n])


def test_transient_steps_match_reference(refo):
    mesh = meshgen.hex_mesh(6)
    n = mesh["nCells"]
    rng = np.random.default_rng(4)
    k = rng.lognormal(0, 1, n)
    rc = rng.uniform(0.5, 2.0, n)
    bcs = {2: ("T", 400.0)}
    fields = {"conductivity": k, "specificHeat": rc}
    amg = _amg(relativeTolerance=1e-10, nMaxIterations=300, nPreSweeps=1, nPostSweeps=1)
    tm, tf, m = gpu_model(mesh, bcs, solver=amg, fields=fields,
                          opts={"transient": True, "timeStep": 1e-3, "relativeTolerance": 1e-10})
    r = ref_model(refo, mesh, bcs, fields=fields, transient=True, dt=1e-3, rel=1e-10, lin_rel=1e-10, max_iter=300,
                  n_pre=1, n_post=1)
    for step in range(3):
        tm.advance(50)
        tm.updateTime()
        r.advance(50)
        r.update_time()
    T = tf.temperature[m.getCells()][:n]
    Tr = r.get_field(0)[:n]
    assert rel_l2(T, Tr) <= TOL_FIELD


def test_csr_residual_matches_reference_order():
    """fvm_csr_residual: r = b + D x + O x in the reference's summation order
    (bit-exact with a scalar restatement); L1 norm to 1e-13 (reduction order)."""
    z = load_fixture("mm226.npz")
    rng = np.random.default_rng(0)
    x = rng.standard_normal(len(z["diag"]))
    r, nrm = fvmbaseExt.csr_residual(z["row"], z["col"], z["diag"], z["off"], x, z["b"])
    row, col, d, o, b = z["row"], z["col"], z["diag"], z["off"], z["b"]
    expect = np.empty(len(d))
    for i in range(len(d)):
        s = float(b[i]) + float(d[i]) * float(x[i])
        for k in range(row[i], row[i + 1]):
            s = s + float(o[k]) * float(x[col[k]])
        expect[i] = s
    np.testing.assert_array_equal(r, expect)
    assert abs(nrm - np.abs(expect).sum()) <= 1e-13 * np.abs(expect).sum()


# ---------------------------------------------------------------------------
# JacobiSolver (fvmbase/JacobiSolver.cpp:27-100): standalone and as the
# preconditioner of CG / BCGStab


def test_jacobi_solver_outer_history_matches_reference(refo):
    """One undamped Jacobi sweep per iteration (bit-identical iterates);
    the outer norms equal the reference's up to the L1 summation order."""
    mesh, f = _synthetic("quad")
    bcs = {gid: v for gid, v in f["bc"].items()}
    fields = {"conductivity": f["k"], "source": f["s"]}
    js = fvmbaseExt.JacobiSolver()
    js.relativeTolerance = 1e-1
    js.nMaxIterations = 20
    tm, tf, m = gpu_model(mesh, bcs, solver=js, fields=fields)
    tm.advance(6)
    hist = tm.getNormHistory()
    r = ref_model(refo, mesh, bcs, fields=fields, solver=3, lin_rel=1e-1, max_iter=20)
    norms, _ = r.advance(6)
    assert len(hist) == len(norms) == 6
    np.testing.assert_allclose(hist, norms, rtol=1e-11, atol=0)
    T = tf.temperature[m.getCells()][: mesh["nCells"]]
    np.testing.assert_allclose(T, r.get_field(0)[: mesh["nCells"]], rtol=1e-12, atol=0)


@pytest.mark.parametrize("kind", ["cg", "bcgstab"])
def test_krylov_with_jacobi_preconditioner_converges_to_reference(refo, kind):
    mesh, f = _synthetic("quad")
    bcs = {gid: v for gid, v in f["bc"].items()}
    fields = {"conductivity": f["k"], "source": f["s"]}
    s = fvmbaseExt.CG() if kind == "cg" else fvmbaseExt.BCGStab()
    s.preconditioner = fvmbaseExt.JacobiSolver()
    s.relativeTolerance = 1e-10
    s.nMaxIterations = 2000
    tm, tf, m = gpu_model(mesh, bcs, solver=s, fields=fields, opts={"relativeTolerance": 1e-10})
    _converge(tm)
    T = tf.temperature[m.getCells()][: mesh["nCells"]]
    r = ref_model(refo, mesh, bcs, fields=fields, solver=4 if kind == "cg" else 5, lin_rel=1e-10, max_iter=2000,
                  rel=1e-10)
    r.advance(200)
    assert rel_l2(T, r.get_field(0)[: mesh["nCells"]]) <= TOL_FIELD


# ---------------------------------------------------------------------------
# every boundary-condition type of ThermalModel::linearize
# (fvmbase/ThermalModel_impl.h:296-398, GenericBCS.h:77-323) and
# getHeatFluxIntegral (ThermalModel_impl.h:400-422)

_ALL_BCS = {  # group -> (bcType, specifiedTemperature, specifiedHeatFlux, h, farFieldTemperature, emissivity)
    1: ("SpecifiedTemperature", 300.0, 0.0, 0.0, 300.0, 1.0),
    2: ("Convective", 0.0, 0.0, 25.0, 350.0, 1.0),
    3: ("Radiative", 0.0, 0.0, 0.0, 310.0, 0.7),
    4: ("Mixed", 0.0, 0.0, 8.0, 320.0, 0.5),
    5: ("SpecifiedHeatFlux", 0.0, 1.5, 0.0, 300.0, 1.0),
    6: ("Symmetry", 0.0, 0.0, 0.0, 300.0, 1.0),
}
_REF_BC = {"SpecifiedTemperature": 0, "SpecifiedHeatFlux": 1, "Symmetry": 2, "Convective": 3, "Radiative": 4,
           "Mixed": 5}


def _all_bc_models(refo, amg, ref_opts):
    from fvm_b200 import models

    mesh, f = meshgen.config1(m=6, seed=4)
    fields = {"conductivity": f["k"], "source": f["s"]}
    tm, tf, m = gpu_model(mesh, {}, solver=amg, fields=None)
    for gid, (t, T, q, h, Tinf, eps) in _ALL_BCS.items():
        bc = tm.getBCMap()[gid]
        bc.bcType = t
        for name, v in zip(models.BC_VARS, (T, q, h, Tinf, eps)):
            bc.setVar(name, v)
    tm.init()
    for name, vals in fields.items():
        getattr(tf, name)[m.getCells()] = vals
    r = ref_model(refo, mesh, {}, fields=None, **ref_opts)
    for gid, (t, T, q, h, Tinf, eps) in _ALL_BCS.items():
        r.set_bc(gid, _REF_BC[t], [T, q, h, Tinf, eps])
    r.init()
    from fvm_b200.meshgen import extend_to_ghosts

    r.set_field(1, extend_to_ghosts(mesh, f["k"]))
    r.set_field(2, extend_to_ghosts(mesh, f["s"]))
    return mesh, tm, tf, m, r


def test_all_boundary_conditions_bit_exact(refo):
    """Matrix, right-hand side, temperatures and boundary heat-flux
    integrals after each of three outer iterations equal the reference's
    bit for bit (reference-ordered Gauss-Seidel); the radiative and mixed
    conditions make the matrix depend on T, so it is rebuilt every
    iteration."""
    amg = _amg(smootherOrdering=fvmbaseExt.AMG.SEQUENTIAL, relativeTolerance=1e-1, nMaxIterations=20)
    mesh, tm, tf, m, r = _all_bc_models(refo, amg, {})
    n = mesh["nCells"]
    for it in range(3):
        diag, off, b = tm.getLinearSystem()
        d_ref, o_ref, b_ref, _ = r.linearize()
        np.testing.assert_array_equal(diag, d_ref[:n], err_msg="diag, outer iteration %d" % it)
        np.testing.assert_array_equal(b, b_ref[:n], err_msg="b, outer iteration %d" % it)
        tm.advance(1)
        r.advance(1)
        np.testing.assert_array_equal(tf.temperature[m.getCells()], r.get_field(0), err_msg="T, iteration %d" % it)
        for gid in _ALL_BCS:
            assert tm.getHeatFluxIntegral(m, gid) == r.heat_flux_integral(gid), (it, gid)


def test_all_boundary_conditions_converge_to_reference(refo):
    amg = _amg(nPreSweeps=1, nPostSweeps=1, relativeTolerance=1e-10, nMaxIterations=500)
    mesh, tm, tf, m, r = _all_bc_models(refo, amg, dict(n_pre=1, n_post=1, lin_rel=1e-10, max_iter=500,
                                                        rel=1e-10))
    tm.getOptions().relativeTolerance = 1e-10
    _converge(tm)
    r.advance(200)
    n = mesh["nCells"]
    T = tf.temperature[m.getCells()][:n]
    assert rel_l2(T, r.get_field(0)[:n]) <= TOL_FIELD
    for gid in _ALL_BCS:
        a, b = tm.getHeatFluxIntegral(m, gid), r.heat_flux_integral(gid)
        assert abs(a - b) <= 1e-8 * max(1.0, abs(b)), gid


@pytest.mark.parametrize("ordering", ["sequential", "multicolor"])
def test_ell_finest_level_matches_reference(refo, ordering):
    """73k tets: the finest level is stored ELL-32 (aligned 32-row groups of
    width 4). Sequential GS: temperatures after two outer iterations equal
    the reference's bit for bit; multicolour: the converged field."""
    mesh, f = meshgen.config1(m=24, seed=2)
    assert mesh["nCells"] >= 32768
    bcs = {gid: v for gid, v in f["bc"].items()}
    fields = {"conductivity": f["k"], "source": f["s"]}
    n = mesh["nCells"]
    if ordering == "sequential":
        amg = _amg(smootherOrdering=fvmbaseExt.AMG.SEQUENTIAL, relativeTolerance=1e-1, nMaxIterations=20)
        tm, tf, m = gpu_model(mesh, bcs, solver=amg, fields=fields)
        r = ref_model(refo, mesh, bcs, fields=fields)
        for it in range(2):
            tm.advance(1)
            r.advance(1)
            np.testing.assert_array_equal(tf.temperature[m.getCells()][:n], r.get_field(0)[:n])
    else:
        amg = _amg(nPreSweeps=1, nPostSweeps=1, relativeTolerance=1e-10, nMaxIterations=500)
        tm, tf, m = gpu_model(mesh, bcs, solver=amg, fields=fields, opts={"relativeTolerance": 1e-10})
        _converge(tm)
        r = ref_model(refo, mesh, bcs, fields=fields, n_pre=1, n_post=1, lin_rel=1e-10, max_iter=500, rel=1e-10)
        r.advance(200)
        assert rel_l2(tf.temperature[m.getCells()][:n], r.get_field(0)[:n]) <= TOL_FIELD


@pytest.mark.gpu
@pytest.mark.parametrize("n", [1000, 3000, 3700, 4096])
def test_gpu_inverse_direct_single_level(n):
    """With no coarse levels and the direct coarse solver, the whole matrix is
    the coarsest level: it is densified on the GPU and inverted by the
    blocked Gauss-Jordan (panels of 8, 8, 7 and 7 columns for these sizes),
    so one cycle is an exact solve. The matrix is not diagonally
    dominant (random-sign couplings on a grid pattern), so row pivoting is
    exercised; the solution is compared with numpy's dense solve."""
    rng = np.random.default_rng(n)
    nx = int(np.ceil(np.sqrt(n)))
    rows = [[] for _ in range(n)]
    for i in range(n):
        for j in (i + 1, i + nx):
            if j < n and (j != i + 1 or (i + 1) % nx):
                v = rng.uniform(-1.0, 1.0)
                rows[i].append((j, v))
                rows[j].append((i, rng.uniform(-1.0, 1.0)))
    row = np.zeros(n + 1, np.int32)
    row[1:] = np.cumsum([len(r) for r in rows])
    col = np.array([j for r in rows for j, _ in r], np.int32)
    off = np.array([v for r in rows for _, v in r])
    diag = -rng.uniform(0.2, 1.0, n)
    b = rng.normal(size=n)
    A = np.diag(diag)
    for i in range(n):
        for k in range(row[i], row[i + 1]):
            A[i, col[k]] += off[k]
    xref = np.linalg.solve(A, -b)  # b + A x = 0
    # condition numbers 3e4-2e5: one exact solve leaves a relative L1
    # residual of 1e-12..1e-11 (measured 3e-12) and a solution error of 4e-13
    amg = _amg(maxCoarseLevels=0, relativeTolerance=1e-10, nMaxIterations=5)
    amg.coarseSolver = fvmbaseExt.AMG.COARSE_DIRECT
    amg.coarsestSize = 4096
    x, info = amg.solve_csr(row, col, diag, off, b)
    assert list(info["levelSizes"]) == []
    assert info["iterations"] == 1
    assert rel_l2(x, xref) <= 1e-11


@pytest.mark.gpu
@pytest.mark.parametrize("symmetric", [False, True], ids=["unsymmetric", "symmetric"])
@pytest.mark.parametrize("n", [1000, 2294, 3000, 4096])
def test_gpu_inverse_dominant_single_level(n, symmetric):
    """A diagonally dominant single level (the shape of every diffusion
    coarsest level) takes the unpivoted blocked Gauss-Jordan: panels of 32
    pivots, the last one partial for all sizes here but 4096; a symmetric
    one the symmetric sweep over the tiles on and above the diagonal. One
    cycle is an exact solve; the solution is compared with numpy's dense
    solve."""
    rng = np.random.default_rng(7 * n)
    nx = int(np.ceil(np.sqrt(n)))
    rows = [[] for _ in range(n)]
    for i in range(n):
        for j in (i + 1, i + nx, i + 3 * nx + 5):
            if j < n and (j != i + 1 or (i + 1) % nx):
                v = rng.uniform(-1.0, 1.0)
                rows[i].append((j, v))
                rows[j].append((i, v if symmetric else rng.uniform(-1.0, 1.0)))
    row = np.zeros(n + 1, np.int32)
    row[1:] = np.cumsum([len(r) for r in rows])
    col = np.array([j for r in rows for j, _ in r], np.int32)
    off = np.array([v for r in rows for _, v in r])
    # weakly dominant rows with a few strict ones, signs of both kinds
    absum = np.array([sum(abs(v) for _, v in r) for r in rows])
    diag = -(absum + np.where(rng.uniform(size=n) < 0.05, rng.uniform(0.01, 0.5, n), 0.0))
    diag[rng.uniform(size=n) < 0.3] *= -1.0
    diag[absum == 0] = -1.0
    b = rng.normal(size=n)
    A = np.diag(diag)
    for i in range(n):
        for k in range(row[i], row[i + 1]):
            A[i, col[k]] += off[k]
    xref = np.linalg.solve(A, -b)
    amg = _amg(maxCoarseLevels=0, relativeTolerance=1e-10, nMaxIterations=5)
    amg.coarseSolver = fvmbaseExt.AMG.COARSE_DIRECT
    amg.coarsestSize = 4096
    x, info = amg.solve_csr(row, col, diag, off, b)
    assert list(info["levelSizes"]) == []
    assert info["iterations"] == 1
    assert rel_l2(x, xref) <= 1e-10


# ---------------------------------------------------------------------------
# config 0 at its stated size: 256 x 256 jittered quads, 65,536 cells


@pytest.fixture(scope="module")
def config0_reference(refo):
    """The reference's own FP64 CPU solve of config 0 (ThermalModel<double>
    + AMG V(1,1), inner relTol 0.1, outer 1e-10), computed once."""
    mesh, f = meshgen.config0(n=256, seed=0)
    bcs = {gid: v for gid, v in f["bc"].items()}
    fields = {"conductivity": f["k"], "source": f["s"]}
    r = ref_model(refo, mesh, bcs, fields=fields, n_pre=1, n_post=1, lin_rel=0.1, max_iter=200, rel=1e-10)
    norms, _ = r.advance(500)
    assert norms[-1] / norms[0] < 1e-10
    return mesh, bcs, fields, r.get_field(0)[: mesh["nCells"]]


@pytest.mark.parametrize("variant", ["plain", "mixed-cg"])
def test_config0_full_size_matches_reference(config0_reference, variant):
    """Config 0 as stated (65,536 cells, AMG V(1,1), coarsening to at most
    100 rows, outer relative residual 1e-10): the plain FP64 GPU AMG and the
    mixed-precision CG + FP32 V(0,2) against the reference's FP64 solve,
    relative L2 <= 1e-8."""
    mesh, bcs, fields, Tr = config0_reference
    amg = _amg(nPreSweeps=1, nPostSweeps=1, relativeTolerance=0.1, nMaxIterations=200, coarsestSize=100)
    solver = amg
    if variant == "mixed-cg":
        amg.precision = fvmbaseExt.AMG.MIXED
        amg.coarseSolver = fvmbaseExt.AMG.COARSE_DIRECT
        amg.coarsestSize = 4096
        amg.coarseJacobiRows = 1 << 30
        amg.nPreSweeps, amg.nPostSweeps = 0, 2
        solver = fvmbaseExt.CG()
        solver.preconditioner = amg
        solver.relativeTolerance = 0.1
        solver.nMaxIterations = 200
    tm, tf, m = gpu_model(mesh, bcs, solver=solver, fields=fields, opts={"relativeTolerance": 1e-10})
    _converge(tm, n_outer=500)
    T = tf.temperature[m.getCells()][: mesh["nCells"]]
    assert rel_l2(T, Tr) <= TOL_FIELD
