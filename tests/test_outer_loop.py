"""advance() with its outer iterations on the device (linear options'
outerOnDevice): one CUDA graph whose conditional while node runs the
linearization, the CG solve (a while node of its own), the outer
convergence test and, under a conditional if node, the solution update.

Bar: the same kernels in the same order as the host loop, so the same outer
and linear iteration counts, bitwise the same outer norm history and
bitwise the same temperature field; the model's state carries across calls
(first outer norm, history) exactly as the host loop carries it; solves
that need the host between iterations (the AMG solver, a learned step,
printing) fall back to the host loop.

Anderson acceleration of the outer iteration (outerAcceleration = depth):
bitwise the same on the device and on the host loop; fewer outer
iterations than the plain loop on the tet mesh; converged field within
1e-8 relative L2 of the reference's plain FP64 solve (ThermalModel::advance,
fvmbase/ThermalModel_impl.h:424-456, compiled here).
"""
import numpy as np
import pytest

from fvm_b200 import fvmbaseExt, meshgen
from helpers import gpu_model, ref_model, rel_l2

pytestmark = pytest.mark.gpu


def _mesh(kind):
    if kind == "tet":
        return meshgen.config1(m=14, seed=1)
    return meshgen.config3(n=16, seed=3)


def _solver(precision, on_device, kind="cg", accel=0):
    a = fvmbaseExt.AMG()
    a.outerAcceleration = accel
    if precision == "mixed":
        a.precision = fvmbaseExt.AMG.MIXED
        a.coarseSolver = fvmbaseExt.AMG.COARSE_DIRECT
        a.coarsestSize = 100
        a.coarseJacobiRows = 1 << 30
        a.nPreSweeps, a.nPostSweeps = 0, 2
        a.setupOnDevice = True
    a.outerOnDevice = on_device
    if kind == "amg":
        a.relativeTolerance = 1e-10
        a.nMaxIterations = 300
        return a
    cg = fvmbaseExt.CG()
    cg.preconditioner = a
    cg.relativeTolerance = 1e-10
    cg.nMaxIterations = 500
    return cg


def _run(kind, precision, on_device, calls, opts=None, fields_extra=None, update_time=False, solver_kind="cg",
         accel=0):
    mesh, f = _mesh(kind)
    bcs = {gid: v for gid, v in f["bc"].items()}
    fields = {"conductivity": f["k"], "source": f["s"]}
    fields.update(fields_extra or {})
    o = {"relativeTolerance": 1e-10}
    o.update(opts or {})
    tm, tf, m = gpu_model(mesh, bcs, solver=_solver(precision, on_device, solver_kind, accel), fields=fields, opts=o)
    reps = []
    for niter in calls:
        tm.advance(niter)
        rep = tm.lastReport()
        reps.append((rep.iterations, rep.linearIterations, bool(rep.converged), bool(rep.outerOnDevice),
                     rep.lastNorm))
        if update_time:
            tm.updateTime()
    T = tf.temperature[m.getCells()][: mesh["nCells"]].copy()
    return T, reps, np.array(tm.getNormHistory())


@pytest.mark.parametrize("precision", ["mixed", "fp64"])
@pytest.mark.parametrize("kind", ["tet", "hex"])
def test_outer_loop_on_device_is_bitwise_neutral(kind, precision):
    T1, r1, h1 = _run(kind, precision, True, [300])
    T0, r0, h0 = _run(kind, precision, False, [300])
    assert r1[0][3] and not r0[0][3]  # the graph ran / the host loop ran
    assert r1[0][2] and r0[0][2]
    assert r1[0][:3] == r0[0][:3]
    assert r1[0][4] == r0[0][4]
    np.testing.assert_array_equal(h1, h0)
    np.testing.assert_array_equal(T1, T0)


def test_outer_loop_state_carries_across_calls():
    """advance(2), advance(1), advance(300): the first outer norm of the
    first call is the reference of every later convergence test, and the
    history grows call by call, as in the host loop."""
    T1, r1, h1 = _run("tet", "mixed", True, [2, 1, 300])
    T0, r0, h0 = _run("tet", "mixed", False, [2, 1, 300])
    assert [r[3] for r in r1] == [True] * 3 and [r[3] for r in r0] == [False] * 3
    assert [r[:3] for r in r1] == [r[:3] for r in r0]
    assert r1[0][0] == 2 and not r1[0][2] and r1[1][0] == 1
    np.testing.assert_array_equal(h1, h0)
    np.testing.assert_array_equal(T1, T0)


def test_outer_loop_transient_steps():
    """Three implicit time steps (advance, then updateTime): the graph is
    built once and replayed with each step's old temperature."""
    mesh, f = _mesh("hex")
    rng = np.random.default_rng(4)
    extra = {"specificHeat": rng.uniform(0.5, 2.0, mesh["nCells"])}
    opts = {"transient": True, "timeStep": 1e-3}
    T1, r1, h1 = _run("hex", "fp64", True, [50, 50, 50], opts=opts, fields_extra=extra, update_time=True)
    T0, r0, h0 = _run("hex", "fp64", False, [50, 50, 50], opts=opts, fields_extra=extra, update_time=True)
    assert all(r[3] for r in r1)
    assert [r[:3] for r in r1] == [r[:3] for r in r0]
    np.testing.assert_array_equal(h1, h0)
    np.testing.assert_array_equal(T1, T0)


def test_outer_loop_falls_back_for_the_amg_solver():
    """The AMG solver tests its residual on the host after every cycle: the
    outer loop stays on the host even with outerOnDevice set."""
    T1, r1, _ = _run("hex", "fp64", True, [300], solver_kind="amg")
    assert not r1[0][3] and r1[0][2]


@pytest.mark.parametrize("depth", [2, 5])
def test_outer_acceleration_device_matches_host(depth):
    """The three acceleration kernels run inside the outer graph's if node
    and from the host loop: bitwise the same, split calls included."""
    T1, r1, h1 = _run("tet", "mixed", True, [3, 300], accel=depth)
    T0, r0, h0 = _run("tet", "mixed", False, [3, 300], accel=depth)
    assert all(r[3] for r in r1) and not any(r[3] for r in r0)
    assert [r[:3] for r in r1] == [r[:3] for r in r0]
    assert r1[-1][2]
    np.testing.assert_array_equal(h1, h0)
    np.testing.assert_array_equal(T1, T0)


@pytest.mark.parametrize("precision", ["mixed", "fp64"])
@pytest.mark.parametrize("kind", ["tet", "hex"])
def test_outer_acceleration_matches_reference(refo, kind, precision):
    mesh, f = _mesh(kind)
    bcs = {gid: v for gid, v in f["bc"].items()}
    fields = {"conductivity": f["k"], "source": f["s"]}
    _, rp, _ = _run(kind, precision, True, [300])
    T, ra, hist = _run(kind, precision, True, [300], accel=2)
    assert ra[0][2] and rp[0][2]
    assert hist[-1] / hist[0] < 1e-10
    if kind == "tet":
        assert ra[0][0] < rp[0][0]  # fewer outer iterations
    r = ref_model(refo, mesh, bcs, fields=fields, n_pre=1, n_post=1, lin_rel=1e-10, max_iter=500, rel=1e-10)
    norms, _ = r.advance(200)
    assert norms[-1] / norms[0] < 1e-10
    assert rel_l2(T, r.get_field(0)[: mesh["nCells"]]) <= 1e-8


def test_outer_acceleration_option_range():
    a = fvmbaseExt.AMG()
    a.outerAcceleration = 6
    with pytest.raises(Exception):
        _ = gpu_model(*_mesh("tet")[:1], {}, solver=a)
