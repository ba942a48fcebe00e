"""Autotuned launch plans of the smoother kernels (threads per row, threads
per block on the SELL-32 levels): the plan changes speed only. Every plan
forms the products of a row in parallel and adds them in stored order, so
solves under any plan -- forced or picked by the autotuner -- give bitwise
the same temperature field."""
import numpy as np
import pytest

from fvm_b200 import fvmbaseExt, meshgen
from helpers import gpu_model


def _solve(mixed, autotune, tpr=0, block=0, ell_rows=0, n=96, device=False):
    mesh, f = meshgen.config0(n=n, seed=3)
    bcs = dict(f["bc"])
    amg = fvmbaseExt.AMG()
    amg.nPreSweeps = 1
    amg.nPostSweeps = 1
    amg.relativeTolerance = 0.1
    amg.nMaxIterations = 200
    if mixed:
        amg.precision = fvmbaseExt.AMG.MIXED
        amg.coarseSolver = fvmbaseExt.AMG.COARSE_DIRECT
        amg.coarsestSize = 1000
        amg.coarseJacobiRows = 1 << 30  # damped Jacobi below the finest level
        amg.setupOnDevice = device
    amg.autotune = autotune
    amg.planThreadsPerRow = tpr
    amg.planBlock = block
    amg.planEllRows = ell_rows
    tm, tf, m = gpu_model(mesh, bcs, solver=amg, fields={"conductivity": f["k"], "source": f["s"]},
                          opts={"relativeTolerance": 1e-10})
    tm.advance(200)
    rep = tm.lastReport()
    assert rep.converged
    return tf.temperature[m.getCells()][: mesh["nCells"]].copy(), tm.getLaunchPlans(), rep.linearIterations


@pytest.mark.gpu
@pytest.mark.parametrize("mixed", [False, True], ids=["fp64-gs", "mixed-jacobi"])
def test_plans_give_bitwise_identical_solves(mixed):
    T0, plans0, c0 = _solve(mixed, autotune=False)
    # default plan everywhere without the tuner
    assert all(p in ((1, 256),) or p[0] < 0 for p in plans0)
    for tpr, block in ((2, 128), (4, 256), (4, 128), (1, 128)):
        T, plans, c = _solve(mixed, autotune=False, tpr=tpr, block=block)
        sell = [p for p in plans if p[0] > 0]
        assert sell and all(p == (tpr, block) for p in sell)
        assert c == c0
        np.testing.assert_array_equal(T, T0)
    T, plans, c = _solve(mixed, autotune=True)
    assert all((p[0] in (1, 2, 4) and p[1] in (128, 256)) or (p[0] < 0 and p[1] in (-1, -2)) for p in plans)
    assert c == c0
    np.testing.assert_array_equal(T, T0)


@pytest.mark.gpu
def test_plans_on_gpu_built_levels_bitwise_identical():
    """Every threads-per-row plan forced on the GPU-built coarse levels
    (natural row order, the last slice of each level partly empty): the
    same iterations and bitwise the same field as the default plan."""
    T0, _, c0 = _solve(True, autotune=False, device=True)
    for tpr, block in ((2, 128), (2, 256), (4, 128), (4, 256), (1, 128)):
        T, plans, c = _solve(True, autotune=False, tpr=tpr, block=block, device=True)
        sell = [p for p in plans if p[0] > 0]
        assert sell and all(p == (tpr, block) for p in sell)
        assert c == c0
        np.testing.assert_array_equal(T, T0)


@pytest.mark.gpu
@pytest.mark.parametrize("mixed", [False, True], ids=["fp64-gs", "mixed"])
def test_ell_rows_per_thread_bitwise_identical(mixed):
    """The ELL-32 finest level (192^2 quads: 36,864 rows) under one and two
    rows per thread of its Gauss-Seidel pass: the same iterations and
    bitwise the same field."""
    T1, plans1, c1 = _solve(mixed, autotune=False, ell_rows=1, n=192)
    T2, plans2, c2 = _solve(mixed, autotune=False, ell_rows=2, n=192)
    assert plans1[0][0] < 0 and plans1[0][1] == -1
    assert plans2[0][0] < 0 and plans2[0][1] == -2
    assert c1 == c2
    np.testing.assert_array_equal(T1, T2)


def test_plan_options_validated():
    a = fvmbaseExt.AMG()
    o = a.options()
    assert o.autotune == 1 and o.planThreadsPerRow == 0 and o.planBlock == 0 and o.planEllRows == 0
    # the finest-level Chebyshev smoother is off by default (Gauss-Seidel)
    assert o.chebyshevDegree == 0 and o.chebyshevFraction == 0.3
