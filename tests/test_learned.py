"""Learned correction: the CPU restatement of the network (oracle/
mpnn_oracle.py) against finite differences; the GPU forward and backward
kernels against that restatement; training on the GPU on pairs harvested
from the plain solver; and the solve with the learned step, whose converged
field must still match the reference FP64 solve.

Tolerances: the restatement's gradient matches central differences to 1e-6
relative (FP64). With the dense layers on the CUDA cores the GPU kernels run
in FP32 with FP32 accumulation, so the forward output is compared at 1e-4
relative (L2) and the gradient at 2e-3 of its largest component. On the
tensor cores (tcgen05 kind::tf32) the layer products read their operands
with a 10-bit mantissa (relative rounding 2^-11) and sum in FP32: forward
output within 1e-2 relative L2, the gradient within 2e-2 (per parameter
block, and max-abs relative to the largest component). Measured on B200:
forward 2.1e-3 to 2.4e-3, gradient blocks 2.5e-3 to 9.6e-3. The converged
field: 1e-8 relative L2."""
import numpy as np
import pytest

from helpers import gpu_model, ref_model, rel_l2
from oracle import mpnn_oracle as mo


def _graph(nx=9, ny=7, seed=0):
    """Symmetric M-matrix on an nx x ny grid with random couplings."""
    rng = np.random.default_rng(seed)
    n = nx * ny
    idx = np.arange(n).reshape(ny, nx)
    pairs = []
    for y in range(ny):
        for x in range(nx):
            if x + 1 < nx:
                pairs.append((idx[y, x], idx[y, x + 1]))
            if y + 1 < ny:
                pairs.append((idx[y, x], idx[y + 1, x]))
    w = rng.uniform(0.1, 2.0, len(pairs))
    rows = [[] for _ in range(n)]
    for (a, b), c in zip(pairs, w):
        rows[a].append((b, c))
        rows[b].append((a, c))
    row = np.zeros(n + 1, np.int32)
    row[1:] = np.cumsum([len(r) for r in rows])
    col = np.array([j for r in rows for j, _ in r], np.int32)
    off = np.array([c for r in rows for _, c in r])
    diag = -np.array([sum(c for _, c in r) for r in rows]) - rng.uniform(0.01, 0.5, n)
    return row, col, diag, off


def _params(seed=1, scale=1.0):
    rng = np.random.default_rng(seed)
    return rng.normal(0, 0.3 * scale, mo.N_PARAMS)


def test_oracle_gradient_matches_finite_differences():
    row, col, diag, off = _graph()
    rng = np.random.default_rng(2)
    r = rng.normal(size=len(diag))
    e = rng.normal(size=len(diag))
    P = _params()
    loss, g = mo.loss_and_gradient(P, row, col, diag, off, r, e)
    assert loss > 0
    h = 1e-6
    for k in rng.choice(mo.N_PARAMS, 60, replace=False).tolist() + [0, 40, mo.DEC_W, mo.N_PARAMS - 1]:
        Pp, Pm = P.copy(), P.copy()
        Pp[k] += h
        Pm[k] -= h
        fd = (mo.loss_and_gradient(Pp, row, col, diag, off, r, e)[0] -
              mo.loss_and_gradient(Pm, row, col, diag, off, r, e)[0]) / (2 * h)
        assert abs(fd - g[k]) <= 1e-6 * max(1.0, abs(g).max()) + 1e-5 * abs(g[k]), k


def test_oracle_output_scales_with_residual():
    """The input is normalised by the mean Jacobi-scaled residual and the
    output rescaled by it: N(c r) = c N(r) for c > 0."""
    row, col, diag, off = _graph(seed=3)
    r = np.random.default_rng(4).normal(size=len(diag))
    P = _params(seed=5)
    a = mo.forward(P, row, col, diag, off, r)
    b = mo.forward(P, row, col, diag, off, 37.5 * r)
    np.testing.assert_allclose(b, 37.5 * a, rtol=1e-12, atol=1e-12 * np.abs(b).max())


# (forward rel. L2, loss rel., gradient max-abs / max|g|, per-block gradient rel. L2)
_TOL = {False: (1e-4, 1e-4, 2e-3, 5e-3), True: (1e-2, 1e-2, 2e-2, 2e-2)}
_BLOCKS = [(0, 64)] + [(64 + l * mo.LAYER, 64 + (l + 1) * mo.LAYER) for l in range(3)] + [(mo.DEC_W, mo.N_PARAMS)]


@pytest.mark.gpu
@pytest.mark.parametrize("tensor_cores", [False, True], ids=["fp32-cuda-cores", "tf32-tcgen05"])
def test_gpu_forward_matches_oracle(tensor_cores):
    from fvm_b200.learned import LearnedCorrection

    row, col, diag, off = _graph(nx=23, ny=19, seed=6)
    lc = LearnedCorrection(seed=3)
    lc.tensorCores = tensor_cores
    assert lc.tensorCores == tensor_cores
    P = lc.getParams().astype(np.float64)
    rng = np.random.default_rng(7)
    for trial in range(3):
        r = rng.normal(size=len(diag)) * 10.0 ** trial
        out = lc.forward_csr(row, col, diag, off, r)
        ref = mo.forward(P, row, col, diag, off, r)
        assert rel_l2(out, ref) <= _TOL[tensor_cores][0]


@pytest.mark.gpu
@pytest.mark.parametrize("tensor_cores", [False, True], ids=["fp32-cuda-cores", "tf32-tcgen05"])
def test_gpu_gradient_matches_oracle(tensor_cores):
    from fvm_b200.learned import LearnedCorrection

    row, col, diag, off = _graph(nx=31, ny=17, seed=8)
    lc = LearnedCorrection(seed=4)
    lc.tensorCores = tensor_cores
    rng = np.random.default_rng(9)
    # random parameters with a spread of signs so that every ReLU path is exercised
    P = rng.normal(0, 0.25, mo.N_PARAMS).astype(np.float32)
    lc.setParams(P)
    r = rng.normal(size=len(diag))
    e = rng.normal(size=len(diag))
    g, loss = lc.gradient_csr(row, col, diag, off, r, e)
    lref, gref = mo.loss_and_gradient(P.astype(np.float64), row, col, diag, off, r, e)
    _, tl, tg, tb = _TOL[tensor_cores]
    assert abs(loss - lref) <= tl * lref
    assert np.abs(g - gref).max() <= tg * np.abs(gref).max()
    # every block of the parameter vector carries gradient
    for a, b in _BLOCKS:
        assert np.abs(gref[a:b]).max() > 0
        assert rel_l2(g[a:b], gref[a:b]) <= tb


@pytest.mark.gpu
def test_tensor_core_wait_runs_out_and_context_survives():
    """The tensor-core layers' bounded completion wait, made to run out: one
    CTA allocates TMEM and waits on an mbarrier that no MMA signals
    (fvm_learned_wait_probe, 1000 tries). The kernel must report the
    timeout through its status flag, release TMEM and return; afterwards the
    tensor-core layers still run and match the FP32 CUDA-core kernels."""
    import ctypes

    from fvm_b200 import _lib
    from fvm_b200.learned import LearnedCorrection

    lib = _lib.load()
    for _ in range(2):
        status = ctypes.c_int(-1)
        assert lib.fvm_learned_wait_probe(1000, ctypes.byref(status)) == 0, lib.fvm_last_error()
        assert status.value == 1
    row, col, diag, off = _graph(nx=40, ny=30, seed=3)
    P = _params(seed=4).astype(np.float32)
    r = np.random.default_rng(5).normal(size=len(diag))
    outs = []
    for tc in (False, True):
        lc = LearnedCorrection(seed=0)
        lc.tensorCores = tc
        lc.setParams(P)
        outs.append(lc.forward_csr(row, col, diag, off, r))
    assert rel_l2(outs[1], outs[0]) <= 1e-2


@pytest.mark.gpu
def test_tensor_core_layers_on_many_tiles():
    """A graph of 50,213 nodes: 393 tiles of 128 nodes, the last one partial,
    so CTAs of the fixed gradient grid (296) accumulate their weight
    gradient over two tiles in TMEM. Tensor-core forward and gradient against
    the FP32 CUDA-core kernels and against the FP64 restatement."""
    from fvm_b200.learned import LearnedCorrection

    row, col, diag, off = _graph(nx=337, ny=149, seed=10)
    n = len(diag)
    assert n % 128 and n > 296 * 128
    rng = np.random.default_rng(11)
    P = rng.normal(0, 0.25, mo.N_PARAMS).astype(np.float32)
    r = rng.normal(size=n)
    e = rng.normal(size=n)
    res = {}
    for tc in (False, True):
        lc = LearnedCorrection(seed=0)
        lc.tensorCores = tc
        lc.setParams(P)
        res[tc] = (lc.forward_csr(row, col, diag, off, r),) + lc.gradient_csr(row, col, diag, off, r, e)
    ref = mo.forward(P.astype(np.float64), row, col, diag, off, r)
    lref, gref = mo.loss_and_gradient(P.astype(np.float64), row, col, diag, off, r, e)
    for tc in (False, True):
        out, g, loss = res[tc]
        tf, tl, tg, tb = _TOL[tc]
        assert rel_l2(out, ref) <= tf
        assert abs(loss - lref) <= tl * lref
        for a, b in _BLOCKS:
            assert rel_l2(g[a:b], gref[a:b]) <= tb, (tc, a)
    assert rel_l2(res[True][1], res[False][1]) <= 2e-2


def _plain(nPre=1, nPost=1):
    from fvm_b200 import fvmbaseExt

    a = fvmbaseExt.AMG()
    a.nPreSweeps, a.nPostSweeps = nPre, nPost
    a.relativeTolerance = 0.1
    a.nMaxIterations = 200
    return a


def _mixed():
    from fvm_b200 import fvmbaseExt

    a = _plain(1, 2)
    a.precision = fvmbaseExt.AMG.MIXED
    a.coarseSolver = fvmbaseExt.AMG.COARSE_DIRECT
    a.coarsestSize = 100
    a.coarseJacobiRows = 1 << 30
    return a


def _case(seed, m=9):
    from fvm_b200 import meshgen

    mesh, f = meshgen.config1(m=m, seed=seed)
    return mesh, f, {gid: v for gid, v in f["bc"].items()}, {"conductivity": f["k"], "source": f["s"]}


@pytest.mark.gpu
def test_training_on_harvested_pairs_and_exact_solve(refo):
    from fvm_b200.learned import LearnedCorrection

    lc = LearnedCorrection(seed=0)
    # training instances: plain-solver runs on two conductivity draws
    for seed in (11, 12):
        mesh, f, bcs, fields = _case(seed)
        tm, tf, m = gpu_model(mesh, bcs, solver=_plain(), fields=fields, opts={"relativeTolerance": 1e-10})
        assert lc.harvest(tm, nOuter=6, perSolve=4, relativeTolerance=1e-10) > 0
    assert lc.numPairs() >= 24
    before = lc.evaluate()
    losses = lc.train(steps=400, lr=2e-3, seed=1)
    after = lc.evaluate()
    assert np.isfinite(losses).all()
    assert after < before
    assert losses[-50:].mean() < losses[:50].mean()
    # held-out draw: mixed solve with the learned step converges to the reference field
    mesh, f, bcs, fields = _case(13)
    tm, tf, m = gpu_model(mesh, bcs, solver=_mixed(), fields=fields, opts={"relativeTolerance": 1e-10})
    tm.setLearnedCorrection(lc)
    tm.advance(300)
    rep = tm.lastReport()
    assert rep.converged
    assert rep.learnedSteps > 0
    T = tf.temperature[m.getCells()][: mesh["nCells"]]
    r = ref_model(refo, mesh, bcs, fields=fields, n_pre=1, n_post=1, lin_rel=1e-10, max_iter=500, rel=1e-10)
    r.advance(300)
    assert rel_l2(T, r.get_field(0)[: mesh["nCells"]]) <= 1e-8


@pytest.mark.gpu
def test_learned_step_never_raises_the_residual():
    """With untrained (random) weights every step is judged by the FP64
    residual: rejected steps leave the iteration as it was, so the solve
    takes the same number of cycles as without the step, and a step that
    keeps failing is retired."""
    from fvm_b200.learned import LearnedCorrection

    mesh, f, bcs, fields = _case(14, m=7)
    counts = []
    for use in (False, True):
        tm, tf, m = gpu_model(mesh, bcs, solver=_mixed(), fields=fields, opts={"relativeTolerance": 1e-10})
        if use:
            lc = LearnedCorrection(seed=99)
            tm.setLearnedCorrection(lc)
        tm.advance(300)
        rep = tm.lastReport()
        assert rep.converged
        counts.append((rep.iterations, rep.linearIterations, rep.learnedSteps, rep.learnedAccepted))
    (o0, c0, s0, a0), (o1, c1, s1, a1) = counts
    # tried after every refinement iteration until it proves useless (useful
    # in fewer than a quarter of its first three tries), then retired
    assert s0 == 0 and 0 < s1 <= c1
    if a1 == 0:
        assert (o1, c1) == (o0, c0)
        assert s1 == 3


def _cg_mixed():
    from fvm_b200 import fvmbaseExt

    a = _plain(0, 2)
    a.precision = fvmbaseExt.AMG.MIXED
    a.coarseSolver = fvmbaseExt.AMG.COARSE_DIRECT
    a.coarsestSize = 100
    a.coarseJacobiRows = 1 << 30
    a.setupOnDevice = True
    cg = fvmbaseExt.CG()
    cg.preconditioner = a
    cg.relativeTolerance = 0.1
    cg.nMaxIterations = 200
    return cg


@pytest.mark.gpu
def test_trained_network_gain_on_held_out_draws():
    """What the trained network gains over the method without it, on draws
    it never saw. Training: the residual objective |r + A d|^2 / |r|^2 on
    the residuals of plain-solver runs of two draws (jittered tets, 9^3-node
    lattice). Use: the flexible post-correction of CG's mixed-precision AMG
    preconditioner (the network corrects the residual the cycle leaves,
    every iteration; kept on throughout, useful factor 1). Scored on three
    held-out draws: the mean number of CG iterations of the whole outer
    solve with the step must be lower than without it, every solve
    converging to outer 1e-10."""
    from fvm_b200.learned import LearnedCorrection

    lc = LearnedCorrection(seed=0)
    lc.setObjective(LearnedCorrection.RESIDUAL)
    lc.setUsefulFactor(1.0)
    for seed in (21, 22):
        mesh, f, bcs, fields = _case(seed)
        tm, tf, m = gpu_model(mesh, bcs, solver=_plain(), fields=fields, opts={"relativeTolerance": 1e-10})
        lc.harvest(tm, nOuter=6, perSolve=4, relativeTolerance=1e-10)
    before = lc.evaluate()
    losses = lc.train(steps=800, lr=2e-3, seed=2)
    after = lc.evaluate()
    assert np.isfinite(losses).all() and after < before
    its = {False: [], True: []}
    for seed in (23, 24, 25):
        mesh, f, bcs, fields = _case(seed)
        for use in (False, True):
            tm, tf, m = gpu_model(mesh, bcs, solver=_cg_mixed(), fields=fields, opts={"relativeTolerance": 1e-10})
            if use:
                tm.setLearnedCorrection(lc)
            tm.advance(300)
            rep = tm.lastReport()
            assert rep.converged
            its[use].append(rep.linearIterations)
            if use:
                assert rep.learnedSteps > 0
    print("residual objective %.4f -> %.4f; CG iterations without / with the learned step on 3 held-out draws: "
          "%s / %s" % (before, after, its[False], its[True]))
    assert np.mean(its[True]) < np.mean(its[False])


@pytest.mark.gpu
def test_trained_network_prediction_on_held_out_draws():
    """The error objective on draws the network never saw: (1) the relative
    squared error of its prediction of the plain solver's error, trained
    weights against the initial ones, on pairs harvested from a held-out
    draw; (2) the standalone mixed AMG solve of that draw with the trained
    step after every refinement iteration (kept only when it lowers the FP64
    residual) against the same solve without it. Measured on B200: held-out
    error 0.999 -> 0.427, cycles 82 without and 83 with the step (3 tries,
    1 kept, then retired): the prediction gain is large, its effect on the
    iteration count within one cycle either way, so the solve is held to at
    most two extra cycles."""
    from fvm_b200.learned import LearnedCorrection

    lc = LearnedCorrection(seed=0)
    init = lc.getParams()
    for seed in (21, 22):
        mesh, f, bcs, fields = _case(seed)
        tm, tf, m = gpu_model(mesh, bcs, solver=_plain(), fields=fields, opts={"relativeTolerance": 1e-10})
        lc.harvest(tm, nOuter=6, perSolve=4, relativeTolerance=1e-10)
    lc.train(steps=600, lr=2e-3, seed=2)
    trained = lc.getParams()
    # held-out pairs, scored with both parameter sets
    mesh, f, bcs, fields = _case(23)
    held = LearnedCorrection(seed=0)
    tm, tf, m = gpu_model(mesh, bcs, solver=_plain(), fields=fields, opts={"relativeTolerance": 1e-10})
    assert held.harvest(tm, nOuter=6, perSolve=4, relativeTolerance=1e-10) > 0
    held.setParams(init)
    loss_init = held.evaluate()
    held.setParams(trained)
    loss_trained = held.evaluate()
    cycles = {}
    for use in (False, True):
        tm, tf, m = gpu_model(mesh, bcs, solver=_mixed(), fields=fields, opts={"relativeTolerance": 1e-10})
        if use:
            tm.setLearnedCorrection(lc)
        tm.advance(300)
        rep = tm.lastReport()
        assert rep.converged
        cycles[use] = (rep.linearIterations, rep.learnedSteps, rep.learnedAccepted)
    print("held-out relative squared error: initial %.4f, trained %.4f; mixed cycles without / with "
          "the learned step: %d / %d (steps %d, kept %d)" % (loss_init, loss_trained, cycles[False][0],
                                                            cycles[True][0], cycles[True][1], cycles[True][2]))
    assert loss_trained < 0.8 * loss_init
    assert cycles[True][0] <= cycles[False][0] + 2
