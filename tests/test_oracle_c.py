"""Pins the C restatement of the reference path (oracle/fvm_oracle.c) two
ways: against the reference's own golden files (tests/golden/, made by
tests/golden/make_golden.py) and against the reference compiled from its own
sources (oracle/_ref/libfvmref.so), bit for bit, on seeded meshes covering
every boundary-condition type, steady and transient assembly, and the AMG,
CG+AMG and BCGStab+AMG solvers with Gauss-Seidel and Jacobi smoothing.
CPU only."""
import numpy as np
import pytest

from helpers import load_fixture


@pytest.fixture(scope="module")
def orc():
    from oracle import oracle_c

    if not oracle_c.available():
        pytest.skip("oracle restatement not built (make -C oracle)")
    return oracle_c


def _meshes():
    from fvm_b200 import meshgen

    return {
        "quad": lambda: meshgen.quad_mesh(12, seed=1),
        "tri": lambda: meshgen.tri_mesh(9, seed=4) if hasattr(meshgen, "tri_mesh") else meshgen.quad_mesh(9, seed=4),
        "tet": lambda: meshgen.tet_mesh(5, seed=2),
        "hex": lambda: meshgen.hex_mesh(5, seed=3),
    }


def _setup(impl, G, bcset, solver, smoother, k, s):
    impl.set_options(solver=solver, n_pre=1, n_post=1, smoother=smoother, lin_rel=1e-3, max_iter=50, rel=1e-10,
                     transient=(bcset == 2), dt=1e-2)
    for g in range(1, G):
        if bcset == 0:  # Dirichlet + Neumann
            impl.set_bc(g, 0 if g <= 2 else 1, [300.0 + 100 * g, 0.5])
        elif bcset == 1:  # every type: T, symmetry, convective, radiative, mixed, flux
            impl.set_bc(g, [0, 2, 3, 4, 5, 1][g % 6], [350.0, 2.0, 3.0, 310.0, 0.7])
        else:  # transient, Dirichlet + flux
            impl.set_bc(g, g % 2, [400.0, -1.0])
    impl.init()
    impl.set_field(1, k)
    impl.set_field(2, s)


def test_mm226_golden(orc):
    """T/testLinearSolver.out: coarse sizes 108/48/20/8 (the serial build
    drops the 3-row level), initial L1 norm 6981.57, serial history."""
    z = load_fixture("mm226.npz")
    x, sizes, hist, cis = orc.amg_csr(z["row"], z["col"], z["diag"], z["off"], z["b"], max_iter=41, rel_tol=1e-30)
    assert sizes == [108, 48, 20, 8]
    assert float("%.6g" % hist[0]) == 6981.57
    assert float("%.6g" % hist[40]) == 6.52597e-05
    np.testing.assert_array_equal(np.concatenate(cis), z["ref_ci"])


def test_mm226_equals_reference(orc, refo):
    z = load_fixture("mm226.npz")
    for smoother in (0, 1):
        for cycle in (0, 1, 2):
            a = orc.amg_csr(z["row"], z["col"], z["diag"], z["off"], z["b"], max_iter=30, rel_tol=1e-30, n_pre=1,
                            cycle=cycle, smoother=smoother)
            b = refo.amg_csr(z["row"], z["col"], z["diag"], z["off"], z["b"], max_iter=30, rel_tol=1e-30, n_pre=1,
                             cycle=cycle, smoother=smoother)
            np.testing.assert_array_equal(a[0], b[0])
            assert a[1] == b[1]
            np.testing.assert_array_equal(a[2], b[2])


def test_cav32_matrix_golden(orc):
    """T/THERMAL_MATRIX/GOLDEN (matrix_mesh0.mat, matrix.rhs), 1e-8."""
    m = load_fixture("cav32_matrix.npz")
    r = orc.OracleThermal(m, group_ids=m["groupId"], group_types=m["groupType"])
    for gid, T in ((3, 400.0), (4, 0.0), (5, 0.0), (6, 0.0)):
        r.set_bc(gid, 0, [T])
    r.init()
    d, o, b, _ = r.linearize()
    n = m["nCells"]
    row, col, _ = r.connectivity()
    mine = {}
    for i in range(n):
        mine[(i, i)] = d[i]
        for k in range(row[i], row[i + 1]):
            if col[k] < n:
                mine[(i, int(col[k]))] = o[k]
    gold = {(int(i), int(j)): v for i, j, v in zip(m["gold_i"], m["gold_j"], m["gold_v"])}
    assert set(mine) == set(gold)
    assert max(abs(mine[k] - gold[k]) for k in gold) <= 1e-8
    assert np.abs(-b[:n] - m["gold_rhs"]).max() <= 1e-8


@pytest.mark.parametrize("case", ["quad_1024", "tri_894", "hexa_10k", "tetra_8k"])
def test_parallel_thermal_golden(orc, case):
    """PARALLEL_TESTS *_THERMALSOLVER np=1 temperatures (1e-5)."""
    m = load_fixture("ptest_%s.npz" % case)
    r = orc.OracleThermal(m, group_ids=m["groupId"], group_types=m["groupType"])
    r.set_options(lin_rel=1e-9, max_iter=2000, max_levels=20)
    for gid, T in ((3, 400.0), (4, 0.0), (5, 0.0), (6, 0.0)):
        if gid in m["groupId"]:
            r.set_bc(gid, 0, [T])
    r.init()
    r.advance(1)
    T = r.get_field(0)[: m["nCells"]]
    assert np.abs(T - m["T_gold"]).max() <= 1e-5


@pytest.mark.parametrize("name", ["quad", "tet", "hex"])
def test_mesh_equals_reference(orc, refo, name):
    mesh = _meshes()[name]()
    r = refo.RefThermal(mesh)
    o = orc.OracleThermal(mesh)
    nf = len(mesh["faceNodeCount"])
    for a, b in zip(r.connectivity(nf), o.connectivity()):
        np.testing.assert_array_equal(a, b)
    g = o.geometry()
    for a, key in zip(r.geometry(nf), ("area", "areaMag", "faceCentroid", "cellCentroid", "volume")):
        np.testing.assert_array_equal(a, g[key])


@pytest.mark.parametrize("name", ["quad", "tet", "hex"])
@pytest.mark.parametrize("bcset", [0, 1, 2])
@pytest.mark.parametrize("solver,smoother", [(0, 0), (0, 1), (1, 0), (2, 0)])
def test_thermal_equals_reference(orc, refo, name, bcset, solver, smoother):
    """Linear system, AMG hierarchy, outer norms and temperature after 8
    outer iterations: identical bits."""
    from fvm_b200.meshgen import extend_to_ghosts

    mesh = _meshes()[name]()
    rng = np.random.default_rng(7)
    n = mesh["nCells"]
    k = extend_to_ghosts(mesh, np.exp(rng.normal(size=n)))
    s = extend_to_ghosts(mesh, rng.random(n))
    G = len(mesh["faceGroupSize"])
    r = refo.RefThermal(mesh)
    o = orc.OracleThermal(mesh)
    for impl in (r, o):
        _setup(impl, G, bcset, solver, smoother, k, s)
    for a, b in zip(r.linearize(), o.linearize()):
        np.testing.assert_array_equal(a, b)
    ha, hb = r.hierarchy(), o.hierarchy()
    assert ha[0] == hb[0]
    for a, b in zip(ha[1], hb[1]):
        np.testing.assert_array_equal(a, b)
    na, _ = r.advance(8)
    nb, cycles = o.advance(8)
    np.testing.assert_array_equal(na, nb)
    np.testing.assert_array_equal(r.get_field(0), o.get_field(0))
    assert cycles > 0


def test_transient_steps_equal_reference(orc, refo):
    from fvm_b200 import meshgen
    from fvm_b200.meshgen import extend_to_ghosts

    mesh = meshgen.hex_mesh(4, seed=5)
    rng = np.random.default_rng(3)
    n = mesh["nCells"]
    k = extend_to_ghosts(mesh, np.exp(rng.normal(size=n)))
    s = extend_to_ghosts(mesh, rng.random(n))
    rc = extend_to_ghosts(mesh, rng.uniform(0.5, 2.0, n))
    G = len(mesh["faceGroupSize"])
    r = refo.RefThermal(mesh)
    o = orc.OracleThermal(mesh)
    for impl in (r, o):
        _setup(impl, G, 2, 0, 0, k, s)
        impl.set_field(3, rc)
    for _ in range(3):
        na, _ = r.advance(20)
        nb, _ = o.advance(20)
        np.testing.assert_array_equal(na, nb)
        r.update_time()
        o.update_time()
    np.testing.assert_array_equal(r.get_field(0), o.get_field(0))
    np.testing.assert_array_equal(r.get_field(4), o.get_field(4))


def test_multicolor_matches_product(orc):
    """The product's level-0 colouring equals the restated definition, and
    is a proper colouring."""
    from fvm_b200 import fvmbaseExt

    z = load_fixture("mm226.npz")
    rng = np.random.default_rng(11)
    cases = [(z["row"], z["col"], z["diag"], z["off"])]
    for n, symmetric in ((50, True), (300, True), (200, False)):
        # random pattern; the unsymmetric one is coloured as A + A^T
        pairs = {(int(a), int(b)) for a, b in rng.integers(0, n, size=(4 * n, 2)) if a != b}
        if symmetric:
            pairs |= {(b, a) for a, b in pairs}
        rows = [[] for _ in range(n)]
        for a, b in sorted(pairs):
            rows[a].append(b)
        row = np.zeros(n + 1, np.int32)
        row[1:] = np.cumsum([len(x) for x in rows])
        col = np.array([c for x in rows for c in x], np.int32)
        off = -rng.random(len(col))
        diag = np.zeros(n)
        np.add.at(diag, np.repeat(np.arange(n), np.diff(row)), off)
        cases.append((row, col, diag - 1.0, off))
    for row, col, diag, off in cases:
        _, _, colors = fvmbaseExt.AMG().hierarchy_csr(row, col, diag, off)
        nc, c = orc.multicolor(row, col)
        np.testing.assert_array_equal(colors[0], c)
        # proper colouring of A + A^T: no stored entry joins two rows of one colour
        rid = np.repeat(np.arange(len(row) - 1), np.diff(row))
        assert not np.any(c[rid] == c[col])
        assert c.max() + 1 == nc
