"""Pins the oracle (the reference solver compiled from its own sources)
against the reference project's own golden files, stored as fixtures under
tests/golden/ by tests/golden/make_golden.py."""
import numpy as np
import pytest

from helpers import load_fixture


def test_mm226_aggregation_and_history(refo):
    z = load_fixture("mm226.npz")
    x, sizes, hist, cis = refo.amg_csr(z["row"], z["col"], z["diag"], z["off"], z["b"], max_iter=41, rel_tol=1e-30)
    text = str(z["golden_text"])
    # testLinearSolver.out (an MPI build): coarse levels 108, 48, 20, 8, 3;
    # the serial build drops the <= 3-row level (AMG.cpp:200-204)
    for s in (108, 48, 20, 8):
        assert "of size %d" % s in text
    assert sizes == [108, 48, 20, 8]
    assert "0: [test : 6981.57]" in text
    assert float("%.6g" % hist[0]) == 6981.57
    # serial reference after 40 cycles (the MPI golden keeps the 3-row level
    # and ends at 5.32223e-05)
    assert float("%.6g" % hist[40]) == 6.52597e-05
    np.testing.assert_array_equal(np.concatenate(cis), z["ref_ci"])


def test_cav32_matrix_golden(refo):
    """THERMAL_MATRIX/GOLDEN: the linearized cav32 system (1e-8 in ptest.py)."""
    m = load_fixture("cav32_matrix.npz")
    r = refo.RefThermal(m, group_ids=m["groupId"], group_types=m["groupType"])
    r.set_options(lin_rel=1e-9, max_iter=2000, max_levels=20)
    for gid, T in ((3, 400.0), (4, 0.0), (5, 0.0), (6, 0.0)):
        r.set_bc(gid, 0, [T])
    r.init()
    d, o, b, _ = r.linearize()
    n = m["nCells"]
    row, col, _ = r.connectivity(len(m["faceNodeCount"]))
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
def test_parallel_thermal_golden(refo, case):
    """PARALLEL_TESTS *_THERMALSOLVER np=1: temperature after advance(1) with
    AMG relTol 1e-9 (tolerance 1e-5 in PARALLEL_TESTS/ptest.py)."""
    m = load_fixture("ptest_%s.npz" % case)
    r = refo.RefThermal(m, group_ids=m["groupId"], group_types=m["groupType"])
    r.set_options(lin_rel=1e-9, max_iter=2000, max_levels=20)
    for gid, T in ((3, 400.0), (4, 0.0), (5, 0.0), (6, 0.0)):
        if gid in m["groupId"]:
            r.set_bc(gid, 0, [T])
    r.init()
    r.advance(1)
    T = r.get_field(0)[: m["nCells"]]
    assert np.abs(T - m["T_gold"]).max() <= 1e-5
