"""Fluent case-file import on the product side (importers.FluentReader over
the library's C++ reader; the reference's FluentReader::readMesh +
getMeshList, src/modules/importers/FluentReader.cpp:572-611, 954-1040).

CPU: the arrays of every reference test mesh -- ASCII (cav32.cas) and
binary double-precision files, 2D and 3D, tri / quad / tet / hex -- are
bit-identical to those the reference's own FluentReader produced
(tests/golden/*.npz, written by tests/golden/make_golden.py from the
compiled reference); malformed and unsupported files raise.
GPU: the PARALLEL_TESTS np=1 cases run end to end from the .cas files
(import, ThermalModel, advance) and reach the golden temperatures within
the tests' 1e-5.
"""
import gzip
import os

import numpy as np
import pytest

from fvm_b200 import fvmbaseExt, importers
from fvm_b200._lib import FvmError
from helpers import GOLDEN, gpu_model, load_fixture

CASES = [("cav32.cas", "cav32_matrix.npz"), ("cav32_thermal.cas", "ptest_quad_1024.npz"),
         ("tri_894.cas", "ptest_tri_894.npz"), ("cav_hexa.cas", "ptest_hexa_10k.npz"),
         ("cav_tetra.cas", "ptest_tetra_8k.npz")]


def _unpack(tmp_path, cas):
    out = tmp_path / cas
    with gzip.open(os.path.join(GOLDEN, cas + ".gz"), "rb") as src:
        out.write_bytes(src.read())
    return str(out)


@pytest.mark.parametrize("cas,npz", CASES)
def test_arrays_equal_reference_reader(tmp_path, cas, npz):
    r = importers.FluentReader(_unpack(tmp_path, cas))
    r.readMesh()
    assert r.getNumCellZones() == 1
    d = r.getMeshArrays(0)
    z = load_fixture(npz)
    for k in ("dim", "nCells"):
        assert int(d[k]) == int(z[k])
    for k in ("nodes", "faceCells", "faceNodes", "faceNodeCount", "faceGroupSize", "groupId"):
        np.testing.assert_array_equal(np.asarray(d[k]).reshape(-1), np.asarray(z[k]).reshape(-1), err_msg=k)
    assert list(d["groupType"]) == [str(t) for t in z["groupType"]]


def test_mesh_list_builds_meshes_with_zone_ids(tmp_path):
    r = importers.FluentReader(_unpack(tmp_path, "cav_tetra.cas"))
    r.readMesh()
    (m,) = r.getMeshList()
    z = load_fixture("ptest_tetra_8k.npz")
    assert m.getCells().getSelfCount() == int(z["nCells"])
    ids = [g.id for g in m.getBoundaryFaceGroups()]
    assert ids == [int(i) for i in z["groupId"][1:]]
    ref = fvmbaseExt.Mesh.from_dict({k: z[k] for k in ("dim", "nCells", "nodes", "faceCells", "faceNodes",
                                                      "faceNodeCount", "faceGroupSize")})
    for a, b in zip(m.getCellCells(), ref.getCellCells()):
        np.testing.assert_array_equal(a, b)


_TWO_QUADS = """(0 "two quads, ASCII")
(2 2)
(10 (0 1 6 0 2))
(10 (1 1 6 1 2)(
0.0 0.0
1.0 0.0
2.0 0.0
0.0 1.0
1.0 1.0
2.0 1.0
))
(12 (0 1 2 0))
(12 (2 1 2 1 3))
(13 (0 1 7 0))
(13 (3 1 1 2 2)(
2 5 1 2
))
(13 (4 2 7 3 2)(
1 2 1 0
2 3 2 0
3 6 2 0
6 5 2 0
5 4 1 0
4 1 1 0
))
(39 (2 fluid fluid 1)())
(39 (3 interior default-interior 1)())
(39 (4 wall outer-wall 1)())
"""


def test_hand_written_ascii_case(tmp_path):
    p = tmp_path / "two.cas"
    p.write_text(_TWO_QUADS)
    r = importers.FluentReader(str(p))
    r.readMesh()
    d = r.getMeshArrays(0)
    assert d["dim"] == 2 and d["nCells"] == 2
    np.testing.assert_array_equal(d["faceGroupSize"], [1, 6])
    assert list(d["groupType"]) == ["interior", "wall"]
    assert list(d["groupId"]) == [0, 4]
    # interior face first; boundary faces get ghosts 2..7 in face order
    np.testing.assert_array_equal(d["faceCells"][:, 1], [1, 2, 3, 4, 5, 6, 7])
    m = r.getMeshList()[0]
    assert m.getCells().getCount() == 8


def test_missing_and_malformed_files_raise(tmp_path):
    with pytest.raises(FvmError):
        importers.FluentReader(str(tmp_path / "none.cas")).readMesh()
    bad = tmp_path / "bad.cas"
    bad.write_text(_TWO_QUADS.replace("(2 2)", "(2 7)"))
    with pytest.raises(FvmError):
        importers.FluentReader(str(bad)).readMesh()
    cut = tmp_path / "cut.cas"
    cut.write_text(_TWO_QUADS[: _TWO_QUADS.index("4 1 1 0")])
    with pytest.raises(FvmError):
        importers.FluentReader(str(cut)).readMesh()
    binary = tmp_path / "bin.cas"
    gz = gzip.open(os.path.join(GOLDEN, "tri_894.cas.gz"), "rb").read()
    binary.write_bytes(gz[: len(gz) // 2])  # a binary section without its end marker
    with pytest.raises(FvmError):
        importers.FluentReader(str(binary)).readMesh()


@pytest.mark.gpu
@pytest.mark.parametrize("cas,case", [("cav32_thermal.cas", "quad_1024"), ("tri_894.cas", "tri_894"),
                                      ("cav_hexa.cas", "hexa_10k"), ("cav_tetra.cas", "tetra_8k")])
def test_parallel_thermal_golden_from_case_file(tmp_path, cas, case):
    """PARALLEL_TESTS np=1 from the .cas file: import, ThermalModel with the
    tests' boundary conditions, reference-ordered AMG to relTol 1e-9,
    advance(1): the golden cell temperatures within 1e-5."""
    r = importers.FluentReader(_unpack(tmp_path, cas))
    r.readMesh()
    d = r.getMeshArrays(0)
    gold = load_fixture("ptest_%s.npz" % case)["T_gold"]
    bcs = {g: ("T", v) for g, v in ((3, 400.0), (4, 0.0), (5, 0.0), (6, 0.0)) if g in d["groupId"]}
    amg = fvmbaseExt.AMG()
    amg.relativeTolerance = 1e-9
    amg.nMaxIterations = 2000
    amg.maxCoarseLevels = 20
    amg.smootherOrdering = fvmbaseExt.AMG.SEQUENTIAL
    tm, tf, mesh = gpu_model(d, bcs, solver=amg, group_ids=d["groupId"], group_types=d["groupType"])
    tm.advance(1)
    T = tf.temperature[mesh.getCells()][: d["nCells"]]
    assert np.abs(T - gold).max() <= 1e-5
