"""Host-side setup of the product (no GPU needed): mesh connectivity,
geometry and AMG aggregation are bit-identical to the reference oracle;
the multicolour ordering is a valid colouring."""
import numpy as np
import pytest

from fvm_b200 import fvmbaseExt, meshgen
from helpers import load_fixture

MESHES = {
    "quad": lambda: meshgen.quad_mesh(12, 0.2, 0),
    "tet": lambda: meshgen.tet_mesh(5, 0.15, 1),
    "hex": lambda: meshgen.hex_mesh(4),
    "tri_894": lambda: load_fixture("ptest_tri_894.npz"),
    "tetra_8k": lambda: load_fixture("ptest_tetra_8k.npz"),
}


@pytest.mark.parametrize("name", sorted(MESHES))
def test_connectivity_and_geometry_bit_exact(refo, name):
    md = MESHES[name]()
    m = fvmbaseExt.Mesh.from_dict(md)
    r = refo.RefThermal(md)
    nf = len(md["faceNodeCount"])
    row, col = m.getCellCells()
    rrow, rcol, rp2c = r.connectivity(nf)
    np.testing.assert_array_equal(row, rrow)
    np.testing.assert_array_equal(col, rcol)
    np.testing.assert_array_equal(m.getPairToColMapping(), rp2c)
    g = m.getGeometry()
    fa, fam, fcn, ccn, vol = r.geometry(nf)
    for a, b in ((g["area"], fa), (g["areaMag"], fam), (g["faceCentroid"], fcn), (g["cellCentroid"], ccn),
                 (g["volume"], vol)):
        np.testing.assert_array_equal(a, b)


def test_mm226_aggregation_matches_reference():
    z = load_fixture("mm226.npz")
    sizes, cis, colors = fvmbaseExt.AMG().hierarchy_csr(z["row"], z["col"], z["diag"], z["off"])
    assert sizes == [108, 48, 20, 8]
    np.testing.assert_array_equal(np.concatenate(cis), z["ref_ci"])


def _random_diffusion_matrix(n, seed):
    rng = np.random.default_rng(seed)
    md = meshgen.quad_mesh(n, 0.25, seed)
    m = fvmbaseExt.Mesh.from_dict(md)
    row, col = m.getCellCells()
    N = md["nCells"]
    r, c, o = [0], [], []
    w = {}
    for i in range(N):
        for k in range(row[i], row[i + 1]):
            j = int(col[k])
            if j < N:
                key = (min(i, j), max(i, j))
                if key not in w:
                    w[key] = float(rng.lognormal(0, 2))
                c.append(j)
                o.append(w[key])
        r.append(len(c))
    o = np.array(o)
    r = np.array(r, np.int32)
    d = np.zeros(N)
    for i in range(N):
        d[i] = -o[r[i]:r[i + 1]].sum() - rng.uniform(0, 0.1)
    return r, np.array(c, np.int32), d, o


@pytest.mark.parametrize("seed", [1, 2, 3])
def test_aggregation_random_matrices(refo, seed):
    row, col, d, o = _random_diffusion_matrix(24, seed)
    b = np.ones(len(d))
    _, rsizes, _, rcis = refo.amg_csr(row, col, d, o, b, max_iter=2)
    sizes, cis, _ = fvmbaseExt.AMG().hierarchy_csr(row, col, d, o)
    assert sizes == rsizes
    for a, b_ in zip(cis, rcis):
        np.testing.assert_array_equal(a, b_)


def test_coloring_is_valid():
    row, col, d, o = _random_diffusion_matrix(20, 7)
    sizes, cis, colors = fvmbaseExt.AMG().hierarchy_csr(row, col, d, o)
    c0 = colors[0]
    for i in range(len(d)):
        for k in range(row[i], row[i + 1]):
            assert c0[i] != c0[col[k]]
    # greedy colouring is deterministic and small
    assert c0.max() + 1 <= 6
