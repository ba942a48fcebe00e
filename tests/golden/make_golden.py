"""Generates the committed golden fixtures under tests/golden/ from the
reference project's own test inputs and golden outputs, using the
reference solver compiled by oracle/Makefile (oracle/_ref/libfvmref.so).

Run in a container where the reference tree exists:

    make -C oracle && python tests/golden/make_golden.py [/path/to/reference]

Fixtures (all inputs are the reference's, converted to plain arrays):
  mm226.npz       src/fvm/test/MatrixMarket226.dat + rhs226.dat as read by
                  MMReader, the golden numbers of src/fvm/test/testLinearSolver.out,
                  and the serial reference AMG run (sizes, L1 history, x,
                  coarseIndex per level).
  cav32_matrix.npz  src/fvm/test/cav32.cas as read by FluentReader, and the
                  golden linear system of src/fvm/test/THERMAL_MATRIX/GOLDEN
                  (matrix_mesh0.mat, matrix.rhs).
  <mesh>.cas.gz   the Fluent case files of those tests (src/fvm/test/cav32.cas,
                  cav32_thermal.cas, tri_894.cas, cav_hexa.cas, cav_tetra.cas),
                  gzip-compressed, as inputs of the product's own importer.
  ptest_<case>.npz  the meshes of src/fvm/test/PARALLEL_TESTS *_THERMALSOLVER
                  np=1 cases and their golden cell temperatures
                  (SOLVER_AMG/ThermalSolver/<CASE>/proc1/GOLDEN/temp_proc0.dat),
                  re-ordered to the FluentReader cell numbering by matching
                  cell centres.
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import ref  # noqa: E402


def mm226(test_dir: str) -> None:
    row, col, d, o, b = ref.mm_read(os.path.join(test_dir, "MatrixMarket226.dat"),
                                    os.path.join(test_dir, "rhs226.dat"))
    x, sizes, hist, cis = ref.amg_csr(row, col, d, o, b, max_iter=41, rel_tol=1e-30)
    golden_txt = open(os.path.join(test_dir, "testLinearSolver.out")).read()
    np.savez_compressed(
        os.path.join(HERE, "mm226.npz"), row=row, col=col, diag=d, off=o, b=b,
        ref_sizes=np.array(sizes), ref_hist=hist, ref_x=x,
        ref_ci=np.concatenate(cis), golden_text=np.array(golden_txt))


def _mesh_arrays(m: dict) -> dict:
    return {k: m[k] for k in ("dim", "nCells", "nodes", "faceCells", "faceNodes", "faceNodeCount",
                              "faceGroupSize", "groupId")} | {"groupType": np.array(m["groupType"])}


def cav32_matrix(test_dir: str) -> None:
    m = ref.fluent_read(os.path.join(test_dir, "cav32.cas"))
    gold = os.path.join(test_dir, "THERMAL_MATRIX", "GOLDEN")
    lines = open(os.path.join(gold, "matrix_mesh0.mat")).read().split("\n")
    n, _, nnz = map(int, lines[1].split())
    ent = np.array([list(map(float, ln.split())) for ln in lines[2: 2 + nnz]])
    rhs = np.array([float(v) for v in open(os.path.join(gold, "matrix.rhs")).read().split()])
    np.savez_compressed(os.path.join(HERE, "cav32_matrix.npz"), **_mesh_arrays(m),
                        gold_i=ent[:, 0].astype(np.int32) - 1, gold_j=ent[:, 1].astype(np.int32) - 1,
                        gold_v=ent[:, 2], gold_rhs=rhs)


def _cell_nodes_centres(m: dict) -> np.ndarray:
    n = m["nCells"]
    fc = m["faceCells"]
    cnt = m["faceNodeCount"]
    ptr = np.concatenate([[0], np.cumsum(cnt)])
    fn = m["faceNodes"]
    nodes = m["nodes"]
    sets = [set() for _ in range(n)]
    for f in range(len(cnt)):
        ns = fn[ptr[f]: ptr[f + 1]]
        for c in fc[f]:
            if c < n:
                sets[c].update(ns.tolist())
    return np.array([nodes[sorted(s)].mean(axis=0) for s in sets])


def _read_tecplot(path: str):
    toks = open(path).read().split("\n")
    head = toks[2]
    nn = int(head.split("N = ")[1].split()[0])
    ne = int(head.split("E = ")[1].split()[0])
    body = " ".join(toks[3:]).split()
    vals = np.array(body[: 3 * nn + 2 * ne], dtype=float)
    x, y, z = vals[:nn], vals[nn: 2 * nn], vals[2 * nn: 3 * nn]
    T = vals[3 * nn: 3 * nn + ne]
    conn_tok = np.array(body[3 * nn + 2 * ne:], dtype=np.int64)
    per = len(conn_tok) // ne
    conn = conn_tok.reshape(ne, per) - 1
    pts = np.stack([x, y, z], axis=1)
    cen = np.array([pts[np.unique(c)].mean(axis=0) for c in conn])
    return T, cen


def ptest(test_dir: str, case: str, cas: str) -> None:
    from scipy.spatial import cKDTree

    m = ref.fluent_read(os.path.join(test_dir, cas))
    T_gold, cen_gold = _read_tecplot(os.path.join(test_dir, "PARALLEL_TESTS", "SOLVER_AMG", "ThermalSolver", case,
                                                  "proc1", "GOLDEN", "temp_proc0.dat"))
    cen = _cell_nodes_centres(m)
    d, idx = cKDTree(cen_gold).query(cen)
    if len(set(idx.tolist())) != len(idx) or d.max() > 1e-6 * max(1.0, np.abs(cen).max()):
        raise RuntimeError("cell matching failed for " + case)
    np.savez_compressed(os.path.join(HERE, "ptest_%s.npz" % case.lower()), **_mesh_arrays(m),
                        T_gold=T_gold[idx])


def fluent_cases(test_dir: str) -> None:
    import gzip
    import shutil

    for cas in ("cav32.cas", "cav32_thermal.cas", "tri_894.cas", "cav_hexa.cas", "cav_tetra.cas"):
        with open(os.path.join(test_dir, cas), "rb") as src, \
                gzip.GzipFile(os.path.join(HERE, cas + ".gz"), "wb", mtime=0) as dst:
            shutil.copyfileobj(src, dst)


def main(reference_root: str = "/root/reference") -> None:
    test_dir = os.path.join(reference_root, "src", "fvm", "test")
    fluent_cases(test_dir)
    mm226(test_dir)
    cav32_matrix(test_dir)
    for case, cas in (("QUAD_1024", "cav32_thermal.cas"), ("TRI_894", "tri_894.cas"),
                      ("HEXA_10K", "cav_hexa.cas"), ("TETRA_8K", "cav_tetra.cas")):
        ptest(test_dir, case, cas)


if __name__ == "__main__":
    main(*sys.argv[1:])
