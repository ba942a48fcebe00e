"""Seeded synthetic meshes and fields for the benchmark configurations.

Every generator returns a dict with exactly the arrays the reference's
7-argument Mesh constructor takes (fvmbase/Mesh.cpp:132-247):

    dim, nCells, nodes (nNodes x 3), faceCells (nFaces x 2),
    faceNodes (flat), faceNodeCount (nFaces), faceGroupSize (interior, then
    one entry per boundary group)

Conventions the reference relies on:
  * interior faces come first, then each boundary group contiguously;
  * every face's area vector points from c0 to c1 (for boundary faces
    outwards from the self cell c0 towards its ghost c1);
  * ghost cells are numbered nCells + t for the t-th boundary face.
Boundary groups are ordered x=0, x=1, y=0, y=1[, z=0, z=1] so that group 1
is x=0 and group 2 is x=1 (Dirichlet 300 / 400 in every configuration).

Meshes:
  quad_mesh(n)         n x n quads on the unit square, interior nodes jittered
  tet_mesh(m)          m^3-node lattice on the unit cube, each hex split into 6 tets
  hex_mesh(n)          n^3 hexes on the unit cube
Fields: lognormal, Gaussian random field (FFT), two-phase spherical inclusions.
"""
from __future__ import annotations

import numpy as np

# ---------------------------------------------------------------------------
# helpers


def _orient_2node(nodes, fn, c0xy, c1xy):
    """Swap node order of 2-node faces whose (dy,-dx) normal points from c1 to c0."""
    p0 = nodes[fn[:, 0], :2]
    p1 = nodes[fn[:, 1], :2]
    dr = p1 - p0
    area = np.stack([dr[:, 1], -dr[:, 0]], axis=1)
    flip = np.einsum("ij,ij->i", area, c1xy - c0xy) < 0
    fn[flip] = fn[flip][:, ::-1]
    return fn


def _orient_poly(nodes, fn, c0, c1):
    """Reverse node order of triangle/quad faces whose area points from c1 to c0."""
    if fn.shape[1] == 3:
        a = np.cross(nodes[fn[:, 1]] - nodes[fn[:, 0]], nodes[fn[:, 2]] - nodes[fn[:, 0]])
    else:
        a = np.cross(nodes[fn[:, 2]] - nodes[fn[:, 0]], nodes[fn[:, 3]] - nodes[fn[:, 1]])
    flip = np.einsum("ij,ij->i", a, c1 - c0) < 0
    fn[flip] = fn[flip][:, ::-1]
    return fn


def _jitter(nodes, h, amount, rng, interior):
    d = nodes.shape[1]
    j = rng.uniform(-amount * h, amount * h, size=(int(interior.sum()), d))
    nodes = nodes.copy()
    nodes[interior] += j
    return nodes


def _pack(dim, n_cells, nodes3, interior_fc, interior_fn, groups_fc, groups_fn):
    """Concatenate interior and boundary groups; number ghosts nCells + t."""
    fcs = [interior_fc]
    fns = [interior_fn]
    sizes = [len(interior_fc)]
    ghost = n_cells
    for fc, fn in zip(groups_fc, groups_fn):
        fc = fc.copy()
        fc[:, 1] = np.arange(ghost, ghost + len(fc))
        ghost += len(fc)
        fcs.append(fc)
        fns.append(fn)
        sizes.append(len(fc))
    fc = np.concatenate(fcs).astype(np.int32)
    fn = np.concatenate(fns).astype(np.int32)
    return {
        "dim": dim,
        "nCells": int(n_cells),
        "nodes": np.ascontiguousarray(nodes3, dtype=np.float64),
        "faceCells": np.ascontiguousarray(fc),
        "faceNodes": np.ascontiguousarray(fn.reshape(-1)),
        "faceNodeCount": np.full(len(fc), fn.shape[1], dtype=np.int32),
        "faceGroupSize": np.asarray(sizes, dtype=np.int32),
    }


# ---------------------------------------------------------------------------
# 2D quads


def quad_mesh(n: int, jitter: float = 0.2, seed: int = 0, ny: int | None = None) -> dict:
    """n x ny quads on [0,1]^2 (stored unstructured); interior nodes moved by
    U(-jitter*h, jitter*h) per axis (seeded)."""
    ny = n if ny is None else ny
    hx, hy = 1.0 / n, 1.0 / ny
    rng = np.random.default_rng(seed)
    I, J = np.meshgrid(np.arange(n + 1), np.arange(ny + 1), indexing="xy")  # node (i,j), i fastest
    xy = np.stack([I.ravel() * hx, J.ravel() * hy], axis=1)
    interior = (I.ravel() > 0) & (I.ravel() < n) & (J.ravel() > 0) & (J.ravel() < ny)
    if jitter > 0:
        j = rng.uniform(-1.0, 1.0, size=(int(interior.sum()), 2)) * np.array([jitter * hx, jitter * hy])
        xy[interior] += j
    nodes = np.zeros((len(xy), 3))
    nodes[:, :2] = xy
    nid = lambda i, j: j * (n + 1) + i  # noqa: E731
    cid = lambda i, j: j * n + i  # noqa: E731
    # interior vertical faces: between (i-1,j) and (i,j), i = 1..n-1
    iv, jv = np.meshgrid(np.arange(1, n), np.arange(ny), indexing="xy")
    iv, jv = iv.ravel(), jv.ravel()
    fc_v = np.stack([cid(iv - 1, jv), cid(iv, jv)], axis=1)
    fn_v = np.stack([nid(iv, jv), nid(iv, jv + 1)], axis=1)
    # interior horizontal faces: between (i,j-1) and (i,j), j = 1..ny-1
    ih, jh = np.meshgrid(np.arange(n), np.arange(1, ny), indexing="xy")
    ih, jh = ih.ravel(), jh.ravel()
    fc_h = np.stack([cid(ih, jh - 1), cid(ih, jh)], axis=1)
    fn_h = np.stack([nid(ih + 1, jh), nid(ih, jh)], axis=1)
    fc_i = np.concatenate([fc_v, fc_h])
    fn_i = np.concatenate([fn_v, fn_h])
    # order interior faces by (c0, c1) for locality
    order = np.lexsort((fc_i[:, 1], fc_i[:, 0]))
    fc_i, fn_i = fc_i[order], fn_i[order]
    cen = _quad_centroids(nodes, n, ny)
    fn_i = _orient_2node(nodes, fn_i, cen[fc_i[:, 0]], cen[fc_i[:, 1]])
    js = np.arange(ny)
    is_ = np.arange(n)
    groups_fc, groups_fn = [], []
    # x=0, x=1, y=0, y=1
    for cells, fn in (
        (cid(0, js), np.stack([nid(0, js + 1), nid(0, js)], axis=1)),
        (cid(n - 1, js), np.stack([nid(n, js), nid(n, js + 1)], axis=1)),
        (cid(is_, 0), np.stack([nid(is_, 0), nid(is_ + 1, 0)], axis=1)),
        (cid(is_, ny - 1), np.stack([nid(is_ + 1, ny), nid(is_, ny)], axis=1)),
    ):
        fc = np.stack([cells, np.zeros_like(cells)], axis=1)
        # outward: from the cell centroid towards the face midpoint
        mid = 0.5 * (nodes[fn[:, 0], :2] + nodes[fn[:, 1], :2])
        fn = _orient_2node(nodes, fn.copy(), cen[cells], mid + (mid - cen[cells]))
        groups_fc.append(fc)
        groups_fn.append(fn)
    return _pack(2, n * ny, nodes, fc_i, fn_i, groups_fc, groups_fn)


def _quad_centroids(nodes, n, ny):
    xy = nodes[:, :2].reshape(ny + 1, n + 1, 2)
    c = 0.25 * (xy[:-1, :-1] + xy[:-1, 1:] + xy[1:, :-1] + xy[1:, 1:])
    return c.reshape(-1, 2)


# ---------------------------------------------------------------------------
# 3D tets (Kuhn split of a hex lattice)

_KUHN = [(0, 1, 2), (0, 2, 1), (1, 0, 2), (1, 2, 0), (2, 0, 1), (2, 1, 0)]


def tet_mesh(m: int, jitter: float = 0.15, seed: int = 1) -> dict:
    """m^3 nodes on [0,1]^3, (m-1)^3 hexes each split into 6 tets along the
    (0,0,0)-(1,1,1) diagonal (conforming), interior nodes jittered by
    U(-jitter*h, jitter*h) per axis."""
    n = m - 1
    h = 1.0 / n
    rng = np.random.default_rng(seed)
    a = np.arange(m)
    X, Y, Z = np.meshgrid(a, a, a, indexing="ij")  # node (i,j,k)
    X, Y, Z = X.transpose(2, 1, 0).ravel(), Y.transpose(2, 1, 0).ravel(), Z.transpose(2, 1, 0).ravel()
    nodes = np.stack([X, Y, Z], axis=1) * h  # node id = (k*m + j)*m + i
    interior = (X > 0) & (X < n) & (Y > 0) & (Y < n) & (Z > 0) & (Z < n)
    if jitter > 0:
        nodes[interior] += rng.uniform(-jitter * h, jitter * h, size=(int(interior.sum()), 3))
    nid = lambda i, j, k: (k * m + j) * m + i  # noqa: E731
    ci, cj, ck = np.meshgrid(np.arange(n), np.arange(n), np.arange(n), indexing="ij")
    ci, cj, ck = ci.transpose(2, 1, 0).ravel(), cj.transpose(2, 1, 0).ravel(), ck.transpose(2, 1, 0).ravel()
    tets = []
    for p in _KUHN:
        v = np.zeros((len(ci), 3), dtype=np.int64)
        off = [np.zeros(3, dtype=np.int64)]
        cur = np.zeros(3, dtype=np.int64)
        for ax in p:
            cur = cur.copy()
            cur[ax] += 1
            off.append(cur)
        verts = [nid(ci + o[0], cj + o[1], ck + o[2]) for o in off]
        tets.append(np.stack(verts, axis=1))
    # cell id = hex id * 6 + permutation index (keeps tets of a hex adjacent)
    tets = np.stack(tets, axis=1).reshape(-1, 4)
    n_cells = len(tets)
    return _simplicial_faces(3, nodes, tets, n_cells, h, n)


def _simplicial_faces(dim, nodes, tets, n_cells, h, n):
    local = np.array([[1, 2, 3], [0, 2, 3], [0, 1, 3], [0, 1, 2]])
    fnodes = tets[:, local].reshape(-1, 3)  # 4 faces per tet
    fcell = np.repeat(np.arange(n_cells, dtype=np.int64), 4)
    s = np.sort(fnodes, axis=1)
    key = (s[:, 0] << 42) | (s[:, 1] << 21) | s[:, 2]
    order = np.argsort(key, kind="stable")
    key_s = key[order]
    same_next = np.concatenate([key_s[1:] == key_s[:-1], [False]])
    first = np.flatnonzero(same_next)  # first of each interior pair
    cent = nodes[tets].mean(axis=1)
    # interior faces
    a, b = order[first], order[first + 1]
    c0 = np.minimum(fcell[a], fcell[b])
    c1 = np.maximum(fcell[a], fcell[b])
    fn_i = fnodes[a].copy()
    o = np.lexsort((c1, c0))
    c0, c1, fn_i = c0[o], c1[o], fn_i[o]
    fn_i = _orient_poly(nodes, fn_i, cent[c0], cent[c1])
    fc_i = np.stack([c0, c1], axis=1)
    # boundary faces: keys that appear once
    paired = np.zeros(len(order), dtype=bool)
    paired[first] = True
    paired[first + 1] = True
    single = order[~paired]
    bfn = fnodes[single]
    bcell = fcell[single]
    fcen = nodes[bfn].mean(axis=1)
    eps = 1e-9
    groups_fc, groups_fn = [], []
    for ax, val in ((0, 0.0), (0, 1.0), (1, 0.0), (1, 1.0), (2, 0.0), (2, 1.0)):
        sel = np.abs(fcen[:, ax] - val) < eps
        idx = np.flatnonzero(sel)
        idx = idx[np.argsort(bcell[idx], kind="stable")]
        cells = bcell[idx]
        fn = bfn[idx].copy()
        outward = fcen[idx] + (fcen[idx] - cent[cells])
        fn = _orient_poly(nodes, fn, cent[cells], outward)
        groups_fc.append(np.stack([cells, np.zeros_like(cells)], axis=1))
        groups_fn.append(fn)
    nb = sum(len(g) for g in groups_fc)
    if nb != len(single):
        raise RuntimeError("boundary faces not on the unit cube planes")
    return _pack(dim, n_cells, nodes, fc_i, fn_i, groups_fc, groups_fn)


# ---------------------------------------------------------------------------
# 3D hexes


def hex_mesh(n: int, jitter: float = 0.0, seed: int = 3) -> dict:
    """n^3 hexes on [0,1]^3 (cell id = (k*n + j)*n + i)."""
    m = n + 1
    h = 1.0 / n
    a = np.arange(m)
    X, Y, Z = np.meshgrid(a, a, a, indexing="ij")
    X, Y, Z = X.transpose(2, 1, 0).ravel(), Y.transpose(2, 1, 0).ravel(), Z.transpose(2, 1, 0).ravel()
    nodes = np.stack([X, Y, Z], axis=1).astype(np.float64) * h
    if jitter > 0:
        rng = np.random.default_rng(seed)
        interior = (X > 0) & (X < n) & (Y > 0) & (Y < n) & (Z > 0) & (Z < n)
        nodes[interior] += rng.uniform(-jitter * h, jitter * h, size=(int(interior.sum()), 3))
    nid = lambda i, j, k: (k * m + j) * m + i  # noqa: E731
    cid = lambda i, j, k: (k * n + j) * n + i  # noqa: E731

    fcs, fns = [], []
    # faces normal to x at i = 1..n-1: quad nodes in the (j,k) plane ordered so the normal is +x
    I, J, K = np.meshgrid(np.arange(1, n), np.arange(n), np.arange(n), indexing="ij")
    I, J, K = I.ravel(), J.ravel(), K.ravel()
    fcs.append(np.stack([cid(I - 1, J, K), cid(I, J, K)], axis=1))
    fns.append(np.stack([nid(I, J, K), nid(I, J + 1, K), nid(I, J + 1, K + 1), nid(I, J, K + 1)], axis=1))
    I, J, K = np.meshgrid(np.arange(n), np.arange(1, n), np.arange(n), indexing="ij")
    I, J, K = I.ravel(), J.ravel(), K.ravel()
    fcs.append(np.stack([cid(I, J - 1, K), cid(I, J, K)], axis=1))
    fns.append(np.stack([nid(I, J, K), nid(I, J, K + 1), nid(I + 1, J, K + 1), nid(I + 1, J, K)], axis=1))
    I, J, K = np.meshgrid(np.arange(n), np.arange(n), np.arange(1, n), indexing="ij")
    I, J, K = I.ravel(), J.ravel(), K.ravel()
    fcs.append(np.stack([cid(I, J, K - 1), cid(I, J, K)], axis=1))
    fns.append(np.stack([nid(I, J, K), nid(I + 1, J, K), nid(I + 1, J + 1, K), nid(I, J + 1, K)], axis=1))
    fc_i = np.concatenate(fcs)
    fn_i = np.concatenate(fns)
    o = np.lexsort((fc_i[:, 1], fc_i[:, 0]))
    fc_i, fn_i = fc_i[o], fn_i[o]
    cent = _hex_centroids(nodes, n)
    fn_i = _orient_poly(nodes, fn_i, cent[fc_i[:, 0]], cent[fc_i[:, 1]])
    groups_fc, groups_fn = [], []
    J, K = np.meshgrid(np.arange(n), np.arange(n), indexing="ij")
    J, K = J.T.ravel(), K.T.ravel()
    for i, cells in ((0, cid(0, J, K)), (n, cid(n - 1, J, K))):
        fn = np.stack([nid(i, J, K), nid(i, J + 1, K), nid(i, J + 1, K + 1), nid(i, J, K + 1)], axis=1)
        groups_fc.append(cells)
        groups_fn.append(fn)
    I, K = np.meshgrid(np.arange(n), np.arange(n), indexing="ij")
    I, K = I.T.ravel(), K.T.ravel()
    for j, cells in ((0, cid(I, 0, K)), (n, cid(I, n - 1, K))):
        fn = np.stack([nid(I, j, K), nid(I, j, K + 1), nid(I + 1, j, K + 1), nid(I + 1, j, K)], axis=1)
        groups_fc.append(cells)
        groups_fn.append(fn)
    I, J = np.meshgrid(np.arange(n), np.arange(n), indexing="ij")
    I, J = I.T.ravel(), J.T.ravel()
    for k, cells in ((0, cid(I, J, 0)), (n, cid(I, J, n - 1))):
        fn = np.stack([nid(I, J, k), nid(I + 1, J, k), nid(I + 1, J + 1, k), nid(I, J + 1, k)], axis=1)
        groups_fc.append(cells)
        groups_fn.append(fn)
    out_fc, out_fn = [], []
    for cells, fn in zip(groups_fc, groups_fn):
        o = np.argsort(cells, kind="stable")
        cells, fn = cells[o], fn[o]
        fcen = nodes[fn].mean(axis=1)
        fn = _orient_poly(nodes, fn.copy(), cent[cells], fcen + (fcen - cent[cells]))
        out_fc.append(np.stack([cells, np.zeros_like(cells)], axis=1))
        out_fn.append(fn)
    return _pack(3, n ** 3, nodes, fc_i, fn_i, out_fc, out_fn)


def _hex_centroids(nodes, n):
    m = n + 1
    p = nodes.reshape(m, m, m, 3)  # [k][j][i]
    c = (p[:-1, :-1, :-1] + p[:-1, :-1, 1:] + p[:-1, 1:, :-1] + p[:-1, 1:, 1:] +
         p[1:, :-1, :-1] + p[1:, :-1, 1:] + p[1:, 1:, :-1] + p[1:, 1:, 1:]) / 8.0
    return c.reshape(-1, 3)


# ---------------------------------------------------------------------------
# geometry helpers for fields


def cell_centers(mesh: dict) -> np.ndarray:
    """Node-average cell centres (self cells), used to sample fields."""
    n = mesh["nCells"]
    fc = mesh["faceCells"]
    fnc = mesh["faceNodeCount"]
    k = int(fnc[0])
    fn = mesh["faceNodes"].reshape(-1, k)
    nodes = mesh["nodes"]
    fcen = nodes[fn].mean(axis=1)
    acc = np.zeros((n, 3))
    cnt = np.zeros(n)
    for s in (0, 1):
        c = fc[:, s]
        ok = c < n
        np.add.at(acc, c[ok], fcen[ok])
        np.add.at(cnt, c[ok], 1)
    return acc / cnt[:, None]


def n_ghost(mesh: dict) -> int:
    return int(mesh["faceGroupSize"][1:].sum())


def extend_to_ghosts(mesh: dict, values: np.ndarray) -> np.ndarray:
    """Self-cell values extended with each ghost taking its neighbour's value."""
    n = mesh["nCells"]
    nb = n_ghost(mesh)
    out = np.empty(n + nb)
    out[:n] = values
    fc = mesh["faceCells"]
    ni = int(mesh["faceGroupSize"][0])
    out[fc[ni:, 1]] = values[fc[ni:, 0]]
    return out


def lognormal_field(n: int, sigma: float, seed: int, mu: float = 0.0) -> np.ndarray:
    return np.random.default_rng(seed).lognormal(mu, sigma, size=n)


def uniform_field(n: int, lo: float, hi: float, seed: int) -> np.ndarray:
    return np.random.default_rng(seed).uniform(lo, hi, size=n)


def gaussian_random_field(points: np.ndarray, corr_len: float, seed: int, grid: int = 64) -> np.ndarray:
    """Gaussian random field with a Gaussian spectrum (correlation length
    corr_len) generated by FFT on a grid^3 lattice of the unit cube, sampled
    at points by trilinear interpolation and scaled to [-1, 1]."""
    rng = np.random.default_rng(seed)
    k = np.fft.fftfreq(grid, d=1.0 / grid) * 2 * np.pi
    KX, KY, KZ = np.meshgrid(k, k, k, indexing="ij")
    spec = np.exp(-0.25 * corr_len ** 2 * (KX ** 2 + KY ** 2 + KZ ** 2))
    noise = rng.standard_normal((grid, grid, grid)) + 1j * rng.standard_normal((grid, grid, grid))
    f = np.real(np.fft.ifftn(np.sqrt(spec) * noise))
    f = (f - f.min()) / (f.max() - f.min()) * 2.0 - 1.0
    g = np.clip(points, 0.0, 1.0) * (grid - 1)
    i0 = np.clip(np.floor(g).astype(np.int64), 0, grid - 2)
    t = g - i0
    out = np.zeros(len(points))
    for dx in (0, 1):
        for dy in (0, 1):
            for dz in (0, 1):
                w = (t[:, 0] if dx else 1 - t[:, 0]) * (t[:, 1] if dy else 1 - t[:, 1]) * \
                    (t[:, 2] if dz else 1 - t[:, 2])
                out += w * f[i0[:, 0] + dx, i0[:, 1] + dy, i0[:, 2] + dz]
    lo, hi = out.min(), out.max()
    return (out - lo) / (hi - lo) * 2.0 - 1.0 if hi > lo else out


def sphere_inclusions(points: np.ndarray, seed: int, fraction: float = 0.3,
                      rmin: float = 0.02, rmax: float = 0.08, k_in: float = 1e4,
                      k_out: float = 1.0) -> np.ndarray:
    """Two-phase conductivity: random spheres (radii U[rmin, rmax]) placed
    until the covered fraction of cells reaches `fraction`."""
    rng = np.random.default_rng(seed)
    inside = np.zeros(len(points), dtype=bool)
    # bin points on a coarse grid to test spheres locally
    nb = 16
    cell = np.clip((points * nb).astype(np.int64), 0, nb - 1)
    key = (cell[:, 0] * nb + cell[:, 1]) * nb + cell[:, 2]
    order = np.argsort(key)
    starts = np.searchsorted(key[order], np.arange(nb ** 3 + 1))
    while inside.mean() < fraction:
        c = rng.uniform(0, 1, 3)
        r = rng.uniform(rmin, rmax)
        lo = np.clip(((c - r) * nb).astype(int), 0, nb - 1)
        hi = np.clip(((c + r) * nb).astype(int), 0, nb - 1)
        for i in range(lo[0], hi[0] + 1):
            for j in range(lo[1], hi[1] + 1):
                for kk in range(lo[2], hi[2] + 1):
                    b = (i * nb + j) * nb + kk
                    idx = order[starts[b]:starts[b + 1]]
                    if len(idx):
                        d2 = ((points[idx] - c) ** 2).sum(axis=1)
                        inside[idx[d2 <= r * r]] = True
    return np.where(inside, k_in, k_out)


# ---------------------------------------------------------------------------
# benchmark workloads


def config0(n: int = 256, seed: int = 0) -> tuple[dict, dict]:
    """Steady 2D heat conduction: n x n jittered quads (20%), k ~ lognormal(0,1),
    s ~ U[0,1]; x=0 -> 300, x=1 -> 400, y faces adiabatic."""
    mesh = quad_mesh(n, jitter=0.2, seed=seed)
    N = mesh["nCells"]
    k = lognormal_field(N, 1.0, seed + 100)
    s = uniform_field(N, 0.0, 1.0, seed + 200)
    return mesh, {"k": k, "s": s, "bc": {1: ("T", 300.0), 2: ("T", 400.0)}}


def config1(m: int = 64, seed: int = 1) -> tuple[dict, dict]:
    """Steady 3D heat conduction on the Kuhn-split m^3-node tet lattice
    (jitter 15%); k = 10^(1.5 g), g a Gaussian random field (corr. length
    0.05) scaled to [-1,1] (contrast 1e3); s ~ U[0,1]."""
    mesh = tet_mesh(m, jitter=0.15, seed=seed)
    N = mesh["nCells"]
    pts = cell_centers(mesh)
    g = gaussian_random_field(pts, 0.05, seed + 100)
    k = 10.0 ** (1.5 * g)
    s = uniform_field(N, 0.0, 1.0, seed + 200)
    return mesh, {"k": k, "s": s, "bc": {1: ("T", 300.0), 2: ("T", 400.0)}}


def config3(n: int = 100, seed: int = 3) -> tuple[dict, dict]:
    """Two-phase 3D hex mesh: spheres (r in [0.02,0.08], 30% volume) with
    k = 1e4 inside, 1 outside; s ~ U[0,1]."""
    mesh = hex_mesh(n)
    N = mesh["nCells"]
    pts = cell_centers(mesh)
    k = sphere_inclusions(pts, seed + 100)
    s = uniform_field(N, 0.0, 1.0, seed + 200)
    return mesh, {"k": k, "s": s, "bc": {1: ("T", 300.0), 2: ("T", 400.0)}}


def config4(n: int = 200, seed: int = 4) -> tuple[dict, dict]:
    """Transient 3D hex mesh: k ~ lognormal(0,1), rho*c ~ U[0.5,2], T0 = 300,
    x=1 Dirichlet 400, other faces adiabatic."""
    mesh = hex_mesh(n)
    N = mesh["nCells"]
    k = lognormal_field(N, 1.0, seed + 100)
    rc = uniform_field(N, 0.5, 2.0, seed + 300)
    return mesh, {"k": k, "s": np.zeros(N), "rc": rc, "bc": {1: ("q", 0.0), 2: ("T", 400.0)}}


def config2(n_meshes: int = 512, seed: int = 2, lo: int = 32, hi: int = 256) -> list[tuple[dict, dict]]:
    """Batch of independent jittered quad meshes with sides drawn from
    U{lo..hi}: mesh i uses seed + i for its jitter and fields; k ~
    lognormal(0, 1.5), s ~ U[0,1], the boundary conditions of config0."""
    rng = np.random.default_rng(seed)
    sides = rng.integers(lo, hi + 1, n_meshes)
    out = []
    for i, n in enumerate(sides):
        sd = seed + i
        mesh = quad_mesh(int(n), jitter=0.2, seed=sd)
        N = mesh["nCells"]
        k = lognormal_field(N, 1.5, sd + 100)
        s = uniform_field(N, 0.0, 1.0, sd + 200)
        out.append((mesh, {"k": k, "s": s, "bc": {1: ("T", 300.0), 2: ("T", 400.0)}}))
    return out
