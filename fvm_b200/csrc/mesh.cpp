// Host mesh setup. Compiled with -ffp-contract=off: every product and sum
// below must round on its own, as the reference's scalar C++ does, so that
// geometry, matrix coefficients and hence the AMG aggregation match it bit
// for bit.
#include "mesh.hpp"

#include <cmath>
#include <cstring>

namespace fvm {

namespace {

inline void sub3(const double* a, const double* b, double* r) {
  r[0] = a[0] - b[0];
  r[1] = a[1] - b[1];
  r[2] = a[2] - b[2];
}
// dot product evaluated left to right, (a0 b0 + a1 b1) + a2 b2
inline double dot3(const double* a, const double* b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }
inline void cross3(const double* a, const double* b, double* c) {
  c[0] = a[1] * b[2] - a[2] * b[1];
  c[1] = a[2] * b[0] - a[0] * b[2];
  c[2] = a[0] * b[1] - a[1] * b[0];
}

}  // namespace

HostMesh* make_mesh(int dim, int nCells, int nNodes, const double* xyz, int nFaces,
                    const int* faceCells, const int* faceNodes, const int* faceNodeCount,
                    int nGroups, const int* groupSize) {
  FVM_REQUIRE(dim == 2 || dim == 3, kBadArgument, "mesh dimension must be 2 or 3");
  FVM_REQUIRE(nCells > 0 && nNodes > 0 && nFaces > 0, kBadArgument, "empty mesh");
  FVM_REQUIRE(nGroups >= 1, kBadArgument, "at least the interior face group is required");
  FVM_REQUIRE(xyz && faceCells && faceNodes && faceNodeCount && groupSize, kBadArgument,
              "null mesh array");
  HostMesh* m = new HostMesh();
  try {
    m->dim = dim;
    m->nCells = nCells;
    m->nNodes = nNodes;
    m->nFaces = nFaces;
    m->xyz.assign(xyz, xyz + 3 * (size_t)nNodes);
    m->faceCells.assign(faceCells, faceCells + 2 * (size_t)nFaces);
    m->faceNodes.nRows = nFaces;
    m->faceNodes.row.resize(nFaces + 1);
    m->faceNodes.row[0] = 0;
    for (int f = 0; f < nFaces; f++) {
      FVM_REQUIRE(faceNodeCount[f] >= 2, kBadMesh, "face with fewer than 2 nodes");
      m->faceNodes.row[f + 1] = m->faceNodes.row[f] + faceNodeCount[f];
    }
    m->faceNodes.col.assign(faceNodes, faceNodes + m->faceNodes.row[nFaces]);
    int offset = 0;
    int nBoundary = 0;
    for (int g = 0; g < nGroups; g++) {
      FaceGroup fg;
      fg.id = g;
      fg.offset = offset;
      fg.size = groupSize[g];
      fg.type = (g == 0) ? "interior" : "wall";
      FVM_REQUIRE(fg.size >= 0, kBadMesh, "negative face group size");
      offset += fg.size;
      if (g > 0) nBoundary += fg.size;
      m->groups.push_back(fg);
    }
    FVM_REQUIRE(offset == nFaces, kBadMesh, "face group sizes do not add up to the face count");
    m->nGhost = nBoundary;
    m->build();
  } catch (...) {
    delete m;
    throw;
  }
  return m;
}

void HostMesh::build() {
  const int nAll = nTotalCells();
  for (int f = 0; f < nFaces; f++) {
    const int c0 = faceCells[2 * f], c1 = faceCells[2 * f + 1];
    FVM_REQUIRE(c0 >= 0 && c0 < nAll && c1 >= 0 && c1 < nAll && c0 != c1, kBadMesh,
                "face-cell index out of range");
  }
  for (int k = 0; k < faceNodes.nnz(); k++)
    FVM_REQUIRE(faceNodes.col[k] >= 0 && faceNodes.col[k] < nNodes, kBadMesh,
                "face-node index out of range");
  for (size_t g = 1; g < groups.size(); g++)
    for (int f = groups[g].offset; f < groups[g].offset + groups[g].size; f++)
      FVM_REQUIRE(faceCells[2 * f] < nCells && faceCells[2 * f + 1] >= nCells, kBadMesh,
                  "boundary face must join a self cell (c0) to a ghost cell (c1)");
  buildConnectivity();
  buildGeometry();
  buildGradientWeights();
}

// cellFaces is the transpose of faceCells (faces ascending within a row);
// cellCells lists, for each cell, the other cells of its faces in the order
// they are first met walking the cell's faces in ascending order and each
// face's (c0, c1) pair -- the column order of the reference's
// CRConnectivity::multiply(faceCells, implicitDiagonal=true).
void HostMesh::buildConnectivity() {
  const int nAll = nTotalCells();
  cellFaces.nRows = nAll;
  cellFaces.row.assign(nAll + 1, 0);
  for (int f = 0; f < nFaces; f++) {
    cellFaces.row[faceCells[2 * f] + 1]++;
    cellFaces.row[faceCells[2 * f + 1] + 1]++;
  }
  for (int i = 0; i < nAll; i++) cellFaces.row[i + 1] += cellFaces.row[i];
  cellFaces.col.resize(cellFaces.row[nAll]);
  {
    std::vector<int> cursor(cellFaces.row.begin(), cellFaces.row.end() - 1);
    for (int f = 0; f < nFaces; f++) {
      cellFaces.col[cursor[faceCells[2 * f]]++] = f;
      cellFaces.col[cursor[faceCells[2 * f + 1]]++] = f;
    }
  }
  cellCells.nRows = nAll;
  cellCells.row.assign(nAll + 1, 0);
  cellCells.col.clear();
  cellCells.col.reserve(cellFaces.col.size());
  std::vector<int> stamp(nAll, -1);
  for (int i = 0; i < nAll; i++) {
    stamp[i] = i;  // the diagonal is implicit
    for (int k = cellFaces.row[i]; k < cellFaces.row[i + 1]; k++) {
      const int f = cellFaces.col[k];
      for (int s = 0; s < 2; s++) {
        const int c = faceCells[2 * f + s];
        if (stamp[c] != i) {
          stamp[c] = i;
          cellCells.col.push_back(c);
        }
      }
    }
    cellCells.row[i + 1] = (int)cellCells.col.size();
  }
  pairToCol.resize(2 * (size_t)nFaces);
  for (int f = 0; f < nFaces; f++) {
    const int c0 = faceCells[2 * f], c1 = faceCells[2 * f + 1];
    int p0 = -1, p1 = -1;
    for (int k = cellCells.row[c0]; k < cellCells.row[c0 + 1]; k++)
      if (cellCells.col[k] == c1) {
        p0 = k;
        break;
      }
    for (int k = cellCells.row[c1]; k < cellCells.row[c1 + 1]; k++)
      if (cellCells.col[k] == c0) {
        p1 = k;
        break;
      }
    FVM_REQUIRE(p0 >= 0 && p1 >= 0, kBadMesh, "face pair missing from cell connectivity");
    pairToCol[2 * f] = p0;
    pairToCol[2 * f + 1] = p1;
  }
}

void HostMesh::buildGeometry() {
  const int nAll = nTotalCells();
  faceArea.assign(3 * (size_t)nFaces, 0.0);
  faceAreaMag.assign(nFaces, 0.0);
  faceCentroid.assign(3 * (size_t)nFaces, 0.0);
  cellCentroid.assign(3 * (size_t)nAll, 0.0);
  cellVolume.assign(nAll, 0.0);
  const double half = 0.5;

  // face area vectors (MeshMetricsCalculator_impl.h:238-304)
  for (int f = 0; f < nFaces; f++) {
    const int nn = faceNodes.count(f);
    const int* fn = &faceNodes.col[faceNodes.row[f]];
    double* fa = &faceArea[3 * f];
    if (nn == 2) {
      double dr[3];
      sub3(&xyz[3 * fn[1]], &xyz[3 * fn[0]], dr);
      fa[0] = dr[1];
      fa[1] = -dr[0];
      fa[2] = 0.;
    } else if (nn == 3) {
      double d10[3], d20[3], c[3];
      sub3(&xyz[3 * fn[1]], &xyz[3 * fn[0]], d10);
      sub3(&xyz[3 * fn[2]], &xyz[3 * fn[0]], d20);
      cross3(d10, d20, c);
      for (int d = 0; d < 3; d++) fa[d] = half * c[d];
    } else if (nn == 4) {
      double d20[3], d31[3], c[3];
      sub3(&xyz[3 * fn[2]], &xyz[3 * fn[0]], d20);
      sub3(&xyz[3 * fn[3]], &xyz[3 * fn[1]], d31);
      cross3(d20, d31, c);
      for (int d = 0; d < 3; d++) fa[d] = half * c[d];
    } else {
      fa[0] = fa[1] = fa[2] = 0.;
      for (int k = 0; k < nn; k++) {
        const double* p0 = &xyz[3 * fn[k]];
        const double* p1 = &xyz[3 * fn[(k + 1) % nn]];
        double xm[3], dr[3];
        for (int d = 0; d < 3; d++) xm[d] = 0.5 * (p1[d] + p0[d]);
        sub3(p1, p0, dr);
        fa[0] += xm[1] * dr[2];
        fa[1] += xm[2] * dr[0];
        fa[2] += xm[0] * dr[1];
      }
    }
    faceAreaMag[f] = std::sqrt(dot3(fa, fa));
  }

  // face centroids with the non-planar correction (:58-120)
  const double twoThirds = 2. / 3.;
  for (int f = 0; f < nFaces; f++) {
    const int nn = faceNodes.count(f);
    const int* fn = &faceNodes.col[faceNodes.row[f]];
    double* fc = &faceCentroid[3 * f];
    for (int d = 0; d < 3; d++) fc[d] = xyz[3 * fn[0] + d];
    for (int k = 1; k < nn; k++)
      for (int d = 0; d < 3; d++) fc[d] += xyz[3 * fn[k] + d];
    for (int d = 0; d < 3; d++) fc[d] /= double(nn);
    if (nn > 3) {
      double en[3];
      for (int d = 0; d < 3; d++) en[d] = faceArea[3 * f + d] / faceAreaMag[f];
      double denom = 0.0;
      double cfc[3] = {0., 0., 0.};
      for (int k = 0; k < nn; k++) {
        const double* p0 = &xyz[3 * fn[k]];
        const double* p1 = &xyz[3 * fn[(k + 1) % nn]];
        double rc0[3], rc1[3], c[3], tri[3], xm[3];
        sub3(p0, fc, rc0);
        sub3(p1, fc, rc1);
        cross3(rc0, rc1, c);
        for (int d = 0; d < 3; d++) tri[d] = half * c[d];
        const double triP = dot3(tri, en);
        for (int d = 0; d < 3; d++) xm[d] = half * (p0[d] + p1[d]);
        for (int d = 0; d < 3; d++) cfc[d] += (twoThirds * (xm[d] - fc[d])) * triP;
        denom += triP;
      }
      for (int d = 0; d < 3; d++) cfc[d] /= denom;
      for (int d = 0; d < 3; d++) fc[d] += cfc[d];
    }
  }

  // cell centroids: area-weighted face centroids (:128-236)
  std::vector<double> weight(nAll, 0.0);
  for (int f = 0; f < nFaces; f++)
    for (int s = 0; s < 2; s++) {
      const int c = faceCells[2 * f + s];
      for (int d = 0; d < 3; d++) cellCentroid[3 * c + d] += faceCentroid[3 * f + d] * faceAreaMag[f];
      weight[c] += faceAreaMag[f];
    }
  for (int c = 0; c < nCells; c++)
    for (int d = 0; d < 3; d++) cellCentroid[3 * c + d] /= weight[c];
  for (size_t g = 1; g < groups.size(); g++) {
    const FaceGroup& fg = groups[g];
    if (!isBoundaryGroupType(fg.type)) continue;
    for (int f = fg.offset; f < fg.offset + fg.size; f++) {
      const int c0 = faceCells[2 * f], c1 = faceCells[2 * f + 1];
      if (fg.type == "symmetry") {
        double en[3], dr0[3], dr1[3];
        for (int d = 0; d < 3; d++) en[d] = faceArea[3 * f + d] / faceAreaMag[f];
        sub3(&faceCentroid[3 * f], &cellCentroid[3 * c0], dr0);
        const double dn = dot3(dr0, en);
        for (int d = 0; d < 3; d++) dr1[d] = dr0[d] - (2. * dn) * en[d];
        for (int d = 0; d < 3; d++)
          cellCentroid[3 * c1 + d] = (cellCentroid[3 * c0 + d] + dr0[d]) - dr1[d];
      } else {
        for (int d = 0; d < 3; d++) cellCentroid[3 * c1 + d] = faceCentroid[3 * f + d];
      }
    }
  }

  // cell volumes by the divergence theorem (:392-460)
  const double dimD = double(dim);
  for (int f = 0; f < nFaces; f++) {
    const int c0 = faceCells[2 * f], c1 = faceCells[2 * f + 1];
    double r[3];
    sub3(&faceCentroid[3 * f], &cellCentroid[3 * c0], r);
    cellVolume[c0] += dot3(r, &faceArea[3 * f]) / dimD;
    sub3(&faceCentroid[3 * f], &cellCentroid[3 * c1], r);
    cellVolume[c1] -= dot3(r, &faceArea[3 * f]) / dimD;
  }
  for (size_t g = 1; g < groups.size(); g++) {
    const FaceGroup& fg = groups[g];
    if (!isBoundaryGroupType(fg.type)) continue;
    for (int f = fg.offset; f < fg.offset + fg.size; f++)
      cellVolume[faceCells[2 * f + 1]] = cellVolume[faceCells[2 * f]];
  }
  for (int c = 0; c < nCells; c++)
    FVM_REQUIRE(cellVolume[c] > 0.0, kBadMesh, "non-positive cell volume (check face orientation)");
}

// Least-squares gradient weights (GradientModel.h:126-436). Entry k of row
// i of cellCells gets a 3-vector w so that grad_i = sum_k w_k (x_j - x_i).
void HostMesh::buildGradientWeights() {
  const int nnzAll = cellCells.nnz();
  gradCoeff.assign(3 * (size_t)nnzAll, 0.0);
  std::vector<char> degenerate(nTotalCells(), 0);
  auto faceDs = [&](int f, double* ds) {
    sub3(&cellCentroid[3 * faceCells[2 * f + 1]], &cellCentroid[3 * faceCells[2 * f]], ds);
    return std::sqrt(dot3(ds, ds));
  };
  for (int f = 0; f < nFaces; f++) {
    double ds[3];
    const double m = faceDs(f, ds);
    double* w01 = &gradCoeff[3 * (size_t)pairToCol[2 * f]];
    double* w10 = &gradCoeff[3 * (size_t)pairToCol[2 * f + 1]];
    for (int d = 0; d < 3; d++) {
      w01[d] = ds[d] / m;
      w10[d] = (-ds[d]) / m;
    }
  }
  for (int c = 0; c < nCells; c++) {
    const int b = cellCells.row[c], e = cellCells.row[c + 1];
    if (dim == 3) {
      double Ixx = 0, Iyy = 0, Izz = 0, Ixy = 0, Ixz = 0, Iyz = 0;
      for (int k = b; k < e; k++) {
        const double* w = &gradCoeff[3 * (size_t)k];
        Ixx += w[0] * w[0];
        Iyy += w[1] * w[1];
        Izz += w[2] * w[2];
        Ixy += w[0] * w[1];
        Ixz += w[0] * w[2];
        Iyz += w[1] * w[2];
      }
      const double det = Ixx * (Iyy * Izz - Iyz * Iyz) - Ixy * (Ixy * Izz - Iyz * Ixz) +
                         Ixz * (Ixy * Iyz - Iyy * Ixz);
      if (det > 1e-6) {
        const double Kxx = (Iyy * Izz - Iyz * Iyz) / det;
        const double Kxy = -(Ixy * Izz - Iyz * Ixz) / det;
        const double Kxz = (Ixy * Iyz - Iyy * Ixz) / det;
        const double Kyy = (Ixx * Izz - Ixz * Ixz) / det;
        const double Kyz = -(Ixx * Iyz - Ixy * Ixz) / det;
        const double Kzz = (Ixx * Iyy - Ixy * Ixy) / det;
        for (int k = b; k < e; k++) {
          double* w = &gradCoeff[3 * (size_t)k];
          const double d0 = w[0], d1 = w[1], d2 = w[2];
          w[0] = Kxx * d0 + Kxy * d1 + Kxz * d2;
          w[1] = Kxy * d0 + Kyy * d1 + Kyz * d2;
          w[2] = Kxz * d0 + Kyz * d1 + Kzz * d2;
        }
      } else {
        degenerate[c] = 1;
      }
    } else {
      double Ixx = 0, Iyy = 0, Ixy = 0;
      for (int k = b; k < e; k++) {
        const double* w = &gradCoeff[3 * (size_t)k];
        Ixx += w[0] * w[0];
        Iyy += w[1] * w[1];
        Ixy += w[0] * w[1];
      }
      const double det = Ixx * Iyy - Ixy * Ixy;
      if (det > 1e-26) {
        const double Kxx = Iyy / det;
        const double Kxy = -Ixy / det;
        const double Kyy = Ixx / det;
        for (int k = b; k < e; k++) {
          double* w = &gradCoeff[3 * (size_t)k];
          const double d0 = w[0], d1 = w[1];
          w[0] = Kxx * d0 + Kxy * d1;
          w[1] = Kxy * d0 + Kyy * d1;
          w[2] = 0;
        }
      } else {
        degenerate[c] = 1;
      }
    }
  }
  for (int f = 0; f < nFaces; f++) {
    double ds[3];
    const double m = faceDs(f, ds);
    double* w01 = &gradCoeff[3 * (size_t)pairToCol[2 * f]];
    double* w10 = &gradCoeff[3 * (size_t)pairToCol[2 * f + 1]];
    for (int d = 0; d < 3; d++) {
      w01[d] /= m;
      w10[d] /= m;
    }
  }
  for (int f = 0; f < nFaces; f++) {
    const int c0 = faceCells[2 * f], c1 = faceCells[2 * f + 1];
    if (degenerate[c0]) {
      double* w = &gradCoeff[3 * (size_t)pairToCol[2 * f]];
      for (int d = 0; d < 3; d++) w[d] = (0.5 * faceArea[3 * f + d]) / cellVolume[c0];
    }
    if (degenerate[c1]) {
      double* w = &gradCoeff[3 * (size_t)pairToCol[2 * f + 1]];
      for (int d = 0; d < 3; d++) w[d] = (-0.5 * faceArea[3 * f + d]) / cellVolume[c1];
    }
  }
}

}  // namespace fvm
