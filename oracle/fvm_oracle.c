/*
 * fvm_oracle.c -- CPU restatement of the reference's scalar heat-diffusion
 * hot path (c-PRIMED/fvm, fvmbase module).
 *
 * TEST INFRASTRUCTURE ONLY. Imported (through oracle/oracle_c.py) by
 * tests/, by __graft_entry__.smoke() and by the CPU-baseline leg of
 * bench.py, as the checker. The product (fvm_b200) never links or calls it.
 *
 * Plain C99, single thread, compiled with -ffp-contract=off so that every
 * product and sum rounds as the reference's scalar C++ does. Every routine
 * follows the reference routine cited beside it, operation for operation,
 * with its visiting order, tie-breaking and floating-point evaluation
 * order, so that integer results (connectivity, aggregation) are identical
 * and floating-point results agree bit for bit with the reference built
 * from its own sources (tests/test_oracle_c.py checks both against it and
 * against the golden vectors).
 *
 * Paths below are relative to src/fvm/src/modules/fvmbase of the reference.
 *
 * The one routine that has no reference counterpart is orc_multicolor: the
 * deterministic colouring used by the GPU multicolour smoothers, restated
 * from its definition (greedy in row order vs greedy in smallest-last
 * order, fewer colours win, row order on a tie) to pin the product's
 * colouring.
 */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#define ORC_API __attribute__((visibility("default")))
#define ORC_MAX_LEVELS 64

static char g_err[256];
ORC_API const char* orc_last_error(void) { return g_err; }
static int fail(const char* msg) {
  snprintf(g_err, sizeof g_err, "%s", msg);
  return 1;
}

static void* xcalloc(size_t n, size_t sz) {
  void* p = calloc(n ? n : 1, sz);
  if (!p) {
    fprintf(stderr, "fvm_oracle: out of memory\n");
    abort();
  }
  return p;
}

/* ------------------------------------------------------------------ */
/* small vector helpers in the reference's evaluation order (Vector.h)  */
/* ------------------------------------------------------------------ */
static double dot3(const double* a, const double* b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }
static double mag3(const double* a) { return sqrt(dot3(a, a)); }
static void cross3(const double* a, const double* b, double* c) {
  c[0] = a[1] * b[2] - a[2] * b[1];
  c[1] = a[2] * b[0] - a[0] * b[2];
  c[2] = a[0] * b[1] - a[1] * b[0];
}

/* ================================================================== */
/* Mesh: sites, connectivity, metrics                                  */
/* ================================================================== */

typedef struct {
  int dim, nCells, nGhost, nNodes, nFaces, nGroups;
  double* xyz;        /* 3 * nNodes */
  int* faceCells;     /* 2 * nFaces */
  int* fnRow;         /* nFaces + 1 */
  int* fnCol;
  int* groupStart;    /* nGroups + 1 face offsets; group 0 interior */
  int* groupId;       /* id of group g (g for the 7-argument constructor) */
  int* groupDefaultT; /* 1: default BC SpecifiedTemperature (inlet/outlet types) */
  /* cellCells over all cells (self + ghost) */
  int* ccRow;
  int* ccCol;
  int* pairToCol;     /* 2 * nFaces */
  /* metrics */
  double *area, *areaMag, *faceCentroid, *cellCentroid, *volume;
} orc_mesh;

/* Mesh::Mesh (Mesh.cpp:132-247): group 0 interior, groups 1.. "wall",
 * cells = nCells self + one ghost per boundary face. cellCells =
 * cellFaces x faceCells with implicit diagonal (Mesh.cpp:453-492,
 * CRConnectivity.cpp:73-94 transpose, :167-270 multiply): per row, columns
 * in first-visit order over the row's faces (ascending face index) and
 * each face's two cells. pair->col by linear search
 * (CRConnectivity.cpp:730-790). */
static void mesh_connectivity(orc_mesh* m) {
  const int nAll = m->nCells + m->nGhost, F = m->nFaces;
  int* cfRow = (int*)xcalloc(nAll + 1, sizeof(int));
  for (int f = 0; f < F; f++) {
    cfRow[m->faceCells[2 * f] + 1]++;
    cfRow[m->faceCells[2 * f + 1] + 1]++;
  }
  for (int c = 0; c < nAll; c++) cfRow[c + 1] += cfRow[c];
  int* cfCol = (int*)xcalloc(cfRow[nAll], sizeof(int));
  int* fill = (int*)xcalloc(nAll, sizeof(int));
  for (int f = 0; f < F; f++)
    for (int k = 0; k < 2; k++) {
      const int c = m->faceCells[2 * f + k];
      cfCol[cfRow[c] + fill[c]++] = f;
    }
  /* two passes as CRConnectivity::multiply: count, then add */
  unsigned char* marker = (unsigned char*)xcalloc(nAll, 1);
  int* marked = (int*)xcalloc(nAll, sizeof(int));
  m->ccRow = (int*)xcalloc(nAll + 1, sizeof(int));
  for (int pass = 0; pass < 2; pass++) {
    for (int i = 0; i < nAll; i++) {
      int nMarked = 0, cnt = 0;
      for (int ir = cfRow[i]; ir < cfRow[i + 1]; ir++) {
        const int f = cfCol[ir];
        for (int k = 0; k < 2; k++) {
          const int jb = m->faceCells[2 * f + k];
          if (!marker[jb]) {
            marker[jb] = 1;
            if (jb != i) {
              if (pass == 0)
                cnt++;
              else
                m->ccCol[m->ccRow[i] + cnt++] = jb;
            }
            marked[nMarked++] = jb;
          }
        }
      }
      for (int n = 0; n < nMarked; n++) marker[marked[n]] = 0;
      if (pass == 0) m->ccRow[i + 1] = cnt;
    }
    if (pass == 0) {
      for (int i = 0; i < nAll; i++) m->ccRow[i + 1] += m->ccRow[i];
      m->ccCol = (int*)xcalloc(m->ccRow[nAll], sizeof(int));
    }
  }
  m->pairToCol = (int*)xcalloc(2 * (size_t)F, sizeof(int));
  for (int f = 0; f < F; f++) {
    const int c0 = m->faceCells[2 * f], c1 = m->faceCells[2 * f + 1];
    m->pairToCol[2 * f] = m->pairToCol[2 * f + 1] = -1;
    for (int k = m->ccRow[c0]; k < m->ccRow[c0 + 1]; k++)
      if (m->ccCol[k] == c1) {
        m->pairToCol[2 * f] = k;
        break;
      }
    for (int k = m->ccRow[c1]; k < m->ccRow[c1 + 1]; k++)
      if (m->ccCol[k] == c0) {
        m->pairToCol[2 * f + 1] = k;
        break;
      }
  }
  free(cfRow);
  free(cfCol);
  free(fill);
  free(marker);
  free(marked);
}

/* MeshMetricsCalculator<double>::init order: face areas
 * (MeshMetricsCalculator_impl.h:234-292), |A| (:335-350), face centroids
 * (:58-114), cell centroids (:121-232, boundary ghosts at the face
 * centroid), volumes (:352-400, ghosts copy their interior neighbour). All
 * groups here are "interior" or "wall". */
static void mesh_metrics(orc_mesh* m) {
  const int F = m->nFaces, nAll = m->nCells + m->nGhost;
  const double* X = m->xyz;
  m->area = (double*)xcalloc(3 * (size_t)F, sizeof(double));
  m->areaMag = (double*)xcalloc(F, sizeof(double));
  m->faceCentroid = (double*)xcalloc(3 * (size_t)F, sizeof(double));
  m->cellCentroid = (double*)xcalloc(3 * (size_t)nAll, sizeof(double));
  m->volume = (double*)xcalloc(nAll, sizeof(double));
  for (int f = 0; f < F; f++) {
    const int* fn = m->fnCol + m->fnRow[f];
    const int nn = m->fnRow[f + 1] - m->fnRow[f];
    double* a = m->area + 3 * f;
    if (nn == 2) {
      double dr[3];
      for (int d = 0; d < 3; d++) dr[d] = X[3 * fn[1] + d] - X[3 * fn[0] + d];
      a[0] = dr[1];
      a[1] = -dr[0];
      a[2] = 0.;
    } else if (nn == 3) {
      double d10[3], d20[3], c[3];
      for (int d = 0; d < 3; d++) {
        d10[d] = X[3 * fn[1] + d] - X[3 * fn[0] + d];
        d20[d] = X[3 * fn[2] + d] - X[3 * fn[0] + d];
      }
      cross3(d10, d20, c);
      for (int d = 0; d < 3; d++) a[d] = 0.5 * c[d];
    } else if (nn == 4) {
      double d20[3], d31[3], c[3];
      for (int d = 0; d < 3; d++) {
        d20[d] = X[3 * fn[2] + d] - X[3 * fn[0] + d];
        d31[d] = X[3 * fn[3] + d] - X[3 * fn[1] + d];
      }
      cross3(d20, d31, c);
      for (int d = 0; d < 3; d++) a[d] = 0.5 * c[d];
    } else if (nn > 0) {
      a[0] = a[1] = a[2] = 0.;
      for (int k = 0; k < nn; k++) {
        const double* p0 = X + 3 * fn[k];
        const double* p1 = X + 3 * fn[(k + 1) % nn];
        double xm[3], dr[3];
        for (int d = 0; d < 3; d++) {
          xm[d] = 0.5 * (p1[d] + p0[d]);
          dr[d] = p1[d] - p0[d];
        }
        a[0] += xm[1] * dr[2];
        a[1] += xm[2] * dr[0];
        a[2] += xm[0] * dr[1];
      }
    }
    m->areaMag[f] = mag3(a);
  }
  for (int f = 0; f < F; f++) {
    const int* fn = m->fnCol + m->fnRow[f];
    const int nn = m->fnRow[f + 1] - m->fnRow[f];
    double* fc = m->faceCentroid + 3 * f;
    if (nn > 0) {
      for (int d = 0; d < 3; d++) fc[d] = X[3 * fn[0] + d];
      for (int k = 1; k < nn; k++)
        for (int d = 0; d < 3; d++) fc[d] += X[3 * fn[k] + d];
      for (int d = 0; d < 3; d++) fc[d] /= (double)nn;
    }
  }
  for (int f = 0; f < F; f++) {
    const int* fn = m->fnCol + m->fnRow[f];
    const int nn = m->fnRow[f + 1] - m->fnRow[f];
    if (nn <= 3) continue;
    double* fc = m->faceCentroid + 3 * f;
    double en[3], cfc[3] = {0, 0, 0}, denom = 0.0;
    for (int d = 0; d < 3; d++) en[d] = m->area[3 * f + d] / m->areaMag[f];
    for (int k = 0; k < nn; k++) {
      const double* p0 = X + 3 * fn[k];
      const double* p1 = X + 3 * fn[(k + 1) % nn];
      double rc0[3], rc1[3], c[3], tri[3], xm[3];
      for (int d = 0; d < 3; d++) {
        rc0[d] = p0[d] - fc[d];
        rc1[d] = p1[d] - fc[d];
      }
      cross3(rc0, rc1, c);
      for (int d = 0; d < 3; d++) tri[d] = 0.5 * c[d];
      const double triP = dot3(tri, en);
      for (int d = 0; d < 3; d++) xm[d] = 0.5 * (p0[d] + p1[d]);
      for (int d = 0; d < 3; d++) cfc[d] += ((2. / 3.) * (xm[d] - fc[d])) * triP;
      denom += triP;
    }
    for (int d = 0; d < 3; d++) cfc[d] /= denom;
    for (int d = 0; d < 3; d++) fc[d] += cfc[d];
  }
  double* weight = (double*)xcalloc(nAll, sizeof(double));
  for (int f = 0; f < F; f++)
    for (int k = 0; k < 2; k++) {
      const int c = m->faceCells[2 * f + k];
      for (int d = 0; d < 3; d++) m->cellCentroid[3 * c + d] += m->faceCentroid[3 * f + d] * m->areaMag[f];
      weight[c] += m->areaMag[f];
    }
  for (int c = 0; c < m->nCells; c++)
    for (int d = 0; d < 3; d++) m->cellCentroid[3 * c + d] /= weight[c];
  for (int f = m->groupStart[1]; f < F; f++) {
    const int c1 = m->faceCells[2 * f + 1];
    for (int d = 0; d < 3; d++) m->cellCentroid[3 * c1 + d] = m->faceCentroid[3 * f + d];
  }
  free(weight);
  const double dim = (double)m->dim;
  for (int f = 0; f < F; f++) {
    const int c0 = m->faceCells[2 * f], c1 = m->faceCells[2 * f + 1];
    double r0[3], r1[3];
    for (int d = 0; d < 3; d++) {
      r0[d] = m->faceCentroid[3 * f + d] - m->cellCentroid[3 * c0 + d];
      r1[d] = m->faceCentroid[3 * f + d] - m->cellCentroid[3 * c1 + d];
    }
    m->volume[c0] += dot3(r0, m->area + 3 * f) / dim;
    m->volume[c1] -= dot3(r1, m->area + 3 * f) / dim;
  }
  for (int f = m->groupStart[1]; f < F; f++) m->volume[m->faceCells[2 * f + 1]] = m->volume[m->faceCells[2 * f]];
}

ORC_API void* orc_mesh_create(int dim, int nCells, int nNodes, const double* xyz, int nFaces, const int* faceCells,
                              const int* faceNodes, const int* faceNodeCount, int nGroups, const int* groupSize) {
  orc_mesh* m = (orc_mesh*)xcalloc(1, sizeof(orc_mesh));
  m->dim = dim;
  m->nCells = nCells;
  m->nNodes = nNodes;
  m->nFaces = nFaces;
  m->nGroups = nGroups;
  m->xyz = (double*)xcalloc(3 * (size_t)nNodes, sizeof(double));
  memcpy(m->xyz, xyz, sizeof(double) * 3 * (size_t)nNodes);
  m->faceCells = (int*)xcalloc(2 * (size_t)nFaces, sizeof(int));
  memcpy(m->faceCells, faceCells, sizeof(int) * 2 * (size_t)nFaces);
  m->fnRow = (int*)xcalloc(nFaces + 1, sizeof(int));
  for (int f = 0; f < nFaces; f++) m->fnRow[f + 1] = m->fnRow[f] + faceNodeCount[f];
  m->fnCol = (int*)xcalloc(m->fnRow[nFaces], sizeof(int));
  memcpy(m->fnCol, faceNodes, sizeof(int) * (size_t)m->fnRow[nFaces]);
  m->groupStart = (int*)xcalloc(nGroups + 1, sizeof(int));
  m->groupId = (int*)xcalloc(nGroups, sizeof(int));
  m->groupDefaultT = (int*)xcalloc(nGroups, sizeof(int));
  for (int g = 0; g < nGroups; g++) {
    m->groupStart[g + 1] = m->groupStart[g] + groupSize[g];
    m->groupId[g] = g;
  }
  m->nGhost = nFaces - groupSize[0];
  mesh_connectivity(m);
  mesh_metrics(m);
  return m;
}

ORC_API void orc_mesh_destroy(void* h) {
  orc_mesh* m = (orc_mesh*)h;
  if (!m) return;
  free(m->xyz);
  free(m->faceCells);
  free(m->fnRow);
  free(m->fnCol);
  free(m->groupStart);
  free(m->groupId);
  free(m->groupDefaultT);
  free(m->ccRow);
  free(m->ccCol);
  free(m->pairToCol);
  free(m->area);
  free(m->areaMag);
  free(m->faceCentroid);
  free(m->cellCentroid);
  free(m->volume);
  free(m);
}

/* Face-group id and type of a mesh read from a file (FluentReader): the id
 * keys the boundary-condition map and the type picks the default condition
 * (ThermalModel_impl.h:41-82). "symmetry" groups, whose ghost centroids and
 * gradients are reflected, are not restated. */
ORC_API int orc_mesh_set_group(void* h, int g, int id, const char* type) {
  orc_mesh* m = (orc_mesh*)h;
  if (g < 1 || g >= m->nGroups) return fail("no such face group");
  if (!strcmp(type, "symmetry")) return fail("symmetry face groups are not restated");
  if (!strcmp(type, "velocity-inlet") || !strcmp(type, "pressure-outlet"))
    m->groupDefaultT[g] = 1;
  else if (!strcmp(type, "wall"))
    m->groupDefaultT[g] = 0;
  else
    return fail("unknown face group type");
  m->groupId[g] = id;
  return 0;
}

/* sizes: nSelf, nGhost, nnz of cellCells over all rows */
ORC_API void orc_mesh_sizes(void* h, int* out) {
  const orc_mesh* m = (const orc_mesh*)h;
  out[0] = m->nCells;
  out[1] = m->nGhost;
  out[2] = m->ccRow[m->nCells + m->nGhost];
}

ORC_API void orc_mesh_connectivity(void* h, int* row, int* col, int* pairToCol) {
  const orc_mesh* m = (const orc_mesh*)h;
  const int nAll = m->nCells + m->nGhost;
  memcpy(row, m->ccRow, sizeof(int) * (nAll + 1));
  memcpy(col, m->ccCol, sizeof(int) * (size_t)m->ccRow[nAll]);
  memcpy(pairToCol, m->pairToCol, sizeof(int) * 2 * (size_t)m->nFaces);
}

ORC_API void orc_mesh_geometry(void* h, double* fa, double* fam, double* fcn, double* ccn, double* vol) {
  const orc_mesh* m = (const orc_mesh*)h;
  const int nAll = m->nCells + m->nGhost;
  memcpy(fa, m->area, sizeof(double) * 3 * (size_t)m->nFaces);
  memcpy(fam, m->areaMag, sizeof(double) * (size_t)m->nFaces);
  memcpy(fcn, m->faceCentroid, sizeof(double) * 3 * (size_t)m->nFaces);
  memcpy(ccn, m->cellCentroid, sizeof(double) * 3 * (size_t)nAll);
  memcpy(vol, m->volume, sizeof(double) * (size_t)nAll);
}

/* ================================================================== */
/* CRMatrix and AMG                                                    */
/* ================================================================== */

typedef struct {
  int nSelf, nAll;
  int *row, *col;
  double *diag, *off;
  unsigned char* isb;
  /* to the next coarser level */
  int* ci;
  int nCoarse;
  int *c2fRow, *c2fCol;
  /* vectors (nAll) */
  double *x, *b, *r, *tmp;
} orc_level;

typedef struct {
  int maxCoarseLevels, nPre, nPost, groupSize, cycleType, smoother;
  double thr;
} orc_amg_opts;

typedef struct {
  int nLevels; /* finest + coarse levels */
  orc_level lv[ORC_MAX_LEVELS + 1];
} orc_hier;

/* CRMatrix::createCoarsening (CRMatrix.h:468-586) */
static int coarsening(const orc_level* a, int groupSize, double thr, int* ci) {
  const int nRows = a->nSelf;
  for (int i = 0; i < a->nAll; i++) ci[i] = -1;
  int nCoarse = 0;
  int* count = (int*)xcalloc(nRows, sizeof(int));
  for (int nr = 0; nr < nRows; nr++) {
    if (ci[nr] != -1 || a->isb[nr]) continue;
    int current = nr, colG = -1, colU = -1, nGrouped;
    ci[current] = nCoarse;
    for (nGrouped = 1; nGrouped < groupSize; nGrouped++) {
      double wU = 0, wG = 0;
      colG = -1;
      colU = -1;
      for (int nb = a->row[current]; nb < a->row[current + 1]; nb++) {
        const int nc = a->col[nb];
        if (nc < nRows && !a->isb[nc]) {
          const double d0 = fabs(a->diag[nr]), d1 = fabs(a->diag[nc]);
          const double w = fabs(fabs(a->off[nb]) / (d0 > d1 ? d0 : d1));
          if (ci[nc] == -1) {
            if (colU == -1 || w > wU) {
              colU = nc;
              wU = w;
            }
          } else if (ci[nc] != ci[nr]) {
            if (colG == -1 || w > wG) {
              colG = nc;
              wG = w;
            }
          }
        }
      }
      if (colU != -1 && (colG == -1 || wU > thr * wG)) {
        ci[colU] = ci[current];
        count[ci[current]]++;
        current = colU;
      } else
        break;
    }
    if (nGrouped > 1 || colG == -1 || count[ci[colG]] > groupSize + 2) {
      count[ci[nr]]++;
      nCoarse++;
    } else {
      ci[nr] = ci[colG];
      count[ci[colG]]++;
    }
  }
  free(count);
  return nCoarse;
}

/* coarse->fine rows (MultiFieldMatrix.cpp:626-667), coarse pattern
 * (CRMatrix.h:597-691) and Galerkin coefficients (CRMatrix.h:699-758). */
static void coarse_level(orc_level* f, orc_level* c) {
  const int nC = f->nCoarse;
  f->c2fRow = (int*)xcalloc(nC + 1, sizeof(int));
  for (int i = 0; i < f->nAll; i++)
    if (f->ci[i] >= 0) f->c2fRow[f->ci[i] + 1]++;
  for (int I = 0; I < nC; I++) f->c2fRow[I + 1] += f->c2fRow[I];
  f->c2fCol = (int*)xcalloc(f->c2fRow[nC], sizeof(int));
  int* fill = (int*)xcalloc(nC, sizeof(int));
  for (int i = 0; i < f->nAll; i++)
    if (f->ci[i] >= 0) f->c2fCol[f->c2fRow[f->ci[i]] + fill[f->ci[i]]++] = i;
  free(fill);

  unsigned char* counted = (unsigned char*)xcalloc(nC, 1);
  c->nSelf = c->nAll = nC;
  c->row = (int*)xcalloc(nC + 1, sizeof(int));
  for (int pass = 0; pass < 2; pass++) {
    for (int I = 0; I < nC; I++) {
      int cnt = 0;
      for (int k = f->c2fRow[I]; k < f->c2fRow[I + 1]; k++) {
        const int i = f->c2fCol[k];
        for (int nb = f->row[i]; nb < f->row[i + 1]; nb++) {
          const int J = f->ci[f->col[nb]];
          if (J >= 0 && J != I && !counted[J]) {
            counted[J] = 1;
            if (pass == 1) c->col[c->row[I] + cnt] = J;
            cnt++;
          }
        }
      }
      for (int k = f->c2fRow[I]; k < f->c2fRow[I + 1]; k++) {
        const int i = f->c2fCol[k];
        for (int nb = f->row[i]; nb < f->row[i + 1]; nb++) {
          const int J = f->ci[f->col[nb]];
          if (J >= 0) counted[J] = 0;
        }
      }
      if (pass == 0) c->row[I + 1] = cnt;
    }
    if (pass == 0) {
      for (int I = 0; I < nC; I++) c->row[I + 1] += c->row[I];
      c->col = (int*)xcalloc(c->row[nC], sizeof(int));
    }
  }
  free(counted);

  c->diag = (double*)xcalloc(nC, sizeof(double));
  c->off = (double*)xcalloc(c->row[nC], sizeof(double));
  int* pos = (int*)xcalloc(nC, sizeof(int));
  for (int I = 0; I < nC; I++) {
    for (int nb = c->row[I]; nb < c->row[I + 1]; nb++) pos[c->col[nb]] = nb;
    for (int k = f->c2fRow[I]; k < f->c2fRow[I + 1]; k++) {
      const int i = f->c2fCol[k];
      c->diag[I] += f->diag[i];
      for (int nb = f->row[i]; nb < f->row[i + 1]; nb++) {
        const int J = f->ci[f->col[nb]];
        if (J < 0) continue;
        if (J != I)
          c->off[pos[J]] += f->off[nb];
        else
          c->diag[I] += f->off[nb];
      }
    }
  }
  free(pos);
  c->isb = (unsigned char*)xcalloc(nC, 1);
}

static void level_vectors(orc_level* l) {
  l->x = (double*)xcalloc(l->nAll, sizeof(double));
  l->b = (double*)xcalloc(l->nAll, sizeof(double));
  l->r = (double*)xcalloc(l->nAll, sizeof(double));
  l->tmp = (double*)xcalloc(l->nAll, sizeof(double));
}

/* AMG::createCoarseLevels, serial build (AMG.cpp:150-210): a level is kept
 * only if it shrank (level 0 compares rows + ghosts) and has > 3 rows. The
 * finest level (index 0) is borrowed from the caller. */
static void build_hierarchy(orc_hier* h, const orc_amg_opts* o) {
  h->nLevels = 1;
  for (int n = 0; n < o->maxCoarseLevels && n < ORC_MAX_LEVELS; n++) {
    orc_level* f = &h->lv[h->nLevels - 1];
    int* ci = (int*)xcalloc(f->nAll, sizeof(int));
    const int nc = coarsening(f, o->groupSize, o->thr, ci);
    if (f->nAll == nc || nc <= 3) {
      free(ci);
      break;
    }
    f->ci = ci;
    f->nCoarse = nc;
    orc_level* c = &h->lv[h->nLevels];
    memset(c, 0, sizeof *c);
    coarse_level(f, c);
    level_vectors(c);
    h->nLevels++;
  }
}

static void free_level(orc_level* l, int ownMatrix) {
  if (ownMatrix) {
    free(l->row);
    free(l->col);
    free(l->diag);
    free(l->off);
    free(l->isb);
    free(l->x);
    free(l->b);
    free(l->r);
    free(l->tmp);
  }
  free(l->ci);
  free(l->c2fRow);
  free(l->c2fCol);
  l->ci = l->c2fRow = l->c2fCol = NULL;
}

static void free_hierarchy(orc_hier* h) {
  for (int l = 0; l < h->nLevels; l++) free_level(&h->lv[l], l > 0);
  h->nLevels = 0;
}

/* CRMatrix::computeResidual (CRMatrix.h:404-426), self rows */
static void residual(const orc_level* a, const double* x, const double* b, double* r) {
  for (int nr = 0; nr < a->nSelf; nr++) {
    r[nr] = b[nr] + a->diag[nr] * x[nr];
    for (int nb = a->row[nr]; nb < a->row[nr + 1]; nb++) r[nr] += a->off[nb] * x[a->col[nb]];
  }
}

/* CRMatrix::multiply (CRMatrix.h:200-216), all rows */
static void multiply(const orc_level* a, const double* x, double* y) {
  for (int nr = 0; nr < a->nAll; nr++) {
    y[nr] = a->diag[nr] * x[nr];
    for (int nb = a->row[nr]; nb < a->row[nr + 1]; nb++) y[nr] += a->off[nb] * x[a->col[nb]];
  }
}

/* CRMatrix::forwardGS / reverseGS (CRMatrix.h:303-346) */
static void gs(const orc_level* a, double* x, const double* b, int reverse) {
  const int n = a->nSelf;
  for (int t = 0; t < n; t++) {
    const int nr = reverse ? n - 1 - t : t;
    double sum = b[nr];
    for (int nb = a->row[nr]; nb < a->row[nr + 1]; nb++) sum += a->off[nb] * x[a->col[nb]];
    x[nr] = -sum / a->diag[nr];
  }
}

/* MultiFieldMatrix::Jacobi + CRMatrix::Jacobi (MultiFieldMatrix.cpp:167-217,
 * CRMatrix.h:353-374): new values for self rows from the old ones, then
 * copied back. */
static void jacobi(const orc_level* a, double* x, const double* b, double* xnew) {
  for (int nr = 0; nr < a->nSelf; nr++) {
    double sum = b[nr];
    for (int nb = a->row[nr]; nb < a->row[nr + 1]; nb++) sum += a->off[nb] * x[a->col[nb]];
    xnew[nr] = -sum / a->diag[nr];
  }
  memcpy(x, xnew, sizeof(double) * (size_t)a->nSelf);
}

/* Array::getOneNorm / dotWith over self rows (Array.h:291-311) */
static double one_norm(const double* v, int n) {
  double s = 0;
  for (int i = 0; i < n; i++) s += fabs(v[i]);
  return s;
}
static double dotp(const double* a, const double* b, int n) {
  double s = 0;
  for (int i = 0; i < n; i++) s += a[i] * b[i];
  return s;
}

/* AMG::doSweeps (AMG.cpp:44-66) */
static void sweeps(orc_level* l, int n, int smoother) {
  for (int i = 0; i < n; i++) {
    if (smoother == 0) {
      gs(l, l->x, l->b, 0);
      gs(l, l->x, l->b, 1);
    } else {
      jacobi(l, l->x, l->b, l->tmp);
      jacobi(l, l->x, l->b, l->tmp);
    }
  }
}

/* AMG::cycle (AMG.cpp:68-135); inject/correct: Array.h:428-467 */
static void cycle(orc_hier* h, const orc_amg_opts* o, int type, int level) {
  orc_level* f = &h->lv[level];
  sweeps(f, o->nPre, o->smoother);
  if (level < h->nLevels - 1) {
    orc_level* c = &h->lv[level + 1];
    residual(f, f->x, f->b, f->r);
    memset(c->b, 0, sizeof(double) * (size_t)c->nAll);
    memset(c->x, 0, sizeof(double) * (size_t)c->nAll);
    for (int i = 0; i < f->nSelf; i++)
      if (f->ci[i] >= 0) c->b[f->ci[i]] += f->r[i];
    cycle(h, o, type, level + 1);
    if (type == 1)
      cycle(h, o, 1, level + 1);
    else if (type == 2)
      cycle(h, o, 0, level + 1);
    for (int i = 0; i < f->nSelf; i++)
      if (f->ci[i] >= 0) f->x[i] += c->x[f->ci[i]];
  }
  sweeps(f, o->nPost, o->smoother);
}

/* AMG::solve (AMG.cpp:228-280) on the finest level's x (delta) and b.
 * hist[0] = initial L1 norm, hist[i] = norm after cycle i. Returns the
 * number of history entries. */
static int amg_solve(orc_hier* h, const orc_amg_opts* o, int maxIter, double relTol, double absTol, double* hist,
                     int* cycles) {
  orc_level* f = &h->lv[0];
  residual(f, f->x, f->b, f->r);
  const double r0 = one_norm(f->r, f->nSelf);
  int nh = 0;
  if (hist) hist[nh] = r0;
  nh++;
  if (r0 < absTol) return nh;
  for (int i = 1; i < maxIter; i++) {
    if (cycles) (*cycles)++;
    cycle(h, o, o->cycleType, 0);
    residual(f, f->x, f->b, f->r);
    const double rn = one_norm(f->r, f->nSelf);
    double ratio = rn;
    if (r0 != 0) ratio /= r0;
    if (hist) hist[nh] = rn;
    nh++;
    if (rn < absTol || ratio < relTol) break;
  }
  return nh;
}

/* CG::solve (CG.cpp:26-139) with one AMG cycle as preconditioner
 * (AMG::smooth, AMG.cpp:283-298). x is the finest delta, b its rhs. */
static int cg_solve(orc_hier* h, const orc_amg_opts* o, int maxIter, double relTol, double absTol, double* hist,
                    int* cycles) {
  orc_level* f = &h->lv[0];
  const int n = f->nAll, ns = f->nSelf;
  double* x = f->x;
  double* bOrig = f->b;
  residual(f, x, bOrig, f->r);
  const double r0 = one_norm(f->r, ns);
  int nh = 0;
  if (hist) hist[nh] = r0;
  nh++;
  double* r = (double*)xcalloc(n, sizeof(double));
  memcpy(r, f->r, sizeof(double) * (size_t)n);
  double* p = NULL;
  double* z = (double*)xcalloc(n, sizeof(double));
  double* q = (double*)xcalloc(n, sizeof(double));
  double rho = 0, rhoPrev = 0;
  for (int i = 0; i < maxIter; i++) {
    memset(z, 0, sizeof(double) * (size_t)n);
    f->x = z;
    f->b = r;
    if (cycles) (*cycles)++;
    cycle(h, o, o->cycleType, 0);
    rhoPrev = rho;
    rho = dotp(r, z, ns);
    if (!p) {
      p = (double*)xcalloc(n, sizeof(double));
      memcpy(p, z, sizeof(double) * (size_t)n);
    } else {
      double beta = rho;
      if (rhoPrev != 0) beta /= rhoPrev;
      for (int k = 0; k < n; k++) p[k] *= beta;
      for (int k = 0; k < n; k++) p[k] += z[k];
    }
    multiply(f, p, q);
    const double ptq = dotp(p, q, ns);
    double alpha = rho;
    if (ptq != 0) alpha /= ptq;
    for (int k = 0; k < n; k++) x[k] -= alpha * p[k];
    for (int k = 0; k < n; k++) r[k] -= alpha * q[k];
    const double rn = one_norm(r, ns);
    double ratio = rn;
    if (r0 != 0) ratio /= r0;
    if (hist) hist[nh] = rn;
    nh++;
    if (rn < absTol || ratio < relTol) break;
  }
  f->x = x;
  f->b = bOrig;
  free(r);
  free(p);
  free(z);
  free(q);
  return nh;
}

/* BCGStab::solve (BCGStab.cpp:27-170); sHat aliases pHat as there. */
static int bcgs_solve(orc_hier* h, const orc_amg_opts* o, int maxIter, double relTol, double absTol, double* hist,
                      int* cycles) {
  orc_level* f = &h->lv[0];
  const int n = f->nAll, ns = f->nSelf;
  double* x = f->x;
  double* bOrig = f->b;
  residual(f, x, bOrig, f->r);
  const double r0 = one_norm(f->r, ns);
  int nh = 0;
  if (hist) hist[nh] = r0;
  nh++;
  double* r = (double*)xcalloc(n, sizeof(double));
  double* rT = (double*)xcalloc(n, sizeof(double));
  memcpy(r, f->r, sizeof(double) * (size_t)n);
  memcpy(rT, f->r, sizeof(double) * (size_t)n);
  double* p = NULL;
  double* pHat = (double*)xcalloc(n, sizeof(double));
  double* v = (double*)xcalloc(n, sizeof(double));
  double* t = (double*)xcalloc(n, sizeof(double));
  double rho = 0, rhoPrev = 0, alpha = 0, omega = 0;
  for (int i = 0; i < maxIter; i++) {
    rhoPrev = rho;
    rho = dotp(r, rT, ns);
    if (!p) {
      p = (double*)xcalloc(n, sizeof(double));
      memcpy(p, r, sizeof(double) * (size_t)n);
    } else {
      double rhoRatio = rho;
      if (rhoPrev != 0) rhoRatio /= rhoPrev;
      double aw = alpha;
      if (omega != 0) aw /= omega;
      const double beta = rhoRatio * aw;
      for (int k = 0; k < n; k++) p[k] -= omega * v[k];
      for (int k = 0; k < n; k++) p[k] *= beta;
      for (int k = 0; k < n; k++) p[k] += r[k];
    }
    memset(pHat, 0, sizeof(double) * (size_t)n);
    f->x = pHat;
    f->b = p;
    if (cycles) (*cycles)++;
    cycle(h, o, o->cycleType, 0);
    multiply(f, pHat, v);
    const double rtv = dotp(rT, v, ns);
    alpha = rho;
    if (rtv != 0) alpha /= rtv;
    for (int k = 0; k < n; k++) x[k] -= alpha * pHat[k];
    for (int k = 0; k < n; k++) r[k] -= alpha * v[k];
    double rn = one_norm(r, ns);
    if (rn < absTol) {
      if (hist) hist[nh] = rn;
      nh++;
      break;
    }
    double* sHat = pHat;
    memset(sHat, 0, sizeof(double) * (size_t)n);
    f->x = sHat;
    f->b = r;
    if (cycles) (*cycles)++;
    cycle(h, o, o->cycleType, 0);
    multiply(f, sHat, t);
    const double tdotr = dotp(t, r, ns);
    const double tdott = dotp(t, t, ns);
    omega = tdotr;
    if (tdott != 0) omega /= tdott;
    for (int k = 0; k < n; k++) x[k] -= omega * sHat[k];
    for (int k = 0; k < n; k++) r[k] -= omega * t[k];
    rn = one_norm(r, ns);
    double ratio = rn;
    if (r0 != 0) ratio /= r0;
    if (hist) hist[nh] = rn;
    nh++;
    if (rn < absTol || ratio < relTol) break;
  }
  f->x = x;
  f->b = bOrig;
  free(r);
  free(rT);
  free(p);
  free(pHat);
  free(v);
  free(t);
  return nh;
}

/* Raw CSR entry point with the argument layout of the compiled reference's
 * driver: opts = {maxCoarseLevels, nPre, nPost, groupSize, cycleType,
 * smootherType, nMaxIterations}, dopts = {weightRatioThreshold, relTol,
 * absTol}. The system has n self rows and no ghosts. Exports the coarse
 * level sizes, the L1 history and the coarseIndex array of every fine
 * level (concatenated, capacity cap). */
ORC_API int orc_amg_csr(int n, const int* row, const int* col, const double* diag, const double* off,
                        const double* b, const int* opts, const double* dopts, double* x, int* nLevels, int* sizes,
                        double* hist, int* nHist, int* ci, int cap) {
  orc_amg_opts o = {opts[0], opts[1], opts[2], opts[3], opts[4], opts[5], dopts[0]};
  orc_hier* h = (orc_hier*)xcalloc(1, sizeof(orc_hier));
  orc_level* f = &h->lv[0];
  f->nSelf = f->nAll = n;
  f->row = (int*)row;
  f->col = (int*)col;
  f->diag = (double*)diag;
  f->off = (double*)off;
  f->isb = (unsigned char*)xcalloc(n, 1);
  f->x = x;
  memset(x, 0, sizeof(double) * (size_t)n);
  f->b = (double*)b;
  f->r = (double*)xcalloc(n, sizeof(double));
  f->tmp = (double*)xcalloc(n, sizeof(double));
  build_hierarchy(h, &o);
  *nLevels = h->nLevels - 1;
  int p = 0;
  for (int l = 0; l + 1 < h->nLevels; l++) {
    sizes[l] = h->lv[l + 1].nSelf;
    for (int i = 0; i < h->lv[l].nSelf && p < cap; i++) ci[p++] = h->lv[l].ci[i];
  }
  *nHist = amg_solve(h, &o, opts[6], dopts[1], dopts[2], hist, NULL);
  free(f->isb);
  free(f->r);
  free(f->tmp);
  f->isb = NULL;
  free_hierarchy(h);
  free(h);
  return 0;
}

/* ================================================================== */
/* Multicolour ordering of the GPU smoothers (no reference counterpart) */
/* ================================================================== */

static int greedy_order(int n, const int* row, const int* col, const int* order, int* color) {
  int* mark = (int*)xcalloc(n + 1, sizeof(int));
  for (int i = 0; i <= n; i++) mark[i] = -1;
  for (int i = 0; i < n; i++) color[i] = -1;
  int nColors = 0;
  for (int t = 0; t < n; t++) {
    const int i = order ? order[t] : t;
    for (int k = row[i]; k < row[i + 1]; k++) {
      const int c = color[col[k]];
      if (c >= 0) mark[c] = i;
    }
    int c = 0;
    while (mark[c] == i) c++;
    color[i] = c;
    if (c + 1 > nColors) nColors = c + 1;
  }
  free(mark);
  return nColors;
}

/* Smallest-last order (Matula & Beck): repeatedly remove a vertex of
 * minimum remaining degree; the colouring order is the reverse of the
 * removal order. Ties, as the product defines them: each degree bucket is
 * a list that starts in ascending index order, a vertex whose degree drops
 * moves to the front of its new bucket, and the vertex removed is the front
 * of the lowest non-empty bucket. Restated with a stamp per vertex (front =
 * largest stamp) and a plain O(n^2) scan: test sizes only. */
static void smallest_last(int n, const int* row, const int* col, int* order) {
  int* deg = (int*)xcalloc(n, sizeof(int));
  long* stamp = (long*)xcalloc(n, sizeof(long));
  unsigned char* gone = (unsigned char*)xcalloc(n, 1);
  long clock = 0;
  for (int i = n - 1; i >= 0; i--) {
    deg[i] = row[i + 1] - row[i];
    stamp[i] = ++clock;
  }
  for (int t = 0; t < n; t++) {
    int v = -1;
    for (int i = 0; i < n; i++)
      if (!gone[i] && (v < 0 || deg[i] < deg[v] || (deg[i] == deg[v] && stamp[i] > stamp[v]))) v = i;
    gone[v] = 1;
    order[n - 1 - t] = v;
    for (int k = row[v]; k < row[v + 1]; k++) {
      const int u = col[k];
      if (gone[u]) continue;
      deg[u]--;
      stamp[u] = ++clock;
    }
  }
  free(deg);
  free(stamp);
  free(gone);
}

/* colour of every row of an n-row symmetric pattern (columns < n):
 * greedy in row order; when that needs more than five colours, also greedy
 * in smallest-last order, keeping the fewer (row order on a tie). Returns
 * the number of colours. */
ORC_API int orc_multicolor(int n, const int* rowIn, const int* colIn, int* color) {
  /* an unsymmetric pattern is coloured as A + A^T: each row keeps its
   * stored columns, followed by the columns present only in the
   * transpose, ascending */
  int* row = (int*)xcalloc(n + 1, sizeof(int));
  int* col = (int*)xcalloc(2 * (size_t)rowIn[n] + 1, sizeof(int));
  for (int i = 0; i < n; i++) {
    int cnt = row[i];
    for (int k = rowIn[i]; k < rowIn[i + 1]; k++) col[cnt++] = colIn[k];
    for (int j = 0; j < n; j++) {
      if (j == i) continue;
      int jHasI = 0, iHasJ = 0;
      for (int k = rowIn[j]; k < rowIn[j + 1]; k++) jHasI |= colIn[k] == i;
      if (!jHasI) continue;
      for (int k = rowIn[i]; k < rowIn[i + 1]; k++) iHasJ |= colIn[k] == j;
      if (!iHasJ) col[cnt++] = j;
    }
    row[i + 1] = cnt;
  }
  const int c1 = greedy_order(n, row, col, NULL, color);
  if (c1 <= 5) {
    free(row);
    free(col);
    return c1;
  }
  int* order = (int*)xcalloc(n, sizeof(int));
  int* color2 = (int*)xcalloc(n, sizeof(int));
  smallest_last(n, row, col, order);
  const int c2 = greedy_order(n, row, col, order, color2);
  if (c2 < c1) memcpy(color, color2, sizeof(int) * (size_t)n);
  free(order);
  free(color2);
  free(row);
  free(col);
  return c2 < c1 ? c2 : c1;
}

/* ================================================================== */
/* ThermalModel<double>                                                 */
/* ================================================================== */

enum { BC_T = 0, BC_FLUX = 1, BC_SYMMETRY = 2, BC_CONVECTIVE = 3, BC_RADIATIVE = 4, BC_MIXED = 5 };

typedef struct {
  orc_mesh* m;
  /* BC per group: type and {T, flux, h, Tinf, emissivity} */
  int* bcType;
  double* bcVal;
  /* options (layout of the compiled reference's driver) */
  int solver, maxIter, transient;
  orc_amg_opts amg;
  double relTol, absTol, linRel, linAbs, t0, dt, kvc, rho, cp;
  /* fields over self + ghost cells */
  double *T, *k, *s, *rhocp, *TN1;
  double* grad; /* 3 per cell */
  double* gcoef; /* LSQ weights, 3 per cellCells entry */
  int niters;
  double initialNorm;
  int haveInitialNorm;
} orc_thermal;

ORC_API void* orc_thermal_create(void* mesh) {
  orc_thermal* t = (orc_thermal*)xcalloc(1, sizeof(orc_thermal));
  t->m = (orc_mesh*)mesh;
  const int G = t->m->nGroups;
  t->bcType = (int*)xcalloc(G, sizeof(int));
  t->bcVal = (double*)xcalloc(5 * (size_t)G, sizeof(double));
  for (int g = 1; g < G; g++) {
    /* walls: SpecifiedHeatFlux, inlets/outlets: SpecifiedTemperature
     * (ThermalModel_impl.h:41-82); every group of a 7-argument mesh is a
     * wall. ThermalBC values (ThermalBC.h:11-18): temperature 300, flux 0,
     * h 0, far-field 300, emissivity 1 */
    t->bcType[g] = t->m->groupDefaultT[g] ? BC_T : BC_FLUX;
    double* v = t->bcVal + 5 * g;
    v[0] = 300.0;
    v[1] = 0.0;
    v[2] = 0.0;
    v[3] = 300.0;
    v[4] = 1.0;
  }
  /* ThermalModelOptions / LinearSolver / AMG defaults */
  t->solver = 0;
  t->maxIter = 20;
  t->amg.maxCoarseLevels = 30;
  t->amg.nPre = 0;
  t->amg.nPost = 1;
  t->amg.groupSize = 2;
  t->amg.cycleType = 0;
  t->amg.smoother = 0;
  t->amg.thr = 0.65;
  t->relTol = 1e-8;
  t->absTol = 1e-16;
  t->linRel = 1e-1;
  t->linAbs = 1e-16;
  t->t0 = 300.0;
  t->dt = 1e-7;
  t->kvc = 1.0;
  t->rho = 1.0;
  t->cp = 1.0;
  return t;
}

ORC_API void orc_thermal_destroy(void* h) {
  orc_thermal* t = (orc_thermal*)h;
  if (!t) return;
  free(t->bcType);
  free(t->bcVal);
  free(t->T);
  free(t->k);
  free(t->s);
  free(t->rhocp);
  free(t->TN1);
  free(t->grad);
  free(t->gcoef);
  free(t);
}

ORC_API int orc_thermal_set_bc(void* h, int groupId, int bcType, const double* vals) {
  orc_thermal* t = (orc_thermal*)h;
  int g = 1;
  while (g < t->m->nGroups && t->m->groupId[g] != groupId) g++;
  if (g >= t->m->nGroups) return fail("no such boundary group");
  if (bcType < 0 || bcType > BC_MIXED) return fail("unknown boundary condition type");
  t->bcType[g] = bcType;
  for (int i = 0; i < 5; i++) t->bcVal[5 * g + i] = vals[i];
  return 0;
}

/* iopts: solver(0 AMG, 1 CG+AMG, 2 BCGStab+AMG), maxCoarseLevels, nPre,
 * nPost, groupSize, cycleType, smootherType, nMaxIterations, transient,
 * verbosity; dopts: outer relTol, outer absTol, linear relTol, linear
 * absTol, weightRatioThreshold, initialTemperature, timeStep,
 * thermalConductivity, density, specificHeat */
ORC_API int orc_thermal_set_options(void* h, const int* io, const double* d) {
  orc_thermal* t = (orc_thermal*)h;
  t->solver = io[0];
  t->amg.maxCoarseLevels = io[1];
  t->amg.nPre = io[2];
  t->amg.nPost = io[3];
  t->amg.groupSize = io[4];
  t->amg.cycleType = io[5];
  t->amg.smoother = io[6];
  t->maxIter = io[7];
  t->transient = io[8] != 0;
  t->relTol = d[0];
  t->absTol = d[1];
  t->linRel = d[2];
  t->linAbs = d[3];
  t->amg.thr = d[4];
  t->t0 = d[5];
  t->dt = d[6];
  t->kvc = d[7];
  t->rho = d[8];
  t->cp = d[9];
  return 0;
}

/* ThermalModel::init (ThermalModel_impl.h:84-173) */
ORC_API int orc_thermal_init(void* h) {
  orc_thermal* t = (orc_thermal*)h;
  const int nAll = t->m->nCells + t->m->nGhost;
  double** fs[] = {&t->T, &t->k, &t->s, &t->rhocp, &t->TN1};
  for (int i = 0; i < 5; i++) {
    free(*fs[i]);
    *fs[i] = (double*)xcalloc(nAll, sizeof(double));
  }
  for (int c = 0; c < nAll; c++) {
    t->T[c] = t->t0;
    t->TN1[c] = t->t0;
    t->k[c] = t->kvc;
    t->s[c] = 0.;
    t->rhocp[c] = t->rho * t->cp;
  }
  free(t->grad);
  t->grad = (double*)xcalloc(3 * (size_t)nAll, sizeof(double));
  t->niters = 0;
  t->haveInitialNorm = 0;
  return 0;
}

/* field: 0 temperature, 1 conductivity, 2 source, 3 rho*cp, 4 temperatureN1 */
static double* field_ptr(orc_thermal* t, int field) {
  double* fs[] = {t->T, t->k, t->s, t->rhocp, t->TN1};
  return (field >= 0 && field < 5) ? fs[field] : NULL;
}
ORC_API int orc_thermal_set_cell_field(void* h, int field, const double* v) {
  orc_thermal* t = (orc_thermal*)h;
  double* p = field_ptr(t, field);
  if (!p) return fail("unknown field (call init first)");
  memcpy(p, v, sizeof(double) * (size_t)(t->m->nCells + t->m->nGhost));
  return 0;
}
ORC_API int orc_thermal_get_cell_field(void* h, int field, double* v) {
  orc_thermal* t = (orc_thermal*)h;
  double* p = field_ptr(t, field);
  if (!p) return fail("unknown field (call init first)");
  memcpy(v, p, sizeof(double) * (size_t)(t->m->nCells + t->m->nGhost));
  return 0;
}

/* GradientModel::getLeastSquaresGradientMatrix{2D,3D}
 * (GradientModel.h:126-436), no immersed boundaries */
static void lsq_weights(orc_thermal* t) {
  const orc_mesh* m = t->m;
  const int F = m->nFaces, N = m->nCells, nAll = N + m->nGhost;
  if (t->gcoef) return;
  t->gcoef = (double*)xcalloc(3 * (size_t)m->ccRow[nAll], sizeof(double));
  double* w = t->gcoef;
  const double* cc = m->cellCentroid;
  unsigned char* degen = (unsigned char*)xcalloc(nAll, 1);
  for (int f = 0; f < F; f++) {
    const int c0 = m->faceCells[2 * f], c1 = m->faceCells[2 * f + 1];
    double ds[3];
    for (int d = 0; d < 3; d++) ds[d] = cc[3 * c1 + d] - cc[3 * c0 + d];
    const double dsMag = mag3(ds);
    double* w01 = w + 3 * m->pairToCol[2 * f];
    double* w10 = w + 3 * m->pairToCol[2 * f + 1];
    for (int d = 0; d < 3; d++) {
      w01[d] = ds[d] / dsMag;
      w10[d] = -ds[d] / dsMag;
    }
  }
  for (int nc = 0; nc < N; nc++) {
    if (m->dim == 3) {
      double Ixx = 0, Iyy = 0, Izz = 0, Ixy = 0, Ixz = 0, Iyz = 0;
      for (int k = m->ccRow[nc]; k < m->ccRow[nc + 1]; k++) {
        const double* ds = w + 3 * k;
        Ixx += ds[0] * ds[0];
        Iyy += ds[1] * ds[1];
        Izz += ds[2] * ds[2];
        Ixy += ds[0] * ds[1];
        Ixz += ds[0] * ds[2];
        Iyz += ds[1] * ds[2];
      }
      const double det = Ixx * (Iyy * Izz - Iyz * Iyz) - Ixy * (Ixy * Izz - Iyz * Ixz) + Ixz * (Ixy * Iyz - Iyy * Ixz);
      if (det > 1e-6) {
        const double Kxx = (Iyy * Izz - Iyz * Iyz) / det;
        const double Kxy = -(Ixy * Izz - Iyz * Ixz) / det;
        const double Kxz = (Ixy * Iyz - Iyy * Ixz) / det;
        const double Kyy = (Ixx * Izz - Ixz * Ixz) / det;
        const double Kyz = -(Ixx * Iyz - Ixy * Ixz) / det;
        const double Kzz = (Ixx * Iyy - Ixy * Ixy) / det;
        for (int k = m->ccRow[nc]; k < m->ccRow[nc + 1]; k++) {
          const double ds0 = w[3 * k], ds1 = w[3 * k + 1], ds2 = w[3 * k + 2];
          w[3 * k] = (Kxx * ds0 + Kxy * ds1 + Kxz * ds2);
          w[3 * k + 1] = (Kxy * ds0 + Kyy * ds1 + Kyz * ds2);
          w[3 * k + 2] = (Kxz * ds0 + Kyz * ds1 + Kzz * ds2);
        }
      } else
        degen[nc] = 1;
    } else {
      double Ixx = 0, Iyy = 0, Ixy = 0;
      for (int k = m->ccRow[nc]; k < m->ccRow[nc + 1]; k++) {
        const double* ds = w + 3 * k;
        Ixx += ds[0] * ds[0];
        Iyy += ds[1] * ds[1];
        Ixy += ds[0] * ds[1];
      }
      const double det = Ixx * Iyy - Ixy * Ixy;
      if (det > 1e-26) {
        const double Kxx = Iyy / det;
        const double Kxy = -Ixy / det;
        const double Kyy = Ixx / det;
        for (int k = m->ccRow[nc]; k < m->ccRow[nc + 1]; k++) {
          const double ds0 = w[3 * k], ds1 = w[3 * k + 1];
          w[3 * k] = Kxx * ds0 + Kxy * ds1;
          w[3 * k + 1] = Kxy * ds0 + Kyy * ds1;
          w[3 * k + 2] = 0.0;
        }
      } else
        degen[nc] = 1;
    }
  }
  for (int f = 0; f < F; f++) {
    const int c0 = m->faceCells[2 * f], c1 = m->faceCells[2 * f + 1];
    double ds[3];
    for (int d = 0; d < 3; d++) ds[d] = cc[3 * c1 + d] - cc[3 * c0 + d];
    const double dsMag = mag3(ds);
    double* w01 = w + 3 * m->pairToCol[2 * f];
    double* w10 = w + 3 * m->pairToCol[2 * f + 1];
    for (int d = 0; d < 3; d++) {
      w01[d] /= dsMag;
      w10[d] /= dsMag;
    }
  }
  for (int f = 0; f < F; f++) {
    const int c0 = m->faceCells[2 * f], c1 = m->faceCells[2 * f + 1];
    if (degen[c0])
      for (int d = 0; d < 3; d++) w[3 * m->pairToCol[2 * f] + d] = 0.5 * m->area[3 * f + d] / m->volume[c0];
    if (degen[c1])
      for (int d = 0; d < 3; d++) w[3 * m->pairToCol[2 * f + 1] + d] = -0.5 * m->area[3 * f + d] / m->volume[c1];
  }
  free(degen);
}

/* GradientMatrix::getGradient + GradientModel::compute
 * (GradientMatrix.h:55-76, GradientModel.h:472-602): self rows, then each
 * boundary ghost takes its interior neighbour's gradient (the reflection
 * there applies to face groups of type "symmetry", which 7-argument meshes
 * never have: the Symmetry boundary condition does not change it). */
static void gradient(orc_thermal* t) {
  const orc_mesh* m = t->m;
  const double* w = t->gcoef;
  for (int nr = 0; nr < m->nCells; nr++) {
    double* g = t->grad + 3 * nr;
    g[0] = g[1] = g[2] = 0.;
    for (int k = m->ccRow[nr]; k < m->ccRow[nr + 1]; k++) {
      const double dx = t->T[m->ccCol[k]] - t->T[nr];
      for (int d = 0; d < 3; d++) g[d] += w[3 * k + d] * dx;
    }
  }
  for (int grp = 1; grp < m->nGroups; grp++)
    for (int f = m->groupStart[grp]; f < m->groupStart[grp + 1]; f++) {
      const int c0 = m->faceCells[2 * f], c1 = m->faceCells[2 * f + 1];
      for (int d = 0; d < 3; d++) t->grad[3 * c1 + d] = t->grad[3 * c0 + d];
    }
}

/* Assembly of one outer iteration over all rows (self + ghost):
 * DiffusionDiscretization::discretize (DiffusionDiscretization.h:65-232),
 * SourceDiscretization (SourceDiscretization.h:39-58),
 * TimeDerivativeDiscretization first order (TimeDerivativeDiscretization.h:
 * 149-155), the boundary conditions of ThermalModel::linearize
 * (ThermalModel_impl.h:296-398, GenericBCS.h:77-323) and
 * CRMatrix::eliminateBoundaryEquations (CRMatrix.h:899-944,1064-1085). */
static void linearize(orc_thermal* t, double* diag, double* off, double* b, unsigned char* isb) {
  orc_mesh* m = t->m;
  const int F = m->nFaces, N = m->nCells, nAll = N + m->nGhost;
  const int nnz = m->ccRow[nAll];
  memset(diag, 0, sizeof(double) * (size_t)nAll);
  memset(off, 0, sizeof(double) * (size_t)nnz);
  memset(b, 0, sizeof(double) * (size_t)nAll);
  memset(isb, 0, (size_t)nAll);
  lsq_weights(t);
  gradient(t);
  const double* cc = m->cellCentroid;
  for (int f = 0; f < F; f++) {
    const int c0 = m->faceCells[2 * f], c1 = m->faceCells[2 * f + 1];
    const double vol0 = m->volume[c0], vol1 = m->volume[c1];
    double ds[3];
    for (int d = 0; d < 3; d++) ds[d] = cc[3 * c1 + d] - cc[3 * c0 + d];
    double kf;
    if (vol0 == 0.)
      kf = t->k[c1];
    else if (vol1 == 0.)
      kf = t->k[c0];
    else {
      const double sum = t->k[c0] + t->k[c1];
      kf = (sum != 0.0) ? 2.0 * t->k[c0] * t->k[c1] / sum : sum;
    }
    const double* A = m->area + 3 * f;
    const double diffMetric = m->areaMag[f] * m->areaMag[f] / dot3(A, ds);
    const double diffCoeff = kf * diffMetric;
    double sc[3], gF[3];
    for (int d = 0; d < 3; d++) sc[d] = kf * (A[d] - ds[d] * diffMetric);
    for (int d = 0; d < 3; d++) gF[d] = (t->grad[3 * c0 + d] * vol0 + t->grad[3 * c1 + d] * vol1) / (vol0 + vol1);
    double sec = 0.0;
    for (int d = 0; d < 3; d++) sec += gF[d] * sc[d];
    const double dFlux = diffCoeff * (t->T[c1] - t->T[c0]) + sec;
    b[c0] += dFlux;
    b[c1] -= dFlux;
    off[m->pairToCol[2 * f]] += diffCoeff;
    off[m->pairToCol[2 * f + 1]] += diffCoeff;
    diag[c0] -= diffCoeff;
    diag[c1] -= diffCoeff;
  }
  for (int c = 0; c < N; c++) b[c] += m->volume[c] * t->s[c];
  if (t->transient)
    for (int c = 0; c < N; c++) {
      const double rhoVbydT = t->rhocp[c] * m->volume[c] / t->dt;
      b[c] -= rhoVbydT * (t->T[c] - t->TN1[c]);
      diag[c] -= rhoVbydT;
    }
  const double sb = 5.670373E-8;
  for (int grp = 1; grp < m->nGroups; grp++) {
    const double* v = t->bcVal + 5 * grp;
    for (int f = m->groupStart[grp]; f < m->groupStart[grp + 1]; f++) {
      const int c0 = m->faceCells[2 * f], c1 = m->faceCells[2 * f + 1];
      const int p01 = m->pairToCol[2 * f], p10 = m->pairToCol[2 * f + 1];
      const double Af = m->areaMag[f];
      switch (t->bcType[grp]) {
        case BC_T: {
          const double dX = v[0] - t->T[c1];
          b[c0] += off[p01] * dX;
          off[p01] = 0.0;
          t->T[c1] = v[0];
          off[p10] = 0.0;
          b[c1] = 0.0;
          diag[c1] = -1.0;
          break;
        }
        case BC_FLUX:
        case BC_SYMMETRY: {
          const double q = t->bcType[grp] == BC_FLUX ? v[1] : 0.0;
          const double fluxB = -b[c1];
          b[c1] = q * Af - fluxB;
          isb[c1] = 1;
          break;
        }
        case BC_CONVECTIVE: {
          const double fluxI = -b[c1];
          const double fluxB = -v[2] * (t->T[c1] - v[3]) * Af;
          b[c1] = fluxB - fluxI;
          diag[c1] -= v[2] * Af;
          isb[c1] = 1;
          break;
        }
        case BC_RADIATIVE: {
          const double x = t->T[c1], xi = v[3], e = v[4];
          const double fluxI = -b[c1];
          const double fluxB = -e * sb * (x * x * x * x - xi * xi * xi * xi) * Af;
          b[c1] = fluxB - fluxI;
          diag[c1] -= 4 * e * sb * x * x * x * Af;
          isb[c1] = 1;
          break;
        }
        case BC_MIXED: {
          const double x = t->T[c1], xi = v[3], e = v[4], hc = v[2];
          const double fluxI = -b[c1];
          const double fluxB = (-e * sb * (x * x * x * x - xi * xi * xi * xi) - hc * (x - xi)) * Af;
          b[c1] = fluxB - fluxI;
          diag[c1] -= (4 * e * sb * x * x * x + hc) * Af;
          isb[c1] = 1;
          break;
        }
      }
    }
  }
  /* eliminate boundary rows j >= N in ascending order: every neighbour i
   * of j (its interior cell) gets d_i -= a_ij (a_ji / a_jj) and
   * b_i -= a_ij (b_j / a_jj), then a_ij = 0 */
  for (int j = N; j < nAll; j++) {
    if (!isb[j]) continue;
    const double ajj = diag[j];
    for (int nb = m->ccRow[j]; nb < m->ccRow[j + 1]; nb++) {
      const int i = m->ccCol[nb];
      int pij = -1;
      for (int k = m->ccRow[i]; k < m->ccRow[i + 1]; k++)
        if (m->ccCol[k] == j) {
          pij = k;
          break;
        }
      for (int nb2 = m->ccRow[j]; nb2 < m->ccRow[j + 1]; nb2++) {
        const int kk = m->ccCol[nb2];
        const double ajk = off[nb2];
        if (i != kk) {
          for (int q = m->ccRow[i]; q < m->ccRow[i + 1]; q++)
            if (m->ccCol[q] == kk) {
              off[q] -= off[pij] * (ajk / ajj);
              break;
            }
        } else
          diag[i] -= off[pij] * (ajk / ajj);
      }
      b[i] -= off[pij] * (b[j] / ajj);
      off[pij] = 0.0;
    }
  }
}

/* one linearization as advance() performs it; exports the matrix over all
 * rows, the right-hand side and the boundary-row flags (0/1 as int) */
ORC_API int orc_thermal_linearize(void* h, double* diag, double* off, double* b, int* isBoundary) {
  orc_thermal* t = (orc_thermal*)h;
  if (!t->T) return fail("call init first");
  const int nAll = t->m->nCells + t->m->nGhost;
  unsigned char* isb = (unsigned char*)xcalloc(nAll, 1);
  linearize(t, diag, off, b, isb);
  if (isBoundary)
    for (int i = 0; i < nAll; i++) isBoundary[i] = isb[i];
  free(isb);
  return 0;
}

/* ThermalModel::advance (ThermalModel_impl.h:424-456): per outer iteration
 * linearize, solve for the delta (AMG, or CG / BCGStab preconditioned by
 * one AMG cycle) with a freshly built hierarchy, solve the boundary rows
 * (CRMatrix::solveBoundary, CRMatrix.h:433-454), x += delta, and stop on
 * the outer test. norms[i] = initial L1 residual of outer iteration i.
 * cycles (optional) accumulates the number of V-cycles. */
ORC_API int orc_thermal_advance(void* h, int niter, double* norms, int* nDone, int* cycles) {
  orc_thermal* t = (orc_thermal*)h;
  if (!t->T) return fail("call init first");
  orc_mesh* m = t->m;
  const int N = m->nCells, nAll = N + m->nGhost, nnz = m->ccRow[nAll];
  double* diag = (double*)xcalloc(nAll, sizeof(double));
  double* off = (double*)xcalloc(nnz, sizeof(double));
  double* b = (double*)xcalloc(nAll, sizeof(double));
  unsigned char* isb = (unsigned char*)xcalloc(nAll, 1);
  double* delta = (double*)xcalloc(nAll, sizeof(double));
  double* r = (double*)xcalloc(nAll, sizeof(double));
  double* tmp = (double*)xcalloc(nAll, sizeof(double));
  if (cycles) *cycles = 0;
  int done = 0;
  for (int n = 0; n < niter; n++) {
    linearize(t, diag, off, b, isb);
    orc_hier* hr = (orc_hier*)xcalloc(1, sizeof(orc_hier));
    orc_level* f = &hr->lv[0];
    f->nSelf = N;
    f->nAll = nAll;
    f->row = m->ccRow;
    f->col = m->ccCol;
    f->diag = diag;
    f->off = off;
    f->isb = isb;
    memset(delta, 0, sizeof(double) * (size_t)nAll);
    memset(r, 0, sizeof(double) * (size_t)nAll);
    f->x = delta;
    f->b = b;
    f->r = r;
    f->tmp = tmp;
    build_hierarchy(hr, &t->amg);
    double rn0 = 0;
    double* hist = (double*)xcalloc((size_t)t->maxIter + 2, sizeof(double));
    if (t->solver == 1)
      cg_solve(hr, &t->amg, t->maxIter, t->linRel, t->linAbs, hist, cycles);
    else if (t->solver == 2)
      bcgs_solve(hr, &t->amg, t->maxIter, t->linRel, t->linAbs, hist, cycles);
    else
      amg_solve(hr, &t->amg, t->maxIter, t->linRel, t->linAbs, hist, cycles);
    rn0 = hist[0];
    free(hist);
    free_hierarchy(hr);
    free(hr);
    /* boundary rows, then x += delta over all rows */
    for (int j = N; j < nAll; j++)
      if (isb[j]) {
        double sum = b[j];
        for (int nb = m->ccRow[j]; nb < m->ccRow[j + 1]; nb++) sum += off[nb] * delta[m->ccCol[nb]];
        delta[j] = -sum / diag[j];
      }
    for (int c = 0; c < nAll; c++) t->T[c] += delta[c];
    if (!t->haveInitialNorm) {
      t->initialNorm = rn0;
      t->haveInitialNorm = 1;
    }
    double ratio = rn0;
    if (t->initialNorm != 0) ratio /= t->initialNorm;
    t->niters++;
    norms[done++] = rn0;
    if (rn0 < t->absTol || ratio < t->relTol) break;
  }
  *nDone = done;
  free(diag);
  free(off);
  free(b);
  free(isb);
  free(delta);
  free(r);
  free(tmp);
  return 0;
}

/* ThermalModel::updateTime (ThermalModel_impl.h:472-495), first order */
ORC_API int orc_thermal_update_time(void* h) {
  orc_thermal* t = (orc_thermal*)h;
  if (!t->T) return fail("call init first");
  memcpy(t->TN1, t->T, sizeof(double) * (size_t)(t->m->nCells + t->m->nGhost));
  return 0;
}

/* AMG hierarchy built for the current linearization: coarse sizes and the
 * concatenated coarseIndex arrays (self rows of every fine level). */
ORC_API int orc_thermal_hierarchy(void* h, int groupSize, double thr, int maxLevels, int* nLevels, int* sizes,
                                  int* coarseIndex) {
  orc_thermal* t = (orc_thermal*)h;
  if (!t->T) return fail("call init first");
  orc_mesh* m = t->m;
  const int N = m->nCells, nAll = N + m->nGhost, nnz = m->ccRow[nAll];
  double* diag = (double*)xcalloc(nAll, sizeof(double));
  double* off = (double*)xcalloc(nnz, sizeof(double));
  double* b = (double*)xcalloc(nAll, sizeof(double));
  unsigned char* isb = (unsigned char*)xcalloc(nAll, 1);
  double* save = (double*)xcalloc(nAll, sizeof(double));
  memcpy(save, t->T, sizeof(double) * (size_t)nAll);
  linearize(t, diag, off, b, isb);
  memcpy(t->T, save, sizeof(double) * (size_t)nAll);
  orc_hier* hr = (orc_hier*)xcalloc(1, sizeof(orc_hier));
  orc_level* f = &hr->lv[0];
  f->nSelf = N;
  f->nAll = nAll;
  f->row = m->ccRow;
  f->col = m->ccCol;
  f->diag = diag;
  f->off = off;
  f->isb = isb;
  orc_amg_opts o = t->amg;
  o.groupSize = groupSize;
  o.thr = thr;
  o.maxCoarseLevels = maxLevels;
  build_hierarchy(hr, &o);
  *nLevels = hr->nLevels - 1;
  int p = 0;
  for (int l = 0; l + 1 < hr->nLevels; l++) {
    sizes[l] = hr->lv[l + 1].nSelf;
    for (int i = 0; i < hr->lv[l].nSelf; i++) coarseIndex[p++] = hr->lv[l].ci[i];
  }
  free_hierarchy(hr);
  free(hr);
  free(diag);
  free(off);
  free(b);
  free(isb);
  free(save);
  return 0;
}
