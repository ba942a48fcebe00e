// AMG hierarchy construction on the host; compiled with -ffp-contract=off so
// that the Galerkin sums round exactly as the reference's do.
#include "amg_setup.hpp"

#include <algorithm>
#include <cmath>

namespace fvm {

int create_coarsening(const RefLevel& a, int groupSize, double thr, std::vector<int>& ci) {
  const int n = a.n;
  const std::vector<int>& row = a.conn.row;
  const std::vector<int>& col = a.conn.col;
  ci.assign(n, -1);
  std::vector<int> count(n, 0);
  int nCoarse = 0;
  for (int nr = 0; nr < n; nr++) {
    if (ci[nr] != -1) continue;
    int current = nr;
    int colMaxGrouped = -1, colMaxUngrouped = -1;
    int nGrouped;
    ci[current] = nCoarse;
    for (nGrouped = 1; nGrouped < groupSize; nGrouped++) {
      double maxWeightUngrouped = 0, maxWeightGrouped = 0;
      colMaxGrouped = -1;
      colMaxUngrouped = -1;
      for (int nb = row[current]; nb < row[current + 1]; nb++) {
        const int nc = col[nb];
        // the weight uses the diagonal of the row that started the group
        const double d0 = std::fabs(a.diag[nr]);
        const double d1 = std::fabs(a.diag[nc]);
        const double w = std::fabs(std::fabs(a.off[nb]) / std::max(d0, d1));
        if (ci[nc] == -1) {
          if (colMaxUngrouped == -1 || w > maxWeightUngrouped) {
            colMaxUngrouped = nc;
            maxWeightUngrouped = w;
          }
        } else if (ci[nc] != ci[nr]) {
          if (colMaxGrouped == -1 || w > maxWeightGrouped) {
            colMaxGrouped = nc;
            maxWeightGrouped = w;
          }
        }
      }
      if (colMaxUngrouped != -1 &&
          (colMaxGrouped == -1 || maxWeightUngrouped > thr * maxWeightGrouped)) {
        ci[colMaxUngrouped] = ci[current];
        count[ci[current]]++;
        current = colMaxUngrouped;
      } else {
        break;
      }
    }
    if (nGrouped > 1 || colMaxGrouped == -1 || count[ci[colMaxGrouped]] > groupSize + 2) {
      count[ci[nr]]++;
      nCoarse++;
    } else {
      ci[nr] = ci[colMaxGrouped];
      count[ci[colMaxGrouped]]++;
    }
  }
  return nCoarse;
}

void create_coarse_level(const RefLevel& fine, RefLevel& coarse, CSR& c2f) {
  const int nc = fine.nCoarse;
  const std::vector<int>& ci = fine.coarseIndex;
  const std::vector<int>& row = fine.conn.row;
  const std::vector<int>& col = fine.conn.col;
  // coarse -> fine rows, fine rows ascending
  c2f.nRows = nc;
  c2f.row.assign(nc + 1, 0);
  for (int i = 0; i < fine.n; i++)
    if (ci[i] >= 0) c2f.row[ci[i] + 1]++;
  for (int I = 0; I < nc; I++) c2f.row[I + 1] += c2f.row[I];
  c2f.col.resize(c2f.row[nc]);
  {
    std::vector<int> cur(c2f.row.begin(), c2f.row.end() - 1);
    for (int i = 0; i < fine.n; i++)
      if (ci[i] >= 0) c2f.col[cur[ci[i]]++] = i;
  }
  // coarse pattern: neighbours in first-visit order
  coarse.n = nc;
  coarse.conn.nRows = nc;
  coarse.conn.row.assign(nc + 1, 0);
  coarse.conn.col.clear();
  std::vector<int> stamp(nc, -1);
  for (int I = 0; I < nc; I++) {
    for (int k = c2f.row[I]; k < c2f.row[I + 1]; k++) {
      const int i = c2f.col[k];
      for (int nb = row[i]; nb < row[i + 1]; nb++) {
        const int J = ci[col[nb]];
        if (J >= 0 && J != I && stamp[J] != I) {
          stamp[J] = I;
          coarse.conn.col.push_back(J);
        }
      }
    }
    coarse.conn.row[I + 1] = (int)coarse.conn.col.size();
  }
  // Galerkin values with piecewise-constant prolongation
  coarse.diag.assign(nc, 0.0);
  coarse.off.assign(coarse.conn.col.size(), 0.0);
  std::vector<int> pos(nc, -1);
  for (int I = 0; I < nc; I++) {
    for (int nb = coarse.conn.row[I]; nb < coarse.conn.row[I + 1]; nb++)
      pos[coarse.conn.col[nb]] = nb;
    for (int k = c2f.row[I]; k < c2f.row[I + 1]; k++) {
      const int i = c2f.col[k];
      coarse.diag[I] += fine.diag[i];
      for (int nb = row[i]; nb < row[i + 1]; nb++) {
        const int J = ci[col[nb]];
        if (J < 0) continue;
        if (J != I)
          coarse.off[pos[J]] += fine.off[nb];
        else
          coarse.diag[I] += fine.off[nb];
      }
    }
  }
}

void build_hierarchy(std::vector<RefLevel>& levels, const HierarchyOptions& opt,
                     std::vector<CSR>& coarseToFine) {
  levels.resize(1);
  coarseToFine.clear();
  for (int n = 0; n < opt.maxCoarseLevels; n++) {
    RefLevel& fine = levels.back();
    std::vector<int> ci;
    const int nc = create_coarsening(fine, opt.groupSize, opt.weightRatioThreshold, ci);
    const int fineLocal = (levels.size() == 1 && opt.finestLocalSize > 0) ? opt.finestLocalSize : fine.n;
    if (fineLocal == nc) break;  // AMG.cpp:161-168
    if (nc <= 3) break;          // AMG.cpp:200-204 (serial: level not kept)
    fine.coarseIndex = ci;
    fine.nCoarse = nc;
    RefLevel coarse;
    CSR c2f;
    create_coarse_level(fine, coarse, c2f);
    levels.push_back(std::move(coarse));
    coarseToFine.push_back(std::move(c2f));
    if (opt.coarsestSize > 0 && nc <= opt.coarsestSize) break;
  }
  levels.back().coarseIndex.clear();
  levels.back().nCoarse = 0;
}

int greedy_coloring(const CSR& conn, std::vector<int>& color) {
  const int n = conn.nRows;
  color.assign(n, -1);
  std::vector<int> mark;
  int nColors = 0;
  for (int i = 0; i < n; i++) {
    // colours taken by already coloured neighbours
    for (int k = conn.row[i]; k < conn.row[i + 1]; k++) {
      const int c = color[conn.col[k]];
      if (c >= 0) {
        if ((int)mark.size() <= c) mark.resize(c + 1, -1);
        mark[c] = i;
      }
    }
    int c = 0;
    while (c < (int)mark.size() && mark[c] == i) c++;
    color[i] = c;
    nColors = std::max(nColors, c + 1);
  }
  return nColors;
}

void pack_level(const RefLevel& lv, SmootherOrdering ordering, PackedLevel& out) {
  const int n = lv.n;
  out.n = n;
  std::vector<int> color;
  if (ordering == kSequential) {
    color.assign(n, 0);
    out.nColors = 1;
  } else {
    out.nColors = greedy_coloring(lv.conn, color);
  }
  // colour-major permutation, stable in reference order
  out.colorStart.assign(out.nColors + 1, 0);
  for (int i = 0; i < n; i++) out.colorStart[color[i] + 1]++;
  for (int c = 0; c < out.nColors; c++) out.colorStart[c + 1] += out.colorStart[c];
  out.perm.resize(n);
  out.iperm.resize(n);
  {
    std::vector<int> cur(out.colorStart.begin(), out.colorStart.end() - 1);
    for (int i = 0; i < n; i++) {
      const int p = cur[color[i]]++;
      out.perm[i] = p;
      out.iperm[p] = i;
    }
  }
  out.diag.resize(n);
  for (int p = 0; p < n; p++) out.diag[p] = lv.diag[out.iperm[p]];
  // SELL-32 slices aligned to colour blocks
  out.colorSliceStart.assign(out.nColors + 1, 0);
  out.sliceRow.clear();
  out.sliceRows.clear();
  for (int c = 0; c < out.nColors; c++) {
    for (int r = out.colorStart[c]; r < out.colorStart[c + 1]; r += 32) {
      out.sliceRow.push_back(r);
      out.sliceRows.push_back(std::min(32, out.colorStart[c + 1] - r));
    }
    out.colorSliceStart[c + 1] = (int)out.sliceRow.size();
  }
  const int nSlices = (int)out.sliceRow.size();
  out.sliceOff.assign(nSlices + 1, 0);
  out.maxWidth = 0;
  for (int s = 0; s < nSlices; s++) {
    int w = 0;
    for (int l = 0; l < out.sliceRows[s]; l++) w = std::max(w, lv.conn.count(out.iperm[out.sliceRow[s] + l]));
    out.maxWidth = std::max(out.maxWidth, w);
    out.sliceOff[s + 1] = out.sliceOff[s] + 32 * w;
  }
  out.cols.assign(out.sliceOff[nSlices], 0);
  out.vals.assign(out.sliceOff[nSlices], 0.0);
  for (int s = 0; s < nSlices; s++) {
    const int w = (out.sliceOff[s + 1] - out.sliceOff[s]) / 32;
    for (int l = 0; l < 32; l++) {
      const int p = out.sliceRow[s] + l;
      const bool live = l < out.sliceRows[s];
      const int i = live ? out.iperm[p] : -1;
      const int cnt = live ? lv.conn.count(i) : 0;
      for (int k = 0; k < w; k++) {
        const size_t e = (size_t)out.sliceOff[s] + (size_t)k * 32 + l;
        if (k < cnt) {
          const int nb = lv.conn.row[i] + k;
          out.cols[e] = out.perm[lv.conn.col[nb]];
          out.vals[e] = lv.off[nb];
        } else {
          out.cols[e] = live ? p : out.sliceRow[s];
          out.vals[e] = 0.0;
        }
      }
    }
  }
}

void pack_transfer(const RefLevel& fine, const CSR& c2f, PackedLevel& pf, const PackedLevel& pc) {
  pf.coarseIndex.assign(fine.n, -1);
  for (int i = 0; i < fine.n; i++)
    if (fine.coarseIndex[i] >= 0) pf.coarseIndex[pf.perm[i]] = pc.perm[fine.coarseIndex[i]];
  const int nc = pc.n;
  pf.c2fRow.assign(nc + 1, 0);
  for (int I = 0; I < nc; I++) pf.c2fRow[pc.perm[I] + 1] = c2f.count(I);
  for (int P = 0; P < nc; P++) pf.c2fRow[P + 1] += pf.c2fRow[P];
  pf.c2fCol.resize(c2f.nnz());
  for (int I = 0; I < nc; I++) {
    const int P = pc.perm[I];
    int o = pf.c2fRow[P];
    for (int k = c2f.row[I]; k < c2f.row[I + 1]; k++) pf.c2fCol[o++] = pf.perm[c2f.col[k]];
  }
}

void dense_inverse(const PackedLevel& lv, std::vector<double>& inv) {
  const int n = lv.n;
  std::vector<double> a((size_t)n * n, 0.0);
  for (int p = 0; p < n; p++) a[(size_t)p * n + p] = lv.diag[p];
  for (size_t s = 0; s + 1 < lv.sliceOff.size(); s++) {
    const int w = (lv.sliceOff[s + 1] - lv.sliceOff[s]) / 32;
    for (int l = 0; l < lv.sliceRows[s]; l++) {
      const int p = lv.sliceRow[s] + l;
      for (int k = 0; k < w; k++) {
        const size_t e = (size_t)lv.sliceOff[s] + (size_t)k * 32 + l;
        if (lv.vals[e] != 0.0) a[(size_t)p * n + lv.cols[e]] += lv.vals[e];
      }
    }
  }
  inv.assign((size_t)n * n, 0.0);
  for (int i = 0; i < n; i++) inv[(size_t)i * n + i] = 1.0;
  for (int c = 0; c < n; c++) {
    int piv = c;
    for (int r = c + 1; r < n; r++)
      if (std::fabs(a[(size_t)r * n + c]) > std::fabs(a[(size_t)piv * n + c])) piv = r;
    FVM_REQUIRE(a[(size_t)piv * n + c] != 0.0, kBadArgument, "singular coarsest-level matrix");
    if (piv != c)
      for (int k = 0; k < n; k++) {
        std::swap(a[(size_t)c * n + k], a[(size_t)piv * n + k]);
        std::swap(inv[(size_t)c * n + k], inv[(size_t)piv * n + k]);
      }
    const double d = a[(size_t)c * n + c];
    for (int k = 0; k < n; k++) {
      a[(size_t)c * n + k] /= d;
      inv[(size_t)c * n + k] /= d;
    }
    for (int r = 0; r < n; r++) {
      if (r == c) continue;
      const double f = a[(size_t)r * n + c];
      if (f == 0.0) continue;
      for (int k = 0; k < n; k++) {
        a[(size_t)r * n + k] -= f * a[(size_t)c * n + k];
        inv[(size_t)r * n + k] -= f * inv[(size_t)c * n + k];
      }
    }
  }
}

}  // namespace fvm
