// AMG hierarchy construction on the host; compiled with -ffp-contract=off so
// that the Galerkin sums round exactly as the reference's do.
#include "amg_setup.hpp"

#include <algorithm>
#include <limits>
#include <memory>
#include <cmath>
#include <thread>

namespace fvm {


namespace {
// The greedy walk over rows [rb, re) with coarse rows numbered from 0; count
// has re - rb entries. On a level whose rows [rb, re) couple to no row
// outside the range, this is exactly the walk of the whole level restricted
// to the range.
int coarsen_range(const RefLevel& a, int rb, int re, int groupSize, double thr, int* ci, int* count) {
  const std::vector<int>& row = a.conn.row;
  const std::vector<int>& col = a.conn.col;
  int nCoarse = 0;
  for (int nr = rb; nr < re; nr++) {
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
}  // namespace

int create_coarsening(const RefLevel& a, int groupSize, double thr, std::vector<int>& ci,
                      std::vector<int>* coarseSegments) {
  const int n = a.n;
  ci.assign(n, -1);
  const std::vector<int>& seg = a.segments;
  if (seg.size() < 3) {  // one block: the reference's walk
    std::vector<int> count(n, 0);
    const int nc = coarsen_range(a, 0, n, groupSize, thr, ci.data(), count.data());
    if (coarseSegments) {
      coarseSegments->clear();
      if (!seg.empty()) *coarseSegments = {0, nc};
    }
    return nc;
  }
  // independent blocks (a batch of meshes): the walks run in parallel, then
  // each block's coarse rows are shifted behind the previous blocks'
  const int ns = (int)seg.size() - 1;
  std::vector<int> nc(ns, 0);
  parallel_chunks(ns, [&](int b, int e) {
    std::vector<int> count;
    for (int s = b; s < e; s++) {
      count.assign(seg[s + 1] - seg[s], 0);
      nc[s] = coarsen_range(a, seg[s], seg[s + 1], groupSize, thr, ci.data(), count.data());
    }
  }, 1);
  std::vector<int> off(ns + 1, 0);
  for (int s = 0; s < ns; s++) off[s + 1] = off[s] + nc[s];
  parallel_chunks(ns, [&](int b, int e) {
    for (int s = b; s < e; s++)
      for (int i = seg[s]; i < seg[s + 1]; i++)
        if (ci[i] >= 0) ci[i] += off[s];
  }, 1);
  if (coarseSegments) *coarseSegments = off;
  return off[ns];
}

void create_coarse_level(const RefLevel& fine, RefLevel& coarse, CSR& c2f) {
  const int nc = fine.nCoarse;
  const std::vector<int>& ci = fine.coarseIndex;
  const std::vector<int>& row = fine.conn.row;
  const std::vector<int>& col = fine.conn.col;
  // coarse -> fine rows, fine rows ascending. Independent blocks (a batch
  // of meshes: fine block s aggregates into coarse rows of block s only)
  // are counted and filled in parallel.
  const std::vector<int>& fseg = fine.segments;
  const bool blocks = fseg.size() >= 3;
  const int nBlocks = blocks ? (int)fseg.size() - 1 : 1;
  auto blockRows = [&](int sg, int& b, int& e) {
    b = blocks ? fseg[sg] : 0;
    e = blocks ? fseg[sg + 1] : fine.n;
  };
  c2f.nRows = nc;
  c2f.row.assign(nc + 1, 0);
  parallel_chunks(nBlocks, [&](int b0, int e0) {
    for (int sg = b0; sg < e0; sg++) {
      int b, e;
      blockRows(sg, b, e);
      for (int i = b; i < e; i++)
        if (ci[i] >= 0) c2f.row[ci[i] + 1]++;
    }
  }, 1);
  for (int I = 0; I < nc; I++) c2f.row[I + 1] += c2f.row[I];
  c2f.col.resize(c2f.row[nc]);
  {
    std::vector<int> cur(c2f.row.begin(), c2f.row.end() - 1);
    parallel_chunks(nBlocks, [&](int b0, int e0) {
      for (int sg = b0; sg < e0; sg++) {
        int b, e;
        blockRows(sg, b, e);
        for (int i = b; i < e; i++)
          if (ci[i] >= 0) c2f.col[cur[ci[i]]++] = i;
      }
    }, 1);
  }
  // Coarse pattern: each coarse row lists the coarse neighbours of its fine
  // rows in first-visit order. Rows are independent, so they are built in
  // parallel: a count pass, a prefix sum, then one pass that lists the
  // columns and sums the values. Stamp arrays replace the reference's marker
  // array and need no clearing between rows.
  coarse.n = nc;
  coarse.symmetricPattern = fine.symmetricPattern;
  coarse.conn.nRows = nc;
  coarse.conn.row.assign(nc + 1, 0);
  // stamp[J - lo] == tag: J already listed in the row being built. Each
  // chunk of coarse rows gets stamp / slot arrays spanning only the coarse
  // columns its rows reach (found by a first pass), so large levels need no
  // nc-sized array per thread.
  auto visit = [&](int I, int* out, int* stamp, int lo, int tag) {
    int cnt = 0;
    for (int k = c2f.row[I]; k < c2f.row[I + 1]; k++) {
      const int i = c2f.col[k];
      for (int nb = row[i]; nb < row[i + 1]; nb++) {
        const int J = ci[col[nb]];
        if (J < 0 || J == I || stamp[J - lo] == tag) continue;
        stamp[J - lo] = tag;
        if (out) out[cnt] = J;
        cnt++;
      }
    }
    return cnt;
  };
  constexpr int kMinRows = 4096;  // coarse rows per level below which the passes run on one thread
  const int nChunks = chunk_count(nc, kMinRows);
  std::vector<int> lo(nChunks, 0), hi(nChunks, -1);
  std::vector<std::vector<int>> stamps(nChunks);
  std::vector<std::unique_ptr<int[]>> slots(nChunks);
  // independent blocks: the columns of coarse rows [b, e) lie in the blocks
  // of rows b and e - 1 (no pass needed to find them)
  const std::vector<int>& cseg = coarse.segments;
  const bool cblocks = cseg.size() >= 3 && cseg.back() == nc;
  parallel_chunks_indexed(nc, [&](int t, int b, int e) {
    int l = std::numeric_limits<int>::max(), h = -1;
    if (cblocks && e > b) {
      l = *(std::upper_bound(cseg.begin(), cseg.end(), b) - 1);
      h = *std::upper_bound(cseg.begin(), cseg.end(), e - 1) - 1;
    } else {
      for (int k = c2f.row[b]; k < c2f.row[e]; k++) {
        const int i = c2f.col[k];
        for (int nb = row[i]; nb < row[i + 1]; nb++) {
          const int J = ci[col[nb]];
          if (J < 0) continue;
          l = std::min(l, J);
          h = std::max(h, J);
        }
      }
    }
    if (h < l) l = h = 0;
    lo[t] = l;
    hi[t] = h;
    stamps[t].assign((size_t)(h - l + 1), -1);
    slots[t].reset(new int[(size_t)(h - l + 1)]);
    for (int I = b; I < e; I++) coarse.conn.row[I + 1] = visit(I, nullptr, stamps[t].data(), l, I);
  }, kMinRows);
  for (int I = 0; I < nc; I++) coarse.conn.row[I + 1] += coarse.conn.row[I];
  coarse.conn.col.resize(coarse.conn.row[nc]);
  coarse.diag.resize(nc);
  coarse.off.resize(coarse.conn.col.size());
  // Galerkin values with piecewise-constant prolongation; every coarse
  // entry receives its fine contributions in the reference's order (fine
  // rows ascending, their entries in stored order), so the sums round
  // exactly as CRMatrix::createCoarseMatrix's do. Row I's columns are listed
  // in the same walk that sums its values: a column gets its slot (pos[J -
  // lo]) when first met, which is the first-visit order (tag I + nc: the
  // stamps of the count pass need no clearing).
  parallel_chunks_indexed(nc, [&](int t, int b, int e) {
    int* stamp = stamps[t].data();
    int* pos = slots[t].get();
    const int l = lo[t];
    for (int I = b; I < e; I++) {
      const int rb = coarse.conn.row[I];
      const int tag = I + nc;
      int cnt = 0;
      double d = 0.0;
      for (int k = c2f.row[I]; k < c2f.row[I + 1]; k++) {
        const int i = c2f.col[k];
        d += fine.diag[i];
        for (int nb = row[i]; nb < row[i + 1]; nb++) {
          const int J = ci[col[nb]];
          if (J < 0) continue;
          if (J != I) {
            if (stamp[J - l] != tag) {
              stamp[J - l] = tag;
              pos[J - l] = rb + cnt;
              coarse.conn.col[rb + cnt] = J;
              coarse.off[rb + cnt] = 0.0;
              cnt++;
            }
            coarse.off[pos[J - l]] += fine.off[nb];
          } else {
            d += fine.off[nb];
          }
        }
      }
      coarse.diag[I] = d;
    }
  }, kMinRows);
}

void build_hierarchy(std::vector<RefLevel>& levels, const HierarchyOptions& opt,
                     std::vector<CSR>& coarseToFine, std::vector<RefLevel>* spareLevels,
                     std::vector<CSR>* spareC2f, const std::function<void(int)>& onLevel) {
  levels.resize(1);
  coarseToFine.clear();
  for (int n = 0; n < opt.maxCoarseLevels; n++) {
    RefLevel& fine = levels.back();
    std::vector<int> ci, coarseSeg;
    const int nc = create_coarsening(fine, opt.groupSize, opt.weightRatioThreshold, ci, &coarseSeg);
    const int fineLocal = (levels.size() == 1 && opt.finestLocalSize > 0) ? opt.finestLocalSize : fine.n;
    if (fineLocal == nc) break;  // AMG.cpp:161-168
    if (nc <= 3) break;          // AMG.cpp:200-204 (serial: level not kept)
    fine.coarseIndex.swap(ci);
    fine.nCoarse = nc;
    const size_t lc = levels.size();
    RefLevel coarse;
    if (spareLevels && lc < spareLevels->size()) coarse = std::move((*spareLevels)[lc]);
    coarse.coarseIndex.clear();
    coarse.nCoarse = 0;
    CSR c2f;
    if (spareC2f && lc - 1 < spareC2f->size()) c2f = std::move((*spareC2f)[lc - 1]);
    coarse.segments = std::move(coarseSeg);
    create_coarse_level(fine, coarse, c2f);
    FVM_REQUIRE(levels.size() < levels.capacity() || !onLevel, kBadArgument,
                "build_hierarchy: no room for another level");
    levels.push_back(std::move(coarse));
    coarseToFine.push_back(std::move(c2f));
    if (onLevel) onLevel((int)levels.size() - 1);
    if (opt.coarsestSize > 0 && nc <= opt.coarsestSize) break;
  }
  levels.back().coarseIndex.clear();
  levels.back().nCoarse = 0;
}

namespace {

// Greedy colouring visiting rows in `order`: each row takes the smallest
// colour unused by its already-coloured neighbours.
int greedy_in_order(const CSR& conn, const std::vector<int>& order, std::vector<int>& color) {
  const int n = conn.nRows;
  color.assign(n, -1);
  std::vector<int> mark;
  int nColors = 0;
  for (int t = 0; t < n; t++) {
    const int i = order[t];
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

// Smallest-last ordering (Matula & Beck): repeatedly remove a vertex of
// minimum remaining degree; colouring in the reverse removal order needs at
// most degeneracy + 1 colours. Ties: each degree bucket is a list that
// starts in ascending index order; a vertex whose degree drops moves to the
// front of its new bucket, and the vertex removed is the front of the
// lowest non-empty bucket.
void smallest_last_order(const CSR& conn, std::vector<int>& order) {
  const int n = conn.nRows;
  std::vector<int> deg(n);
  int maxDeg = 0;
  for (int i = 0; i < n; i++) {
    deg[i] = conn.count(i);
    maxDeg = std::max(maxDeg, deg[i]);
  }
  // bucket lists by degree (doubly linked), kept in ascending index order
  std::vector<int> head(maxDeg + 1, -1), next(n, -1), prev(n, -1);
  for (int i = n - 1; i >= 0; i--) {
    next[i] = head[deg[i]];
    if (head[deg[i]] >= 0) prev[head[deg[i]]] = i;
    head[deg[i]] = i;
  }
  std::vector<char> removed(n, 0);
  std::vector<int> removal;
  removal.reserve(n);
  int d = 0;
  for (int t = 0; t < n; t++) {
    if (d > 0) d--;
    while (head[d] < 0) d++;
    const int v = head[d];
    head[d] = next[v];
    if (next[v] >= 0) prev[next[v]] = -1;
    removed[v] = 1;
    removal.push_back(v);
    for (int k = conn.row[v]; k < conn.row[v + 1]; k++) {
      const int u = conn.col[k];
      if (removed[u]) continue;
      // unlink u from bucket deg[u], push to the front of deg[u]-1
      if (prev[u] >= 0)
        next[prev[u]] = next[u];
      else
        head[deg[u]] = next[u];
      if (next[u] >= 0) prev[next[u]] = prev[u];
      deg[u]--;
      prev[u] = -1;
      next[u] = head[deg[u]];
      if (head[deg[u]] >= 0) prev[head[deg[u]]] = u;
      head[deg[u]] = u;
    }
  }
  order.assign(removal.rbegin(), removal.rend());
}

}  // namespace

// Deterministic colouring for the multicolour smoothers: greedy in row
// order; when that needs more than kFewColors colours, also greedy in
// smallest-last order, keeping whichever needs fewer (row order on a tie).
// Fewer colours mean fewer dependent passes per sweep; the smallest-last
// pass costs several greedy passes and rarely improves a colouring that is
// already this small (finest tetrahedral and hexahedral levels).
bool pattern_is_symmetric(const CSR& a) {
  for (int i = 0; i < a.nRows; i++)
    for (int k = a.row[i]; k < a.row[i + 1]; k++) {
      const int j = a.col[k];
      bool found = false;
      for (int q = a.row[j]; q < a.row[j + 1] && !found; q++) found = a.col[q] == i;
      if (!found) return false;
    }
  return true;
}

bool symmetrize_pattern(const CSR& a, CSR& out) {
  const int n = a.nRows;
  // transpose, rows in ascending source order
  std::vector<int> tr(n + 1, 0), tc(a.col.size());
  for (int c : a.col) tr[c + 1]++;
  for (int i = 0; i < n; i++) tr[i + 1] += tr[i];
  {
    std::vector<int> cur(tr.begin(), tr.end() - 1);
    for (int i = 0; i < n; i++)
      for (int k = a.row[i]; k < a.row[i + 1]; k++) tc[cur[a.col[k]]++] = i;
  }
  std::vector<int> mark(n, -1);
  out.nRows = n;
  out.row.assign(n + 1, 0);
  out.col.clear();
  out.col.reserve(2 * a.col.size());
  bool extra = false;
  for (int i = 0; i < n; i++) {
    for (int k = a.row[i]; k < a.row[i + 1]; k++) {
      out.col.push_back(a.col[k]);
      mark[a.col[k]] = i;
    }
    for (int k = tr[i]; k < tr[i + 1]; k++)
      if (mark[tc[k]] != i && tc[k] != i) {
        out.col.push_back(tc[k]);
        mark[tc[k]] = i;
        extra = true;
      }
    out.row[i + 1] = (int)out.col.size();
  }
  return extra;
}

int multicolor(const CSR& connIn, std::vector<int>& color, bool symmetricPattern, const std::vector<int>* segments) {
  CSR sym;
  const CSR& conn = (!symmetricPattern && symmetrize_pattern(connIn, sym)) ? sym : connIn;
  constexpr int kFewColors = 5;
  const int n = conn.nRows;
  if (segments && segments->size() >= 3) {
    // independent blocks: the row-order greedy colouring of each block is
    // the global one restricted to it (no edge leaves a block), so the
    // blocks are coloured in parallel with the same result
    const std::vector<int>& sg = *segments;
    const int nb = (int)sg.size() - 1;
    color.assign(n, -1);
    std::vector<int> ncol(nb, 0);
    parallel_chunks(nb, [&](int b0, int e0) {
      std::vector<int> mark;
      for (int q = b0; q < e0; q++) {
        int nc = 0;
        for (int i = sg[q]; i < sg[q + 1]; i++) {
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
          nc = std::max(nc, c + 1);
        }
        ncol[q] = nc;
      }
    }, 1);
    const int c1 = *std::max_element(ncol.begin(), ncol.end());
    if (c1 <= kFewColors) return c1;
  }
  std::vector<int> natural(n);
  for (int i = 0; i < n; i++) natural[i] = i;
  const int c1 = greedy_in_order(conn, natural, color);
  if (c1 <= kFewColors) return c1;
  std::vector<int> order, color2;
  smallest_last_order(conn, order);
  const int c2 = greedy_in_order(conn, order, color2);
  if (c2 < c1) {
    color.swap(color2);
    return c2;
  }
  return c1;
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

namespace {
// The colouring, colour-major permutation, slices and packed slots of a
// level. With values, diag and off give the diagonal and the stored
// entries; without, the pattern alone is packed. pos (optional) gets the
// CSR entry index of every packed slot (-1: padding).
void pack_core(const CSR& conn, bool symmetricPattern, const std::vector<int>& segments, bool values,
               const double* diag, const double* off, SmootherOrdering ordering, PackedLevel& out,
               std::unique_ptr<int[]>* colsOut, std::unique_ptr<int[]>* pos, size_t* slotsOut) {
  const int n = conn.nRows;
  out.n = n;
  // (out may be a reused object: pack_transfer refills these for all but
  // the coarsest level)
  out.coarseIndex.clear();
  out.c2fRow.clear();
  out.c2fCol.clear();
  std::vector<int> color;
  if (ordering == kSequential) {
    color.assign(n, 0);
    out.nColors = 1;
  } else {
    out.nColors = multicolor(conn, color, symmetricPattern, &segments);
  }
  // colour-major permutation, stable in reference order: per-chunk colour
  // counts, then every chunk places its rows behind the earlier chunks'
  const int C = out.nColors;
  int nt = (int)std::thread::hardware_concurrency();
  nt = std::max(1, std::min(nt, 32));
  if (n < 200000) nt = 1;
  const int chunk = (n + nt - 1) / nt;
  std::vector<int> cnt((size_t)nt * C, 0);
  parallel_chunks(nt, [&](int t0, int t1) {
    for (int t = t0; t < t1; t++)
      for (int i = t * chunk; i < std::min(n, (t + 1) * chunk); i++) cnt[(size_t)t * C + color[i]]++;
  }, 1);
  out.colorStart.assign(C + 1, 0);
  std::vector<int> base((size_t)nt * C);
  {
    int pos = 0;
    for (int c = 0; c < C; c++) {
      out.colorStart[c] = pos;
      for (int t = 0; t < nt; t++) {
        base[(size_t)t * C + c] = pos;
        pos += cnt[(size_t)t * C + c];
      }
    }
    out.colorStart[C] = pos;
  }
  out.perm.resize(n);
  out.iperm.resize(n);
  if (values)
    out.diag.resize(n);
  else
    out.diag.clear();
  parallel_chunks(nt, [&](int t0, int t1) {
    for (int t = t0; t < t1; t++) {
      int* cur = &base[(size_t)t * C];
      for (int i = t * chunk; i < std::min(n, (t + 1) * chunk); i++) {
        const int p = cur[color[i]]++;
        out.perm[i] = p;
        out.iperm[p] = i;
        if (values) out.diag[p] = diag[i];
      }
    }
  }, 1);
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
  parallel_chunks(nSlices, [&](int b, int e) {
    for (int s = b; s < e; s++) {
      int w = 0;
      for (int l = 0; l < out.sliceRows[s]; l++) w = std::max(w, conn.count(out.iperm[out.sliceRow[s] + l]));
      out.sliceOff[s + 1] = w;
    }
  });
  for (int s = 0; s < nSlices; s++) {
    out.maxWidth = std::max(out.maxWidth, out.sliceOff[s + 1]);
    out.sliceOff[s + 1] = out.sliceOff[s] + 32 * out.sliceOff[s + 1];
  }
  // A large level whose rows all have about the same short length (the
  // finest level of a tet, hex or quad mesh) is stored ELL-32: aligned
  // 32-row groups of one width, ignoring colour boundaries, so the kernels
  // compute a slice's position instead of loading it (one dependent load
  // less per row) at the cost of a little padding.
  const long long ellEntries = (long long)((n + 31) / 32) * 32 * out.maxWidth;
  out.ellWidth = 0;
  if (n >= 32768 && out.maxWidth <= 8 && ellEntries * 100 <= (long long)out.sliceOff[nSlices] * 115) {
    const int W = out.maxWidth, groups = (n + 31) / 32;
    out.ellWidth = W;
    out.sliceRow.resize(groups);
    out.sliceRows.resize(groups);
    out.sliceOff.resize(groups + 1);
    for (int s = 0; s < groups; s++) {
      out.sliceRow[s] = 32 * s;
      out.sliceRows[s] = std::min(32, n - 32 * s);
      out.sliceOff[s] = 32 * W * s;
    }
    out.sliceOff[groups] = 32 * W * groups;
    // colour passes of an ELL-32 level run over colorStart rows
    out.colorSliceStart = out.colorStart;
  }
  const int nPacked = (int)out.sliceRow.size();
  const size_t slots = (size_t)out.sliceOff[nPacked];
  // the pattern's arrays are not zero-filled first: the parallel fill below
  // writes every slot (and first-touches the pages on many threads)
  int* cols = nullptr;
  if (colsOut) {
    colsOut->reset(new int[slots > 0 ? slots : 1]);
    cols = colsOut->get();
    out.cols.clear();
  } else {
    out.cols.resize(slots);
    cols = out.cols.data();
  }
  if (values)
    out.vals.resize(slots);
  else
    out.vals.clear();
  int* posp = nullptr;
  if (pos) {
    pos->reset(new int[slots > 0 ? slots : 1]);
    posp = pos->get();
  }
  if (slotsOut) *slotsOut = slots;
  parallel_chunks(nPacked, [&](int sBegin, int sEnd) {
    for (int s = sBegin; s < sEnd; s++) {
      const int w = (out.sliceOff[s + 1] - out.sliceOff[s]) / 32;
      for (int l = 0; l < 32; l++) {
        const int p = out.sliceRow[s] + l;
        const bool live = l < out.sliceRows[s];
        const int i = live ? out.iperm[p] : -1;
        const int cnt = live ? conn.count(i) : 0;
        for (int k = 0; k < w; k++) {
          const size_t e = (size_t)out.sliceOff[s] + (size_t)k * 32 + l;
          if (k < cnt) {
            const int nb = conn.row[i] + k;
            cols[e] = out.perm[conn.col[nb]];
            if (values) out.vals[e] = off[nb];
            if (posp) posp[e] = nb;
          } else {
            cols[e] = live ? p : out.sliceRow[s];
            if (values) out.vals[e] = 0.0;
            if (posp) posp[e] = -1;
          }
        }
      }
    }
  });
}
}  // namespace

void pack_level(const RefLevel& lv, SmootherOrdering ordering, PackedLevel& out) {
  pack_core(lv.conn, lv.symmetricPattern, lv.segments, true, lv.diag.data(), lv.off.data(), ordering, out,
            nullptr, nullptr, nullptr);
}

void pack_pattern(const CSR& conn, bool symmetricPattern, const std::vector<int>& segments,
                  SmootherOrdering ordering, PackedLevel& out, std::unique_ptr<int[]>& cols,
                  std::unique_ptr<int[]>& pos, size_t& slots) {
  pack_core(conn, symmetricPattern, segments, false, nullptr, nullptr, ordering, out, &cols, &pos, &slots);
}

void pack_transfer(const RefLevel& fine, const CSR& c2f, PackedLevel& pf, const PackedLevel& pc) {
  pf.coarseIndex.resize(fine.n);
  parallel_chunks(fine.n, [&](int b, int e) {
    for (int i = b; i < e; i++)
      pf.coarseIndex[pf.perm[i]] = fine.coarseIndex[i] >= 0 ? pc.perm[fine.coarseIndex[i]] : -1;
  }, 1 << 17);
  const int nc = pc.n;
  pf.c2fRow.assign(nc + 1, 0);
  parallel_chunks(nc, [&](int b, int e) {
    for (int I = b; I < e; I++) pf.c2fRow[pc.perm[I] + 1] = c2f.count(I);
  }, 1 << 17);
  for (int P = 0; P < nc; P++) pf.c2fRow[P + 1] += pf.c2fRow[P];
  pf.c2fCol.resize(c2f.nnz());
  parallel_chunks(nc, [&](int b, int e) {
    for (int I = b; I < e; I++) {
      int o = pf.c2fRow[pc.perm[I]];
      for (int k = c2f.row[I]; k < c2f.row[I + 1]; k++) pf.c2fCol[o++] = pf.perm[c2f.col[k]];
    }
  }, 1 << 17);
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
