// Device-built AMG hierarchy: aggregation, coarse-to-fine lists, Galerkin
// products and SELL-32 packing as sm_100a kernels (amg_device.cuh), and the
// host orchestration AmgHierarchy::buildDevice.
//
// Every result is deterministic: each output element is written by one
// thread (or one warp) that reads its inputs in a fixed order; the only
// atomics place fine rows into coarse-row lists, which are then sorted.
#include "amg_device.cuh"

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>

#include "common.hpp"
#include "solver.hpp"

namespace fvm {
namespace dev {

namespace {

constexpr int kT = 256;
constexpr int kScanTile = 1024;  // 256 threads x 4 elements
constexpr unsigned kFull = 0xffffffffu;

inline int cdiv(long long a, long long b) { return (int)((a + b - 1) / b); }

__device__ __forceinline__ void row_range(const LevelRows& a, int i, int& base, int& w) {
  if (a.ellWidth) {
    base = ((i >> 5) << 5) * a.ellWidth + (i & 31);
    w = a.ellWidth;
  } else {
    const int4 m = a.meta[a.rowSlice[i]];
    base = m.z + (i - m.x);
    w = m.w;
  }
}

// exclusive scan of one int per thread over a 256-thread block
__device__ __forceinline__ int block_exclusive_scan(int v, int& total) {
  __shared__ int wsum[kT / 32];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  int x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int y = __shfl_up_sync(kFull, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) wsum[wid] = x;
  __syncthreads();
  if (wid == 0) {
    int s = lane < kT / 32 ? wsum[lane] : 0;
#pragma unroll
    for (int o = 1; o < kT / 32; o <<= 1) {
      const int y = __shfl_up_sync(kFull, s, o);
      if (lane >= o) s += y;
    }
    if (lane < kT / 32) wsum[lane] = s;
  }
  __syncthreads();
  const int off = wid > 0 ? wsum[wid - 1] : 0;
  total = wsum[kT / 32 - 1];
  __syncthreads();
  return off + x - v;
}

__global__ void k_scan_tiles(const int* __restrict__ in, int* out, int n, int* tileSum) {
  const int base = blockIdx.x * kScanTile + threadIdx.x * 4;
  int v[4];
  int s = 0;
#pragma unroll
  for (int q = 0; q < 4; q++) {
    v[q] = base + q < n ? in[base + q] : 0;
    s += v[q];
  }
  int total;
  int e = block_exclusive_scan(s, total);
#pragma unroll
  for (int q = 0; q < 4; q++) {
    if (base + q < n) out[base + q] = e;
    e += v[q];
  }
  if (threadIdx.x == 0) tileSum[blockIdx.x] = total;
}

// one block: exclusive scan of the tile sums in place, total at [nTiles]
__global__ void k_scan_tile_sums(int* tileSum, int nTiles) {
  const int per = (nTiles + kT - 1) / kT;
  const int b = threadIdx.x * per;
  int s = 0;
  for (int q = 0; q < per; q++)
    if (b + q < nTiles) s += tileSum[b + q];
  int total;
  int e = block_exclusive_scan(s, total);
  for (int q = 0; q < per; q++)
    if (b + q < nTiles) {
      const int t = tileSum[b + q];
      tileSum[b + q] = e;
      e += t;
    }
  if (threadIdx.x == 0) tileSum[nTiles] = total;
}

__global__ void k_scan_add(int* out, int n, const int* tileSum, int nTiles) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] += tileSum[i / kScanTile];
  if (i == 0) out[n] = tileSum[nTiles];
}

__global__ void k_fill_finest_vals(long long entries, const int* __restrict__ posSrc, const double* __restrict__ src,
                                   double* vals, float* valsF) {
  const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= entries) return;
  const int s = posSrc[p];
  const double v = s >= 0 ? src[s] : 0.0;
  vals[p] = v;
  if (valsF) valsF[p] = (float)v;
}

__global__ void k_fill_finest_diag(int n, const int* __restrict__ iperm, const double* __restrict__ diagSrc,
                                   double* diag, float* diagF) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n) return;
  const double d = diagSrc[iperm[p]];
  diag[p] = d;
  if (diagF) diagF[p] = (float)d;
}

// ---- aggregation -------------------------------------------------------------

__device__ __forceinline__ double strength(double v, double di, double dj) { return fabs(v) / fmax(di, dj); }

// The matching kernels take a row's entries in chunks of kAggChunk: the
// chunk's column and value loads are issued together, then its neighbour
// loads (only for the entries that one at a time would load them for), then
// the entries are taken in stored order, so the result is the one-at-a-time
// result with a quarter of the dependent round trips to memory.
constexpr int kAggChunk = 4;

__global__ void k_agg_init(LevelRows a, double* maxw, int* partner) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= a.n) return;
  int base, w;
  row_range(a, i, base, w);
  const double di = fabs(a.diag[i]);
  double m = 0.0;
  for (int k0 = 0; k0 < w; k0 += kAggChunk) {
    int jj[kAggChunk];
    double vv[kAggChunk], dj[kAggChunk];
    bool use[kAggChunk];
#pragma unroll
    for (int u = 0; u < kAggChunk; u++) {
      use[u] = false;
      if (k0 + u < w) {
        jj[u] = a.cols[base + 32 * (k0 + u)];
        vv[u] = a.vals[base + 32 * (k0 + u)];
        use[u] = !(jj[u] == i || vv[u] == 0.0);
      }
    }
#pragma unroll
    for (int u = 0; u < kAggChunk; u++)
      if (use[u]) dj[u] = fabs(a.diag[jj[u]]);
#pragma unroll
    for (int u = 0; u < kAggChunk; u++)
      if (use[u]) m = fmax(m, strength(vv[u], di, dj[u]));
  }
  maxw[i] = m;
  partner[i] = -1;
}

// the strongest candidate of row i among its entries whose neighbour j has
// (paired ? partner[j] >= 0 : partner[j] == -1), strength at least thr
// (ties: smaller index); -1 when none
template <bool Paired>
__device__ __forceinline__ int agg_strongest(const LevelRows& a, int i, double thr, const int* __restrict__ partner) {
  int base, w;
  row_range(a, i, base, w);
  const double di = fabs(a.diag[i]);
  int bj = -1;
  double bw = 0.0;
  for (int k0 = 0; k0 < w; k0 += kAggChunk) {
    int jj[kAggChunk];
    double vv[kAggChunk], dj[kAggChunk];
    bool use[kAggChunk];
#pragma unroll
    for (int u = 0; u < kAggChunk; u++) {
      use[u] = false;
      if (k0 + u < w) {
        jj[u] = a.cols[base + 32 * (k0 + u)];
        vv[u] = a.vals[base + 32 * (k0 + u)];
        use[u] = !(jj[u] == i || vv[u] == 0.0);
      }
    }
#pragma unroll
    for (int u = 0; u < kAggChunk; u++)
      if (use[u]) {
        const int p = partner[jj[u]];
        use[u] = Paired ? p >= 0 : p == -1;
      }
#pragma unroll
    for (int u = 0; u < kAggChunk; u++)
      if (use[u]) dj[u] = fabs(a.diag[jj[u]]);
#pragma unroll
    for (int u = 0; u < kAggChunk; u++) {
      if (!use[u]) continue;
      const double s = strength(vv[u], di, dj[u]);
      if (!(s > 0.0) || s < thr) continue;
      if (s > bw || (s == bw && jj[u] < bj)) {
        bw = s;
        bj = jj[u];
      }
    }
  }
  return bj;
}

// strongest unpaired candidate of every unpaired row (ties: smaller index)
__global__ void k_agg_best(LevelRows a, const double* __restrict__ maxw, double beta, const int* __restrict__ partner,
                           int* best) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= a.n) return;
  if (partner[i] != -1) {
    best[i] = -1;
    return;
  }
  best[i] = agg_strongest<false>(a, i, beta * maxw[i], partner);
}

// handshake: i and j pair when each is the other's strongest candidate
__global__ void k_agg_match(int n, const int* __restrict__ best, int* partner) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n || partner[i] != -1) return;
  const int j = best[i];
  if (j >= 0 && best[j] == i) partner[i] = j;
}

// an unpaired row joins the pair of its strongest paired candidate
__global__ void k_agg_join(LevelRows a, const double* __restrict__ maxw, double beta, const int* __restrict__ partner,
                           int* join) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= a.n) return;
  if (partner[i] != -1) {
    join[i] = -1;
    return;
  }
  join[i] = agg_strongest<true>(a, i, beta * maxw[i], partner);
}

__device__ __forceinline__ bool is_leader(int i, const int* partner, const int* join) {
  const int p = partner[i];
  return p >= 0 ? i < p : join[i] < 0;
}

__global__ void k_agg_flags(int n, const int* __restrict__ partner, const int* __restrict__ join,
                            const int* __restrict__ order, int* flag) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  flag[order ? order[i] : i] = is_leader(i, partner, join) ? 1 : 0;
}

__global__ void k_agg_ci_leaders(int n, const int* __restrict__ partner, const int* __restrict__ join,
                                 const int* __restrict__ order, const int* __restrict__ pos, int* ci) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n || !is_leader(i, partner, join)) return;
  ci[i] = pos[order ? order[i] : i];
}

__global__ void k_agg_ci_rest(int n, const int* __restrict__ partner, const int* __restrict__ join, int* ci) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n || is_leader(i, partner, join)) return;
  const int p = partner[i];
  if (p >= 0) {
    ci[i] = ci[p];  // the pair's leader is its smaller row
  } else {
    const int j = join[i];
    const int q = partner[j];
    ci[i] = ci[j < q ? j : q];
  }
}

// ---- coarse-to-fine lists ------------------------------------------------------

__global__ void k_c2f_count(int n, const int* __restrict__ ci, int* cnt) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) atomicAdd(&cnt[ci[i]], 1);
}

__global__ void k_c2f_place(int n, const int* __restrict__ ci, const int* __restrict__ c2fRow, int* cursor,
                            int* c2fCol) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int c = ci[i];
  c2fCol[c2fRow[c] + atomicAdd(&cursor[c], 1)] = i;
}

__global__ void k_c2f_sort(int nc, const int* __restrict__ c2fRow, int* c2fCol) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= nc) return;
  const int b = c2fRow[c], e = c2fRow[c + 1];
  for (int q = b + 1; q < e; q++) {
    const int v = c2fCol[q];
    int r = q - 1;
    while (r >= b && c2fCol[r] > v) {
      c2fCol[r + 1] = c2fCol[r];
      r--;
    }
    c2fCol[r + 1] = v;
  }
}

// ---- Galerkin ----------------------------------------------------------------------

constexpr int kGalWarps = 4;

template <bool kFill>
__global__ void __launch_bounds__(32 * kGalWarps) k_galerkin(LevelRows a, int nc, const int* __restrict__ ci,
                                                             const int* __restrict__ c2fRow,
                                                             const int* __restrict__ c2fCol, int* count,
                                                             int* overflow, const int* __restrict__ sliceOff,
                                                             int* ccols, double* cvals, float* cvalsF,
                                                             double* cdiag, float* cdiagF) {
  __shared__ int sJ[kGalWarps][kGalerkinCap];
  __shared__ double sV[kGalWarps][kGalerkinCap];
  __shared__ int sOff[kGalWarps][32], sBase[kGalWarps][32], sRow[kGalWarps][32];
  __shared__ double sDiag[kGalWarps][32];
  const int wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int I = blockIdx.x * kGalWarps + wid;
  if (I >= nc) return;  // the whole warp leaves together
  int* J = sJ[wid];
  double* V = sV[wid];
  const int f0 = c2fRow[I], f1 = c2fRow[I + 1];
  // the coarse diagonal (fill pass, lane 0): fine diagonals plus the entries
  // inside the aggregate, fine rows ascending, entries in stored order,
  // summed chunk by chunk from the values staged in shared memory
  double dsum = 0.0;
  // every entry of the aggregate's fine rows, fine rows ascending, entries
  // in stored order; J = coarse column (-1: padding). Up to 32 fine rows at
  // a time: each lane looks up one row's range, a warp scan places the rows,
  // and the lanes then gather all their entries at once.
  int L = 0;
  bool over = false;
  for (int q0 = f0; q0 < f1; q0 += 32) {
    const int nq = min(32, f1 - q0);
    int base = 0, w = 0, f = -1;
    if (lane < nq) {
      f = c2fCol[q0 + lane];
      row_range(a, f, base, w);
      if (kFill) sDiag[wid][lane] = a.diag[f];
    }
    int incl = w;
    for (int o = 1; o < 32; o <<= 1) {
      const int t = __shfl_up_sync(kFull, incl, o);
      if (lane >= o) incl += t;
    }
    const int tot = __shfl_sync(kFull, incl, 31);
    if (L + tot > kGalerkinCap) {
      over = true;
      break;
    }
    sOff[wid][lane] = incl - w;
    sBase[wid][lane] = base;
    sRow[wid][lane] = f;
    __syncwarp();
    for (int e = lane; e < tot; e += 32) {
      // the last row q < nq whose range starts at or before e
      int lo = 0, hi = nq - 1;
      while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (sOff[wid][mid] <= e)
          lo = mid;
        else
          hi = mid - 1;
      }
      const int idx = sBase[wid][lo] + 32 * (e - sOff[wid][lo]);
      const int j = a.cols[idx];
      const double v = a.vals[idx];
      J[L + e] = (j == sRow[wid][lo] || v == 0.0) ? -1 : ci[j];
      V[L + e] = v;
    }
    __syncwarp();
    if (kFill && lane == 0) {
      int e = L;
      for (int q = 0; q < nq; q++) {
        dsum += sDiag[wid][q];
        const int we = (q + 1 < nq ? sOff[wid][q + 1] : tot) - sOff[wid][q];
        for (int k = 0; k < we; k++, e++)
          if (J[e] == I) dsum += V[e];
      }
    }
    __syncwarp();
    L += tot;
  }
  __syncwarp();
  if (over) {
    if (lane == 0) {
      atomicExch(overflow, 1);
      if (!kFill) count[I] = 0;
    }
    return;
  }
  int cbase = 0, cw = 0;
  if (kFill) {
    const int s = I >> 5;
    cbase = sliceOff[s] + (I & 31);
    cw = (sliceOff[s + 1] - sliceOff[s]) >> 5;
  }
  // off-diagonal coarse columns in first-visit order; each first visit sums
  // every later entry of its column in stored order
  int nUnique = 0;
  for (int e0 = 0; e0 < L; e0 += 32) {
    const int e = e0 + lane;
    bool first = false;
    int Je = -1;
    if (e < L) {
      Je = J[e];
      if (Je >= 0 && Je != I) {
        first = true;
        for (int e2 = 0; e2 < e; e2++)
          if (J[e2] == Je) {
            first = false;
            break;
          }
      }
    }
    const unsigned m = __ballot_sync(kFull, first);
    if (kFill && first) {
      const int slot = nUnique + __popc(m & ((1u << lane) - 1u));
      double s = 0.0;
      for (int e2 = e; e2 < L; e2++)
        if (J[e2] == Je) s += V[e2];
      const size_t o = (size_t)cbase + 32 * (size_t)slot;
      ccols[o] = Je;
      cvals[o] = s;
      if (cvalsF) cvalsF[o] = (float)s;
    }
    nUnique += __popc(m);
  }
  if constexpr (!kFill) {
    if (lane == 0) count[I] = nUnique;
    return;
  } else {
    for (int slot = nUnique + lane; slot < cw; slot += 32) {
      const size_t o = (size_t)cbase + 32 * (size_t)slot;
      ccols[o] = I;
      cvals[o] = 0.0;
      if (cvalsF) cvalsF[o] = 0.f;
    }
  }
  if (lane == 0) {
    cdiag[I] = dsum;
    if (cdiagF) cdiagF[I] = (float)dsum;
  }
}

__global__ void k_slice_widths(int n, const int* __restrict__ count, int* width32) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  const int ns = (n + 31) >> 5;
  if (s >= ns) return;
  int w = 0;
  for (int r = s << 5; r < min(n, (s + 1) << 5); r++) w = max(w, count[r]);
  width32[s] = 32 * w;
}

__global__ void k_slice_meta(int n, const int* __restrict__ sliceOff, int4* meta, int* sliceRow, int* sliceRows,
                             int* rowSlice, int* maxWidth) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  const int ns = (n + 31) >> 5;
  if (s >= ns) return;
  const int r0 = s << 5, rows = min(32, n - r0);
  const int w = (sliceOff[s + 1] - sliceOff[s]) >> 5;
  meta[s] = make_int4(r0, rows, sliceOff[s], w);
  sliceRow[s] = r0;
  sliceRows[s] = rows;
  for (int r = 0; r < rows; r++) rowSlice[r0 + r] = s;
  atomicMax(maxWidth, w);
}

__global__ void k_compose(int n, int* ci, const int* __restrict__ ci2) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) ci[i] = ci2[ci[i]];
}

__global__ void k_dominance(LevelRows a, int* flag) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= a.n) return;
  int base, w;
  row_range(a, i, base, w);
  double s = 0.0;
  for (int k = 0; k < w; k++) {
    const int j = a.cols[base + 32 * k];
    if (j != i) s += fabs(a.vals[base + 32 * k]);
  }
  const double d = a.diag[i];
  if (!(d != 0.0 && s <= fabs(d) * (1.0 + 1e-8))) atomicOr(flag, 1);
}

// ---- level-0 pattern of a mesh on the device -------------------------------
// Self-column entries per self row of cellCells.
__global__ void k_ip_count(int n, const int* __restrict__ ccRow, const int* __restrict__ ccCol, int* cnt) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  int c = 0;
  for (int k = ccRow[i]; k < ccRow[i + 1]; k++) c += ccCol[k] < n ? 1 : 0;
  cnt[i] = c;
}

// The self-column entries in cellCells order, with the face behind each:
// the last of the row's faces (ascending) joining the two cells, as the
// face -> entry map of cellCells assigns it. *bad is set when no face joins
// an entry's cells.
__global__ void k_ip_fill(int n, const int* __restrict__ ccRow, const int* __restrict__ ccCol,
                          const int* __restrict__ cfRow, const int* __restrict__ cfCol,
                          const int* __restrict__ fc, const int* __restrict__ rowOff, int* col, int* face,
                          int* bad) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  int q = rowOff[i];
  for (int k = ccRow[i]; k < ccRow[i + 1]; k++) {
    const int j = ccCol[k];
    if (j >= n) continue;
    int f = -1;
    for (int t = cfRow[i]; t < cfRow[i + 1]; t++) {
      const int g = cfCol[t];
      const int a = fc[2 * g], b = fc[2 * g + 1];
      if ((a == i && b == j) || (a == j && b == i)) f = g;
    }
    if (f < 0) atomicOr(bad, 1);
    col[q] = j;
    face[q] = f;
    q++;
  }
}

// One in-place sweep towards the row-order greedy colouring: color[i] =
// the smallest colour no neighbour j < i holds. That colouring is the
// unique fixed point of the update (row i's value depends only on rows
// below it), and a sweep in which no row changes has read only settled
// values, so it is the fixed point. *changed is set when a row changes;
// *overflow when a row would need colour 32 or more.
__global__ void k_greedy_sweep(int n, const int* __restrict__ rowOff, const int* __restrict__ col, int* color,
                               int* changed, int* overflow) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  unsigned used = 0u;
  for (int q = rowOff[i]; q < rowOff[i + 1]; q++) {
    const int j = col[q];
    if (j < i) {
      const int c = __ldcg(color + j);
      if (c < 32) used |= 1u << c;
    }
  }
  if (used == 0xffffffffu) {
    atomicOr(overflow, 1);
    return;
  }
  const int c = __ffs(~used) - 1;
  if (c != __ldcg(color + i)) {
    __stcg(color + i, c);
    atomicOr(changed, 1);
  }
}

// per-colour row counts (colours < 32), one atomic per block and colour
__global__ void k_color_hist(int n, const int* __restrict__ color, int* hist) {
  __shared__ int h[32];
  if (threadIdx.x < 32) h[threadIdx.x] = 0;
  __syncthreads();
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) atomicAdd(&h[color[i] & 31], 1);
  __syncthreads();
  if (threadIdx.x < 32 && h[threadIdx.x]) atomicAdd(&hist[threadIdx.x], h[threadIdx.x]);
}

__global__ void k_color_flags(int n, const int* __restrict__ color, int c, int* flag) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) flag[i] = color[i] == c ? 1 : 0;
}

// rows of colour c in ascending order after those of the colours below it
__global__ void k_color_place(int n, const int* __restrict__ color, int c, const int* __restrict__ pos, int start,
                              int* perm, int* iperm) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n || color[i] != c) return;
  const int p = start + pos[i];
  perm[i] = p;
  iperm[p] = i;
}

// largest row length (atomicMax) and the SELL-32 size of colour-aligned
// slices (one warp per slice; slice s of colour c starts at row
// colorStart[c] + 32 (s - sliceStart[c]))
__global__ void k_row_max(int n, const int* __restrict__ rowOff, int* maxLen) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  int w = i < n ? rowOff[i + 1] - rowOff[i] : 0;
  for (int o = 16; o > 0; o >>= 1) w = max(w, __shfl_xor_sync(kFull, w, o));
  if ((threadIdx.x & 31) == 0 && w > 0) atomicMax(maxLen, w);
}

__global__ void k_sell_size(int nSlices, int nColors, const int* __restrict__ colorStart,
                            const int* __restrict__ sliceStart, const int* __restrict__ iperm,
                            const int* __restrict__ rowOff, unsigned long long* total) {
  const int s = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  if (s >= nSlices) return;  // whole warp
  int c = 0;
  while (c + 1 < nColors && sliceStart[c + 1] <= s) c++;
  const int r0 = colorStart[c] + 32 * (s - sliceStart[c]);
  const int rows = min(32, colorStart[c + 1] - r0);
  int w = 0;
  if (lane < rows) {
    const int i = iperm[r0 + lane];
    w = rowOff[i + 1] - rowOff[i];
  }
  for (int o = 16; o > 0; o >>= 1) w = max(w, __shfl_xor_sync(kFull, w, o));
  if (lane == 0) atomicAdd(total, 32ull * (unsigned long long)w);
}

// ELL-32 slots of every packed row p (groups x 32 rows, rows past n are
// padding): the permuted column and the face of each entry, padding (own
// row, no face); rowSlice of every row
__global__ void k_ell_fill(int n, int rowsPadded, int W, const int* __restrict__ iperm,
                           const int* __restrict__ rowOff, const int* __restrict__ col, const int* __restrict__ face,
                           const int* __restrict__ perm, int* cols, int* posSrc, int* rowSlice) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= rowsPadded) return;
  const bool live = p < n;
  const int g = p >> 5;
  const size_t base = (size_t)g * 32 * W + (p & 31);
  int i = 0, q0 = 0, cnt = 0;
  if (live) {
    i = iperm[p];
    q0 = rowOff[i];
    cnt = rowOff[i + 1] - q0;
    rowSlice[p] = g;
  }
  for (int k = 0; k < W; k++) {
    const size_t e = base + 32 * (size_t)k;
    if (k < cnt) {
      cols[e] = perm[col[q0 + k]];
      posSrc[e] = face[q0 + k];
    } else {
      cols[e] = live ? p : 32 * g;
      posSrc[e] = -1;
    }
  }
}

}  // namespace

int scan_scratch_ints(int n) { return cdiv(n, kScanTile) + 1; }

void scan_exclusive(const int* in, int* out, int n, int* scratch, cudaStream_t st) {
  const int tiles = std::max(1, cdiv(n, kScanTile));
  k_scan_tiles<<<tiles, kT, 0, st>>>(in, out, n, scratch);
  k_scan_tile_sums<<<1, kT, 0, st>>>(scratch, tiles);
  k_scan_add<<<std::max(1, cdiv(n, kT)), kT, 0, st>>>(out, n, scratch, tiles);
}

void fill_finest(long long entries, const int* posSrc, const double* src, double* vals, float* valsF, int n,
                 const int* iperm, const double* diagSrc, double* diag, float* diagF, cudaStream_t st) {
  if (entries > 0) k_fill_finest_vals<<<cdiv(entries, kT), kT, 0, st>>>(entries, posSrc, src, vals, valsF);
  if (n > 0) k_fill_finest_diag<<<cdiv(n, kT), kT, 0, st>>>(n, iperm, diagSrc, diag, diagF);
}

void aggregate_pairs(const LevelRows& a, double beta, int rounds, const int* order, const AggWork& w, int* ci,
                     cudaStream_t st) {
  const int n = a.n, g = cdiv(n, kT);
  k_agg_init<<<g, kT, 0, st>>>(a, w.maxw, w.partner);
  for (int r = 0; r < rounds; r++) {
    k_agg_best<<<g, kT, 0, st>>>(a, w.maxw, beta, w.partner, w.best);
    k_agg_match<<<g, kT, 0, st>>>(n, w.best, w.partner);
  }
  k_agg_join<<<g, kT, 0, st>>>(a, w.maxw, beta, w.partner, w.join);
  k_agg_flags<<<g, kT, 0, st>>>(n, w.partner, w.join, order, w.flag);
  scan_exclusive(w.flag, w.pos, n, w.scan, st);
  k_agg_ci_leaders<<<g, kT, 0, st>>>(n, w.partner, w.join, order, w.pos, ci);
  k_agg_ci_rest<<<g, kT, 0, st>>>(n, w.partner, w.join, ci);
}

void coarse_to_fine(int n, int nc, const int* ci, int* cnt, int* c2fRow, int* c2fCol, int* scanScratch,
                    cudaStream_t st) {
  cudaMemsetAsync(cnt, 0, sizeof(int) * (size_t)nc, st);
  k_c2f_count<<<cdiv(n, kT), kT, 0, st>>>(n, ci, cnt);
  scan_exclusive(cnt, c2fRow, nc, scanScratch, st);
  cudaMemsetAsync(cnt, 0, sizeof(int) * (size_t)nc, st);
  k_c2f_place<<<cdiv(n, kT), kT, 0, st>>>(n, ci, c2fRow, cnt, c2fCol);
  k_c2f_sort<<<cdiv(nc, kT), kT, 0, st>>>(nc, c2fRow, c2fCol);
}

void galerkin_count(const LevelRows& a, int nc, const int* ci, const int* c2fRow, const int* c2fCol, int* count,
                    int* overflow, cudaStream_t st) {
  k_galerkin<false><<<cdiv(nc, kGalWarps), 32 * kGalWarps, 0, st>>>(a, nc, ci, c2fRow, c2fCol, count, overflow,
                                                                      nullptr, nullptr, nullptr, nullptr, nullptr,
                                                                      nullptr);
}

void galerkin_fill(const LevelRows& a, int nc, const int* ci, const int* c2fRow, const int* c2fCol,
                   const int* sliceOff, int* cols, double* vals, float* valsF, double* diag, float* diagF,
                   cudaStream_t st) {
  k_galerkin<true><<<cdiv(nc, kGalWarps), 32 * kGalWarps, 0, st>>>(a, nc, ci, c2fRow, c2fCol, nullptr, nullptr,
                                                                     sliceOff, cols, vals, valsF, diag, diagF);
}

void slice_widths(int n, const int* count, int* width32, cudaStream_t st) {
  const int ns = cdiv(n, 32);
  k_slice_widths<<<cdiv(ns, kT), kT, 0, st>>>(n, count, width32);
}

void slice_meta_fill(int n, const int* sliceOff, int4* meta, int* sliceRow, int* sliceRows, int* rowSlice,
                     int* maxWidth, cudaStream_t st) {
  const int ns = cdiv(n, 32);
  k_slice_meta<<<cdiv(ns, kT), kT, 0, st>>>(n, sliceOff, meta, sliceRow, sliceRows, rowSlice, maxWidth);
}

void compose_index(int n, int* ci, const int* ci2, cudaStream_t st) {
  if (n > 0) k_compose<<<cdiv(n, kT), kT, 0, st>>>(n, ci, ci2);
}

void dominance_check(const LevelRows& a, int* flag, cudaStream_t st) {
  k_dominance<<<cdiv(a.n, kT), kT, 0, st>>>(a, flag);
}

}  // namespace dev
}  // namespace fvm

// ===========================================================================
// Host orchestration
namespace fvm {

#define CUDA_OK(call)                                                                            \
  do {                                                                                           \
    cudaError_t e_ = (call);                                                                     \
    if (e_ != cudaSuccess)                                                                       \
      throw ::fvm::Error(::fvm::kDeviceError, std::string(#call ": ") + cudaGetErrorString(e_)); \
  } while (0)

namespace {
// Device blocks of a rebuilt hierarchy are recycled by exact size; sizes
// rounded up to 1/8 of their power of two let a rebuild whose level sizes
// moved a little (another conductivity field) reuse them too.
size_t size_class(size_t bytes) {
  if (bytes <= 4096) return 4096;
  size_t p = 1;
  while (p < bytes) p <<= 1;
  const size_t g = p >> 3;
  return (bytes + g - 1) / g * g;
}
}  // namespace

bool AmgHierarchy::prepareFinestPatternDevice(const FinestDevice& in) {
  TraceRange traceRange("level-0 pattern on the device");
  const int n = in.conn->nRows;
  // ELL-32 needs at least 32768 rows (the host packing's rule); smaller
  // levels are packed on the host, where they take a few milliseconds
  if (n < 32768 || !in.ccRow || !in.ccCol || !in.cfRow || !in.cfCol || !in.faceCells || !in.symmetricPattern)
    return false;
  constexpr int kFewColors = 5;
  cudaStream_t st = setupStream_;
  const bool trace = getenv("FVM_TRACE") != nullptr;
  auto t0 = std::chrono::steady_clock::now();
  auto lap = [&](const char* what) {
    if (!trace) return;
    CUDA_OK(cudaStreamSynchronize(st));
    const auto t1 = std::chrono::steady_clock::now();
    fprintf(stderr, "[fvm device pattern] %-28s %8.2f ms\n", what,
            std::chrono::duration<double, std::milli>(t1 - t0).count());
    t0 = t1;
  };
  std::unique_ptr<FinestPattern> fpp(new FinestPattern());
  FinestPattern& fp = *fpp;
  DeviceArena tmp;  // work arrays of this build only
  int* flags = (int*)tmp.alloc(64 * sizeof(int));  // [0] bad face, [1] changed, [2] overflow, [3] max len, [8..39] hist
  unsigned long long* sellTotal = (unsigned long long*)tmp.alloc(sizeof(unsigned long long));
  CUDA_OK(cudaMemsetAsync(flags, 0, 64 * sizeof(int), st));
  CUDA_OK(cudaMemsetAsync(sellTotal, 0, sizeof(unsigned long long), st));
  int* h = reinterpret_cast<int*>(pinnedScalars());
  // self-column entries of cellCells with the face behind each
  int* cnt = (int*)tmp.alloc(sizeof(int) * ((size_t)n + 1));
  int* rowOff = (int*)tmp.alloc(sizeof(int) * ((size_t)n + 1));
  int* scan = (int*)tmp.alloc(sizeof(int) * (dev::scan_scratch_ints(n + 1) + 1));
  dev::k_ip_count<<<dev::cdiv(n, dev::kT), dev::kT, 0, st>>>(n, in.ccRow, in.ccCol, cnt);
  dev::scan_exclusive(cnt, rowOff, n, scan, st);
  CUDA_OK(cudaMemcpyAsync(h, rowOff + n, sizeof(int), cudaMemcpyDeviceToHost, st));
  CUDA_OK(cudaStreamSynchronize(st));
  const int nnz = h[0];
  if (nnz != in.conn->nnz()) return false;
  int* col = (int*)tmp.alloc(sizeof(int) * (size_t)std::max(nnz, 1));
  int* face = (int*)tmp.alloc(sizeof(int) * (size_t)std::max(nnz, 1));
  dev::k_ip_fill<<<dev::cdiv(n, dev::kT), dev::kT, 0, st>>>(n, in.ccRow, in.ccCol, in.cfRow, in.cfCol, in.faceCells,
                                                           rowOff, col, face, flags);
  // row-order greedy colouring: sweeps until one changes nothing, read back
  // every 32 sweeps (the flag is cleared before the last sweep of a batch)
  lap("entries and faces");
  int* color = cnt;  // the counts are no longer needed
  CUDA_OK(cudaMemsetAsync(color, 0, sizeof(int) * (size_t)n, st));
  constexpr int kBatch = 32, kMaxBatches = 128;
  bool settled = false;
  int batches = 0;
  for (int b = 0; b < kMaxBatches && !settled; b++, batches++) {
    for (int k = 0; k < kBatch; k++) {
      if (k == kBatch - 1) CUDA_OK(cudaMemsetAsync(flags + 1, 0, sizeof(int), st));
      dev::k_greedy_sweep<<<dev::cdiv(n, dev::kT), dev::kT, 0, st>>>(n, rowOff, col, color, flags + 1, flags + 2);
    }
    CUDA_OK(cudaMemcpyAsync(h, flags, 3 * sizeof(int), cudaMemcpyDeviceToHost, st));
    CUDA_OK(cudaStreamSynchronize(st));
    if (h[0] || h[2]) return false;  // an entry without a face, or a colour >= 32
    settled = h[1] == 0;
  }
  if (trace) fprintf(stderr, "[fvm device pattern] colouring settled within %d sweeps\n", 32 * batches);
  lap("colouring");
  if (!settled) return false;
  dev::k_color_hist<<<dev::cdiv(n, dev::kT), dev::kT, 0, st>>>(n, color, flags + 8);
  dev::k_row_max<<<dev::cdiv(n, dev::kT), dev::kT, 0, st>>>(n, rowOff, flags + 3);
  CUDA_OK(cudaMemcpyAsync(h, flags, 40 * sizeof(int), cudaMemcpyDeviceToHost, st));
  CUDA_OK(cudaStreamSynchronize(st));
  int C = 0;
  for (int c = 0; c < 32; c++)
    if (h[8 + c] > 0) C = c + 1;
  const int maxWidth = h[3];
  if (C < 1 || C > kFewColors || maxWidth > 8) return false;
  PackedLevel& pk = fp.packed;
  pk.n = n;
  pk.nColors = C;
  pk.colorStart.assign(C + 1, 0);
  for (int c = 0; c < C; c++) pk.colorStart[c + 1] = pk.colorStart[c] + h[8 + c];
  // colour-major permutation, ascending rows within a colour
  fp.perm = (int*)fp.arena.alloc(sizeof(int) * (size_t)n);
  fp.iperm = (int*)fp.arena.alloc(sizeof(int) * (size_t)n);
  int* flag = (int*)tmp.alloc(sizeof(int) * (size_t)n);
  int* pos = (int*)tmp.alloc(sizeof(int) * ((size_t)n + 1));
  for (int c = 0; c < C; c++) {
    dev::k_color_flags<<<dev::cdiv(n, dev::kT), dev::kT, 0, st>>>(n, color, c, flag);
    dev::scan_exclusive(flag, pos, n, scan, st);
    dev::k_color_place<<<dev::cdiv(n, dev::kT), dev::kT, 0, st>>>(n, color, c, pos, pk.colorStart[c], fp.perm,
                                                                 fp.iperm);
  }
  lap("permutation");
  // ELL-32 when the colour-aligned SELL-32 slices would not save more than
  // 15 % (the host packing's rule)
  std::vector<int> sliceStart(C + 1, 0);
  for (int c = 0; c < C; c++) sliceStart[c + 1] = sliceStart[c] + dev::cdiv(pk.colorStart[c + 1] - pk.colorStart[c], 32);
  const int nSellSlices = sliceStart[C];
  int* dStarts = (int*)tmp.alloc(sizeof(int) * 2 * (C + 1));
  std::vector<int> starts(pk.colorStart);
  starts.insert(starts.end(), sliceStart.begin(), sliceStart.end());
  CUDA_OK(cudaMemcpyAsync(dStarts, starts.data(), sizeof(int) * starts.size(), cudaMemcpyHostToDevice, st));
  dev::k_sell_size<<<dev::cdiv((long long)nSellSlices * 32, dev::kT), dev::kT, 0, st>>>(
      nSellSlices, C, dStarts, dStarts + C + 1, fp.iperm, rowOff, sellTotal);
  unsigned long long sellEntries = 0;
  CUDA_OK(cudaMemcpyAsync(&sellEntries, sellTotal, sizeof(sellEntries), cudaMemcpyDeviceToHost, st));
  CUDA_OK(cudaStreamSynchronize(st));
  const int groups = dev::cdiv(n, 32), W = maxWidth;
  const long long ellEntries = (long long)groups * 32 * W;
  if (W < 1 || ellEntries * 100 > (long long)sellEntries * 115) return false;
  pk.maxWidth = W;
  pk.ellWidth = W;
  pk.colorSliceStart = pk.colorStart;
  pk.sliceRow.resize(groups);
  pk.sliceRows.resize(groups);
  pk.sliceOff.resize(groups + 1);
  std::vector<int4> meta(groups);
  for (int g = 0; g < groups; g++) {
    pk.sliceRow[g] = 32 * g;
    pk.sliceRows[g] = std::min(32, n - 32 * g);
    pk.sliceOff[g] = 32 * W * g;
    meta[g] = make_int4(32 * g, pk.sliceRows[g], 32 * W * g, W);
  }
  pk.sliceOff[groups] = 32 * W * groups;
  fp.entries = (size_t)ellEntries;
  fp.cols = (int*)fp.arena.alloc(sizeof(int) * fp.entries);
  fp.posSrc = (int*)fp.arena.alloc(sizeof(int) * fp.entries);
  fp.rowSlice = (int*)fp.arena.alloc(sizeof(int) * (size_t)n);
  dev::k_ell_fill<<<dev::cdiv((long long)groups * 32, dev::kT), dev::kT, 0, st>>>(
      n, groups * 32, W, fp.iperm, rowOff, col, face, fp.perm, fp.cols, fp.posSrc, fp.rowSlice);
  lap("ELL-32 slots");
  fp.sliceRow = fp.arena.upload(pk.sliceRow);
  fp.sliceRows = fp.arena.upload(pk.sliceRows);
  fp.sliceOff = fp.arena.upload(pk.sliceOff);
  fp.meta = fp.arena.upload(meta);
  // the permutation on the host too (exports of level 0 use it)
  pk.perm.resize(n);
  pk.iperm.resize(n);
  CUDA_OK(cudaMemcpyAsync(pk.perm.data(), fp.perm, sizeof(int) * (size_t)n, cudaMemcpyDeviceToHost, st));
  CUDA_OK(cudaMemcpyAsync(pk.iperm.data(), fp.iperm, sizeof(int) * (size_t)n, cudaMemcpyDeviceToHost, st));
  CUDA_OK(cudaStreamSynchronize(st));
  lap("slices and host permutation");
  fp.key = in.key;
  fp.ordering = (int)kMulticolor;
  finest_ = std::move(fpp);
  return true;
}

void AmgHierarchy::prepareFinestPattern(const FinestDevice& in, int ordering) {
  if (finest_ && in.key != 0 && finest_->key == in.key && finest_->ordering == ordering) return;
  finest_.reset(new FinestPattern());
  FinestPattern& fp = *finest_;
  fp.key = in.key;
  fp.ordering = ordering;
  const CSR& c = *in.conn;
  const int n = c.nRows;
  // colours, permutation and slices of the pattern, with the CSR entry
  // stored in every packed slot
  std::unique_ptr<int[]> cols, posSrc;
  size_t E = 0;
  pack_pattern(c, in.symmetricPattern, in.segments, (SmootherOrdering)ordering, fp.packed, cols, posSrc, E);
  PackedLevel& p = fp.packed;
  fp.entries = E;
  if (in.entrySrc) {
    const std::vector<int>& src = *in.entrySrc;
    int* ps = posSrc.get();
    parallel_chunks((int)E, [&](int b, int e) {
      for (int q = b; q < e; q++)
        if (ps[q] >= 0) ps[q] = src[ps[q]];
    }, 1 << 18);
  }
  const int nSlices = (int)p.sliceRow.size();
  std::vector<int> rs(n);
  std::vector<int4> meta(nSlices);
  for (int s = 0; s < nSlices; s++) {
    for (int k = 0; k < p.sliceRows[s]; k++) rs[p.sliceRow[s] + k] = s;
    meta[s] = make_int4(p.sliceRow[s], p.sliceRows[s], p.sliceOff[s], (p.sliceOff[s + 1] - p.sliceOff[s]) / 32);
  }
  fp.sliceRow = fp.arena.upload(p.sliceRow);
  fp.sliceRows = fp.arena.upload(p.sliceRows);
  fp.sliceOff = fp.arena.upload(p.sliceOff);
  fp.cols = fp.arena.upload(cols.get(), E);
  fp.rowSlice = fp.arena.upload(rs);
  fp.meta = fp.arena.upload(meta);
  fp.posSrc = fp.arena.upload(posSrc.get(), E);
  fp.iperm = fp.arena.upload(p.iperm);
  fp.perm = fp.arena.upload(p.perm);
}

void AmgHierarchy::allocVectors(DevLevel& d, bool mixed) {
  const size_t nb = (size_t)d.n * sizeof(double);
  d.x = (double*)arena_.alloc(size_class(nb));
  d.b = (double*)arena_.alloc(size_class(nb));
  d.r = (double*)arena_.alloc(size_class(nb));
  d.tmp = (double*)arena_.alloc(size_class(nb));
  CUDA_OK(cudaMemsetAsync(d.x, 0, nb, setupStream_));
  CUDA_OK(cudaMemsetAsync(d.b, 0, nb, setupStream_));
  CUDA_OK(cudaMemsetAsync(d.tmp, 0, nb, setupStream_));
  d.nPartials = dev::residual_partials(d.nSlices, d.n, d.ellWidth);
  d.partials = (double*)arena_.alloc(size_class(sizeof(double) * (d.nPartials + 1)));
  if (mixed) {
    const size_t fb = (size_t)d.n * sizeof(float);
    d.xF = (float*)arena_.alloc(size_class(fb));
    d.bF = (float*)arena_.alloc(size_class(fb));
    d.rF = (float*)arena_.alloc(size_class(fb));
    d.tmpF = (float*)arena_.alloc(size_class(fb));
    CUDA_OK(cudaMemsetAsync(d.xF, 0, fb, setupStream_));
    CUDA_OK(cudaMemsetAsync(d.tmpF, 0, fb, setupStream_));
  }
}

int* AmgHierarchy::pendingStatus() { return reinterpret_cast<int*>(pinnedScalars() + 31); }

void AmgHierarchy::finishBuild() {
  if (!setupStream_) return;
  CUDA_OK(cudaStreamSynchronize(setupStream_));
  if (!inversePending_) return;
  inversePending_ = false;
  FVM_REQUIRE(*pendingStatus() == 0, kBadArgument, "singular coarsest-level matrix");
}

void AmgHierarchy::buildDevice(const FinestDevice& in, const SolverOptions& opt, bool deferCheck) {
  TraceRange traceRange("AMG hierarchy on the device");
  const bool trace = getenv("FVM_TRACE") != nullptr;
  auto t0 = std::chrono::steady_clock::now();
  auto lap = [&](const char* what) {
    if (!trace) return;
    CUDA_OK(cudaStreamSynchronize(setupStream_));
    const auto t1 = std::chrono::steady_clock::now();
    fprintf(stderr, "[fvm device setup] %-30s %8.2f ms\n", what,
            std::chrono::duration<double, std::milli>(t1 - t0).count());
    t0 = t1;
  };
  FVM_REQUIRE(in.conn && in.offSrc && in.diag, kBadArgument, "device-built hierarchy: missing level-0 input");
  FVM_REQUIRE(!opt.finestOnly(), kUnsupported, "device-built hierarchy: not for the Jacobi solver or preconditioner");
  release();
  opt_ = opt;
  if (!setupStream_) CUDA_OK(cudaStreamCreateWithFlags(&setupStream_, cudaStreamNonBlocking));
  cudaStream_t st = setupStream_;
  const bool mixed = opt.precision == kMixed;
  {
    const bool cached = finest_ && in.key != 0 && finest_->key == in.key && finest_->ordering == (int)opt.ordering;
    if (!cached && !(opt.patternOnDevice && opt.ordering == kMulticolor && prepareFinestPatternDevice(in)))
      prepareFinestPattern(in, (int)opt.ordering);
  }
  deviceBuilt_ = true;
  lap("level-0 pattern");
  const FinestPattern& fp = *finest_;
  const PackedLevel& p0 = fp.packed;
  const int n0 = p0.n;
  const size_t maxL = (size_t)std::max(1, opt.maxCoarseLevels) + 2;
  lv_.clear();
  lv_.reserve(maxL);
  lv_.emplace_back();
  {
    DevLevel& d = lv_[0];
    d.n = n0;
    d.nColors = p0.nColors;
    d.nSlices = (int)p0.sliceRow.size();
    d.maxWidth = p0.maxWidth;
    d.ellWidth = p0.ellWidth;
    d.colorSliceStart = p0.colorSliceStart;
    d.entries = fp.entries;
    d.sliceRow = fp.sliceRow;
    d.sliceRows = fp.sliceRows;
    d.sliceOff = fp.sliceOff;
    d.cols = fp.cols;
    d.rowSlice = fp.rowSlice;
    d.meta = fp.meta;
    d.vals = (double*)arena_.alloc(size_class(sizeof(double) * d.entries));
    d.diag = (double*)arena_.alloc(size_class(sizeof(double) * n0));
    if (mixed) {
      d.valsF = (float*)arena_.alloc(size_class(sizeof(float) * d.entries));
      d.diagF = (float*)arena_.alloc(size_class(sizeof(float) * n0));
    }
    lap("level 0 allocations");
    dev::fill_finest((long long)d.entries, fp.posSrc, in.offSrc, d.vals, d.valsF, n0, fp.iperm, in.diag, d.diag,
                     d.diagF, st);
    lap("level 0 values filled");
    allocVectors(d, mixed);
  }
  // work arrays sized by level 0, shared by every level
  dev::AggWork w;
  w.maxw = (double*)arena_.alloc(size_class(sizeof(double) * n0));
  w.best = (int*)arena_.alloc(size_class(sizeof(int) * n0));
  w.partner = (int*)arena_.alloc(size_class(sizeof(int) * n0));
  w.join = (int*)arena_.alloc(size_class(sizeof(int) * n0));
  w.flag = (int*)arena_.alloc(size_class(sizeof(int) * n0));
  w.pos = (int*)arena_.alloc(size_class(sizeof(int) * (n0 + 1)));
  w.scan = (int*)arena_.alloc(size_class(sizeof(int) * (dev::scan_scratch_ints(n0 + 1) + 1)));
  int* flags = (int*)arena_.alloc(4096);  // [0] overflow, [1] max width, [2] not dominant
  int* hflags = reinterpret_cast<int*>(pinnedScalars());
  lap("level 0 values");

  // Coarse level of `fine` under the aggregation ci (nc rows): coarse-to-fine
  // lists into fine's c2fRow / c2fCol, then counts, slice widths and
  // offsets, then the Galerkin entries into c (FP32 copies when f32).
  auto galerkin = [&](DevLevel& fine, int* ci, int nc, DevLevel& c, bool f32) -> long long {
    fine.ci = ci;
    fine.nCoarse = nc;
    fine.c2fRow = (int*)arena_.alloc(size_class(sizeof(int) * (nc + 1)));
    fine.c2fCol = (int*)arena_.alloc(size_class(sizeof(int) * fine.n));
    dev::coarse_to_fine(fine.n, nc, ci, w.flag, fine.c2fRow, fine.c2fCol, w.scan, st);
    const dev::LevelRows af{fine.n, fine.cols, fine.vals, fine.diag, fine.meta, fine.rowSlice, fine.ellWidth};
    const int nSlices = (nc + 31) / 32;
    int* sliceOff = (int*)arena_.alloc(size_class(sizeof(int) * (nSlices + 1)));
    CUDA_OK(cudaMemsetAsync(flags, 0, 3 * sizeof(int), st));
    dev::galerkin_count(af, nc, ci, fine.c2fRow, fine.c2fCol, w.best, flags, st);
    dev::slice_widths(nc, w.best, w.join, st);
    dev::scan_exclusive(w.join, sliceOff, nSlices, w.scan, st);
    CUDA_OK(cudaMemcpyAsync(hflags, sliceOff + nSlices, sizeof(int), cudaMemcpyDeviceToHost, st));
    CUDA_OK(cudaMemcpyAsync(hflags + 1, flags, sizeof(int), cudaMemcpyDeviceToHost, st));
    CUDA_OK(cudaStreamSynchronize(st));
    const long long E = hflags[0];
    FVM_REQUIRE(hflags[1] == 0, kUnsupported,
                "device-built hierarchy: an aggregate's entries exceed the Galerkin kernel's capacity");
    const size_t e1 = (size_t)std::max<long long>(E, 1);
    c.n = nc;
    c.nColors = 1;
    c.nSlices = nSlices;
    c.colorSliceStart = {0, nSlices};
    c.entries = (size_t)E;
    c.ellWidth = 0;
    c.sliceOff = sliceOff;
    c.cols = (int*)arena_.alloc(size_class(sizeof(int) * e1));
    c.vals = (double*)arena_.alloc(size_class(sizeof(double) * e1));
    c.diag = (double*)arena_.alloc(size_class(sizeof(double) * nc));
    c.valsF = f32 ? (float*)arena_.alloc(size_class(sizeof(float) * e1)) : nullptr;
    c.diagF = f32 ? (float*)arena_.alloc(size_class(sizeof(float) * nc)) : nullptr;
    c.meta = (int4*)arena_.alloc(size_class(sizeof(int4) * nSlices));
    c.sliceRow = (int*)arena_.alloc(size_class(sizeof(int) * nSlices));
    c.sliceRows = (int*)arena_.alloc(size_class(sizeof(int) * nSlices));
    c.rowSlice = (int*)arena_.alloc(size_class(sizeof(int) * nc));
    // the fill writes every row's entries and padding; the lanes of the last
    // slice past the last row keep these (column 0) so that no index in the
    // level is undefined
    CUDA_OK(cudaMemsetAsync(c.cols, 0, sizeof(int) * e1, st));
    dev::galerkin_fill(af, nc, ci, fine.c2fRow, fine.c2fCol, sliceOff, c.cols, c.vals, c.valsF, c.diag, c.diagF,
                       st);
    dev::slice_meta_fill(nc, sliceOff, c.meta, c.sliceRow, c.sliceRows, c.rowSlice, flags + 1, st);
    CUDA_OK(cudaMemcpyAsync(hflags, flags + 1, sizeof(int), cudaMemcpyDeviceToHost, st));
    CUDA_OK(cudaStreamSynchronize(st));
    c.maxWidth = hflags[0];
    return E;
  };
  // one matching: coarse size of `a`'s pairs (ci written)
  auto match = [&](const dev::LevelRows& a, const int* order, int* ci) {
    dev::aggregate_pairs(a, opt.matchBeta, opt.matchRounds, order, w, ci, st);
    CUDA_OK(cudaMemcpyAsync(hflags, w.pos + a.n, sizeof(int), cudaMemcpyDeviceToHost, st));
    CUDA_OK(cudaStreamSynchronize(st));
    return hflags[0];
  };
  for (int l = 0;; l++) {
    if (l >= opt.maxCoarseLevels || lv_.size() + 1 > maxL) break;
    {
      const DevLevel& f = lv_[l];
      if (opt.coarsestSize > 0 ? f.n <= opt.coarsestSize : f.n <= 3) break;
    }
    DevLevel& f = lv_[l];
    const dev::LevelRows a{f.n, f.cols, f.vals, f.diag, f.meta, f.rowSlice, f.ellWidth};
    int* ci = (int*)arena_.alloc(size_class(sizeof(int) * f.n));
    int nc = match(a, l == 0 ? fp.iperm : nullptr, ci);
    // a level that no longer shrinks is the coarsest
    if (nc <= 0 || nc >= f.n || (double)nc > 0.9 * f.n) break;
    if (opt.matchPasses == 2 && (opt.coarsestSize <= 0 || nc > opt.coarsestSize)) {
      // pairs of pairs: the pairs' Galerkin matrix (not kept) is matched
      // again and the two aggregations composed
      DevLevel t;
      galerkin(f, ci, nc, t, false);
      const dev::LevelRows at{t.n, t.cols, t.vals, t.diag, t.meta, t.rowSlice, t.ellWidth};
      int* ci2 = (int*)arena_.alloc(size_class(sizeof(int) * t.n));
      const int nc2 = match(at, nullptr, ci2);
      if (nc2 > 0 && nc2 < nc) {
        dev::compose_index(f.n, ci, ci2, st);
        nc = nc2;
      }
    }
    lv_.emplace_back();
    const long long E = galerkin(lv_[l], ci, nc, lv_.back(), mixed);
    allocVectors(lv_.back(), mixed);
    if (trace) {
      char msg[96];
      snprintf(msg, sizeof msg, "level %d: %d rows, %lld entries", l + 1, nc, E);
      lap(msg);
    }
  }
  const int L = (int)lv_.size();
  // launch plans before the coarsest inverse (the tuning does not run the
  // coarsest level): the inverse is the last GPU work of the build, and the
  // host may queue or prepare other work while it runs
  CUDA_OK(cudaStreamSynchronize(st));
  prepareChebyshev();
  tunePlans();
  lap("launch plans");
  // coarsest direct solve: dense inverse built on the GPU (no pivoting when
  // the level is diagonally dominant), FP32 copy for the FP32 cycle
  if (opt.coarseSolver == kCoarseDirect) {
    DevLevel& c = lv_[L - 1];
    FVM_REQUIRE(c.n <= 4096, kTooLarge,
                "coarsest level too large for the dense direct solve (max 4096 rows); set coarsestSize");
    const size_t nn = (size_t)c.n * c.n;
    if (c.n <= 128) {
      // small: inverted on the host (a launch sequence costs more)
      PackedLevel h;
      h.n = c.n;
      const int ns = c.nSlices;
      std::vector<int4> meta(ns);
      if (c.ellWidth == 0) {
        CUDA_OK(cudaMemcpyAsync(meta.data(), c.meta, sizeof(int4) * ns, cudaMemcpyDeviceToHost, st));
      } else {
        for (int s = 0; s < ns; s++)
          meta[s] = make_int4(32 * s, std::min(32, c.n - 32 * s), 32 * s * c.ellWidth, c.ellWidth);
      }
      h.cols.resize(c.entries);
      h.vals.resize(c.entries);
      h.diag.resize(c.n);
      CUDA_OK(cudaMemcpyAsync(h.cols.data(), c.cols, sizeof(int) * c.entries, cudaMemcpyDeviceToHost, st));
      CUDA_OK(cudaMemcpyAsync(h.vals.data(), c.vals, sizeof(double) * c.entries, cudaMemcpyDeviceToHost, st));
      CUDA_OK(cudaMemcpyAsync(h.diag.data(), c.diag, sizeof(double) * c.n, cudaMemcpyDeviceToHost, st));
      CUDA_OK(cudaStreamSynchronize(st));
      h.sliceRow.resize(ns);
      h.sliceRows.resize(ns);
      h.sliceOff.resize(ns + 1);
      for (int s = 0; s < ns; s++) {
        h.sliceRow[s] = meta[s].x;
        h.sliceRows[s] = meta[s].y;
        h.sliceOff[s] = meta[s].z;
      }
      h.sliceOff[ns] = (int)c.entries;
      std::vector<double> inv;
      dense_inverse(h, inv);
      coarseInv_ = arena_.upload(inv);
    } else {
      FVM_REQUIRE(c.ellWidth == 0, kUnsupported, "coarsest level in ELL-32 layout");
      const dev::LevelRows a{c.n, c.cols, c.vals, c.diag, c.meta, c.rowSlice, c.ellWidth};
      CUDA_OK(cudaMemsetAsync(flags + 2, 0, sizeof(int), st));
      dev::dominance_check(a, flags + 2, st);
      CUDA_OK(cudaMemcpyAsync(hflags, flags + 2, sizeof(int), cudaMemcpyDeviceToHost, st));
      CUDA_OK(cudaStreamSynchronize(st));
      const bool dominant = hflags[0] == 0;
      void* gjScratch = arena_.alloc(size_class(dev::gauss_jordan_scratch_bytes(c.n)));
      coarseInv_ = (double*)arena_.alloc(size_class(sizeof(double) * nn));
      if (dominant) {
        dev::dense_from_sell(c.view64(), c.nSlices, coarseInv_, st);
        // a symmetric level (a diffusion operator's Galerkin level) takes
        // the symmetric sweep: half the products
        CUDA_OK(cudaMemsetAsync(flags + 2, 0, sizeof(int), st));
        dev::dense_symmetry_check(c.n, coarseInv_, flags + 2, st);
        CUDA_OK(cudaMemcpyAsync(hflags, flags + 2, sizeof(int), cudaMemcpyDeviceToHost, st));
        CUDA_OK(cudaStreamSynchronize(st));
        if (hflags[0] == 0)
          dev::gauss_jordan_inverse_symmetric(c.n, coarseInv_, gjScratch, st);
        else
          dev::gauss_jordan_inverse_dominant(c.n, coarseInv_, gjScratch, st);
      } else {
        double* dA = (double*)arena_.alloc(size_class(sizeof(double) * nn));
        dev::dense_from_sell(c.view64(), c.nSlices, dA, st);
        dev::gauss_jordan_inverse(c.n, dA, coarseInv_, gjScratch, st);
      }
      // the status is read by finishBuild
      CUDA_OK(cudaMemcpyAsync(pendingStatus(), dev::gauss_jordan_status(c.n, gjScratch), sizeof(int),
                              cudaMemcpyDeviceToHost, st));
      inversePending_ = true;
    }
    if (mixed) {
      coarseInvF_ = (float*)arena_.alloc(size_class(sizeof(float) * nn));
      dev::cast_d2f(nn, coarseInv_, coarseInvF_, st);
    }
    if (trace) {
      finishBuild();
      lap("coarsest inverse");
    }
  }
  if (!deferCheck) finishBuild();
  if (trace) {
    fprintf(stderr, "[fvm device setup] levels:");
    for (int l = 0; l < L; l++) fprintf(stderr, " %d", lv_[l].n);
    fprintf(stderr, "\n");
  }
}

std::vector<int> AmgHierarchy::coarseIndexHost(int l) const {
  FVM_REQUIRE(l >= 0 && l + 1 < (int)lv_.size(), kBadArgument, "no coarser level");
  if (!deviceBuilt_) return ref_[l].coarseIndex;
  const DevLevel& d = lv_[l];
  std::vector<int> ci(d.n);
  CUDA_OK(cudaMemcpy(ci.data(), d.ci, sizeof(int) * d.n, cudaMemcpyDeviceToHost));
  if (l > 0) return ci;
  std::vector<int> ref(d.n);
  const PackedLevel& p = finest_->packed;
  for (int i = 0; i < d.n; i++) ref[i] = ci[p.perm[i]];
  return ref;
}

}  // namespace fvm
