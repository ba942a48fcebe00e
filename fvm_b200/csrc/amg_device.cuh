// Device-built AMG hierarchy for the mixed-precision path: parallel
// pairwise aggregation by handshake matching, Galerkin coarse matrices and
// their SELL-32 packing, all as sm_100a kernels. The reference's greedy
// walk (CRMatrix::createCoarsening, fvmbase/CRMatrix.h:468-586) is
// sequential by construction; this path replaces it where the aggregation
// need not be bit-exact (the FP32 preconditioner under FP64 refinement is
// judged only by the converged field).
#pragma once

#include <cuda_runtime.h>

#include "kernels.cuh"

namespace fvm {
namespace dev {

// Row access to a level matrix (SELL-32 or ELL-32 layout, FP64 values).
struct LevelRows {
  int n;
  const int* cols;
  const double* vals;
  const double* diag;
  const int4* meta;      // SELL-32: per slice {first row, rows, offset, width}
  const int* rowSlice;   // SELL-32: row -> slice
  int ellWidth;          // > 0: ELL-32 (aligned 32-row groups of this width)
};

// Exclusive prefix sum of n ints: out[0..n], out[n] = total. scratch holds
// scan_scratch_ints(n) ints. Asynchronous on st.
int scan_scratch_ints(int n);
void scan_exclusive(const int* in, int* out, int n, int* scratch, cudaStream_t st);

// Level-0 values of a cached pattern: vals[p] = src[posSrc[p]] (0 where
// posSrc < 0, the padding), diag[p] = diagSrc[iperm[p]]; FP32 copies too.
void fill_finest(long long entries, const int* posSrc, const double* src, double* vals, float* valsF, int n,
                 const int* iperm, const double* diagSrc, double* diag, float* diagF, cudaStream_t st);

// Parallel pairwise aggregation of one level. Strength of (i, j): |a_ij| /
// max(|a_ii|, |a_jj|) (the reference's weight); a neighbour is a candidate
// when its strength is at least beta times the row's strongest. `rounds`
// handshake rounds pair rows that are each other's strongest unpaired
// candidate; a row left over joins the pair of its strongest paired
// candidate, or stays alone. Coarse rows are numbered by their leading
// (smallest) fine row in `order` (null: the level's own order): ci[i] is
// the coarse row of fine row i. Work arrays: 4 n ints + n doubles + the
// scan scratch. Returns nothing; *nCoarse (device) gets the coarse size.
struct AggWork {
  double* maxw;
  int *best, *partner, *join, *flag, *pos, *scan;
};
void aggregate_pairs(const LevelRows& a, double beta, int rounds, const int* order, const AggWork& w, int* ci,
                     cudaStream_t st);

// coarse-to-fine lists: c2fRow (nc + 1) and c2fCol (n), each list ascending;
// cnt holds nc ints of scratch
void coarse_to_fine(int n, int nc, const int* ci, int* cnt, int* c2fRow, int* c2fCol, int* scanScratch,
                    cudaStream_t st);

// Galerkin product Ac = P^T A P for piecewise-constant P, one warp per
// coarse row. Pass 1 (count != null): unique off-diagonal coarse columns
// per row into count[I]. Pass 2: the row's columns (first-visit order over
// its fine rows ascending, entries in stored order) and sums into the
// coarse SELL-32 level (natural row order, 32-row slices described by
// sliceOff), padding (own row, 0); diagonal = sum of the fine diagonals and
// of the entries inside the aggregate. FP64 values, and FP32 copies where
// valsF / diagF are not null. *overflow is set when an aggregate's entries
// exceed the per-warp capacity.
constexpr int kGalerkinCap = 512;
void galerkin_count(const LevelRows& a, int nc, const int* ci, const int* c2fRow, const int* c2fCol, int* count,
                    int* overflow, cudaStream_t st);
void galerkin_fill(const LevelRows& a, int nc, const int* ci, const int* c2fRow, const int* c2fCol,
                   const int* sliceOff, int* cols, double* vals, float* valsF, double* diag, float* diagF,
                   cudaStream_t st);

// Natural-order SELL-32 structure from per-row counts: width[s] = max count
// in slice s (nSlices = ceil(n / 32)); after a scan of 32 * width into
// sliceOff: meta, sliceRow, sliceRows, rowSlice.
void slice_widths(int n, const int* count, int* width32, cudaStream_t st);
void slice_meta_fill(int n, const int* sliceOff, int4* meta, int* sliceRow, int* sliceRows, int* rowSlice,
                     int* maxWidth, cudaStream_t st);

// ci[i] = ci2[ci[i]]: two aggregations composed
void compose_index(int n, int* ci, const int* ci2, cudaStream_t st);

// *flag = 1 unless every row is diagonally dominant (|a_ii| >= sum |a_ij|
// up to a relative slack of 1e-8); *flag must be 0 on entry
void dominance_check(const LevelRows& a, int* flag, cudaStream_t st);

}  // namespace dev
}  // namespace fvm
