// AMG hierarchy construction on the host.
//
// The integer work (greedy pairwise aggregation, coarse-to-fine map,
// coarse sparsity pattern) and the FP64 Galerkin coarse matrices follow
// the reference's CRMatrix routines operation for operation, so level
// sizes, aggregation indices and coarse coefficients are bit-identical to
// the reference on the same fine matrix. On top of that each level gets a
// deterministic greedy colouring and a colour-major row permutation, and
// is packed into SELL-32 slices for the GPU smoothers.
#pragma once

#include <functional>
#include <memory>
#include <vector>

#include "common.hpp"

namespace fvm {

// One level in the reference's row order: self rows only, implicit
// diagonal, columns restricted to self rows (ghost couplings of the
// finest level are zero after boundary elimination and are dropped).
struct RefLevel {
  int n = 0;
  CSR conn;
  std::vector<double> diag;
  std::vector<double> off;
  // to the next coarser level (empty on the coarsest)
  std::vector<int> coarseIndex;  // fine row -> coarse row (reference CRMatrix.h:468-586)
  int nCoarse = 0;
  // the column pattern is known to be structurally symmetric (cellCells and
  // the Galerkin levels built from a symmetric level); otherwise the
  // colouring uses the pattern of A + A^T
  bool symmetricPattern = false;
  // optional row offsets of independent diagonal blocks (a batch of
  // meshes; no entry couples two blocks): the aggregation of each block
  // runs in parallel, with the same result as the sequential walk
  std::vector<int> segments;
};

// Greedy aggregation (reference CRMatrix::createCoarsening). Returns the
// number of coarse rows.
int create_coarsening(const RefLevel& a, int groupSize, double weightRatioThreshold,
                      std::vector<int>& coarseIndex, std::vector<int>* coarseSegments = nullptr);

// Coarse-to-fine rows (MultiFieldMatrix::createCoarseToFineMapping), coarse
// connectivity (CRMatrix::createCoarseConnectivity) and Galerkin values
// (CRMatrix::createCoarseMatrix).
void create_coarse_level(const RefLevel& fine, RefLevel& coarse, CSR& coarseToFine);

struct HierarchyOptions {
  int maxCoarseLevels = 30;
  int groupSize = 2;
  double weightRatioThreshold = 0.65;
  // stop once a kept level has at most this many rows (0: the reference's
  // rule only -- stop when a level fails to shrink or reaches <= 3 rows)
  int coarsestSize = 0;
  // count of rows+ghosts of the finest system, used by the reference's
  // "did this level shrink" test on level 0
  int finestLocalSize = 0;
};

// Builds levels[1..] from levels[0]; levels.size() - 1 coarse levels are
// kept, following AMG::createCoarseLevels (serial build, AMG.cpp:150-210).
// spareLevels / spareC2f (optional, indexed by level): objects of an earlier
// build whose buffers the new levels reuse. onLevel (optional) is called
// with the index of each new coarse level once its matrix is complete (the
// caller may then read its conn / diag / off from another thread while the
// next levels are built; levels must have capacity for every level).
void build_hierarchy(std::vector<RefLevel>& levels, const HierarchyOptions& opt,
                     std::vector<CSR>& coarseToFine, std::vector<RefLevel>* spareLevels = nullptr,
                     std::vector<CSR>* spareC2f = nullptr,
                     const std::function<void(int)>& onLevel = nullptr);

// Packed, colour-permuted form of one level for the GPU.
struct PackedLevel {
  int n = 0;
  int nColors = 0;
  std::vector<int> colorStart;       // nColors+1 row offsets (permuted order)
  std::vector<int> colorSliceStart;  // nColors+1 slice offsets
  std::vector<int> sliceRow;         // first row of each slice
  std::vector<int> sliceRows;        // rows in each slice (<= 32)
  std::vector<int> sliceOff;         // nSlices+1 offsets into cols/vals (32 per width unit)
  std::vector<int> cols;             // permuted columns, slice-column-major; padding = own row
  std::vector<double> vals;          // padding = 0
  std::vector<double> diag;          // permuted
  std::vector<int> perm;             // reference row -> permuted row
  std::vector<int> iperm;            // permuted row -> reference row
  // transfer to the next coarser level, in permuted numbering of both
  std::vector<int> coarseIndex;      // fine row -> coarse row
  std::vector<int> c2fRow, c2fCol;   // coarse row -> fine rows, ascending reference order
  int maxWidth = 0;
  // > 0: ELL-32 layout (slices = aligned 32-row groups of this width, not
  // aligned to colours; colour passes use colorStart rows)
  int ellWidth = 0;
};

enum SmootherOrdering { kMulticolor = 0, kSequential = 1 };

// Greedy colouring in reference row order: each row takes the smallest
// colour unused by its already-coloured neighbours.
int greedy_coloring(const CSR& conn, std::vector<int>& color);
// The colouring the multicolour smoothers use: row-order greedy, or when
// that needs more than five colours the better (fewer colours) of it and
// smallest-last-order greedy; deterministic.
// With segments (row offsets of independent diagonal blocks) the blocks
// are coloured in parallel, with the same result.
int multicolor(const CSR& conn, std::vector<int>& color, bool symmetricPattern = true,
               const std::vector<int>* segments = nullptr);
// Pattern of A + A^T: each row keeps its stored columns, followed by the
// columns present only in the transpose, ascending. Returns false (and
// leaves out untouched) when the pattern is already symmetric.
bool symmetrize_pattern(const CSR& a, CSR& out);
// true when every stored (i, j) has a stored (j, i)
bool pattern_is_symmetric(const CSR& a);

void pack_level(const RefLevel& lv, SmootherOrdering ordering, PackedLevel& out);
// The same colouring, permutation and slices for a pattern alone: out gets
// everything but cols, vals and diag; cols (the packed columns) and pos
// (the CSR entry index of every packed slot, -1 for padding) are filled in
// parallel into fresh arrays of `slots` ints, never zero-initialised.
void pack_pattern(const CSR& conn, bool symmetricPattern, const std::vector<int>& segments,
                  SmootherOrdering ordering, PackedLevel& out, std::unique_ptr<int[]>& cols,
                  std::unique_ptr<int[]>& pos, size_t& slots);
void pack_transfer(const RefLevel& fine, const CSR& coarseToFine, PackedLevel& pf,
                   const PackedLevel& pc);

// Dense inverse of a (small) level matrix by Gauss-Jordan elimination with
// partial pivoting, in the level's permuted numbering, row-major.
void dense_inverse(const PackedLevel& lv, std::vector<double>& inv);

}  // namespace fvm
