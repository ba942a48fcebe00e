// Launch wrappers for the sm_100a kernels of the thermal/AMG hot path.
// Every wrapper enqueues on the given stream and never synchronises, so
// sequences of them can be captured into CUDA graphs.
#pragma once

#include <cuda_runtime.h>

namespace fvm {
namespace dev {

// A level matrix in colour-permuted SELL-32 form (see amg_setup.hpp).
template <class T>
struct SellView {
  int n;
  const int* sliceRow;
  const int* sliceRows;
  const int* sliceOff;
  const int* cols;
  const T* vals;
  const T* diag;
  // per slice, packed for a single 16-byte load: first row, rows (<= 32),
  // offset of its first entry, width (entries per row, padded)
  const int4* meta;
  // > 0: ELL-32 layout -- the slices are the aligned 32-row groups, all of
  // this width, so a slice's metadata and a row's slice are computed, not
  // loaded (colour passes then take row ranges instead of slice ranges)
  int ellWidth = 0;
};

// ---- smoothers -----------------------------------------------------------
// One Gauss-Seidel pass over the rows of slices [s0, s1) (one colour block;
// on an ELL-32 level s0, s1 are the colour's first and end ROWS):
// x_i = -(b_i + sum_j a_ij x_j) / a_ii
// Launch plan of the SELL-32 smoother kernels, picked per level by the
// autotuner: threads per row (1, 2 or 4: the entries of a row are split
// round-robin over the threads, their products are formed in parallel and
// summed in stored order, so every plan gives bitwise the same result) and
// threads per block (128 or 256). ELL-32 levels ignore it.
struct RowPlan {
  int tpr = 1;
  int block = 256;
  int ellRows = 1;  // ELL-32 levels: rows per thread of the Gauss-Seidel pass (1 or 2)
  bool isDefault() const { return tpr == 1 && block == 256 && ellRows == 1; }
};

// With xc (ELL-32 levels only): the pass is part of the first forward
// sweep after a prolongation that would have assigned x = xc[ci]; rows of
// later colours are read from xc (bitwise that prolongation + the pass)
template <class T>
void gs_color(const SellView<T>& a, int s0, int s1, T* x, const T* b, cudaStream_t st, RowPlan plan = RowPlan(),
              const T* xc = nullptr, const int* ci = nullptr);
// Lexicographic Gauss-Seidel by a single thread in row order (reverse when
// asked): the reference's CRMatrix::forwardGS / reverseGS, for parity runs.
template <class T>
void gs_sequential(const SellView<T>& a, T* x, const T* b, bool reverse, cudaStream_t st);
// Jacobi: xnew_i = -(b_i + sum_j a_ij xold_j) / a_ii over all rows
template <class T>
void jacobi(const SellView<T>& a, int nSlices, const T* xold, T* xnew, const T* b, cudaStream_t st);
// damped Jacobi: xnew = xold + w (Jacobi update - xold). With xc (and ci),
// xold is taken as the prolongation xc[ci] (the values a prolongation that
// assigns would have written; xold unused): bitwise the result of that
// prolongation followed by this pass, one launch and one x round trip less.
template <class T>
void jacobi_damped(const SellView<T>& a, int nSlices, const T* xold, T* xnew, const T* b, T w, cudaStream_t st,
                   RowPlan plan = RowPlan(), const T* xc = nullptr, const int* ci = nullptr);
// one step of a Chebyshev smoother on D^-1 A over all rows: res = b + A x,
// dv = c1 dv + c2 (-res / a_ii) (first: dv = c2 (-res / a_ii), dv not read),
// xnew = x + dv; x and xnew distinct
template <class T>
void chebyshev_step(const SellView<T>& a, int nSlices, const T* x, T* xnew, T* dv, const T* b, T c1, T c2,
                    bool first, cudaStream_t st);
// Gershgorin bound of the spectrum of D^-1 A, max_i 1 + sum_j |a_ij / a_ii|,
// into *out (device; asynchronous)
void gershgorin_bound(const SellView<double>& a, int nSlices, double* out, cudaStream_t st);

// ---- residual / products ---------------------------------------------------
// r = b + D x + O x over all rows; when partials != null each block also
// writes the L1 sum of its rows' r to partials[blockIdx] (FP64).
template <class T>
void residual(const SellView<T>& a, int nSlices, const T* x, const T* b, T* r, double* partials,
              cudaStream_t st);
// y = D x + O x (FP64 only)
void spmv(const SellView<double>& a, int nSlices, const double* x, double* y, cudaStream_t st);
int reduce_blocks(int nSlices);  // grid of the SELL-32 whole-level row kernels

// ---- fused Krylov vector steps (CG) -------------------------------------------
// y = A x with one partial of x.y per block (spmv_dot_blocks of them)
int spmv_dot_blocks(const SellView<double>& a, int nSlices);
void spmv_dot(const SellView<double>& a, int nSlices, const double* x, double* y, double* partials, cudaStream_t st);
// the same with p = p_old * beta + z formed on the fly (spmv_dot_blocks
// partials); cg_update_pby then writes that p and updates x and r
void spmv_dot_pby(const SellView<double>& a, int nSlices, const double* z, const double* p, const double* beta,
                  double* y, double* partials, cudaStream_t st);
void cg_update_pby(int n, const double* alpha, const double* z, const double* beta, double* p, const double* q,
                   double* x, double* r, double* partials, cudaStream_t st, float* rF = nullptr);
// z <- src (converted to FP64) with per-block partials of r.z_old and
// r.z_new (interleaved, vec_blocks(n) pairs)
template <class S>
void cg_take_z(int n, const S* src, const double* r, double* z, double* partials, cudaStream_t st);
// from those pairs: *rhoPrev <- *rho, *rho <- (r, z_new), *beta <- *rho /
// *rhoPrev, or with flexible (Polak-Ribiere) (*rho - (r, z_old)) / *rhoPrev
void cg_beta(int np, const double* partials, double* rho, double* rhoPrev, double* beta, bool flexible,
             cudaStream_t st);
// *alpha = *rho / (sum of np partials)
void cg_alpha(int np, const double* partials, const double* rho, double* alpha, cudaStream_t st);
// x += -alpha p, r += -alpha q, and per-block L1 partials of the new r
// (vec_blocks(n) of them); rF (optional) gets the new r in FP32, the
// right-hand side of the next FP32 cycle
void cg_update(int n, const double* alpha, const double* p, const double* q, double* x, double* r, double* partials,
               cudaStream_t st, float* rF = nullptr);
// number of L1 partials residual() writes for a level (one per block)
int residual_partials(int nSlices, int n, int ellWidth);

// r = b + D x + O x on a plain CSR matrix (implicit diagonal, reference
// column order), one thread per row; block k writes the L1 sum of its 256
// rows to partials[k] (csr_residual_blocks(n) of them), then
// csr_residual_finish sums them in a fixed order into *l1.
int csr_residual_blocks(int n);
void csr_residual(int n, const int* row, const int* col, const double* diag, const double* off,
                  const double* x, const double* b, double* r, double* partials, cudaStream_t st);
void csr_residual_finish(int nPartials, const double* partials, double* l1, cudaStream_t st);

// ---- transfers ---------------------------------------------------------------
// bc[I] = sum over fine rows i of aggregate I (ascending reference order) of r[i]
template <class T>
void restrict_sum(int nc, const int* c2fRow, const int* c2fCol, const T* r, T* bc, cudaStream_t st);
// bc = restriction of the fine residual b + A x; also zeroes the coarse x
// (xc may be null). r == null: one kernel, each coarse row computes its fine
// rows' residuals itself (r never stored; the fine rows of an aggregate are
// scattered over the matrix, so its loads are gathers). r != null: the
// residual pass writes r with coalesced row loads, then a second kernel
// gathers it per aggregate. Both sum the same products in the same order:
// bitwise the same bc.
template <class T>
void residual_restrict(const SellView<T>& a, int nSlices, const int* rowSlice, int nc, const int* c2fRow,
                       const int* c2fCol, const T* x, const T* b, T* bc, T* xc, T* r, cudaStream_t st);
// bc[I] = sum of b over the fine rows of aggregate I (ascending order) and
// xc = 0: the restricted residual of a level whose x is zero (r = b)
template <class T>
void restrict_rhs(int nc, const int* c2fRow, const int* c2fCol, const T* b, T* bc, T* xc, cudaStream_t st);
template <class T>
void zero(int n, T* x, cudaStream_t st);
// x[i] += xc[ci[i]] (assign: x[i] = xc[ci[i]], for an x that is zero)
template <class T>
void prolong(int n, const int* ci, const T* xc, T* x, cudaStream_t st, bool assign = false);

// ---- coarsest level --------------------------------------------------------
// x = -Ainv b with a dense FP64 inverse (n x n, row-major)
template <class T>
void dense_solve(int n, const double* ainv, const T* b, T* x, cudaStream_t st);
// same with an FP32 copy of the inverse (half the bytes; FP32 V-cycle)
void dense_solve_f32(int n, const float* ainv, const float* b, float* x, cudaStream_t st);
// Inverse of the dense n x n matrix `a` (row-major, FP64, device;
// overwritten) by blocked in-place Gauss-Jordan elimination with partial
// (row) pivoting; result in `inv` (n^2 doubles). scratch must hold
// gauss_jordan_scratch_bytes(n); *status (device int inside scratch, see
// gauss_jordan_status) becomes 1 if a pivot was exactly zero. Asynchronous
// on st.
// a = the dense n x n form (row-major) of a SELL-32 level (not ELL-32):
// diagonal plus every nonzero stored entry; asynchronous on st.
void dense_from_sell(const SellView<double>& m, int nSlices, double* a, cudaStream_t st);
size_t gauss_jordan_scratch_bytes(int n);
void gauss_jordan_inverse(int n, double* a, double* inv, void* scratch, cudaStream_t st);
// device address of the status flag inside scratch
const int* gauss_jordan_status(int n, const void* scratch);
// In-place inverse of a diagonally dominant (by rows or by columns) dense
// matrix `a` by blocked Gauss-Jordan without pivoting: one kernel per panel
// of 16 pivots. Same scratch and status as gauss_jordan_inverse.
void gauss_jordan_inverse_dominant(int n, double* a, void* scratch, cudaStream_t st);
// The same for a symmetric diagonally dominant matrix: the sweep operator,
// which keeps the matrix symmetric, on the tiles on and above the diagonal
// only (half the products), then the lower triangle mirrored. Same scratch
// and status.
void gauss_jordan_inverse_symmetric(int n, double* a, void* scratch, cudaStream_t st);
// *flag = 1 unless the dense n x n matrix is symmetric to a relative 1e-12
// entry by entry (*flag must be 0 on entry)
void dense_symmetry_check(int n, const double* a, int* flag, cudaStream_t st);
void cast_d2f(size_t n, const double* a, float* b, cudaStream_t st);

// ---- vector ops ------------------------------------------------------------
void convert_d2f(int n, const double* a, float* b, cudaStream_t st);
void add_f2d(int n, const float* a, double* b, cudaStream_t st);  // b += a
// partial sums of |a| or a*b per block, finalised by sum_partials
int vec_blocks(int n);
void l1_partials(int n, const double* a, double* partials, cudaStream_t st);
void dot_partials(int n, const double* a, const double* b, double* partials, cudaStream_t st);
// out[0] = sum of the partials in a fixed order
void sum_partials(int np, const double* partials, double* out, cudaStream_t st);
// r = b (the residual at x = 0), rF = (float) b when rF is not null, and the
// |b|_1 partials of l1_partials (vec_blocks(n) of them)
void cg_start(int n, const double* b, double* r, float* rF, double* partials, cudaStream_t st);
// scalar recurrences for the Krylov solvers, all on the device:
// out = num / den (out, num, den are device scalars)
void scalar_div(const double* num, const double* den, double* out, cudaStream_t st);
// out = (rho - rzPrev) / rhoPrev (flexible CG's beta)
void scalar_flex_beta(const double* rho, const double* rzPrev, const double* rhoPrev, double* out, cudaStream_t st);
// out = (a / b) * (c / d)
void scalar_ratio_product(const double* a, const double* b, const double* c, const double* d,
                          double* out, cudaStream_t st);
// y += s * x (s a device scalar, sign +1/-1)
void axpy_dev(int n, const double* s, double sign, const double* x, double* y, cudaStream_t st);
// p = z + beta * p
void xpby_dev(int n, const double* z, const double* beta, double* p, cudaStream_t st);
// p = (p - omega v) * beta + r   (BiCGStab direction update)
void bicg_p_update(int n, const double* r, const double* v, const double* omega,
                   const double* beta, double* p, cudaStream_t st);
void copy_d(int n, const double* a, double* b, cudaStream_t st);

// ---- thermal linearization (original cell order) -----------------------------
struct FaceGeom {
  int nFaces;
  int nCells;  // self cells
  const int* faceCells;       // 2 per face
  const double* faceArea;     // 3 per face
  const double* faceAreaMag;  // per face
  const double* cellCentroid; // 3 per cell (self + ghost)
  const double* cellVolume;   // per cell (self + ghost)
};
// c_f and the secondary (non-orthogonal) coefficient per face; secCoeff
// holds one 32-byte record per face (x, y, z, pad), 32-byte aligned
void face_coefficients(const FaceGeom& g, const double* k, double* coeff, double* secCoeff,
                       cudaStream_t st);
// least-squares gradient of x on self rows, then boundary ghosts copy c0;
// grad holds one 32-byte record per cell (x, y, z, pad), 32-byte aligned
void gradient(int nCells, const int* ccRow, const int* ccCol, const double* w, const double* x,
              double* grad, cudaStream_t st);
void ghost_gradient(int nBFaces, const int* bFaces, const int* faceCells, double* grad,
                    cudaStream_t st);
// flux_f = c_f (x1 - x0) + gradF . sec_f
void face_flux(const FaceGeom& g, const double* coeff, const double* secCoeff,
               const double* grad, const double* x, double* flux, cudaStream_t st);

// Per boundary face (in face order): the condition and what the
// linearization records for the post-solve update (GenericBCS.h:77-323,
// LinearSystem::postSolve).
enum BoundaryKind { kBkDirichlet = 0, kBkFlux = 1, kBkConvective = 2, kBkRadiative = 3, kBkMixed = 4 };
struct BoundaryData {
  int nBFaces;
  const int* bFace;     // face index of each boundary face
  const int* kind;      // BoundaryKind; Symmetry is a zero specified flux
  const double* value;  // specified temperature or heat flux
  const double* param;  // 3 per face: convective coefficient, far-field temperature, emissivity
  double* ghostRhs;     // per face: the ghost row's rhs after the condition (not Dirichlet)
  double* ghostDiag;    // per face: the ghost row's diagonal after the condition (not Dirichlet)
  double* hf;           // 4 per face: heat flux at linearization, its rhs, d/dx0, d/dx1
  double* heatFlux;     // per face: heat flux after the update
};
struct CellFaceView {
  const int* row;  // cellFaces over self cells
  const int* col;
  const int* bRow;   // per self cell: range into the boundary-face lists
  const int* bCol;   // boundary faces, ascending face index (BC application order)
  const int* bColG;  // the same faces by ascending ghost index (elimination order)
};
// Assembles the delta-form right-hand side of every self cell exactly as
// DiffusionDiscretization + Source + TimeDerivative + GenericBCS +
// eliminateBoundaryEquations produce it, writing b[perm[i]]; also records
// the Neumann ghost rhs (bGhost) and sets Dirichlet ghosts of x to the
// boundary value. transient: rhoVdt != null.
void assemble_rhs(int nCells, const CellFaceView& cf, const int* faceCells, const double* flux,
                  const double* coeff, const double* faceAreaMag, const double* vol,
                  const double* source, const double* rhoVdt, const double* xN1,
                  const BoundaryData& bd, const int* bIndexOfFace, double* x, const int* perm, double* b,
                  cudaStream_t st);
// The matrix part (constant while conductivity, geometry and time step are):
// diagonal of every self cell and the off-diagonals through entryFace.
void assemble_matrix(int nCells, const CellFaceView& cf, const int* faceCells, const double* coeff,
                     const double* faceAreaMag, const double* rhoVdt, const BoundaryData& bd,
                     const int* bIndexOfFace, const double* x, double* diagOrig, cudaStream_t st);
// rhoVdt_i = rho c_i V_i / dt
void transient_coeff(int nCells, const double* rhoCp, const double* vol, double dt, double* out,
                     cudaStream_t st);
// off-diagonal value of entry e = coeff[entryFace[e]] (gathered into the SELL layout)
void gather_offdiag(int nEntries, const int* entryFace, const double* coeff, double* vals,
                    cudaStream_t st);
void gather_diag(int n, const int* iperm, const double* diagOrig, double* diag, cudaStream_t st);
void cast_d2f_vals(int n, const double* a, float* b, cudaStream_t st);
// T_i += delta[perm[i]] on self cells; the ghosts of flux-type conditions
// solve their boundary row and update too, and every boundary face's heat
// flux takes its update (LinearSystem::postSolve + updateSolution)
void update_solution(int nCells, const int* perm, const double* delta, const BoundaryData& bd,
                     const int* faceCells, const double* coeff, double* x, cudaStream_t st);

}  // namespace dev
}  // namespace fvm
