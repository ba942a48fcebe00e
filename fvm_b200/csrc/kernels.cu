// sm_100a kernels for the thermal linearization and the AMG / Krylov solve.
//
// Build note: this file is compiled with -fmad=false. Every FP64 product
// and sum then rounds on its own, exactly as the reference's scalar C++
// does on x86-64, which keeps the face coefficients, the matrix and the
// right-hand side bit-identical to the reference and lets the sequential
// Gauss-Seidel and Jacobi smoothers reproduce its iterates. The kernels are
// memory-bound, so fused multiply-adds would buy no speed here.
//
// Layout: level matrices are colour-permuted SELL-32 (32 rows per slice,
// entries stored column-major inside the slice, so a warp reads 32
// consecutive cols/vals per step: fully coalesced 128 B / 256 B lines).
#include <cuda_runtime.h>

#include <cstdint>

#include "kernels.cuh"

namespace fvm {
namespace dev {

namespace {

constexpr int kBlock = 256;           // threads per block for row kernels
constexpr int kSlicesPerBlock = kBlock / 32;
constexpr int kRowGridCap = 148 * 8;
constexpr int kReduceBlocks = 1184;   // 148 SMs x 8: vector reductions

inline int ceil_div(long long a, long long b) { return (int)((a + b - 1) / b); }

__device__ __forceinline__ double warp_sum(double v) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  return v;
}

// Block-wide sum of one double per thread; result valid in thread 0.
__device__ __forceinline__ double block_sum(double v) {
  __shared__ double sh[32];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  v = warp_sum(v);
  if (lane == 0) sh[wid] = v;
  __syncthreads();
  const int nw = (blockDim.x + 31) >> 5;
  v = (threadIdx.x < nw) ? sh[threadIdx.x] : 0.0;
  if (wid == 0) v = warp_sum(v);
  return v;
}

// The value of column j a row sum gathers: x[j], or, for a pass that
// starts right after a prolongation that assigned x = xc[ci], xc[ci[j]]
// (the same value, without the prolongation's launch and x round trip)
template <class T>
struct XDirect {
  const T* __restrict__ x;
  __device__ __forceinline__ T operator()(int j) const { return x[j]; }
};
// CG's new search direction read where it is needed: p_j = p_old_j * beta +
// z_j, rounded as k_xpby_dev rounds it (contraction off in this file)
struct XPby {
  const double* __restrict__ z;
  const double* __restrict__ p;
  double beta;
  __device__ __forceinline__ double operator()(int j) const { return p[j] * beta + z[j]; }
};
template <class T>
struct XProlonged {
  const T* __restrict__ xc;
  const int* __restrict__ ci;
  __device__ __forceinline__ T operator()(int j) const { return xc[ci[j]]; }
};

// Up to K entries of a row: every column and value load is issued, then
// every x gather, then the products are accumulated in stored order -- two
// dependent round trips to memory for the whole chunk.
template <class T, int K, class X>
__device__ __forceinline__ T row_chunk_g(const SellView<T>& a, int e0, int cnt, const X& xg, T sum) {
  int c[K];
  T v[K];
  T xv[K];
#pragma unroll
  for (int k = 0; k < K; k++)
    if (k < cnt) {
      c[k] = a.cols[e0 + (k << 5)];
      v[k] = a.vals[e0 + (k << 5)];
    }
#pragma unroll
  for (int k = 0; k < K; k++)
    if (k < cnt) xv[k] = xg(c[k]);
#pragma unroll
  for (int k = 0; k < K; k++)
    if (k < cnt) sum = sum + v[k] * xv[k];
  return sum;
}
template <class T, int K>
__device__ __forceinline__ T row_chunk(const SellView<T>& a, int e0, int cnt, const T* __restrict__ x, T sum) {
  return row_chunk_g<T, K>(a, e0, cnt, XDirect<T>{x}, sum);
}

// Sum over one row of a slice (m = the slice's packed metadata) in stored
// order, in chunks of four entries with all loads of a chunk in flight
// together; the summation order is the stored order.
template <class T, class X>
__device__ __forceinline__ T row_sum_g(const SellView<T>& a, const int4 m, int lane, const X& xg, T sum) {
  // four entries in flight per chunk: wider chunks (8 or 16) raised the
  // register count to 63 and halved the occupancy of the finest-level
  // passes (ncu: 42 % warps active, 22 % of DRAM peak)
  const int o = m.z + lane;
  const int w = m.w;
  int k = 0;
  for (; k + 4 <= w; k += 4) sum = row_chunk_g<T, 4>(a, o + (k << 5), 4, xg, sum);
  if (k < w) sum = row_chunk_g<T, 4>(a, o + (k << 5), w - k, xg, sum);
  return sum;
}
template <class T>
__device__ __forceinline__ T row_sum(const SellView<T>& a, const int4 m, int lane, const T* __restrict__ x,
                                     T sum) {
  return row_sum_g(a, m, lane, XDirect<T>{x}, sum);
}


// Programmatic dependent launch: every hot-path kernel lets the next
// kernel in the stream be scheduled as soon as all of its own blocks are
// running (launch_dependents), and waits for its predecessor's completion
// and memory before touching any data (griddepcontrol.wait). The launch
// latency of the next kernel then overlaps this one. Kernels launched
// without the attribute see both instructions as no-ops.
#define FVM_PDL()                                                  \
  do {                                                             \
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); \
    asm volatile("griddepcontrol.wait;" ::: "memory");             \
  } while (0)

// A slice's {first row, rows, offset, width}: loaded (SELL-32) or computed
// (ELL-32: aligned 32-row groups of one width)
template <class T>
__device__ __forceinline__ int4 slice_meta(const SellView<T>& a, int s) {
  if (a.ellWidth) {
    const int r0 = s << 5;
    return make_int4(r0, min(32, a.n - r0), r0 * a.ellWidth, a.ellWidth);
  }
  return a.meta[s];
}
template <class T>
__device__ __forceinline__ int slice_of(const SellView<T>& a, const int* rowSlice, int i) {
  return a.ellWidth ? (i >> 5) : rowSlice[i];
}

template <class T>
__global__ void k_zero(int n, T* x) {
  FVM_PDL();
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) x[i] = T(0);
}

// ---------------------------------------------------------------------------
template <class T>
__global__ void __launch_bounds__(kBlock, 8) k_gs_color(SellView<T> a, int s0, int s1, T* x, const T* __restrict__ b) {
  FVM_PDL();
  const int lane = threadIdx.x & 31;
  if (a.ellWidth) {
    // rows [s0, s1) of the aligned 32-row groups
    const int s = (s0 >> 5) + blockIdx.x * kSlicesPerBlock + (threadIdx.x >> 5);
    const int i = (s << 5) + lane;
    if (i < s0 || i >= s1) return;
    const T sum = row_sum(a, slice_meta(a, s), lane, x, b[i]);
    x[i] = -sum / a.diag[i];
    return;
  }
  const int s = s0 + blockIdx.x * kSlicesPerBlock + (threadIdx.x >> 5);
  if (s >= s1) return;
  const int4 m = slice_meta(a, s);
  if (lane >= m.y) return;
  const int i = m.x + lane;
  const T sum = row_sum(a, m, lane, x, b[i]);
  x[i] = -sum / a.diag[i];
}

template <class T>
__global__ void k_gs_sequential(SellView<T> a, T* x, const T* __restrict__ b, int reverse) {
  FVM_PDL();
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  for (int t = 0; t < a.n; t++) {
    const int i = reverse ? a.n - 1 - t : t;
    const int s = i >> 5, lane = i & 31;  // one colour: slices are consecutive 32-row blocks
    const T sum = row_sum(a, slice_meta(a, s), lane, x, b[i]);
    x[i] = -sum / a.diag[i];
  }
}

template <class T>
__global__ void __launch_bounds__(kBlock, 8) k_jacobi(SellView<T> a, int nSlices, const T* __restrict__ xold, T* xnew,
                         const T* __restrict__ b) {
  FVM_PDL();
  const int lane = threadIdx.x & 31;
  for (int s = blockIdx.x * kSlicesPerBlock + (threadIdx.x >> 5); s < nSlices; s += gridDim.x * kSlicesPerBlock) {
    const int4 m = slice_meta(a, s);
    if (lane >= m.y) continue;
    const int i = m.x + lane;
    const T sum = row_sum(a, m, lane, xold, b[i]);
    xnew[i] = -sum / a.diag[i];
  }
}

// damped Jacobi: xnew = xold + w (xJacobi - xold); Pro: xold is the
// prolongation xc[ci] a pass would otherwise have assigned first
template <class T, bool Pro>
__global__ void __launch_bounds__(kBlock, 8) k_jacobi_damped(SellView<T> a, int nSlices, const T* __restrict__ xold,
                                                             T* xnew, const T* __restrict__ b, T w,
                                                             const T* __restrict__ xc, const int* __restrict__ ci) {
  FVM_PDL();
  const int lane = threadIdx.x & 31;
  for (int s = blockIdx.x * kSlicesPerBlock + (threadIdx.x >> 5); s < nSlices; s += gridDim.x * kSlicesPerBlock) {
    const int4 m = slice_meta(a, s);
    if (lane >= m.y) continue;
    const int i = m.x + lane;
    T sum, xo;
    if constexpr (Pro) {
      sum = row_sum_g(a, m, lane, XProlonged<T>{xc, ci}, b[i]);
      xo = xc[ci[i]];
    } else {
      sum = row_sum(a, m, lane, xold, b[i]);
      xo = xold[i];
    }
    xnew[i] = xo + w * (-sum / a.diag[i] - xo);
  }
}

// One step of a Chebyshev polynomial smoother on D^-1 A: with the row's
// residual res = b + A x, dv = c1 dv + c2 (-res / a_ii) (First: dv is
// written, not read) and xnew = x + dv. dv is indexed by row only, so it
// is updated in place; x and xnew are distinct.
template <class T, bool First>
__global__ void __launch_bounds__(kBlock, 8) k_cheb(SellView<T> a, int nSlices, const T* __restrict__ x, T* xnew,
                                                    T* dv, const T* __restrict__ b, T c1, T c2) {
  FVM_PDL();
  const int lane = threadIdx.x & 31;
  for (int s = blockIdx.x * kSlicesPerBlock + (threadIdx.x >> 5); s < nSlices; s += gridDim.x * kSlicesPerBlock) {
    const int4 m = slice_meta(a, s);
    if (lane >= m.y) continue;
    const int i = m.x + lane;
    const T xi = x[i];
    const T res = row_sum(a, m, lane, x, b[i] + a.diag[i] * xi);
    const T z = -res / a.diag[i];
    const T d = First ? c2 * z : c1 * dv[i] + c2 * z;
    dv[i] = d;
    xnew[i] = xi + d;
  }
}

// Gershgorin bound of the spectrum of D^-1 A: max over rows of
// 1 + sum_j |a_ij / a_ii|, by atomicMax on the bits of a non-negative double
__global__ void __launch_bounds__(kBlock) k_gershgorin(SellView<double> a, int nSlices, unsigned long long* out) {
  const int lane = threadIdx.x & 31;
  double best = 0.0;
  for (int s = blockIdx.x * kSlicesPerBlock + (threadIdx.x >> 5); s < nSlices; s += gridDim.x * kSlicesPerBlock) {
    const int4 m = slice_meta(a, s);
    if (lane >= m.y) continue;
    const int i = m.x + lane;
    double sum = 0.0;
    for (int k = 0; k < m.w; k++) sum += fabs(a.vals[m.z + (k << 5) + lane]);
    best = fmax(best, 1.0 + sum / fabs(a.diag[i]));
  }
  for (int o = 16; o > 0; o >>= 1) best = fmax(best, __shfl_xor_sync(0xffffffffu, best, o));
  if (lane == 0 && best > 0.0) atomicMax(out, (unsigned long long)__double_as_longlong(best));
}

template <class T>
__global__ void __launch_bounds__(kBlock, 8) k_residual(SellView<T> a, int nSlices, const T* __restrict__ x,
                           const T* __restrict__ b, T* r, double* partials) {
  FVM_PDL();
  const int lane = threadIdx.x & 31;
  double l1 = 0.0;
  for (int s = blockIdx.x * kSlicesPerBlock + (threadIdx.x >> 5); s < nSlices; s += gridDim.x * kSlicesPerBlock) {
    const int4 m = slice_meta(a, s);
    if (lane < m.y) {
      const int i = m.x + lane;
      // reference order: r = b + d x, then r += a_ij x_j
      const T ri = row_sum(a, m, lane, x, b[i] + a.diag[i] * x[i]);
      r[i] = ri;
      l1 += fabs((double)ri);
    }
  }
  if (partials) {
    const double t = block_sum(l1);
    if (threadIdx.x == 0) partials[blockIdx.x] = t;
  }
}

__global__ void k_csr_residual(int n, const int* __restrict__ row, const int* __restrict__ col,
                               const double* __restrict__ diag, const double* __restrict__ off,
                               const double* __restrict__ x, const double* __restrict__ b, double* r,
                               double* partials) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  double l1 = 0.0;
  if (i < n) {
    double s = b[i] + diag[i] * x[i];
    for (int k = row[i]; k < row[i + 1]; k++) s = s + off[k] * x[col[k]];
    if (r) r[i] = s;
    l1 = fabs(s);
  }
  const double t = block_sum(l1);
  if (threadIdx.x == 0) partials[blockIdx.x] = t;
}

__global__ void __launch_bounds__(kBlock, 8) k_spmv(SellView<double> a, int nSlices, const double* __restrict__ x, double* y) {
  FVM_PDL();
  const int lane = threadIdx.x & 31;
  for (int s = blockIdx.x * kSlicesPerBlock + (threadIdx.x >> 5); s < nSlices; s += gridDim.x * kSlicesPerBlock) {
    const int4 m = slice_meta(a, s);
    if (lane >= m.y) continue;
    const int i = m.x + lane;
    y[i] = row_sum(a, m, lane, x, a.diag[i] * x[i]);
  }
}

// ---- ELL-32 levels: compile-time width, one aligned 32-row group per warp ----
// Row i lives in group i / 32 at lane i % 32, its entries at (i / 32) * 32 W
// + i % 32 + 32 k. With the width known at compile time every column and
// value load of the row is issued at once, then every x gather: one
// dependent round trip per row (W <= 6; W = 7, 8 take two chunks to stay at
// 32 registers). One group per warp and no grid-stride loop: on B200 this
// beat a resident-sized striding grid by 7-45 % (8M-row width-6 pass:
// 5.8 vs 4.4 TB/s, 1M rows: 3.9 vs 2.7 TB/s). Summation in stored order,
// as row_sum.
template <class T, int W, class X>
__device__ __forceinline__ T ell_row_g(const SellView<T>& a, int i, const X& xg, T sum) {
  const int o = (i >> 5) * (32 * W) + (i & 31);
  if constexpr (W <= 6) {
    return row_chunk_g<T, W>(a, o, W, xg, sum);
  } else {
    sum = row_chunk_g<T, 4>(a, o, 4, xg, sum);
    return row_chunk_g<T, W - 4>(a, o + 128, W - 4, xg, sum);
  }
}
template <class T, int W>
__device__ __forceinline__ T ell_row(const SellView<T>& a, int i, const T* __restrict__ x, T sum) {
  return ell_row_g<T, W>(a, i, XDirect<T>{x}, sum);
}

// The first forward Gauss-Seidel sweep after a prolongation that would
// assign x = xc[ci]: rows of earlier colours (below r0 in the colour-major
// order) already hold their new values, rows of later colours still the
// prolonged ones, read from xc
template <class T>
struct XSweepProlonged {
  const T* x;
  const T* __restrict__ xc;
  const int* __restrict__ ci;
  int r0;
  __device__ __forceinline__ T operator()(int j) const { return j < r0 ? x[j] : xc[ci[j]]; }
};

// rows [r0, r1) of one colour
template <class T, int W>
__global__ void __launch_bounds__(kBlock, 8) k_gs_color_ell(SellView<T> a, int r0, int r1, T* x,
                                                            const T* __restrict__ b) {
  FVM_PDL();
  const int i = (((r0 >> 5) + blockIdx.x * kSlicesPerBlock) << 5) + threadIdx.x;
  if (i < r0 || i >= r1) return;
  const T sum = ell_row<T, W>(a, i, x, b[i]);
  x[i] = -sum / a.diag[i];
}

// the same colour pass in the first forward sweep after a fused
// prolongation (XSweepProlonged): bitwise the values of prolongation + pass
template <class T, int W>
__global__ void __launch_bounds__(kBlock, 8) k_gs_color_ell_pro(SellView<T> a, int r0, int r1, T* x,
                                                                const T* __restrict__ b, const T* __restrict__ xc,
                                                                const int* __restrict__ ci) {
  FVM_PDL();
  const int i = (((r0 >> 5) + blockIdx.x * kSlicesPerBlock) << 5) + threadIdx.x;
  if (i < r0 || i >= r1) return;
  const T sum = ell_row_g<T, W>(a, i, XSweepProlonged<T>{x, xc, ci, r0}, b[i]);
  x[i] = -sum / a.diag[i];
}

// The same pass with two rows per thread (32-row groups g and g + 8 of a
// block's 16): both rows' column, value, b and diagonal loads are issued
// first, then both rows' x gathers, then the two sums, so a thread keeps
// twice the loads in flight and a colour of a few hundred thousand rows
// fits in one wave. Each row sums b then its products in stored order, as
// ell_row does, and rows of one colour never read each other, so the
// result is bitwise that of k_gs_color_ell.
template <class T, int W>
__global__ void __launch_bounds__(kBlock) k_gs_color_ell2(SellView<T> a, int r0, int r1, T* x,
                                                          const T* __restrict__ b) {
  FVM_PDL();
  const int g0 = (r0 >> 5) + blockIdx.x * (2 * kSlicesPerBlock) + (threadIdx.x >> 5);
  const int i0 = (g0 << 5) + (threadIdx.x & 31);
  const int i1 = i0 + (kSlicesPerBlock << 5);
  const bool v0 = i0 >= r0 && i0 < r1, v1 = i1 >= r0 && i1 < r1;
  const int o0 = (i0 >> 5) * (32 * W) + (i0 & 31), o1 = (i1 >> 5) * (32 * W) + (i1 & 31);
  int c0[W], c1[W];
  T a0[W], a1[W], x0[W], x1[W];
#pragma unroll
  for (int k = 0; k < W; k++) {
    c0[k] = v0 ? a.cols[o0 + (k << 5)] : 0;
    a0[k] = v0 ? a.vals[o0 + (k << 5)] : T(0);
    c1[k] = v1 ? a.cols[o1 + (k << 5)] : 0;
    a1[k] = v1 ? a.vals[o1 + (k << 5)] : T(0);
  }
  T s0 = v0 ? b[i0] : T(0), s1 = v1 ? b[i1] : T(0);
  const T d0 = v0 ? a.diag[i0] : T(1), d1 = v1 ? a.diag[i1] : T(1);
#pragma unroll
  for (int k = 0; k < W; k++) {
    x0[k] = v0 ? x[c0[k]] : T(0);
    x1[k] = v1 ? x[c1[k]] : T(0);
  }
#pragma unroll
  for (int k = 0; k < W; k++) {
    s0 = s0 + a0[k] * x0[k];
    s1 = s1 + a1[k] * x1[k];
  }
  if (v0) x[i0] = -s0 / d0;
  if (v1) x[i1] = -s1 / d1;
}

template <class T, int W>
__global__ void __launch_bounds__(kBlock, 8) k_jacobi_ell(SellView<T> a, const T* __restrict__ xold, T* xnew,
                                                          const T* __restrict__ b) {
  FVM_PDL();
  const int i = blockIdx.x * kBlock + threadIdx.x;
  if (i >= a.n) return;
  const T sum = ell_row<T, W>(a, i, xold, b[i]);
  xnew[i] = -sum / a.diag[i];
}

template <class T, int W>
__global__ void __launch_bounds__(kBlock, 8) k_jacobi_damped_ell(SellView<T> a, const T* __restrict__ xold, T* xnew,
                                                                 const T* __restrict__ b, T w) {
  FVM_PDL();
  const int i = blockIdx.x * kBlock + threadIdx.x;
  if (i >= a.n) return;
  const T sum = ell_row<T, W>(a, i, xold, b[i]);
  const T xo = xold[i];
  xnew[i] = xo + w * (-sum / a.diag[i] - xo);
}

template <class T, int W, bool First>
__global__ void __launch_bounds__(kBlock, 8) k_cheb_ell(SellView<T> a, const T* __restrict__ x, T* xnew, T* dv,
                                                        const T* __restrict__ b, T c1, T c2) {
  FVM_PDL();
  const int i = blockIdx.x * kBlock + threadIdx.x;
  if (i >= a.n) return;
  const T xi = x[i];
  const T res = ell_row<T, W>(a, i, x, b[i] + a.diag[i] * xi);
  const T z = -res / a.diag[i];
  const T d = First ? c2 * z : c1 * dv[i] + c2 * z;
  dv[i] = d;
  xnew[i] = xi + d;
}

// residual with one L1 partial per block (256 rows)
template <class T, int W>
__global__ void __launch_bounds__(kBlock, 8) k_residual_ell(SellView<T> a, const T* __restrict__ x,
                                                            const T* __restrict__ b, T* r, double* partials) {
  FVM_PDL();
  const int i = blockIdx.x * kBlock + threadIdx.x;
  double l1 = 0.0;
  if (i < a.n) {
    const T ri = ell_row<T, W>(a, i, x, b[i] + a.diag[i] * x[i]);
    r[i] = ri;
    l1 = fabs((double)ri);
  }
  if (partials) {
    const double t = block_sum(l1);
    if (threadIdx.x == 0) partials[blockIdx.x] = t;
  }
}

template <int W>
__global__ void __launch_bounds__(kBlock, 8) k_spmv_ell(SellView<double> a, const double* __restrict__ x, double* y) {
  FVM_PDL();
  const int i = blockIdx.x * kBlock + threadIdx.x;
  if (i >= a.n) return;
  y[i] = ell_row<double, W>(a, i, x, a.diag[i] * x[i]);
}

// ---- fused Krylov vector steps ---------------------------------------------

// Block-wide sums of two doubles per thread; results valid in thread 0.
__device__ __forceinline__ void block_sum2(double& a, double& b) {
  __shared__ double sh[2][32];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  a = warp_sum(a);
  b = warp_sum(b);
  if (lane == 0) {
    sh[0][wid] = a;
    sh[1][wid] = b;
  }
  __syncthreads();
  const int nw = (blockDim.x + 31) >> 5;
  a = (threadIdx.x < nw) ? sh[0][threadIdx.x] : 0.0;
  b = (threadIdx.x < nw) ? sh[1][threadIdx.x] : 0.0;
  if (wid == 0) {
    a = warp_sum(a);
    b = warp_sum(b);
  }
}

// y = A x over an ELL-32 level, with one partial of x.y per block
template <int W>
__global__ void __launch_bounds__(kBlock, 8) k_spmv_dot_ell(SellView<double> a, const double* __restrict__ x, double* y,
                                                            double* partials) {
  FVM_PDL();
  const int i = blockIdx.x * kBlock + threadIdx.x;
  double d = 0.0;
  if (i < a.n) {
    const double xi = x[i];
    const double yi = ell_row<double, W>(a, i, x, a.diag[i] * xi);
    y[i] = yi;
    d = xi * yi;
  }
  d = block_sum(d);
  if (threadIdx.x == 0) partials[blockIdx.x] = d;
}

// q = A p with p = p_old * beta + z formed on the fly (p itself is written
// by k_cg_update_pby, after every row has read its neighbours' p_old), one
// partial of p.q per block
template <int W>
__global__ void __launch_bounds__(kBlock, 8) k_spmv_dot_pby_ell(SellView<double> a, const double* __restrict__ z,
                                                                const double* __restrict__ p, const double* beta,
                                                                double* y, double* partials) {
  FVM_PDL();
  const int i = blockIdx.x * kBlock + threadIdx.x;
  const XPby pg{z, p, beta[0]};
  double d = 0.0;
  if (i < a.n) {
    const double xi = pg(i);
    const double yi = ell_row_g<double, W>(a, i, pg, a.diag[i] * xi);
    y[i] = yi;
    d = xi * yi;
  }
  d = block_sum(d);
  if (threadIdx.x == 0) partials[blockIdx.x] = d;
}

__global__ void __launch_bounds__(kBlock, 8) k_spmv_dot_pby(SellView<double> a, int nSlices,
                                                            const double* __restrict__ z, const double* __restrict__ p,
                                                            const double* beta, double* y, double* partials) {
  FVM_PDL();
  const int lane = threadIdx.x & 31;
  const XPby pg{z, p, beta[0]};
  double d = 0.0;
  for (int s = blockIdx.x * kSlicesPerBlock + (threadIdx.x >> 5); s < nSlices; s += gridDim.x * kSlicesPerBlock) {
    const int4 m = slice_meta(a, s);
    if (lane >= m.y) continue;
    const int i = m.x + lane;
    const double xi = pg(i);
    const double yi = row_sum_g(a, m, lane, pg, a.diag[i] * xi);
    y[i] = yi;
    d += xi * yi;
  }
  d = block_sum(d);
  if (threadIdx.x == 0) partials[blockIdx.x] = d;
}

// the same over a SELL-32 level (grid-stride over slices)
__global__ void __launch_bounds__(kBlock, 8) k_spmv_dot(SellView<double> a, int nSlices, const double* __restrict__ x,
                                                        double* y, double* partials) {
  FVM_PDL();
  const int lane = threadIdx.x & 31;
  double d = 0.0;
  for (int s = blockIdx.x * kSlicesPerBlock + (threadIdx.x >> 5); s < nSlices; s += gridDim.x * kSlicesPerBlock) {
    const int4 m = slice_meta(a, s);
    if (lane >= m.y) continue;
    const int i = m.x + lane;
    const double xi = x[i];
    const double yi = row_sum(a, m, lane, x, a.diag[i] * xi);
    y[i] = yi;
    d += xi * yi;
  }
  d = block_sum(d);
  if (threadIdx.x == 0) partials[blockIdx.x] = d;
}

// z <- src (as FP64), with block partials of r.z_old and r.z_new
template <class S>
__global__ void k_cg_take_z(int n, const S* __restrict__ src, const double* __restrict__ r, double* z,
                            double* partials) {
  FVM_PDL();
  double a = 0.0, b = 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const double ri = r[i];
    const double zo = z[i];
    const double zn = (double)src[i];
    z[i] = zn;
    a += ri * zo;
    b += ri * zn;
  }
  block_sum2(a, b);
  if (threadIdx.x == 0) {
    partials[2 * blockIdx.x] = a;
    partials[2 * blockIdx.x + 1] = b;
  }
}

// rho_prev <- rho, rho <- (r, z_new), beta (flexible: (rho - (r, z_old)) / rho_prev)
__global__ void k_cg_beta(int np, const double* __restrict__ p, double* rho, double* rhoPrev, double* beta,
                          int flexible) {
  FVM_PDL();
  double a = 0.0, b = 0.0;
  for (int i = threadIdx.x; i < np; i += blockDim.x) {
    a += p[2 * i];
    b += p[2 * i + 1];
  }
  block_sum2(a, b);
  if (threadIdx.x == 0) {
    const double prev = rho[0];
    rhoPrev[0] = prev;
    rho[0] = b;
    beta[0] = flexible ? (b - a) / prev : b / prev;
  }
}

// alpha = rho / sum of the partials (p.Ap)
__global__ void k_cg_alpha(int np, const double* __restrict__ p, const double* rho, double* alpha) {
  FVM_PDL();
  double s = 0.0;
  for (int i = threadIdx.x; i < np; i += blockDim.x) s += p[i];
  s = block_sum(s);
  if (threadIdx.x == 0) alpha[0] = rho[0] / s;
}

// x += -alpha p; r += -alpha q; block partials of |r|
__global__ void k_cg_update(int n, const double* alpha, const double* __restrict__ p, const double* __restrict__ q,
                            double* x, double* r, double* partials, float* rF) {
  FVM_PDL();
  const double am = -1.0 * alpha[0];
  double l1 = 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    x[i] = x[i] + am * p[i];
    const double ri = r[i] + am * q[i];
    r[i] = ri;
    if (rF) rF[i] = (float)ri;
    l1 += fabs(ri);
  }
  l1 = block_sum(l1);
  if (threadIdx.x == 0) partials[blockIdx.x] = l1;
}

// p = p_old * beta + z (written here), x += -alpha p; r += -alpha q; block
// partials of |r|
__global__ void k_cg_update_pby(int n, const double* alpha, const double* __restrict__ z, const double* beta,
                                double* p, const double* __restrict__ q, double* x, double* r, double* partials,
                                float* rF) {
  FVM_PDL();
  const double am = -1.0 * alpha[0];
  const double b = beta[0];
  double l1 = 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const double pi = p[i] * b + z[i];
    p[i] = pi;
    x[i] = x[i] + am * pi;
    const double ri = r[i] + am * q[i];
    r[i] = ri;
    if (rF) rF[i] = (float)ri;
    l1 += fabs(ri);
  }
  l1 = block_sum(l1);
  if (threadIdx.x == 0) partials[blockIdx.x] = l1;
}

// ---- SELL-32 smoothers with several threads per row (autotuned plans) ---------
// A warp covers 32 / TPR rows of one slice; thread `sub` of a row's group
// takes the entries k = sub, sub + TPR, ... Four entries per thread are in
// flight per step; the group's products are then added to the row sum in
// stored order (k ascending), one shuffle per product, so the sum rounds
// exactly as row_sum's does.
// Lanes of rows past the slice's last row (live = false) take part in the
// shuffles but load nothing: their slots of the slice hold no entries.
template <class T, int TPR, class X>
__device__ __forceinline__ T row_sum_tpr(const SellView<T>& a, const int4 m, int l, bool live, const X& xg,
                                         T sum) {
  constexpr int C = 4;
  const int lane = threadIdx.x & 31, sub = lane & (TPR - 1), g0 = lane & ~(TPR - 1);
  const int o = m.z + l, w = m.w;
  for (int k0 = 0; k0 < w; k0 += TPR * C) {
    int c[C];
    T v[C], p[C];
#pragma unroll
    for (int q = 0; q < C; q++) {
      const int k = k0 + q * TPR + sub;
      const bool ok = live && k < w;
      c[q] = ok ? a.cols[o + (k << 5)] : 0;
      v[q] = ok ? a.vals[o + (k << 5)] : T(0);
    }
#pragma unroll
    for (int q = 0; q < C; q++) p[q] = v[q] * xg(c[q]);
#pragma unroll
    for (int q = 0; q < C; q++)
#pragma unroll
      for (int s2 = 0; s2 < TPR; s2++) {
        const T pv = __shfl_sync(0xffffffffu, p[q], g0 + s2);
        if (k0 + q * TPR + s2 < w) sum = sum + pv;
      }
  }
  return sum;
}

// global warp gw -> (slice, row within the slice) for TPR threads per row
template <int TPR>
__device__ __forceinline__ void tpr_row(int gw, int& sliceOffset, int& l) {
  sliceOffset = gw / TPR;
  l = (gw % TPR) * (32 / TPR) + ((threadIdx.x & 31) / TPR);
}

template <class T, int TPR, int BLOCK>
__global__ void __launch_bounds__(BLOCK) k_gs_color_tpr(SellView<T> a, int s0, int s1, T* x,
                                                        const T* __restrict__ b) {
  FVM_PDL();
  int so, l;
  tpr_row<TPR>(blockIdx.x * (BLOCK / 32) + (threadIdx.x >> 5), so, l);
  const int s = s0 + so;
  if (s >= s1) return;  // whole warp
  const int4 m = a.meta[s];
  const bool live = l < m.y;
  const int i = m.x + (live ? l : 0);
  const T sum = row_sum_tpr<T, TPR>(a, m, l, live, XDirect<T>{x}, live ? b[i] : T(0));
  if (live && (threadIdx.x & (TPR - 1)) == 0) x[i] = -sum / a.diag[i];
}

// Pro: the pass right after a prolongation that would assign x = xc[ci]
// reads those values from xc directly (xold unused)
template <class T, int TPR, int BLOCK, bool Pro>
__global__ void __launch_bounds__(BLOCK) k_jacobi_damped_tpr(SellView<T> a, int nSlices, const T* __restrict__ xold,
                                                             T* xnew, const T* __restrict__ b, T w,
                                                             const T* __restrict__ xc, const int* __restrict__ ci) {
  FVM_PDL();
  int s, l;
  tpr_row<TPR>(blockIdx.x * (BLOCK / 32) + (threadIdx.x >> 5), s, l);
  if (s >= nSlices) return;  // whole warp
  const int4 m = a.meta[s];
  const bool live = l < m.y;
  const int i = m.x + (live ? l : 0);
  T sum;
  if constexpr (Pro)
    sum = row_sum_tpr<T, TPR>(a, m, l, live, XProlonged<T>{xc, ci}, live ? b[i] : T(0));
  else
    sum = row_sum_tpr<T, TPR>(a, m, l, live, XDirect<T>{xold}, live ? b[i] : T(0));
  if (live && (threadIdx.x & (TPR - 1)) == 0) {
    const T xo = Pro ? xc[ci[i]] : xold[i];
    xnew[i] = xo + w * (-sum / a.diag[i] - xo);
  }
}

// Calls LAUNCH(TPR, BLOCK) for a supported plan; false otherwise.
#define FVM_PLAN_SWITCH(plan, LAUNCH)                              \
  [&]() -> bool {                                                  \
    const int key_ = (plan).tpr * 1000 + (plan).block;             \
    switch (key_) {                                                \
      case 1128: LAUNCH(1, 128); return true;                      \
      case 1256: LAUNCH(1, 256); return true;                      \
      case 2128: LAUNCH(2, 128); return true;                      \
      case 2256: LAUNCH(2, 256); return true;                      \
      case 4128: LAUNCH(4, 128); return true;                      \
      case 4256: LAUNCH(4, 256); return true;                      \
      default: return false;                                       \
    }                                                              \
  }()

// Calls LAUNCH(W) with the compile-time width of an ELL level (1..8);
// false for wider levels (they take the generic kernels).
#define FVM_ELL_SWITCH(width, LAUNCH) \
  [&]() -> bool {                     \
    switch (width) {                  \
      case 1: LAUNCH(1); return true; \
      case 2: LAUNCH(2); return true; \
      case 3: LAUNCH(3); return true; \
      case 4: LAUNCH(4); return true; \
      case 5: LAUNCH(5); return true; \
      case 6: LAUNCH(6); return true; \
      case 7: LAUNCH(7); return true; \
      case 8: LAUNCH(8); return true; \
      default: return false;          \
    }                                 \
  }()

template <class T>
__global__ void k_restrict(int nc, const int* __restrict__ c2fRow, const int* __restrict__ c2fCol,
                           const T* __restrict__ r, T* bc, T* xc) {
  FVM_PDL();
  const int I = blockIdx.x * blockDim.x + threadIdx.x;
  if (I >= nc) return;
  T s = T(0);
  for (int k = c2fRow[I]; k < c2fRow[I + 1]; k++) s = s + r[c2fCol[k]];
  bc[I] = s;
  if (xc) xc[I] = T(0);
}

// Fine-row residuals computed inside the restriction: rowSlice maps a fine
// row to its slice (lane = row - sliceRow).
template <class T>
__global__ void __launch_bounds__(kBlock, 4) k_residual_restrict(SellView<T> a, const int* __restrict__ rowSlice, int nc,
                                    const int* __restrict__ c2fRow, const int* __restrict__ c2fCol,
                                    const T* __restrict__ x, const T* __restrict__ b, T* bc, T* xc) {
  FVM_PDL();
  const int I = blockIdx.x * blockDim.x + threadIdx.x;
  if (I >= nc) return;
  T s = T(0);
  for (int k = c2fRow[I]; k < c2fRow[I + 1]; k++) {
    const int i = c2fCol[k];
    const int4 m = slice_meta(a, slice_of(a, rowSlice, i));
    const int lane = i - m.x;
    const T ri = row_sum(a, m, lane, x, b[i] + a.diag[i] * x[i]);
    s = s + ri;
  }
  bc[I] = s;
  if (xc) xc[I] = T(0);
}

template <class T>
__global__ void k_prolong(int n, const int* __restrict__ ci, const T* __restrict__ xc, T* x, int assign) {
  FVM_PDL();
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int c = ci[i];
  if (assign)
    x[i] = c >= 0 ? xc[c] : T(0);
  else if (c >= 0)
    x[i] = x[i] + xc[c];
}

template <class T>
__global__ void k_dense_solve(int n, const double* __restrict__ ainv, const T* __restrict__ b, T* x) {
  FVM_PDL();
  // one warp per row
  const int row = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  const int lane = threadIdx.x & 31;
  if (row >= n) return;
  double s = 0.0;
  for (int j = lane; j < n; j += 32) s += ainv[(size_t)row * n + j] * (double)b[j];
  s = warp_sum(s);
  if (lane == 0) x[row] = (T)(-s);
}

__global__ void k_dense_solve_f32(int n, const float* __restrict__ ainv, const float* __restrict__ b,
                                  float* x) {
  FVM_PDL();
  const int row = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  const int lane = threadIdx.x & 31;
  if (row >= n) return;
  float s = 0.0f;
  for (int j = lane; j < n; j += 32) s += ainv[(size_t)row * n + j] * b[j];
  for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
  if (lane == 0) x[row] = -s;
}

// Blocked in-place Gauss-Jordan inversion with partial (row) pivoting.
// For each panel of B columns [k0, k0+nb): one CTA factors the panel (all n
// rows, held column-major in shared memory), choosing pivot rows, applying
// the row swaps to the panel and eliminating above and below each pivot;
// the panel then holds the columns k0.. of the accumulated transform M.
// The swaps are applied to the other columns and their pivot rows copied
// out (k_gj_swap_rows); every other column j is then updated as
// a'[i] = (i not a pivot row ? a[i] : 0) + sum_t M[i][t] a[k0+t]
// (k_gj_update), a rank-nb update instead of nb sweeps over the matrix.
// The row interchanges become a column permutation of the result
// (k_gj_colperm, k_gj_gather).
template <int B>
__global__ void __launch_bounds__(1024) k_gj_panel(int n, int k0, int nb, double* __restrict__ A,
                                                    int* __restrict__ piv, int* __restrict__ status) {
  extern __shared__ double P[];  // P[t * n + i] = A[i][k0 + t]
  __shared__ double redV[32];
  __shared__ int redI[32];
  __shared__ int sPiv;
  const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5, nw = blockDim.x >> 5;
  for (int idx = tid; idx < n * B; idx += blockDim.x) {
    const int t = idx / n, i = idx - t * n;
    P[idx] = t < nb ? A[(size_t)i * n + k0 + t] : 0.0;
  }
  __syncthreads();
  for (int t = 0; t < nb; t++) {
    const int k = k0 + t;
    double best = -1.0;
    int bi = n;
    for (int r = k + tid; r < n; r += blockDim.x) {
      const double v = fabs(P[t * n + r]);
      if (v > best) {  // rows visited in ascending order: ties keep the lowest
        best = v;
        bi = r;
      }
    }
    for (int o = 16; o > 0; o >>= 1) {
      const double v2 = __shfl_down_sync(0xffffffffu, best, o);
      const int i2 = __shfl_down_sync(0xffffffffu, bi, o);
      if (v2 > best || (v2 == best && i2 < bi)) {
        best = v2;
        bi = i2;
      }
    }
    if (lane == 0) {
      redV[w] = best;
      redI[w] = bi;
    }
    __syncthreads();
    if (w == 0) {
      best = lane < nw ? redV[lane] : -1.0;
      bi = lane < nw ? redI[lane] : n;
      for (int o = 16; o > 0; o >>= 1) {
        const double v2 = __shfl_down_sync(0xffffffffu, best, o);
        const int i2 = __shfl_down_sync(0xffffffffu, bi, o);
        if (v2 > best || (v2 == best && i2 < bi)) {
          best = v2;
          bi = i2;
        }
      }
      if (lane == 0) sPiv = (bi >= k && bi < n) ? bi : k;
    }
    __syncthreads();
    const int p = sPiv;
    if (tid == 0) piv[k] = p;
    if (p != k && tid < nb) {
      const double a = P[tid * n + k];
      P[tid * n + k] = P[tid * n + p];
      P[tid * n + p] = a;
    }
    __syncthreads();
    const double pv = P[t * n + k];
    if (pv == 0.0 && tid == 0) atomicExch(status, 1);
    __syncthreads();
    if (tid < nb) P[tid * n + k] = (tid == t ? 1.0 : P[tid * n + k]) / pv;
    __syncthreads();
    for (int i = tid; i < n; i += blockDim.x) {
      if (i == k) continue;
      const double f = P[t * n + i];
      if (f != 0.0) {
        P[t * n + i] = 0.0;
        for (int s = 0; s < nb; s++) P[s * n + i] = P[s * n + i] - f * P[s * n + k];
      }
    }
    __syncthreads();
  }
  for (int idx = tid; idx < n * nb; idx += blockDim.x) {
    const int t = idx / n, i = idx - t * n;
    A[(size_t)i * n + k0 + t] = P[idx];
  }
}

// Applies the panel's row swaps to every column outside the panel and
// copies the pivot rows (old values) to Bt[t * n + j]; panel columns get 0.
__global__ void k_gj_swap_rows(int n, int k0, int nb, double* __restrict__ A, const int* __restrict__ piv,
                               double* __restrict__ Bt) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= n) return;
  const bool inPanel = j >= k0 && j < k0 + nb;
  if (!inPanel)
    for (int t = 0; t < nb; t++) {
      const int k = k0 + t, p = piv[k];
      if (p != k) {
        const double a = A[(size_t)k * n + j];
        A[(size_t)k * n + j] = A[(size_t)p * n + j];
        A[(size_t)p * n + j] = a;
      }
    }
  for (int t = 0; t < nb; t++) Bt[(size_t)t * n + j] = inPanel ? 0.0 : A[(size_t)(k0 + t) * n + j];
}

// columns [jlo, jhi) outside the panel [k0, k0 + nb) and outside [s0, s1)
__global__ void k_gj_update(int n, int k0, int nb, double* __restrict__ A, const double* __restrict__ Bt, int jlo,
                            int jhi, int s0, int s1) {
  const int j = jlo + blockIdx.x * blockDim.x + threadIdx.x;
  const int i = blockIdx.y;
  if (j >= jhi || (j >= k0 && j < k0 + nb) || (j >= s0 && j < s1)) return;
  const double* Mi = A + (size_t)i * n + k0;
  double s = 0.0;
  for (int t = 0; t < nb; t++) s = s + Mi[t] * Bt[(size_t)t * n + j];
  const size_t e = (size_t)i * n + j;
  A[e] = (i >= k0 && i < k0 + nb) ? s : A[e] + s;
}

// column order of the inverse: the row swaps undone in reverse order
__global__ void k_gj_colperm(int n, const int* __restrict__ piv, int* __restrict__ idx) {
  if (blockIdx.x != 0 || threadIdx.x != 0) return;
  for (int j = 0; j < n; j++) idx[j] = j;
  for (int k = n - 1; k >= 0; k--) {
    const int p = piv[k];
    const int a = idx[k];
    idx[k] = idx[p];
    idx[p] = a;
  }
}

__global__ void k_gj_gather(int n, const double* __restrict__ X, const int* __restrict__ idx, double* inv) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  const int i = blockIdx.y;
  if (j >= n) return;
  inv[(size_t)i * n + j] = X[(size_t)i * n + idx[j]];
}

__global__ void k_cast_d2f_big(size_t n, const double* __restrict__ a, float* b) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) b[i] = (float)a[i];
}

__global__ void k_convert_d2f(int n, const double* __restrict__ a, float* b) {
  FVM_PDL();
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) b[i] = (float)a[i];
}
__global__ void k_add_f2d(int n, const float* __restrict__ a, double* b) {
  FVM_PDL();
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) b[i] = b[i] + (double)a[i];
}
__global__ void k_l1_partials(int n, const double* __restrict__ a, double* partials) {
  FVM_PDL();
  double s = 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) s += fabs(a[i]);
  s = block_sum(s);
  if (threadIdx.x == 0) partials[blockIdx.x] = s;
}
// The start of a CG solve from x = 0: r = b + A x is b itself. r, its FP32
// copy (the FP32 cycle's right-hand side; null: none) and the |r|_1
// partials in k_l1_partials' layout, in one pass over b.
__global__ void k_cg_start(int n, const double* __restrict__ b, double* __restrict__ r, float* __restrict__ rF,
                           double* partials) {
  FVM_PDL();
  double s = 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const double v = b[i];
    r[i] = v;
    if (rF) rF[i] = (float)v;
    s += fabs(v);
  }
  s = block_sum(s);
  if (threadIdx.x == 0) partials[blockIdx.x] = s;
}
__global__ void k_dot_partials(int n, const double* __restrict__ a, const double* __restrict__ b,
                               double* partials) {
  FVM_PDL();
  double s = 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) s += a[i] * b[i];
  s = block_sum(s);
  if (threadIdx.x == 0) partials[blockIdx.x] = s;
}
__global__ void k_sum_partials(int np, const double* __restrict__ p, double* out) {
  FVM_PDL();
  // four independent loads in flight per thread (ELL residuals leave one
  // partial per 256 rows: 31k partials for 8M rows); fixed order
  double s = 0.0;
  const int bd = blockDim.x;
  int i = threadIdx.x;
  for (; i + 3 * bd < np; i += 4 * bd) {
    const double a0 = p[i], a1 = p[i + bd], a2 = p[i + 2 * bd], a3 = p[i + 3 * bd];
    s += a0;
    s += a1;
    s += a2;
    s += a3;
  }
  for (; i < np; i += bd) s += p[i];
  s = block_sum(s);
  if (threadIdx.x == 0) out[0] = s;
}
__global__ void k_scalar_div(const double* num, const double* den, double* out) {
  FVM_PDL();
  out[0] = num[0] / den[0];
}
// flexible (Polak-Ribiere) CG: beta = (r_k+1, z_k+1 - z_k) / (r_k, z_k)
__global__ void k_scalar_flex_beta(const double* rho, const double* rzPrev, const double* rhoPrev, double* out) {
  FVM_PDL();
  out[0] = (rho[0] - rzPrev[0]) / rhoPrev[0];
}
__global__ void k_scalar_ratio_product(const double* a, const double* b, const double* c,
                                       const double* d, double* out) {
  FVM_PDL();
  out[0] = (a[0] / b[0]) * (c[0] / d[0]);
}
__global__ void k_axpy_dev(int n, const double* s, double sign, const double* __restrict__ x, double* y) {
  FVM_PDL();
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) y[i] = y[i] + (sign * s[0]) * x[i];
}
__global__ void k_xpby_dev(int n, const double* __restrict__ z, const double* beta, double* p) {
  FVM_PDL();
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) p[i] = p[i] * beta[0] + z[i];
}
__global__ void k_bicg_p(int n, const double* __restrict__ r, const double* __restrict__ v,
                         const double* omega, const double* beta, double* p) {
  FVM_PDL();
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) p[i] = (p[i] - omega[0] * v[i]) * beta[0] + r[i];
}
__global__ void k_copy_d(int n, const double* __restrict__ a, double* b) {
  FVM_PDL();
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) b[i] = a[i];
}

// ---------------------------------------------------------------------------
// thermal linearization
__device__ __forceinline__ double harmonic_average(double x0, double x1) {
  const double sum = x0 + x1;
  if (x0 + x1 != 0.0) return 2.0 * x0 * x1 / sum;
  return sum;
}

__global__ void k_face_coefficients(FaceGeom g, const double* __restrict__ k, double* coeff,
                                    double* secCoeff) {
  const int f = blockIdx.x * blockDim.x + threadIdx.x;
  if (f >= g.nFaces) return;
  const int c0 = g.faceCells[2 * f], c1 = g.faceCells[2 * f + 1];
  const double vol0 = g.cellVolume[c0], vol1 = g.cellVolume[c1];
  double ds[3];
  for (int d = 0; d < 3; d++) ds[d] = g.cellCentroid[3 * c1 + d] - g.cellCentroid[3 * c0 + d];
  double kf;
  if (vol0 == 0.)
    kf = k[c1];
  else if (vol1 == 0.)
    kf = k[c0];
  else
    kf = harmonic_average(k[c0], k[c1]);
  const double* A = &g.faceArea[3 * f];
  const double am = g.faceAreaMag[f];
  const double dm = am * am / (A[0] * ds[0] + A[1] * ds[1] + A[2] * ds[2]);
  coeff[f] = kf * dm;
  // one 32-byte record per face (the fourth entry pads)
  reinterpret_cast<double4*>(secCoeff)[f] =
      make_double4(kf * (A[0] - ds[0] * dm), kf * (A[1] - ds[1] * dm), kf * (A[2] - ds[2] * dm), 0.0);
}

__global__ void k_gradient(int nCells, const int* __restrict__ row, const int* __restrict__ col,
                           const double* __restrict__ w, const double* __restrict__ x, double* grad) {
  FVM_PDL();
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nCells) return;
  double g0 = 0.0, g1 = 0.0, g2 = 0.0;
  const double xi = x[i];
  for (int k = row[i]; k < row[i + 1]; k++) {
    const double dx = x[col[k]] - xi;
    g0 += w[3 * k] * dx;
    g1 += w[3 * k + 1] * dx;
    g2 += w[3 * k + 2] * dx;
  }
  // one 32-byte record per cell (the fourth entry pads)
  reinterpret_cast<double4*>(grad)[i] = make_double4(g0, g1, g2, 0.0);
}

__global__ void k_ghost_gradient(int nB, const int* __restrict__ bFaces, const int* __restrict__ fc,
                                 double* grad) {
  FVM_PDL();
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nB) return;
  const int f = bFaces[t];
  const int c0 = fc[2 * f], c1 = fc[2 * f + 1];
  double4* g4 = reinterpret_cast<double4*>(grad);
  g4[c1] = g4[c0];
}

__global__ void k_face_flux(FaceGeom g, const double* __restrict__ coeff,
                            const double* __restrict__ sec, const double* __restrict__ grad,
                            const double* __restrict__ x, double* flux) {
  FVM_PDL();
  const int f = blockIdx.x * blockDim.x + threadIdx.x;
  if (f >= g.nFaces) return;
  // faceCells as one 8-byte load, the two gradients and the secondary
  // coefficient as 32-byte records (vector loads); same arithmetic order
  const int2 cc = reinterpret_cast<const int2*>(g.faceCells)[f];
  const int c0 = cc.x, c1 = cc.y;
  const double vol0 = g.cellVolume[c0], vol1 = g.cellVolume[c1];
  const double4 ga = reinterpret_cast<const double4*>(grad)[c0];
  const double4 gb = reinterpret_cast<const double4*>(grad)[c1];
  const double4 sc = reinterpret_cast<const double4*>(sec)[f];
  const double vs = vol0 + vol1;
  double s = 0.0;
  s += ((ga.x * vol0 + gb.x * vol1) / vs) * sc.x;
  s += ((ga.y * vol0 + gb.y * vol1) / vs) * sc.y;
  s += ((ga.z * vol0 + gb.z * vol1) / vs) * sc.z;
  flux[f] = coeff[f] * (x[c1] - x[c0]) + s;
}

// Ghost row of a flux-type boundary face as GenericBCS leaves it
// (GenericBCS.h:111-323), from the face flux of the face loop: the ghost's
// rhs bj and diagonal ajj, and the boundary heat flux with its derivative
// with respect to the ghost value (the post-solve flux update).
__device__ __forceinline__ void flux_bc(int kind, double q, const double* p, double x1, double flux, double am,
                                        double c, double& bj, double& ajj, double& hfB, double& hfR) {
  const double sb = 5.670373E-8;
  const double fluxI = -(0.0 - flux);
  ajj = 0.0 - c;
  hfR = 0.0;
  if (kind == kBkFlux) {
    bj = q * am - fluxI;
    hfB = q * am;
  } else if (kind == kBkConvective) {
    const double h = p[0], xi = p[1];
    const double fb = -h * (x1 - xi) * am;
    bj = fb - fluxI;
    ajj -= h * am;
    hfB = fb;
    hfR = -h * am;
  } else if (kind == kBkRadiative) {
    const double xi = p[1], e = p[2];
    const double fb = -e * sb * (x1 * x1 * x1 * x1 - xi * xi * xi * xi) * am;
    bj = fb - fluxI;
    ajj -= 4 * e * sb * x1 * x1 * x1 * am;
    hfB = fb;
    hfR = -4 * e * sb * x1 * x1 * x1 * am;
  } else {  // mixed; its flux derivative omits h, as the reference's does
    const double h = p[0], xi = p[1], e = p[2];
    const double fb = (-e * sb * (x1 * x1 * x1 * x1 - xi * xi * xi * xi) - h * (x1 - xi)) * am;
    bj = fb - fluxI;
    ajj -= (4 * e * sb * x1 * x1 * x1 + h) * am;
    hfB = fb;
    hfR = -4 * e * sb * x1 * x1 * x1 * am;
  }
}

__global__ void k_assemble_rhs(int nCells, CellFaceView cf, const int* __restrict__ fc,
                               const double* __restrict__ flux, const double* __restrict__ coeff,
                               const double* __restrict__ am, const double* __restrict__ vol,
                               const double* __restrict__ source, const double* __restrict__ rhoVdt,
                               const double* __restrict__ xN1, BoundaryData bd,
                               const int* __restrict__ bIndexOfFace, double* x,
                               const int* __restrict__ perm, double* b) {
  FVM_PDL();
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nCells) return;
  // DiffusionDiscretization: r0 += flux, r1 -= flux, faces ascending
  double r = 0.0;
  for (int k = cf.row[i]; k < cf.row[i + 1]; k++) {
    const int f = cf.col[k];
    if (fc[2 * f] == i)
      r += flux[f];
    else
      r -= flux[f];
  }
  // SourceDiscretization
  r += vol[i] * source[i];
  // TimeDerivativeDiscretization (first order)
  if (rhoVdt) r -= rhoVdt[i] * (x[i] - xN1[i]);
  // GenericBCS::applyDirichletBC: r0 += a01 (Tb - x1); ghost takes Tb; the
  // boundary heat flux is the face flux plus a01 (Tb - x1) - a01 dx0
  for (int k = cf.bRow[i]; k < cf.bRow[i + 1]; k++) {
    const int f = cf.bCol[k];
    const int t = bIndexOfFace[f];
    if (bd.kind[t] == kBkDirichlet) {
      const int c1 = fc[2 * f + 1];
      const double dX = bd.value[t] - x[c1];
      r += coeff[f] * dX;
      bd.hf[4 * t] = -(0.0 - flux[f]);
      bd.hf[4 * t + 1] = -(0.0 - coeff[f]) * dX;
      bd.hf[4 * t + 2] = -coeff[f];
      bd.hf[4 * t + 3] = 0.0;
      x[c1] = bd.value[t];
    }
  }
  // flux-type conditions set the ghost row; eliminateBoundaryEquations then
  // folds it into the interior row, ghosts by ascending index:
  // b_i -= a_ij (b_j / a_jj)
  for (int k = cf.bRow[i]; k < cf.bRow[i + 1]; k++) {
    const int f = cf.bColG[k];
    const int t = bIndexOfFace[f];
    const int kind = bd.kind[t];
    if (kind != kBkDirichlet) {
      double bj, ajj, hfB, hfR;
      flux_bc(kind, bd.value[t], bd.param + 3 * t, x[fc[2 * f + 1]], flux[f], am[f], coeff[f], bj, ajj, hfB, hfR);
      bd.ghostRhs[t] = bj;
      bd.ghostDiag[t] = ajj;
      bd.hf[4 * t] = hfB;
      bd.hf[4 * t + 1] = 0.0;
      bd.hf[4 * t + 2] = 0.0;
      bd.hf[4 * t + 3] = hfR;
      r -= coeff[f] * (bj / ajj);
    }
  }
  b[perm[i]] = r;
}

__global__ void k_assemble_matrix(int nCells, CellFaceView cf, const int* __restrict__ fc,
                                  const double* __restrict__ coeff, const double* __restrict__ am,
                                  const double* __restrict__ rhoVdt, BoundaryData bd,
                                  const int* __restrict__ bIndexOfFace, const double* __restrict__ x,
                                  double* diag) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nCells) return;
  double d = 0.0;
  for (int k = cf.row[i]; k < cf.row[i + 1]; k++) d -= coeff[cf.col[k]];
  if (rhoVdt) d -= rhoVdt[i];
  for (int k = cf.bRow[i]; k < cf.bRow[i + 1]; k++) {
    const int f = cf.bColG[k];
    const int t = bIndexOfFace[f];
    const int kind = bd.kind[t];
    if (kind != kBkDirichlet) {
      double bj, ajj, hfB, hfR;
      flux_bc(kind, bd.value[t], bd.param + 3 * t, x[fc[2 * f + 1]], 0.0, am[f], coeff[f], bj, ajj, hfB, hfR);
      const double aij = coeff[f];
      d -= aij * (aij / ajj);
    }
  }
  diag[i] = d;
}

__global__ void k_transient_coeff(int n, const double* __restrict__ rc, const double* __restrict__ vol,
                                  double dt, double* out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] = rc[i] * vol[i] / dt;
}

__global__ void k_cast_d2f(int n, const double* __restrict__ a, float* b) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) b[i] = (float)a[i];
}

__global__ void k_update_self(int nCells, const int* __restrict__ perm, const double* __restrict__ delta,
                              double* x) {
  FVM_PDL();
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < nCells) x[i] = x[i] + delta[perm[i]];
}

// Ghost rows of flux-type conditions: delta_j = -(b_j + a_ji delta_i) / a_jj
// with a_ji = c_f (CRMatrix::solveBoundary); Dirichlet ghosts keep delta 0.
// Then the boundary heat flux: q += -(r_q + (L dx0 + R dx1)) / (-1)
// (FluxJacobianMatrix::multiplyAndAdd, DiagonalMatrix::solveBoundary).
__global__ void k_update_ghosts(BoundaryData bd, const int* __restrict__ perm,
                                const double* __restrict__ delta, const int* __restrict__ fc,
                                const double* __restrict__ coeff, double* x) {
  FVM_PDL();
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= bd.nBFaces) return;
  const int f = bd.bFace[t];
  const int c0 = fc[2 * f], c1 = fc[2 * f + 1];
  const double dx0 = delta[perm[c0]];
  double dx1 = 0.0;
  if (bd.kind[t] != kBkDirichlet) {
    const double sum = bd.ghostRhs[t] + coeff[f] * dx0;
    dx1 = -sum / bd.ghostDiag[t];
    x[c1] = x[c1] + dx1;
  }
  const double* h = bd.hf + 4 * t;
  const double rq = h[1] + (h[2] * dx0 + h[3] * dx1);
  bd.heatFlux[t] = h[0] + (-rq / -1.0);
}

}  // namespace

// ---------------------------------------------------------------------------
// wrappers

namespace {
template <typename... KArgs, typename... Args>
void pdl_launch(void (*kernel)(KArgs...), dim3 grid, dim3 block, cudaStream_t st, Args... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = 0;
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  cudaLaunchKernelEx(&cfg, kernel, static_cast<KArgs>(args)...);
}
}  // namespace
template <class T>
void gs_color(const SellView<T>& a, int s0, int s1, T* x, const T* b, cudaStream_t st, RowPlan plan, const T* xc,
              const int* ci) {
  if (s1 <= s0) return;
  // ELL-32: s0, s1 are rows; the launch covers the 32-row groups they touch
  const int groups = a.ellWidth ? ((s1 - 1) >> 5) - (s0 >> 5) + 1 : s1 - s0;
  const int g = ceil_div(groups, kSlicesPerBlock);
  if (xc) {
#define FVM_L(W) pdl_launch(k_gs_color_ell_pro<T, W>, g, kBlock, st, a, s0, s1, x, b, xc, ci)
    if (a.ellWidth && FVM_ELL_SWITCH(a.ellWidth, FVM_L)) return;
#undef FVM_L
  }
  if (a.ellWidth && plan.ellRows == 2) {
#define FVM_L(W) pdl_launch(k_gs_color_ell2<T, W>, ceil_div(groups, 2 * kSlicesPerBlock), kBlock, st, a, s0, s1, x, b)
    if (FVM_ELL_SWITCH(a.ellWidth, FVM_L)) return;
#undef FVM_L
  }
#define FVM_L(W) pdl_launch(k_gs_color_ell<T, W>, g, kBlock, st, a, s0, s1, x, b)
  if (a.ellWidth && FVM_ELL_SWITCH(a.ellWidth, FVM_L)) return;
#undef FVM_L
  if (!a.ellWidth && !plan.isDefault()) {
#define FVM_P(TPR, BLOCK) \
  pdl_launch(k_gs_color_tpr<T, TPR, BLOCK>, ceil_div((long long)groups * TPR, BLOCK / 32), BLOCK, st, a, s0, s1, x, b)
    if (FVM_PLAN_SWITCH(plan, FVM_P)) return;
#undef FVM_P
  }
  pdl_launch(k_gs_color<T>, g, kBlock, st, a, s0, s1, x, b);
}
template <class T>
void gs_sequential(const SellView<T>& a, T* x, const T* b, bool reverse, cudaStream_t st) {
  pdl_launch(k_gs_sequential<T>, 1, 32, st, a, x, b, reverse ? 1 : 0);
}
template <class T>
void jacobi(const SellView<T>& a, int nSlices, const T* xold, T* xnew, const T* b, cudaStream_t st) {
#define FVM_L(W) pdl_launch(k_jacobi_ell<T, W>, ceil_div(a.n, kBlock), kBlock, st, a, xold, xnew, b)
  if (a.ellWidth && FVM_ELL_SWITCH(a.ellWidth, FVM_L)) return;
#undef FVM_L
  pdl_launch(k_jacobi<T>, reduce_blocks(nSlices), kBlock, st, a, nSlices, xold, xnew, b);
}
template <class T>
void jacobi_damped(const SellView<T>& a, int nSlices, const T* xold, T* xnew, const T* b, T w, cudaStream_t st,
                   RowPlan plan, const T* xc, const int* ci) {
  const bool pro = xc != nullptr;
  if (a.ellWidth && !pro) {
#define FVM_L(W) pdl_launch(k_jacobi_damped_ell<T, W>, ceil_div(a.n, kBlock), kBlock, st, a, xold, xnew, b, w)
    if (FVM_ELL_SWITCH(a.ellWidth, FVM_L)) return;
#undef FVM_L
  }
  if (!a.ellWidth && !plan.isDefault()) {
#define FVM_P(TPR, BLOCK)                                                                                          \
  (pro ? pdl_launch(k_jacobi_damped_tpr<T, TPR, BLOCK, true>, ceil_div((long long)nSlices * TPR, BLOCK / 32), BLOCK, \
                    st, a, nSlices, xold, xnew, b, w, xc, ci)                                                        \
       : pdl_launch(k_jacobi_damped_tpr<T, TPR, BLOCK, false>, ceil_div((long long)nSlices * TPR, BLOCK / 32), BLOCK, \
                    st, a, nSlices, xold, xnew, b, w, xc, ci))
    if (FVM_PLAN_SWITCH(plan, FVM_P)) return;
#undef FVM_P
  }
  if (pro)
    pdl_launch(k_jacobi_damped<T, true>, reduce_blocks(nSlices), kBlock, st, a, nSlices, xold, xnew, b, w, xc, ci);
  else
    pdl_launch(k_jacobi_damped<T, false>, reduce_blocks(nSlices), kBlock, st, a, nSlices, xold, xnew, b, w, xc, ci);
}
template <class T>
void chebyshev_step(const SellView<T>& a, int nSlices, const T* x, T* xnew, T* dv, const T* b, T c1, T c2,
                    bool first, cudaStream_t st) {
  if (a.ellWidth) {
#define FVM_L(W)                                                                                          \
  (first ? pdl_launch(k_cheb_ell<T, W, true>, ceil_div(a.n, kBlock), kBlock, st, a, x, xnew, dv, b, c1, c2) \
         : pdl_launch(k_cheb_ell<T, W, false>, ceil_div(a.n, kBlock), kBlock, st, a, x, xnew, dv, b, c1, c2))
    if (FVM_ELL_SWITCH(a.ellWidth, FVM_L)) return;
#undef FVM_L
  }
  if (first)
    pdl_launch(k_cheb<T, true>, reduce_blocks(nSlices), kBlock, st, a, nSlices, x, xnew, dv, b, c1, c2);
  else
    pdl_launch(k_cheb<T, false>, reduce_blocks(nSlices), kBlock, st, a, nSlices, x, xnew, dv, b, c1, c2);
}

void gershgorin_bound(const SellView<double>& a, int nSlices, double* out, cudaStream_t st) {
  cudaMemsetAsync(out, 0, sizeof(double), st);
  k_gershgorin<<<reduce_blocks(nSlices), kBlock, 0, st>>>(a, nSlices, reinterpret_cast<unsigned long long*>(out));
}

template <class T>
void residual(const SellView<T>& a, int nSlices, const T* x, const T* b, T* r, double* partials,
              cudaStream_t st) {
#define FVM_L(W) pdl_launch(k_residual_ell<T, W>, ceil_div(a.n, kBlock), kBlock, st, a, x, b, r, partials)
  if (a.ellWidth && FVM_ELL_SWITCH(a.ellWidth, FVM_L)) return;
#undef FVM_L
  pdl_launch(k_residual<T>, reduce_blocks(nSlices), kBlock, st, a, nSlices, x, b, r, partials);
}
// Row kernels over a whole SELL-32 level run a grid of at most 8 resident
// blocks per SM (148 SMs at 32 registers), each striding over slices: no
// partial last wave, and one L1 partial per block.
int reduce_blocks(int nSlices) {
  const int b = ceil_div(nSlices, kSlicesPerBlock);
  return b < kRowGridCap ? (b < 1 ? 1 : b) : kRowGridCap;
}
int residual_partials(int nSlices, int n, int ellWidth) {
  if (ellWidth >= 1 && ellWidth <= 8) return ceil_div(n, kBlock) < 1 ? 1 : ceil_div(n, kBlock);
  return reduce_blocks(nSlices);
}
int csr_residual_blocks(int n) { return ceil_div(n, kBlock); }
void csr_residual(int n, const int* row, const int* col, const double* diag, const double* off,
                  const double* x, const double* b, double* r, double* partials, cudaStream_t st) {
  k_csr_residual<<<csr_residual_blocks(n), kBlock, 0, st>>>(n, row, col, diag, off, x, b, r, partials);
}
void csr_residual_finish(int nPartials, const double* partials, double* l1, cudaStream_t st) {
  pdl_launch(k_sum_partials, 1, 1024, st, nPartials, partials, l1);
}
void spmv(const SellView<double>& a, int nSlices, const double* x, double* y, cudaStream_t st) {
#define FVM_L(W) pdl_launch(k_spmv_ell<W>, ceil_div(a.n, kBlock), kBlock, st, a, x, y)
  if (a.ellWidth && FVM_ELL_SWITCH(a.ellWidth, FVM_L)) return;
#undef FVM_L
  pdl_launch(k_spmv, reduce_blocks(nSlices), kBlock, st, a, nSlices, x, y);
}
int spmv_dot_blocks(const SellView<double>& a, int nSlices) {
  return (a.ellWidth >= 1 && a.ellWidth <= 8) ? ceil_div(a.n, kBlock) : reduce_blocks(nSlices);
}
void spmv_dot(const SellView<double>& a, int nSlices, const double* x, double* y, double* partials, cudaStream_t st) {
#define FVM_L(W) pdl_launch(k_spmv_dot_ell<W>, ceil_div(a.n, kBlock), kBlock, st, a, x, y, partials)
  if (a.ellWidth && FVM_ELL_SWITCH(a.ellWidth, FVM_L)) return;
#undef FVM_L
  pdl_launch(k_spmv_dot, reduce_blocks(nSlices), kBlock, st, a, nSlices, x, y, partials);
}
void spmv_dot_pby(const SellView<double>& a, int nSlices, const double* z, const double* p, const double* beta,
                  double* y, double* partials, cudaStream_t st) {
#define FVM_L(W) pdl_launch(k_spmv_dot_pby_ell<W>, ceil_div(a.n, kBlock), kBlock, st, a, z, p, beta, y, partials)
  if (a.ellWidth && FVM_ELL_SWITCH(a.ellWidth, FVM_L)) return;
#undef FVM_L
  pdl_launch(k_spmv_dot_pby, reduce_blocks(nSlices), kBlock, st, a, nSlices, z, p, beta, y, partials);
}
void cg_update_pby(int n, const double* alpha, const double* z, const double* beta, double* p, const double* q,
                   double* x, double* r, double* partials, cudaStream_t st, float* rF) {
  pdl_launch(k_cg_update_pby, vec_blocks(n), kBlock, st, n, alpha, z, beta, p, q, x, r, partials, rF);
}
template <class S>
void cg_take_z(int n, const S* src, const double* r, double* z, double* partials, cudaStream_t st) {
  pdl_launch(k_cg_take_z<S>, vec_blocks(n), kBlock, st, n, src, r, z, partials);
}
template void cg_take_z<float>(int, const float*, const double*, double*, double*, cudaStream_t);
template void cg_take_z<double>(int, const double*, const double*, double*, double*, cudaStream_t);
void cg_beta(int np, const double* partials, double* rho, double* rhoPrev, double* beta, bool flexible,
             cudaStream_t st) {
  pdl_launch(k_cg_beta, 1, 1024, st, np, partials, rho, rhoPrev, beta, flexible ? 1 : 0);
}
void cg_alpha(int np, const double* partials, const double* rho, double* alpha, cudaStream_t st) {
  pdl_launch(k_cg_alpha, 1, 1024, st, np, partials, rho, alpha);
}
void cg_update(int n, const double* alpha, const double* p, const double* q, double* x, double* r, double* partials,
               cudaStream_t st, float* rF) {
  pdl_launch(k_cg_update, vec_blocks(n), kBlock, st, n, alpha, p, q, x, r, partials, rF);
}
template <class T>
void restrict_sum(int nc, const int* c2fRow, const int* c2fCol, const T* r, T* bc, cudaStream_t st) {
  pdl_launch(k_restrict<T>, ceil_div(nc, kBlock), kBlock, st, nc, c2fRow, c2fCol, r, bc, (T*)nullptr);
}
template <class T>
void restrict_rhs(int nc, const int* c2fRow, const int* c2fCol, const T* b, T* bc, T* xc, cudaStream_t st) {
  pdl_launch(k_restrict<T>, ceil_div(nc, kBlock), kBlock, st, nc, c2fRow, c2fCol, b, bc, xc);
}
template <class T>
void residual_restrict(const SellView<T>& a, int nSlices, const int* rowSlice, int nc, const int* c2fRow,
                       const int* c2fCol, const T* x, const T* b, T* bc, T* xc, T* r, cudaStream_t st) {
  if (r) {
    residual<T>(a, nSlices, x, b, r, nullptr, st);
    pdl_launch(k_restrict<T>, ceil_div(nc, kBlock), kBlock, st, nc, c2fRow, c2fCol, (const T*)r, bc, xc);
    return;
  }
  pdl_launch(k_residual_restrict<T>, ceil_div(nc, kBlock), kBlock, st, a, rowSlice, nc, c2fRow, c2fCol, x, b, bc, xc);
}
template <class T>
void zero(int n, T* x, cudaStream_t st) {
  pdl_launch(k_zero<T>, ceil_div(n, kBlock), kBlock, st, n, x);
}
template <class T>
void prolong(int n, const int* ci, const T* xc, T* x, cudaStream_t st, bool assign) {
  pdl_launch(k_prolong<T>, ceil_div(n, kBlock), kBlock, st, n, ci, xc, x, assign ? 1 : 0);
}
template <class T>
void dense_solve(int n, const double* ainv, const T* b, T* x, cudaStream_t st) {
  pdl_launch(k_dense_solve<T>, ceil_div(n, kBlock / 32), kBlock, st, n, ainv, b, x);
}
void dense_solve_f32(int n, const float* ainv, const float* b, float* x, cudaStream_t st) {
  pdl_launch(k_dense_solve_f32, ceil_div(n, kBlock / 32), kBlock, st, n, ainv, b, x);
}
namespace {
constexpr int kGjMaxPanel = 8;
// the panel's shared memory: the 227 KB a CTA may hold, less 2 KB for the
// kernel's static reduction arrays
constexpr size_t kGjSmemLimit = 227 * 1024 - 2048;
size_t gj_align(size_t b) { return (b + 255) & ~size_t(255); }

// ---- Gauss-Jordan without pivoting (diagonally dominant matrices) ----------
// The in-place sweep over a panel K = [k0, k0 + nb) of pivots, with
// D = A[K][K]:
//   A[K][K] <- D^-1          A[K][j] <- D^-1 A[K][j]                 (j not in K)
//   A[i][K] <- -A[i][K] D^-1 A[i][j] <- A[i][j] - A[i][K] D^-1 A[K][j] (i, j not in K)
// After all panels A holds its inverse. Without pivot searches each panel
// is two kernels over the matrix: k_gjd_rows forms the panel's new pivot
// rows Rp = D^-1 A[K][:] once, then k_gjd_update sweeps 64 x 64 tiles,
// each thread 4 x 4 entries, with the tile's 64 x 32 panel columns and
// 32 x 64 pivot rows staged in shared memory by asynchronous copies
// (cp.async, issued after the tile's own loads, so the latencies of both
// overlap and no register holds a staged value; 16 fused multiply-adds per
// 8 shared loads). The panel's old rows and columns are read from side
// buffers (R, C) that the previous panel's update filled while writing
// them, so no CTA reads a value another CTA of the same launch writes;
// D^-1 comes ready-made: the last CTA of the previous launch to finish (a
// fence and a ticket counter, no waiting) inverts the next panel's block.
// Side buffers use padded strides: rows of R and Rp hold ld = n rounded up
// to 64 doubles, C holds ld rows of 32, and their padding stays zero (the
// buffers are cleared once), so every staged copy is 16-byte aligned and in
// bounds. Diagonal dominance keeps every pivot away from zero and the
// growth bounded, which is why the caller takes this path only for
// diagonally dominant levels. This is not a reference computation, so the
// products use fused multiply-adds (__fma_rn) although the file is built
// without contraction.
constexpr int kGdB = 32;   // panel width
constexpr int kGdT = 64;   // tile rows / columns
constexpr int kGdPad = 2;  // shared row padding (keeps 16-byte row alignment)

int gjd_ld(int n) { return (n + kGdT - 1) / kGdT * kGdT; }

__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
  const unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem));
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

// The inverse of the nb x nb block src[r * stride + c] (padded to kGdB with
// the identity) into Dout; D: shared memory of 2 x kGdB x (kGdB + 1)
// doubles (double-buffered block)
__device__ void gjd_invert_block(const double* src, size_t stride, int nb, double* Dout, int* status,
                                 double (*D)[kGdB][kGdB + 1]) {
  const int tid = threadIdx.x, nt = blockDim.x;
  for (int e = tid; e < kGdB * kGdB; e += nt) {
    const int r = e / kGdB, c = e % kGdB;
    D[0][r][c] = (r < nb && c < nb) ? __ldcg(src + (size_t)r * stride + c) : (r == c ? 1.0 : 0.0);
  }
  __syncthreads();
  int cur = 0;
  for (int t = 0; t < kGdB; t++) {
    const double pv = D[cur][t][t];
    const double ip = 1.0 / pv;
    for (int e = tid; e < kGdB * kGdB; e += nt) {
      const int r = e / kGdB, c = e % kGdB;
      const double drt = D[cur][r][t], dtc = D[cur][t][c], drc = D[cur][r][c];
      double v;
      if (r == t && c == t)
        v = ip;
      else if (r == t)
        v = dtc * ip;
      else if (c == t)
        v = -drt * ip;
      else
        v = __fma_rn(-drt, dtc * ip, drc);
      D[cur ^ 1][r][c] = v;
    }
    if (pv == 0.0 && tid == 0) atomicExch(status, 1);
    cur ^= 1;
    __syncthreads();
  }
  for (int e = tid; e < kGdB * kGdB; e += nt) Dout[e] = D[cur][e / kGdB][e % kGdB];
}

// C[i * kGdB + t] = A[i][k0 + t], R[t * ld + j] = A[k0 + t][j] (t < nb; 0 beyond)
__global__ void k_gjd_extract(int n, int ld, int k0, int nb, const double* __restrict__ A, double* __restrict__ C,
                              double* __restrict__ R) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= n) return;
  for (int t = 0; t < kGdB; t++) {
    R[(size_t)t * ld + j] = t < nb ? A[(size_t)(k0 + t) * n + j] : 0.0;
    C[(size_t)j * kGdB + t] = t < nb ? A[(size_t)j * n + k0 + t] : 0.0;
  }
}

__global__ void __launch_bounds__(256) k_gjd_first(const double* __restrict__ src, size_t stride, int nb,
                                                   double* Dout, int* status) {
  __shared__ double D[2][kGdB][kGdB + 1];
  gjd_invert_block(src, stride, nb, Dout, status, D);
}

// Rp[t][j] = sum_u D[t][u] R[u][j]: the panel's new pivot rows; one CTA
// (256 threads) per 32 columns stages R's 32 x 32 block, each thread forms
// four outputs (grid ceil(n / 32); the padding columns come out zero)
__global__ void __launch_bounds__(256) k_gjd_rows(int ld, int nb, const double* __restrict__ R,
                                                  const double* __restrict__ Dinv, double* __restrict__ Rp) {
  __shared__ double D[kGdB][kGdB + 1];
  __shared__ double Rs[kGdB][kGdB + 1];
  const int tid = threadIdx.x, c = tid & 31, w = tid >> 5;
  const int j = blockIdx.x * kGdB + c;
#pragma unroll
  for (int q = 0; q < 4; q++) {
    const int u = w + 8 * q;
    Rs[u][c] = u < nb ? R[(size_t)u * ld + j] : 0.0;
    D[u][c] = Dinv[u * kGdB + c];
  }
  __syncthreads();
#pragma unroll
  for (int q = 0; q < 4; q++) {
    const int t = w + 8 * q;
    double acc = 0.0;
#pragma unroll
    for (int u = 0; u < kGdB; u++) acc = __fma_rn(D[t][u], Rs[u][c], acc);
    Rp[(size_t)t * ld + j] = t < nb ? acc : 0.0;
  }
}

// One panel [k0, k0 + nb) over the whole matrix in 64 x 64 tiles, 256
// threads. Unsymmetric (Sym = false): grid (ceil(n / 64), ceil(n / 64)),
// the Gauss-Jordan sweep; fills Cn / Rn with the next panel's [k1, k1 +
// nb1) columns / rows. Symmetric (Sym = true): one CTA per tile on or above
// the diagonal (grid T (T + 1) / 2, T = ceil(n / 64)), the sweep operator
// (pivot block -D^-1, panel columns C D^-1 unnegated), which keeps the
// matrix symmetric; Cn gets the next panel's columns from the column strip
// and, transposed, from the row strip of the off-diagonal tiles (Rn is not
// used). In both the launch's last CTA inverts the next pivot block into
// Dnext. *ticket is 0 on entry and left 0.
template <bool Sym>
__global__ void __launch_bounds__(256, 3) k_gjd_update(int n, int ld, int k0, int nb, double* __restrict__ A,
                                                    const double* __restrict__ C, const double* __restrict__ Rp,
                                                    const double* __restrict__ Dinv, double* __restrict__ Cn,
                                                    double* __restrict__ Rn, double* __restrict__ Dnext, int k1,
                                                    int nb1, unsigned* ticket, int* status) {
  // Cs doubles as the last CTA's pivot-block workspace (2 x 32 x 33 doubles)
  static_assert(kGdT * (kGdB + kGdPad) >= 2 * kGdB * (kGdB + 1), "block inverse workspace");
  __shared__ __align__(16) double Cs[kGdT][kGdB + kGdPad];
  __shared__ __align__(16) double Rs[kGdB][kGdT + kGdPad];
  __shared__ __align__(16) double Ds[kGdB][kGdB + kGdPad];
  __shared__ bool last;
  const int tid = threadIdx.x;
  int bi = blockIdx.y, bj = blockIdx.x;
  if (Sym) {
    // the p-th tile of the upper triangle, row by row
    const int T = (n + kGdT - 1) / kGdT;
    int p = blockIdx.x;
    bi = 0;
    while (p >= T - bi) {
      p -= T - bi;
      bi++;
    }
    bj = bi + p;
  }
  const int i0 = bi * kGdT, j0 = bj * kGdT;
  const int ty = tid >> 4, tx = tid & 15;
  // does the tile meet the panel's rows / columns?
  const bool rowsK = i0 < k0 + nb && i0 + kGdT > k0;
  const bool colsK = j0 < k0 + nb && j0 + kGdT > k0;
  // the tile's own entries are loaded first, so their latency overlaps the
  // staging of the panel columns and pivot rows (they do not depend on it)
  double acc[4][4];
#pragma unroll
  for (int a = 0; a < 4; a++) {
    const int i = i0 + ty + 16 * a;
#pragma unroll
    for (int b = 0; b < 4; b++) {
      const int j = j0 + tx + 16 * b;
      acc[a][b] = (i < n && j < n) ? A[(size_t)i * n + j] : 0.0;
    }
  }
  // 16-byte copies: Cs 64 rows x 16, Rs 32 rows x 32, Ds 32 rows x 16;
  // i0 + 64 <= ld and j0 + 64 <= ld keep every source inside the buffers
#pragma unroll
  for (int q = 0; q < 4; q++) {
    const int e = tid + 256 * q;
    const int r = e >> 4, k = (e & 15) * 2;
    cp_async16(&Cs[r][k], C + (size_t)(i0 + r) * kGdB + k);
  }
#pragma unroll
  for (int q = 0; q < 4; q++) {
    const int e = tid + 256 * q;
    const int t = e >> 5, k = (e & 31) * 2;
    cp_async16(&Rs[t][k], Rp + (size_t)t * ld + j0 + k);
  }
  if (colsK || rowsK) {
#pragma unroll
    for (int q = 0; q < 2; q++) {
      const int e = tid + 256 * q;
      const int r = e >> 4, k = (e & 15) * 2;
      cp_async16(&Ds[r][k], Dinv + r * kGdB + k);
    }
  }
  cp_async_wait_all();
  __syncthreads();
#pragma unroll 4
  for (int t = 0; t < kGdB; t++) {
    double c[4], r[4];
#pragma unroll
    for (int a = 0; a < 4; a++) c[a] = Cs[ty + 16 * a][t];
#pragma unroll
    for (int b = 0; b < 4; b++) r[b] = Rs[t][tx + 16 * b];
#pragma unroll
    for (int a = 0; a < 4; a++)
#pragma unroll
      for (int b = 0; b < 4; b++) acc[a][b] = __fma_rn(-c[a], r[b], acc[a][b]);
  }
#pragma unroll
  for (int a = 0; a < 4; a++) {
    const int r = ty + 16 * a;
    const int i = i0 + r;
    if (i >= n) continue;
    const bool iK = i >= k0 && i < k0 + nb;
#pragma unroll
    for (int b = 0; b < 4; b++) {
      const int cix = tx + 16 * b;
      const int j = j0 + cix;
      if (j >= n) continue;
      const bool jK = j >= k0 && j < k0 + nb;
      double v = acc[a][b];
      if (iK && jK) {
        v = Sym ? -Ds[i - k0][j - k0] : Ds[i - k0][j - k0];
      } else if (iK) {
        v = Rs[i - k0][cix];
      } else if (jK) {
        double s = 0.0;
        for (int t = 0; t < kGdB; t++) s = __fma_rn(Cs[r][t], Ds[t][j - k0], s);
        v = Sym ? s : -s;
      }
      A[(size_t)i * n + j] = v;
      if (j >= k1 && j < k1 + nb1) Cn[(size_t)i * kGdB + (j - k1)] = v;
      if (i >= k1 && i < k1 + nb1) {
        if (!Sym)
          Rn[(size_t)(i - k1) * ld + j] = v;
        else if (bi != bj)  // the diagonal tile's own column strip covers it
          Cn[(size_t)j * kGdB + (i - k1)] = v;
      }
    }
  }
  if (nb1 <= 0) return;  // the last panel: no next block to invert
  // the last CTA to finish inverts the next panel's pivot block: the
  // barrier orders the CTA's writes before thread 0's fence, which makes
  // them visible device-wide before its ticket increment (fences are
  // cumulative in the PTX memory model; the CUDA cooperative-groups grid
  // barrier relies on the same CTA barrier + one-thread fence pattern).
  // A fence in every thread measured one membar stall per issued
  // instruction here.
  __syncthreads();
  if (tid == 0) {
    __threadfence();
    const unsigned done = atomicAdd(ticket, 1u);
    last = done == gridDim.x * gridDim.y - 1;
  }
  __syncthreads();
  if (!last) return;
  __threadfence();
  double(*ws)[kGdB][kGdB + 1] = reinterpret_cast<double(*)[kGdB][kGdB + 1]>(&Cs[0][0]);
  if (Sym)
    gjd_invert_block(Cn + (size_t)k1 * kGdB, kGdB, nb1, Dnext, status, ws);
  else
    gjd_invert_block(Rn + k1, (size_t)ld, nb1, Dnext, status, ws);
  if (tid == 0) *ticket = 0u;
}

// Symmetric sweep: C[j * kGdB + t] = A[j][t] (t < nb; 0 beyond)
__global__ void k_gjs_extract(int n, int nb, const double* __restrict__ A, double* __restrict__ C) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= n) return;
  for (int t = 0; t < kGdB; t++) C[(size_t)j * kGdB + t] = t < nb ? A[(size_t)j * n + t] : 0.0;
}

// Symmetric sweep: the pivot rows Rp[t][j] = sum_u D[t][u] A[K + u][j], with
// A[K + u][j] = C[j][u] by symmetry; one CTA (256 threads) per 32 columns
__global__ void __launch_bounds__(256) k_gjs_rows(int ld, int nb, const double* __restrict__ C,
                                                  const double* __restrict__ Dinv, double* __restrict__ Rp) {
  __shared__ double D[kGdB][kGdB + 1];
  __shared__ double Ct[kGdB][kGdB + 1];  // Ct[c][u] = C[j0 + c][u]
  const int tid = threadIdx.x, c = tid & 31, w = tid >> 5;
  const int j0 = blockIdx.x * kGdB;
#pragma unroll
  for (int q = 0; q < 4; q++) {
    const int rr = w + 8 * q;
    Ct[rr][c] = C[(size_t)(j0 + rr) * kGdB + c];
    D[rr][c] = Dinv[rr * kGdB + c];
  }
  __syncthreads();
#pragma unroll
  for (int q = 0; q < 4; q++) {
    const int t = w + 8 * q;
    double acc = 0.0;
#pragma unroll
    for (int u = 0; u < kGdB; u++) acc = __fma_rn(D[t][u], u < nb ? Ct[c][u] : 0.0, acc);
    Rp[(size_t)t * ld + j0 + c] = t < nb ? acc : 0.0;
  }
}

// Symmetric sweep, last step: the upper triangle holds -A^-1; negate it and
// mirror it to the lower triangle (32 x 32 tiles on and above the diagonal,
// grid T (T + 1) / 2 with T = ceil(n / 32), block 32 x 8). Each CTA reads
// only its own upper tile and writes it and its mirror, so no two CTAs
// touch the same entry.
__global__ void __launch_bounds__(256) k_gjs_finish(int n, double* A) {
  __shared__ double S[32][33];
  const int T = (n + 31) / 32;
  int p = blockIdx.x, bi = 0;
  while (p >= T - bi) {
    p -= T - bi;
    bi++;
  }
  const int bj = bi + p;
  const int i0 = bi * 32, j0 = bj * 32;
  const int c = threadIdx.x;
  for (int r = threadIdx.y; r < 32; r += 8) {
    const int i = i0 + r, j = j0 + c;
    S[r][c] = (i < n && j < n) ? A[(size_t)i * n + j] : 0.0;
  }
  __syncthreads();
  for (int r = threadIdx.y; r < 32; r += 8) {
    const int i = i0 + r, j = j0 + c;
    if (i < n && j < n) A[(size_t)i * n + j] = -(bi == bj && r > c ? S[c][r] : S[r][c]);
    if (bi != bj) {
      const int i2 = j0 + r, j2 = i0 + c;  // mirror tile: A[j0 + r][i0 + c] = -S[c][r]
      if (i2 < n && j2 < n) A[(size_t)i2 * n + j2] = -S[c][r];
    }
  }
}

// *flag = 1 unless |a_ij - a_ji| <= 1e-12 max(|a_ij|, |a_ji|) everywhere
// (one thread per entry above the diagonal; *flag must be 0 on entry)
__global__ void k_dense_symmetry(int n, const double* __restrict__ A, int* flag) {
  const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= (long long)n * n) return;
  const int i = (int)(e / n), j = (int)(e % n);
  if (j <= i) return;
  const double a = A[(size_t)i * n + j], b = A[(size_t)j * n + i];
  if (!(fabs(a - b) <= 1e-12 * fmax(fabs(a), fabs(b)))) atomicExch(flag, 1);
}

// Look-ahead: after panel p's row swaps, the next panel's columns are
// updated first and factored on stream st while the rest of the matrix
// takes panel p's update on a second stream (disjoint columns); panel p+1's
// row swaps then wait for that update. The single-CTA panel factorization
// thus overlaps the whole-GPU update instead of following it.
template <int B>
void gj_run(int n, double* a, double* inv, double* Bt, int* piv, int* idx, int* status, cudaStream_t st) {
  const size_t smem = sizeof(double) * (size_t)B * n;
  cudaFuncSetAttribute(k_gj_panel<B>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  cudaStream_t us = nullptr;
  cudaEvent_t swapped = nullptr, updated = nullptr;
  const bool split = cudaStreamCreateWithFlags(&us, cudaStreamNonBlocking) == cudaSuccess &&
                     cudaEventCreateWithFlags(&swapped, cudaEventDisableTiming) == cudaSuccess &&
                     cudaEventCreateWithFlags(&updated, cudaEventDisableTiming) == cudaSuccess;
  const dim3 ug(ceil_div(n, kBlock), n);
  k_gj_panel<B><<<1, 1024, smem, st>>>(n, 0, n < B ? n : B, a, piv, status);
  for (int k0 = 0; k0 < n; k0 += B) {
    const int nb = n - k0 < B ? n - k0 : B;
    const int k1 = k0 + nb;                          // next panel [k1, k1 + nb1)
    const int nb1 = n - k1 < B ? n - k1 : B;
    if (split && k0 > 0) cudaStreamWaitEvent(st, updated, 0);  // previous panel's update done
    k_gj_swap_rows<<<ceil_div(n, kBlock), kBlock, 0, st>>>(n, k0, nb, a, piv, Bt);
    if (!split || nb1 <= 0) {
      k_gj_update<<<ug, kBlock, 0, st>>>(n, k0, nb, a, Bt, 0, n, 0, 0);
      if (nb1 > 0) k_gj_panel<B><<<1, 1024, smem, st>>>(n, k1, nb1, a, piv, status);
      continue;
    }
    cudaEventRecord(swapped, st);
    const dim3 ul(ceil_div(nb1, kBlock), n);
    k_gj_update<<<ul, kBlock, 0, st>>>(n, k0, nb, a, Bt, k1, k1 + nb1, 0, 0);
    k_gj_panel<B><<<1, 1024, smem, st>>>(n, k1, nb1, a, piv, status);
    cudaStreamWaitEvent(us, swapped, 0);
    k_gj_update<<<ug, kBlock, 0, us>>>(n, k0, nb, a, Bt, 0, n, k1, k1 + nb1);
    cudaEventRecord(updated, us);
  }
  if (split) {
    cudaStreamWaitEvent(st, updated, 0);
    cudaEventDestroy(swapped);
    cudaEventDestroy(updated);
    cudaStreamDestroy(us);
  }
  k_gj_colperm<<<1, 1, 0, st>>>(n, piv, idx);
  k_gj_gather<<<ug, kBlock, 0, st>>>(n, a, idx, inv);
}
}  // namespace

// scratch: [panel doubles][piv: n ints][idx: n ints][status]; the panel
// doubles hold the pivoted path's Bt (kGjMaxPanel x n) or the unpivoted
// path's side buffers (C, R of two panels and Rp, 5 x kGdB x ld, ld = n
// rounded up to 64), plus its two inverted pivot blocks and its ticket
// counter
size_t gj_panel_bytes(int n) {
  const size_t ld = (size_t)gjd_ld(n);
  const size_t unpiv = 5 * (size_t)kGdB * ld + 2 * kGdB * kGdB + 2;
  const size_t piv = (size_t)kGjMaxPanel * n;
  return gj_align(sizeof(double) * (unpiv > piv ? unpiv : piv));
}
size_t gauss_jordan_scratch_bytes(int n) {
  return gj_panel_bytes(n) + 2 * gj_align(sizeof(int) * (size_t)n) + gj_align(sizeof(int));
}
const int* gauss_jordan_status(int n, const void* scratch) {
  const char* s = (const char*)scratch;
  return (const int*)(s + gj_panel_bytes(n) + 2 * gj_align(sizeof(int) * (size_t)n));
}
void gauss_jordan_inverse_dominant(int n, double* a, void* scratch, cudaStream_t st) {
  double* sb = (double*)scratch;
  const int ld = gjd_ld(n);
  const size_t pn = (size_t)kGdB * ld;
  double* C[2] = {sb, sb + pn};
  double* R[2] = {sb + 2 * pn, sb + 3 * pn};
  double* Rp = sb + 4 * pn;
  double* Dv[2] = {sb + 5 * pn, sb + 5 * pn + kGdB * kGdB};
  unsigned* ticket = (unsigned*)(sb + 5 * pn + 2 * kGdB * kGdB);
  int* status = (int*)gauss_jordan_status(n, scratch);
  cudaMemsetAsync(status, 0, sizeof(int), st);
  // side buffers, blocks and ticket: the padding must read as zero
  cudaMemsetAsync(sb, 0, sizeof(double) * (5 * pn + 2 * kGdB * kGdB + 2), st);
  if (n <= 0) return;
  const int nb0 = n < kGdB ? n : kGdB;
  k_gjd_extract<<<ceil_div(n, kBlock), kBlock, 0, st>>>(n, ld, 0, nb0, a, C[0], R[0]);
  k_gjd_first<<<1, 256, 0, st>>>(R[0], (size_t)ld, nb0, Dv[0], status);
  const dim3 grid(ceil_div(n, kGdT), ceil_div(n, kGdT));
  int cur = 0;
  for (int k0 = 0; k0 < n; k0 += kGdB) {
    const int nb = n - k0 < kGdB ? n - k0 : kGdB;
    const int k1 = k0 + nb;
    const int nb1 = n - k1 < kGdB ? n - k1 : kGdB;
    k_gjd_rows<<<ceil_div(n, kGdB), 256, 0, st>>>(ld, nb, R[cur], Dv[cur], Rp);
    k_gjd_update<false><<<grid, 256, 0, st>>>(n, ld, k0, nb, a, C[cur], Rp, Dv[cur], C[cur ^ 1], R[cur ^ 1],
                                              Dv[cur ^ 1], k1, nb1 > 0 ? nb1 : 0, ticket, status);
    cur ^= 1;
  }
}
void gauss_jordan_inverse_symmetric(int n, double* a, void* scratch, cudaStream_t st) {
  double* sb = (double*)scratch;
  const int ld = gjd_ld(n);
  const size_t pn = (size_t)kGdB * ld;
  double* C[2] = {sb, sb + pn};
  double* Rp = sb + 4 * pn;
  double* Dv[2] = {sb + 5 * pn, sb + 5 * pn + kGdB * kGdB};
  unsigned* ticket = (unsigned*)(sb + 5 * pn + 2 * kGdB * kGdB);
  int* status = (int*)gauss_jordan_status(n, scratch);
  cudaMemsetAsync(status, 0, sizeof(int), st);
  cudaMemsetAsync(sb, 0, sizeof(double) * (5 * pn + 2 * kGdB * kGdB + 2), st);
  if (n <= 0) return;
  const int nb0 = n < kGdB ? n : kGdB;
  k_gjs_extract<<<ceil_div(n, kBlock), kBlock, 0, st>>>(n, nb0, a, C[0]);
  k_gjd_first<<<1, 256, 0, st>>>(C[0], (size_t)kGdB, nb0, Dv[0], status);
  const int T = ceil_div(n, kGdT);
  int cur = 0;
  for (int k0 = 0; k0 < n; k0 += kGdB) {
    const int nb = n - k0 < kGdB ? n - k0 : kGdB;
    const int k1 = k0 + nb;
    const int nb1 = n - k1 < kGdB ? n - k1 : kGdB;
    k_gjs_rows<<<ceil_div(n, kGdB), 256, 0, st>>>(ld, nb, C[cur], Dv[cur], Rp);
    k_gjd_update<true><<<T * (T + 1) / 2, 256, 0, st>>>(n, ld, k0, nb, a, C[cur], Rp, Dv[cur], C[cur ^ 1], nullptr,
                                                         Dv[cur ^ 1], k1, nb1 > 0 ? nb1 : 0, ticket, status);
    cur ^= 1;
  }
  const int T32 = ceil_div(n, 32);
  k_gjs_finish<<<T32 * (T32 + 1) / 2, dim3(32, 8), 0, st>>>(n, a);
}
void dense_symmetry_check(int n, const double* a, int* flag, cudaStream_t st) {
  if (n > 0) k_dense_symmetry<<<ceil_div((long long)n * n, kBlock), kBlock, 0, st>>>(n, a, flag);
}
namespace {
// a (n x n, row-major, zeroed) += the SELL-32 level: one thread per row
__global__ void k_dense_from_sell(SellView<double> m, int nSlices, double* a) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  const int s = t >> 5, lane = t & 31;
  if (s >= nSlices) return;
  const int4 mt = m.meta[s];
  if (lane >= mt.y) return;
  const int i = mt.x + lane;
  double* ai = a + (size_t)i * m.n;
  ai[i] += m.diag[i];
  for (int k = 0; k < mt.w; k++) {
    const int e = mt.z + (k << 5) + lane;
    const double v = m.vals[e];
    if (v != 0.0) ai[m.cols[e]] += v;
  }
}
}  // namespace

void dense_from_sell(const SellView<double>& m, int nSlices, double* a, cudaStream_t st) {
  cudaMemsetAsync(a, 0, sizeof(double) * (size_t)m.n * m.n, st);
  k_dense_from_sell<<<ceil_div((long long)nSlices * 32, kBlock), kBlock, 0, st>>>(m, nSlices, a);
}

void gauss_jordan_inverse(int n, double* a, double* inv, void* scratch, cudaStream_t st) {
  char* s = (char*)scratch;
  double* Bt = (double*)s;
  int* piv = (int*)(s + gj_panel_bytes(n));
  int* idx = piv + gj_align(sizeof(int) * (size_t)n) / sizeof(int);
  int* status = (int*)gauss_jordan_status(n, scratch);
  cudaMemsetAsync(status, 0, sizeof(int), st);
  // the widest panel (up to 8 columns) whose n x B block fits in shared
  // memory: every panel streams the whole matrix once, so fewer, wider panels
  // stream less (4096 rows: 7 columns, 586 panels instead of 1024 of 4);
  // wider than 8, the single-CTA panel factorization costs more than the
  // passes it saves (2294 rows: 20.5 ms with 12 columns, 14.5 ms with 8)
  const size_t col = sizeof(double) * (size_t)n;
  if (8 * col <= kGjSmemLimit)
    gj_run<8>(n, a, inv, Bt, piv, idx, status, st);
  else if (7 * col <= kGjSmemLimit)
    gj_run<7>(n, a, inv, Bt, piv, idx, status, st);
  else if (6 * col <= kGjSmemLimit)
    gj_run<6>(n, a, inv, Bt, piv, idx, status, st);
  else if (4 * col <= kGjSmemLimit)
    gj_run<4>(n, a, inv, Bt, piv, idx, status, st);
  else
    gj_run<2>(n, a, inv, Bt, piv, idx, status, st);
}
void cast_d2f(size_t n, const double* a, float* b, cudaStream_t st) {
  k_cast_d2f_big<<<(unsigned)((n + kBlock - 1) / kBlock), kBlock, 0, st>>>(n, a, b);
}
void convert_d2f(int n, const double* a, float* b, cudaStream_t st) {
  pdl_launch(k_convert_d2f, ceil_div(n, kBlock), kBlock, st, n, a, b);
}
void add_f2d(int n, const float* a, double* b, cudaStream_t st) {
  pdl_launch(k_add_f2d, ceil_div(n, kBlock), kBlock, st, n, a, b);
}
int vec_blocks(int n) {
  const int b = ceil_div(n, kBlock);
  return b < kReduceBlocks ? (b < 1 ? 1 : b) : kReduceBlocks;
}
void l1_partials(int n, const double* a, double* partials, cudaStream_t st) {
  pdl_launch(k_l1_partials, vec_blocks(n), kBlock, st, n, a, partials);
}
void cg_start(int n, const double* b, double* r, float* rF, double* partials, cudaStream_t st) {
  pdl_launch(k_cg_start, vec_blocks(n), kBlock, st, n, b, r, rF, partials);
}
void dot_partials(int n, const double* a, const double* b, double* partials, cudaStream_t st) {
  pdl_launch(k_dot_partials, vec_blocks(n), kBlock, st, n, a, b, partials);
}
void sum_partials(int np, const double* partials, double* out, cudaStream_t st) {
  pdl_launch(k_sum_partials, 1, 1024, st, np, partials, out);
}
void scalar_div(const double* num, const double* den, double* out, cudaStream_t st) {
  pdl_launch(k_scalar_div, 1, 1, st, num, den, out);
}
void scalar_flex_beta(const double* rho, const double* rzPrev, const double* rhoPrev, double* out, cudaStream_t st) {
  pdl_launch(k_scalar_flex_beta, 1, 1, st, rho, rzPrev, rhoPrev, out);
}
void scalar_ratio_product(const double* a, const double* b, const double* c, const double* d,
                          double* out, cudaStream_t st) {
  pdl_launch(k_scalar_ratio_product, 1, 1, st, a, b, c, d, out);
}
void axpy_dev(int n, const double* s, double sign, const double* x, double* y, cudaStream_t st) {
  pdl_launch(k_axpy_dev, ceil_div(n, kBlock), kBlock, st, n, s, sign, x, y);
}
void xpby_dev(int n, const double* z, const double* beta, double* p, cudaStream_t st) {
  pdl_launch(k_xpby_dev, ceil_div(n, kBlock), kBlock, st, n, z, beta, p);
}
void bicg_p_update(int n, const double* r, const double* v, const double* omega, const double* beta,
                   double* p, cudaStream_t st) {
  pdl_launch(k_bicg_p, ceil_div(n, kBlock), kBlock, st, n, r, v, omega, beta, p);
}
void copy_d(int n, const double* a, double* b, cudaStream_t st) {
  pdl_launch(k_copy_d, ceil_div(n, kBlock), kBlock, st, n, a, b);
}

void face_coefficients(const FaceGeom& g, const double* k, double* coeff, double* secCoeff,
                       cudaStream_t st) {
  k_face_coefficients<<<ceil_div(g.nFaces, kBlock), kBlock, 0, st>>>(g, k, coeff, secCoeff);
}
void gradient(int nCells, const int* ccRow, const int* ccCol, const double* w, const double* x,
              double* grad, cudaStream_t st) {
  pdl_launch(k_gradient, ceil_div(nCells, kBlock), kBlock, st, nCells, ccRow, ccCol, w, x, grad);
}
void ghost_gradient(int nB, const int* bFaces, const int* faceCells, double* grad, cudaStream_t st) {
  if (nB > 0) pdl_launch(k_ghost_gradient, ceil_div(nB, kBlock), kBlock, st, nB, bFaces, faceCells, grad);
}
void face_flux(const FaceGeom& g, const double* coeff, const double* secCoeff, const double* grad,
               const double* x, double* flux, cudaStream_t st) {
  pdl_launch(k_face_flux, ceil_div(g.nFaces, kBlock), kBlock, st, g, coeff, secCoeff, grad, x, flux);
}
void assemble_rhs(int nCells, const CellFaceView& cf, const int* faceCells, const double* flux,
                  const double* coeff, const double* faceAreaMag, const double* vol,
                  const double* source, const double* rhoVdt, const double* xN1,
                  const BoundaryData& bd, const int* bIndexOfFace, double* x, const int* perm, double* b,
                  cudaStream_t st) {
  pdl_launch(k_assemble_rhs, ceil_div(nCells, kBlock), kBlock, st, nCells, cf, faceCells, flux, coeff,
                                                              faceAreaMag, vol, source, rhoVdt, xN1,
                                                              bd, bIndexOfFace, x, perm, b);
}
void assemble_matrix(int nCells, const CellFaceView& cf, const int* faceCells, const double* coeff,
                     const double* faceAreaMag, const double* rhoVdt, const BoundaryData& bd,
                     const int* bIndexOfFace, const double* x, double* diagOrig, cudaStream_t st) {
  k_assemble_matrix<<<ceil_div(nCells, kBlock), kBlock, 0, st>>>(nCells, cf, faceCells, coeff, faceAreaMag,
                                                                 rhoVdt, bd, bIndexOfFace, x, diagOrig);
}
void transient_coeff(int n, const double* rhoCp, const double* vol, double dt, double* out,
                     cudaStream_t st) {
  k_transient_coeff<<<ceil_div(n, kBlock), kBlock, 0, st>>>(n, rhoCp, vol, dt, out);
}
void cast_d2f_vals(int n, const double* a, float* b, cudaStream_t st) {
  k_cast_d2f<<<ceil_div(n, kBlock), kBlock, 0, st>>>(n, a, b);
}
void update_solution(int nCells, const int* perm, const double* delta, const BoundaryData& bd,
                     const int* faceCells, const double* coeff, double* x, cudaStream_t st) {
  pdl_launch(k_update_self, ceil_div(nCells, kBlock), kBlock, st, nCells, perm, delta, x);
  if (bd.nBFaces > 0)
    pdl_launch(k_update_ghosts, ceil_div(bd.nBFaces, kBlock), kBlock, st, bd, perm, delta, faceCells, coeff, x);
}

// explicit instantiations
#define FVM_INST(T)                                                                              \
  template void gs_color<T>(const SellView<T>&, int, int, T*, const T*, cudaStream_t, RowPlan, const T*,  \
                            const int*);                                                                \
  template void gs_sequential<T>(const SellView<T>&, T*, const T*, bool, cudaStream_t);          \
  template void jacobi<T>(const SellView<T>&, int, const T*, T*, const T*, cudaStream_t);        \
  template void jacobi_damped<T>(const SellView<T>&, int, const T*, T*, const T*, T, cudaStream_t, RowPlan,     \
                                 const T*, const int*);                                                          \
  template void chebyshev_step<T>(const SellView<T>&, int, const T*, T*, T*, const T*, T, T, bool, cudaStream_t); \
  template void residual<T>(const SellView<T>&, int, const T*, const T*, T*, double*, cudaStream_t); \
  template void restrict_sum<T>(int, const int*, const int*, const T*, T*, cudaStream_t);        \
  template void restrict_rhs<T>(int, const int*, const int*, const T*, T*, T*, cudaStream_t);    \
  template void residual_restrict<T>(const SellView<T>&, int, const int*, int, const int*,        \
                                     const int*, const T*, const T*, T*, T*, T*, cudaStream_t);   \
  template void zero<T>(int, T*, cudaStream_t);                                                  \
  template void prolong<T>(int, const int*, const T*, T*, cudaStream_t, bool);                         \
  template void dense_solve<T>(int, const double*, const T*, T*, cudaStream_t);
FVM_INST(double)
FVM_INST(float)
#undef FVM_INST

}  // namespace dev
}  // namespace fvm
