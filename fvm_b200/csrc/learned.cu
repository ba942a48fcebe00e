// Kernels of the learned correction (learned.hpp): forward, backward and
// Adam with fixed reduction orders (deterministic). Message passing,
// encoder, decoder and Adam run on the CUDA cores in FP32; the dense 64 ->
// 32 layer products (forward, and the backward's input and weight
// gradients) run on the tensor cores (tcgen05, TF32 inputs, FP32 sums), or
// optionally in FP32 on the CUDA cores.
//
// Layout: activations node-major, h[i * 32 + c]; one warp per node, lane =
// channel, so a neighbour's activations are one coalesced 128-byte load.
// The graph is the finest level's SELL-32 matrix (neighbours j of row i:
// its stored columns, padding entries carry a zero coupling).
#include <cmath>
#include <stdexcept>

#include "common.hpp"
#include "learned.hpp"
#include "umma.cuh"

namespace fvm {
namespace nn {

namespace {

constexpr int kBlock = 256;
constexpr int kWarps = kBlock / 32;
// Fixed grid of the gradient kernels: the assignment of nodes to warps, and
// so every floating-point summation order, does not depend on the device.
constexpr int kGradBlocks = 296;
constexpr unsigned kFull = 0xffffffffu;

int ceil_div(long long a, long long b) { return (int)((a + b - 1) / b); }
int node_blocks(int n) {
  const int b = ceil_div(n, kWarps);
  return b < 148 * 16 ? (b < 1 ? 1 : b) : 148 * 16;
}

__device__ __forceinline__ float relu(float x) { return x > 0.f ? x : 0.f; }

__device__ __forceinline__ double block_sum(double v) {
  __shared__ double red[kWarps];
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(kFull, v, o);
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  if (lane == 0) red[w] = v;
  __syncthreads();
  double s = 0.0;
  if (threadIdx.x == 0)
    for (int k = 0; k < kWarps; k++) s += red[k];
  __syncthreads();
  return s;
}

// sum_i |r_i| / |a_ii| per block (input scale)
__global__ void k_scale_partials(int n, const double* __restrict__ r, const double* __restrict__ diag,
                                 double* partials) {
  double s = 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    s += fabs(r[i]) / fabs(diag[i]);
  s = block_sum(s);
  if (threadIdx.x == 0) partials[blockIdx.x] = s;
}

// sum_i e_i^2 per block
__global__ void k_sq_partials(int n, const double* __restrict__ e, double* partials) {
  double s = 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) s += e[i] * e[i];
  s = block_sum(s);
  if (threadIdx.x == 0) partials[blockIdx.x] = s;
}

// u_i = r_i / (|a_ii| s), s = sum / n; s stored as scal[0] = sum / n
__global__ void k_input(int n, const double* __restrict__ r, const double* __restrict__ diag,
                        const double* __restrict__ sum, float* u, double* scale) {
  const double s = sum[0] / (double)n;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i == 0) scale[0] = s;
  if (i >= n) return;
  u[i] = s > 0.0 ? (float)(r[i] / (fabs(diag[i]) * s)) : 0.f;
}

__global__ void k_encode(int n, const float* __restrict__ u, const float* __restrict__ P, float* H0) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)n * 32) return;
  const int i = (int)(t >> 5), c = (int)(t & 31);
  H0[t] = relu(__fmaf_rn(P[kEncW + c], u[i], P[kEncB + c]));
}

struct GraphArgs {
  const int* cols;
  const double* vals;
  const double* diag;
  const int4* meta;
  const int* rowSlice;
  const float* wf;  // per stored entry (i, j): |a_ij| / |a_ii| (message weight)
  const float* wb;  // per stored entry (i, j): |a_ij| / |a_jj| (its transpose's weight)
};

// The message weights of every stored entry, computed once per pass (the
// same FP64 quotient rounded to FP32 that the layers used to form inline).
__global__ void k_edge_weights(int nSlices, const int4* __restrict__ meta, const int* __restrict__ cols,
                               const double* __restrict__ vals, const double* __restrict__ diag, float* wf,
                               float* wb) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  const int s = t >> 5, lane = t & 31;
  if (s >= nSlices) return;
  const int4 m = meta[s];
  if (lane >= m.y) return;
  const double di = fabs(diag[m.x + lane]);
  for (int k = 0; k < m.w; k++) {
    const int e = m.z + (k << 5) + lane;
    const double a = fabs(vals[e]);
    wf[e] = (float)(a / di);
    wb[e] = (float)(a / fabs(diag[cols[e]]));
  }
}

// sum_k w[e_k] X[j_k][lane] over the entries e_k = base + 32 k (k < width)
// of one row, in stored order, with the loads of four entries in flight
__device__ __forceinline__ float gather_row(const int* __restrict__ cols, const float* __restrict__ w, int base,
                                            int width, const float* __restrict__ X, int lane, float acc) {
  int k = 0;
  for (; k + 4 <= width; k += 4) {
    int j[4];
    float wk[4], x[4];
#pragma unroll
    for (int q = 0; q < 4; q++) {
      j[q] = cols[base + ((k + q) << 5)];
      wk[q] = w[base + ((k + q) << 5)];
    }
#pragma unroll
    for (int q = 0; q < 4; q++) x[q] = X[(size_t)j[q] * 32 + lane];
#pragma unroll
    for (int q = 0; q < 4; q++) acc = __fmaf_rn(wk[q], x[q], acc);
  }
  for (; k < width; k++) {
    const int e = base + (k << 5);
    acc = __fmaf_rn(w[e], X[(size_t)cols[e] * 32 + lane], acc);
  }
  return acc;
}

// h_out = relu(Ws h + Wm m + b), m_i = sum_j w_ij h_j
__global__ void __launch_bounds__(kBlock) k_layer(int n, GraphArgs g, const float* __restrict__ P,
                                                  const float* __restrict__ Hin, float* __restrict__ Hout,
                                                  float* __restrict__ Mout) {
  __shared__ float sWsT[32 * 32], sWmT[32 * 32], sb[32];
  for (int t = threadIdx.x; t < 1024; t += blockDim.x) {
    const int c = t >> 5, k = t & 31;
    sWsT[k * 32 + c] = P[t];
    sWmT[k * 32 + c] = P[1024 + t];
  }
  if (threadIdx.x < 32) sb[threadIdx.x] = P[2048 + threadIdx.x];
  __syncthreads();
  const int lane = threadIdx.x & 31;
  const int nw = (gridDim.x * blockDim.x) >> 5;
  for (int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < n; i += nw) {
    const int4 m = g.meta[g.rowSlice[i]];
    const float msg = gather_row(g.cols, g.wf, m.z + (i - m.x), m.w, Hin, lane, 0.f);
    const float h = Hin[(size_t)i * 32 + lane];
    float z = sb[lane];
#pragma unroll
    for (int k = 0; k < 32; k++) {
      z = __fmaf_rn(sWsT[k * 32 + lane], __shfl_sync(kFull, h, k), z);
      z = __fmaf_rn(sWmT[k * 32 + lane], __shfl_sync(kFull, msg, k), z);
    }
    Hout[(size_t)i * 32 + lane] = relu(z);
    if (Mout) Mout[(size_t)i * 32 + lane] = msg;
  }
}

// ---- dense layers on the tensor cores (tcgen05, kind tf32) ------------------
//
// A tile is 128 nodes (the MMA's M). Operands are staged in shared memory in
// the no-swizzle K-major layout: element (row r, k) of a K-wide operand at
// float offset (r/8)*8K + (k/4)*32 + (r%8)*4 + k%4, i.e. 8 x 4 core
// matrices of 128 bytes, K-adjacent ones 128 B apart (LBO) and 8-row groups
// 32K bytes apart (SBO). The FP32 accumulator lives in TMEM (lane = row,
// column = output) and is read back with tcgen05.ld for the epilogue. The
// MMA reads its operands as TF32 (10-bit mantissa); sums are FP32.

constexpr int kTcRows = 128;
constexpr int kTcThreads = 256;
constexpr uint32_t kTcWaitLimit = 1u << 22;  // tries of the completion wait before the kernel gives up

__device__ __forceinline__ int kmajor(int r, int k, int K) {
  return (r >> 3) * (K << 3) + ((k >> 2) << 5) + ((r & 7) << 2) + (k & 3);
}

// The same layer as k_layer: the message gather on the CUDA cores (warp per
// node, FP32, same order), then [h_i, m_i] (128 x 64) times [Ws Wm]^T (64 x
// 32) as 8 MMAs of K = 8 into TMEM, bias + ReLU in the epilogue. status
// gets 1 if a completion wait runs out (outputs of that tile not written).
__global__ void __launch_bounds__(kTcThreads, 4) k_layer_tc(int n, GraphArgs g, const float* __restrict__ P,
                                                            const float* __restrict__ Hin, float* __restrict__ Hout,
                                                            float* __restrict__ Mout, int* status) {
  __shared__ __align__(128) float sA[kTcRows * 64];
  __shared__ __align__(128) float sB[32 * 64];
  __shared__ float sBias[32];
  __shared__ __align__(8) uint64_t bar;
  __shared__ uint32_t sTmem;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  // B = [Ws Wm]: row = output channel, K = the 64 inputs (h then m)
  for (int t = threadIdx.x; t < 2048; t += blockDim.x) {
    const int o = t >> 6, k = t & 63;
    sB[kmajor(o, k, 64)] = k < 32 ? P[o * 32 + k] : P[1024 + o * 32 + (k - 32)];
  }
  if (threadIdx.x < 32) sBias[threadIdx.x] = P[2048 + threadIdx.x];
  if (warp == 0) umma::tmem_alloc(&sTmem, 32);
  if (threadIdx.x == 32) umma::mbar_init(&bar, 1);
  umma::fence_smem_for_mma();
  umma::fence_before_sync();
  __syncthreads();
  umma::fence_after_sync();
  const uint32_t tmem = sTmem;
  const uint32_t idesc = umma::idesc_tf32(kTcRows, 32);
  const uint32_t aBase = umma::smem_addr(sA), bBase = umma::smem_addr(sB);
  const int nTiles = (n + kTcRows - 1) / kTcRows;
  uint32_t parity = 0;
  bool pending = false;
  for (int tile = blockIdx.x; tile < nTiles; tile += gridDim.x) {
    const int row0 = tile * kTcRows;
    for (int r = warp; r < kTcRows; r += kTcThreads / 32) {
      const int i = row0 + r;
      float h = 0.f, msg = 0.f;
      if (i < n) {
        const int4 m = g.meta[g.rowSlice[i]];
        h = Hin[(size_t)i * 32 + lane];
        msg = gather_row(g.cols, g.wf, m.z + (i - m.x), m.w, Hin, lane, 0.f);
        if (Mout) Mout[(size_t)i * 32 + lane] = msg;
      }
      sA[kmajor(r, lane, 64)] = h;
      sA[kmajor(r, 32 + lane, 64)] = msg;
    }
    umma::fence_smem_for_mma();
    __syncthreads();
    if (threadIdx.x == 0) {
      umma::fence_after_sync();
#pragma unroll
      for (int s = 0; s < 8; s++)
        umma::mma_tf32(tmem, umma::smem_desc(aBase + s * 256, 128, 2048), umma::smem_desc(bBase + s * 256, 128, 2048),
                       idesc, s > 0);
      umma::commit(&bar);
    }
    pending = true;
    const bool done = __syncthreads_and(umma::mbar_wait(&bar, parity, kTcWaitLimit));
    if (!done) {
      if (threadIdx.x == 0) atomicOr(status, 1);
      break;
    }
    pending = false;
    parity ^= 1u;
    umma::fence_after_sync();
    // warp w reads TMEM lanes 32 (w % 4) .. +31 (its rows), columns 16 (w / 4) .. +15
    const int q = warp & 3, half = warp >> 2;
    float z[16];
    umma::ld16(umma::tmem_at(tmem, 32 * q, 16 * half), z);
    const int i = row0 + 32 * q + lane;
    if (i < n) {
      float4* out = reinterpret_cast<float4*>(Hout + (size_t)i * 32 + 16 * half);
#pragma unroll
      for (int c = 0; c < 4; c++) {
        const float* b = sBias + 16 * half + 4 * c;
        out[c] = make_float4(relu(z[4 * c] + b[0]), relu(z[4 * c + 1] + b[1]), relu(z[4 * c + 2] + b[2]),
                             relu(z[4 * c + 3] + b[3]));
      }
    }
    umma::fence_before_sync();
    __syncthreads();
  }
  // after a wait that ran out, give the MMAs in flight one more bounded wait
  // before their accumulator is released
  if (pending) __syncthreads_and(umma::mbar_wait(&bar, parity, kTcWaitLimit));
  umma::fence_after_sync();
  if (warp == 0) umma::tmem_free(tmem, 32);
}

// Failure path of the bounded completion wait of the tensor-core layers:
// TMEM is allocated as the layers allocate it and an mbarrier is armed, but
// no MMA commits to it, so the wait runs out after `limit` tries; the
// kernel then sets *status, releases TMEM and returns, as the layers do.
__global__ void k_tc_wait_probe(uint32_t limit, int* status) {
  __shared__ __align__(8) uint64_t bar;
  __shared__ uint32_t sTmem;
  const int warp = threadIdx.x >> 5;
  if (warp == 0) umma::tmem_alloc(&sTmem, 32);
  if (threadIdx.x == 32) umma::mbar_init(&bar, 1);
  umma::fence_before_sync();
  __syncthreads();
  umma::fence_after_sync();
  const bool done = __syncthreads_and(umma::mbar_wait(&bar, 0u, limit));
  if (!done && threadIdx.x == 0) atomicOr(status, 1);
  umma::fence_after_sync();
  if (warp == 0) umma::tmem_free(sTmem, 32);
}

__device__ __forceinline__ float warp_sum(float v) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(kFull, v, o);
  return __shfl_sync(kFull, v, 0);
}

__global__ void __launch_bounds__(kBlock) k_decode(int n, const float* __restrict__ P, const float* __restrict__ H3,
                                                   const double* __restrict__ scale, double* out) {
  const int lane = threadIdx.x & 31;
  const int nw = (gridDim.x * blockDim.x) >> 5;
  const float wd = P[kDecW + lane], bd = P[kDecB];
  const double s = scale[0];
  for (int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < n; i += nw) {
    const float y = warp_sum(wd * H3[(size_t)i * 32 + lane]) + bd;
    if (lane == 0) out[i] = s * (double)y;
  }
}

// ---- backward -----------------------------------------------------------------

// Writes this block's sums over its warps (fixed order) of nv per-warp
// values sv[warp * nv + p] into gp[blockIdx * kParams + off + p].
__device__ void block_grad_store(const float* sv, int nv, float* gp, int off) {
  __syncthreads();
  for (int p = threadIdx.x; p < nv; p += blockDim.x) {
    float s = 0.f;
    for (int w = 0; w < kWarps; w++) s += sv[w * nv + p];
    gp[(size_t)blockIdx.x * kParams + off + p] = s;
  }
}

__global__ void __launch_bounds__(kBlock) k_decode_bwd(int n, const float* __restrict__ P,
                                                       const float* __restrict__ H3, const double* __restrict__ scale,
                                                       const double* __restrict__ e, const double* __restrict__ e2,
                                                       float* __restrict__ dH3, float* gp, double* lossPartials) {
  __shared__ float sv[kWarps * 33];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int nw = (gridDim.x * blockDim.x) >> 5;
  const float wd = P[kDecW + lane], bd = P[kDecB];
  const double s = scale[0];
  const double E2 = e2[0] > 0.0 ? e2[0] : 1.0;
  float gwd = 0.f, gbd = 0.f;
  double loss = 0.0;
  for (int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < n; i += nw) {
    const float h = H3[(size_t)i * 32 + lane];
    const float y = warp_sum(wd * h) + bd;
    const double diff = s * (double)y - e[i];
    const float gy = (float)(2.0 * s * diff / E2);
    dH3[(size_t)i * 32 + lane] = gy * wd;
    gwd = __fmaf_rn(gy, h, gwd);
    gbd += gy;
    if (lane == 0) loss += diff * diff / E2;
  }
  sv[w * 33 + lane] = gwd;
  if (lane == 0) sv[w * 33 + 32] = gbd;
  block_grad_store(sv, 33, gp, kDecW);
  loss = block_sum(loss);
  if (threadIdx.x == 0) lossPartials[blockIdx.x] = loss;
}

// Decoder backward from a given gradient of the loss with respect to the
// FP64 output d = s y: gd[i] * gdScale[0] (dL/dy = s dL/dd).
__global__ void __launch_bounds__(kBlock) k_decode_bwd_grad(int n, const float* __restrict__ P,
                                                            const float* __restrict__ H3,
                                                            const double* __restrict__ scale,
                                                            const double* __restrict__ gd,
                                                            const double* __restrict__ gdScale,
                                                            float* __restrict__ dH3, float* gp) {
  __shared__ float sv[kWarps * 33];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int nw = (gridDim.x * blockDim.x) >> 5;
  const float wd = P[kDecW + lane];
  const double s = scale[0] * gdScale[0];
  float gwd = 0.f, gbd = 0.f;
  for (int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < n; i += nw) {
    const float h = H3[(size_t)i * 32 + lane];
    const float gy = (float)(s * gd[i]);
    dH3[(size_t)i * 32 + lane] = gy * wd;
    gwd = __fmaf_rn(gy, h, gwd);
    gbd += gy;
  }
  sv[w * 33 + lane] = gwd;
  if (lane == 0) sv[w * 33 + 32] = gbd;
  block_grad_store(sv, 33, gp, kDecW);
}

// t = r + q in place of q, with block partials of t.t and r.r
__global__ void k_residual_loss(int n, const double* __restrict__ r, double* q, double* partials) {
  double a = 0.0, b = 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const double ri = r[i];
    const double t = ri + q[i];
    q[i] = t;
    a += t * t;
    b += ri * ri;
  }
  a = block_sum(a);
  b = block_sum(b);
  if (threadIdx.x == 0) {
    partials[2 * blockIdx.x] = a;
    partials[2 * blockIdx.x + 1] = b;
  }
}

// loss = sum t.t / sum r.r; gscale = 2 / sum r.r
__global__ void k_residual_loss_finish(int np, const double* __restrict__ partials, double* loss, double* gscale) {
  double a = 0.0, b = 0.0;
  for (int k = threadIdx.x; k < np; k += blockDim.x) {
    a += partials[2 * k];
    b += partials[2 * k + 1];
  }
  a = block_sum(a);
  b = block_sum(b);
  if (threadIdx.x == 0) {
    const double r2 = b > 0.0 ? b : 1.0;
    loss[0] = a / r2;
    gscale[0] = 2.0 / r2;
  }
}

// dz = dHout * [Hout > 0]; dS = Ws^T dz; dM = Wm^T dz; gradients of Ws, Wm, b
__global__ void __launch_bounds__(kBlock) k_layer_bwd_a(int n, const float* __restrict__ P,
                                                        const float* __restrict__ Hin, const float* __restrict__ Hout,
                                                        const float* __restrict__ Min, const float* __restrict__ dHout,
                                                        float* __restrict__ dS, float* __restrict__ dM, float* gp,
                                                        int off) {
  extern __shared__ float sv[];  // kWarps * kLayerSize (per-warp gradient sums)
  __shared__ float sWs[1024], sWm[1024];
  for (int t = threadIdx.x; t < 1024; t += blockDim.x) {
    sWs[t] = P[t];
    sWm[t] = P[1024 + t];
  }
  __syncthreads();
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int nw = (gridDim.x * blockDim.x) >> 5;
  float gWs[32], gWm[32], gb = 0.f;
#pragma unroll
  for (int k = 0; k < 32; k++) gWs[k] = gWm[k] = 0.f;
  for (int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < n; i += nw) {
    const size_t o = (size_t)i * 32 + lane;
    const float dz = Hout[o] > 0.f ? dHout[o] : 0.f;
    const float h = Hin[o], m = Min[o];
    float ds = 0.f, dm = 0.f;
#pragma unroll
    for (int c = 0; c < 32; c++) {
      const float dzc = __shfl_sync(kFull, dz, c);
      ds = __fmaf_rn(sWs[c * 32 + lane], dzc, ds);
      dm = __fmaf_rn(sWm[c * 32 + lane], dzc, dm);
    }
    dS[o] = ds;
    dM[o] = dm;
#pragma unroll
    for (int k = 0; k < 32; k++) {
      gWs[k] = __fmaf_rn(dz, __shfl_sync(kFull, h, k), gWs[k]);
      gWm[k] = __fmaf_rn(dz, __shfl_sync(kFull, m, k), gWm[k]);
    }
    gb += dz;
  }
  float* mine = sv + w * kLayerSize;
#pragma unroll
  for (int k = 0; k < 32; k++) {
    mine[lane * 32 + k] = gWs[k];
    mine[1024 + lane * 32 + k] = gWm[k];
  }
  mine[2048 + lane] = gb;
  block_grad_store(sv, kLayerSize, gp, off);
}

// dHin_i = dS_i + sum_j w_ji dM_j (w_ji = |a_ji| / |a_jj|; symmetric couplings)
__global__ void __launch_bounds__(kBlock) k_layer_bwd_b(int n, GraphArgs g, const float* __restrict__ dS,
                                                        const float* __restrict__ dM, float* __restrict__ dHin) {
  const int lane = threadIdx.x & 31;
  const int nw = (gridDim.x * blockDim.x) >> 5;
  for (int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < n; i += nw) {
    const int4 m = g.meta[g.rowSlice[i]];
    const float acc = gather_row(g.cols, g.wb, m.z + (i - m.x), m.w, dM, lane, dS[(size_t)i * 32 + lane]);
    dHin[(size_t)i * 32 + lane] = acc;
  }
}

// k_layer_bwd_a on the tensor cores. Per 128-node tile:
//   [dS dM] (128 x 64) = dz (128 x 32) [Ws Wm]            4 MMAs, K = 8 channels each
//   G (128 x 32)      += [h m 1 0]^T (128 x 128 nodes) dz 16 MMAs, K = 8 nodes each
// G accumulates in TMEM over all tiles of the CTA: row f < 32 is the
// gradient of Ws[., f], 32 <= f < 64 of Wm[., f - 32], row 64 (the constant
// 1 feature) of the bias; rows 65..127 multiply zeros. Every operand is
// staged K-major, so the products that contract over nodes get transposed
// copies: XT (128 features x 128 nodes), Z (128 nodes x 32 channels), ZT
// (32 channels x 128 nodes), W^T (64 inputs x 32 channels).
constexpr int kBwdSmem = (128 * kTcRows + kTcRows * 32 + 32 * kTcRows + 64 * 32) * (int)sizeof(float);

__global__ void __launch_bounds__(kTcThreads, 2) k_layer_bwd_tc(int n, const float* __restrict__ P,
                                                                const float* __restrict__ Hin,
                                                                const float* __restrict__ Hout,
                                                                const float* __restrict__ Min,
                                                                const float* __restrict__ dHout,
                                                                float* __restrict__ dS, float* __restrict__ dM,
                                                                float* gp, int off, int* status) {
  extern __shared__ __align__(1024) float smem[];
  float* sXT = smem;                // 128 x 128
  float* sZ = sXT + 128 * kTcRows;  // 128 x 32
  float* sZT = sZ + kTcRows * 32;   // 32 x 128
  float* sW = sZT + 32 * kTcRows;   // 64 x 32
  __shared__ __align__(8) uint64_t bar;
  __shared__ uint32_t sTmem;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int t = threadIdx.x; t < 2048; t += blockDim.x) {
    const int f = t >> 5, c = t & 31;  // W^T[f][c] = Ws[c][f] or Wm[c][f - 32]
    sW[kmajor(f, c, 32)] = f < 32 ? P[c * 32 + f] : P[1024 + c * 32 + (f - 32)];
  }
  for (int t = threadIdx.x; t < 64 * kTcRows; t += blockDim.x) {
    const int f = 64 + (t >> 7), r = t & 127;
    sXT[kmajor(f, r, kTcRows)] = f == 64 ? 1.f : 0.f;
  }
  if (warp == 0) umma::tmem_alloc(&sTmem, 128);
  if (threadIdx.x == 32) umma::mbar_init(&bar, 1);
  umma::fence_smem_for_mma();
  umma::fence_before_sync();
  __syncthreads();
  umma::fence_after_sync();
  const uint32_t tmem = sTmem;  // columns 0..63: [dS dM]; 64..95: G
  const uint32_t idescD = umma::idesc_tf32(kTcRows, 64);
  const uint32_t idescG = umma::idesc_tf32(128, 32);
  const uint32_t xtBase = umma::smem_addr(sXT), zBase = umma::smem_addr(sZ), ztBase = umma::smem_addr(sZT),
                 wBase = umma::smem_addr(sW);
  const int nTiles = (n + kTcRows - 1) / kTcRows;
  uint32_t parity = 0;
  bool pending = false, any = false, failed = false;
  for (int tile = blockIdx.x; tile < nTiles; tile += gridDim.x) {
    const int row0 = tile * kTcRows;
    for (int r = warp; r < kTcRows; r += kTcThreads / 32) {
      const int i = row0 + r;
      float dz = 0.f, h = 0.f, m = 0.f;
      if (i < n) {
        const size_t o = (size_t)i * 32 + lane;
        dz = Hout[o] > 0.f ? dHout[o] : 0.f;
        h = Hin[o];
        m = Min[o];
      }
      sZ[kmajor(r, lane, 32)] = dz;
      sZT[kmajor(lane, r, kTcRows)] = dz;
      sXT[kmajor(lane, r, kTcRows)] = h;
      sXT[kmajor(32 + lane, r, kTcRows)] = m;
    }
    umma::fence_smem_for_mma();
    __syncthreads();
    if (threadIdx.x == 0) {
      umma::fence_after_sync();
#pragma unroll
      for (int s = 0; s < 4; s++)
        umma::mma_tf32(tmem, umma::smem_desc(zBase + s * 256, 128, 1024), umma::smem_desc(wBase + s * 256, 128, 1024),
                       idescD, s > 0);
#pragma unroll
      for (int s = 0; s < 16; s++)
        umma::mma_tf32(tmem + 64, umma::smem_desc(xtBase + s * 256, 128, 4096),
                       umma::smem_desc(ztBase + s * 256, 128, 4096), idescG, any || s > 0);
      umma::commit(&bar);
    }
    pending = true;
    any = true;
    const bool done = __syncthreads_and(umma::mbar_wait(&bar, parity, kTcWaitLimit));
    if (!done) {
      failed = true;
      break;
    }
    pending = false;
    parity ^= 1u;
    umma::fence_after_sync();
    // warp w: rows 32 (w % 4) .., columns 32 (w / 4) ..: dS for w < 4, dM for w >= 4
    const int q = warp & 3, half = warp >> 2;
    float v[16];
    const int i = row0 + 32 * q + lane;
    float* dst = (half ? dM : dS) + (size_t)i * 32;
#pragma unroll
    for (int p = 0; p < 2; p++) {
      umma::ld16(umma::tmem_at(tmem, 32 * q, 32 * half + 16 * p), v);
      if (i < n) {
        float4* o4 = reinterpret_cast<float4*>(dst + 16 * p);
#pragma unroll
        for (int c = 0; c < 4; c++) o4[c] = make_float4(v[4 * c], v[4 * c + 1], v[4 * c + 2], v[4 * c + 3]);
      }
    }
    umma::fence_before_sync();
    __syncthreads();
  }
  if (pending) __syncthreads_and(umma::mbar_wait(&bar, parity, kTcWaitLimit));
  umma::fence_after_sync();
  // gradient partials of this CTA: warps 0..3 hold features 32 w + lane
  float* gb = gp + (size_t)blockIdx.x * kParams + off;
  if (warp < 4) {
    const int f = 32 * warp + lane;
    float v[16];
#pragma unroll
    for (int p = 0; p < 2; p++) {
      if (any && !failed) {
        umma::ld16(umma::tmem_at(tmem, 32 * warp, 64 + 16 * p), v);
      } else {
#pragma unroll
        for (int c = 0; c < 16; c++) v[c] = 0.f;
      }
#pragma unroll
      for (int c = 0; c < 16; c++) {
        const int ch = 16 * p + c;
        if (f < 32) gb[ch * 32 + f] = v[c];
        else if (f < 64) gb[1024 + ch * 32 + (f - 32)] = v[c];
        else if (f == 64) gb[2048 + ch] = v[c];
      }
    }
  }
  if (failed && threadIdx.x == 0) atomicOr(status, 1);
  umma::fence_before_sync();
  __syncthreads();
  umma::fence_after_sync();
  if (warp == 0) umma::tmem_free(tmem, 128);
}

__global__ void __launch_bounds__(kBlock) k_encode_bwd(int n, const float* __restrict__ u, const float* __restrict__ H0,
                                                       const float* __restrict__ dH0, float* gp) {
  __shared__ float sv[kWarps * 64];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int nw = (gridDim.x * blockDim.x) >> 5;
  float gw = 0.f, gb = 0.f;
  for (int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < n; i += nw) {
    const size_t o = (size_t)i * 32 + lane;
    const float dz = H0[o] > 0.f ? dH0[o] : 0.f;
    gw = __fmaf_rn(dz, u[i], gw);
    gb += dz;
  }
  sv[w * 64 + lane] = gw;
  sv[w * 64 + 32 + lane] = gb;
  block_grad_store(sv, 64, gp, kEncW);
}

__global__ void k_grad_reduce(int nBlocks, const float* __restrict__ gp, float* grad) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= kParams) return;
  float s = 0.f;
  for (int b = 0; b < nBlocks; b++) s += gp[(size_t)b * kParams + p];
  grad[p] = s;
}

__global__ void k_adam(float* P, const float* __restrict__ g, float* m, float* v, float lr, float c1, float c2) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= kParams) return;
  const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
  const float gp = g[p];
  const float mp = b1 * m[p] + (1.f - b1) * gp;
  const float vp = b2 * v[p] + (1.f - b2) * gp * gp;
  m[p] = mp;
  v[p] = vp;
  P[p] -= lr * (mp / c1) / (sqrtf(vp / c2) + eps);
}

GraphArgs args(const Graph& g, const Workspace& w) {
  return {g.a.cols, g.a.vals, g.a.diag, g.a.meta, g.rowSlice, w.wf, w.wb};
}

void check(cudaError_t e, const char* what) {
  if (e != cudaSuccess) throw Error(kDeviceError, std::string(what) + ": " + cudaGetErrorString(e));
}

constexpr int kReduceBlocks = 592;

// persistent grid of the forward tensor-core layer: up to 4 CTAs per SM
int tc_blocks(int n) {
  const int t = ceil_div(n, kTcRows);
  return t < 148 * 4 ? (t < 1 ? 1 : t) : 148 * 4;
}

void run_forward(const Graph& g, const float* P, const double* r, Workspace& w, double* scal, bool keepMessages,
                 cudaStream_t st) {
  const int n = w.n;
  k_scale_partials<<<kReduceBlocks, kBlock, 0, st>>>(n, r, g.a.diag, w.partials);
  dev::sum_partials(kReduceBlocks, w.partials, scal + 1, st);
  k_input<<<ceil_div(n, kBlock), kBlock, 0, st>>>(n, r, g.a.diag, scal + 1, w.u, scal);
  k_encode<<<ceil_div((long long)n * 32, kBlock), kBlock, 0, st>>>(n, w.u, P, w.H[0]);
  FVM_REQUIRE(g.entries > 0 && g.entries <= w.wcap, kBadArgument,
              "learned correction: workspace not prepared for this graph's entries");
  k_edge_weights<<<ceil_div((long long)g.nSlices * 32, kBlock), kBlock, 0, st>>>(g.nSlices, g.a.meta, g.a.cols,
                                                                               g.a.vals, g.a.diag, w.wf, w.wb);
  const GraphArgs ga = args(g, w);
  for (int l = 0; l < kLayers; l++) {
    const float* Pl = P + kLayer0 + l * kLayerSize;
    float* Ml = keepMessages ? w.M[l] : nullptr;
    if (w.tensorCores)
      k_layer_tc<<<tc_blocks(n), kTcThreads, 0, st>>>(n, ga, Pl, w.H[l], w.H[l + 1], Ml, w.status);
    else
      k_layer<<<node_blocks(n), kBlock, 0, st>>>(n, ga, Pl, w.H[l], w.H[l + 1], Ml);
  }
}

}  // namespace

void Workspace::allocate(int n_, bool training, long long entries) {
  if (!(n_ <= cap && (!training || M[0]))) {
    release();
    n = cap = n_;
    const size_t hb = sizeof(float) * (size_t)n * 32;
    check(cudaMalloc(&u, sizeof(float) * (size_t)n), "cudaMalloc");
    for (int l = 0; l <= kLayers; l++) check(cudaMalloc(&H[l], hb), "cudaMalloc");
    check(cudaMalloc(&partials, sizeof(double) * (kReduceBlocks + 8)), "cudaMalloc");
    check(cudaMalloc(&status, sizeof(int)), "cudaMalloc");
    check(cudaMemset(status, 0, sizeof(int)), "cudaMemset");
    if (training) {
      for (int l = 0; l < kLayers; l++) check(cudaMalloc(&M[l], hb), "cudaMalloc");
      check(cudaMalloc(&dA, hb), "cudaMalloc");
      check(cudaMalloc(&dB, hb), "cudaMalloc");
      check(cudaMalloc(&dS, hb), "cudaMalloc");
      gradBlocks = kGradBlocks;
      check(cudaMalloc(&gradPartials, sizeof(float) * (size_t)kGradBlocks * kParams), "cudaMalloc");
      check(cudaMalloc(&dv, 2 * sizeof(double) * (size_t)n), "cudaMalloc");
    }
  }
  n = n_;
  if (entries > wcap) {
    cudaFree(wf);
    cudaFree(wb);
    wf = wb = nullptr;
    wcap = 0;
    check(cudaMalloc(&wf, sizeof(float) * (size_t)entries), "cudaMalloc");
    check(cudaMalloc(&wb, sizeof(float) * (size_t)entries), "cudaMalloc");
    wcap = entries;
  }
}

void Workspace::release() {
  cudaFree(u);
  for (auto& h : H) cudaFree(h);
  for (auto& m : M) cudaFree(m);
  cudaFree(dA);
  cudaFree(dB);
  cudaFree(dS);
  cudaFree(partials);
  cudaFree(gradPartials);
  cudaFree(status);
  cudaFree(wf);
  cudaFree(wb);
  wf = wb = nullptr;
  wcap = 0;
  u = dA = dB = dS = gradPartials = nullptr;
  partials = nullptr;
  status = nullptr;
  for (auto& h : H) h = nullptr;
  for (auto& m : M) m = nullptr;
  n = cap = 0;
  cudaFree(dv);
  dv = nullptr;
}

void Workspace::checkStatus() {
  if (!status) return;
  int h = 0;
  check(cudaMemcpy(&h, status, sizeof(int), cudaMemcpyDeviceToHost), "status copy");
  if (h) {
    check(cudaMemset(status, 0, sizeof(int)), "cudaMemset");
    throw Error(kDeviceError, "learned correction: a tensor-core completion wait ran out");
  }
}

void forward(const Graph& g, const float* params, const double* r, double* out, Workspace& w, double* scal,
             cudaStream_t st) {
  run_forward(g, params, r, w, scal, false, st);
  k_decode<<<node_blocks(w.n), kBlock, 0, st>>>(w.n, params, w.H[kLayers], scal, out);
}

void forward_backward(const Graph& g, const float* P, const double* r, const double* e, float* grad, double* loss,
                      Workspace& w, double* scal, cudaStream_t st) {
  const int n = w.n;
  run_forward(g, P, r, w, scal, true, st);
  k_sq_partials<<<kReduceBlocks, kBlock, 0, st>>>(n, e, w.partials);
  dev::sum_partials(kReduceBlocks, w.partials, scal + 2, st);
  k_decode_bwd<<<kGradBlocks, kBlock, 0, st>>>(n, P, w.H[kLayers], scal, e, scal + 2, w.dA, w.gradPartials,
                                               w.partials);
  dev::sum_partials(kGradBlocks, w.partials, loss, st);
  const GraphArgs ga = args(g, w);
  const size_t smem = sizeof(float) * kWarps * kLayerSize;
  check(cudaFuncSetAttribute(k_layer_bwd_a, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem),
        "k_layer_bwd_a shared memory");
  check(cudaFuncSetAttribute(k_layer_bwd_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, kBwdSmem),
        "k_layer_bwd_tc shared memory");
  for (int l = kLayers - 1; l >= 0; l--) {
    const int off = kLayer0 + l * kLayerSize;
    if (w.tensorCores)
      k_layer_bwd_tc<<<kGradBlocks, kTcThreads, kBwdSmem, st>>>(n, P + off, w.H[l], w.H[l + 1], w.M[l], w.dA, w.dS,
                                                                 w.dB, w.gradPartials, off, w.status);
    else
      k_layer_bwd_a<<<kGradBlocks, kBlock, smem, st>>>(n, P + off, w.H[l], w.H[l + 1], w.M[l], w.dA, w.dS, w.dB,
                                                       w.gradPartials, off);
    check(cudaGetLastError(), "layer backward launch");
    k_layer_bwd_b<<<node_blocks(n), kBlock, 0, st>>>(n, ga, w.dS, w.dB, w.dA);
  }
  k_encode_bwd<<<kGradBlocks, kBlock, 0, st>>>(n, w.u, w.H[0], w.dA, w.gradPartials);
  k_grad_reduce<<<ceil_div(kParams, kBlock), kBlock, 0, st>>>(kGradBlocks, w.gradPartials, grad);
}

void forward_backward_residual(const Graph& g, const float* P, const double* r, float* grad, double* loss,
                               Workspace& w, double* scal, cudaStream_t st) {
  const int n = w.n;
  double* d = w.dv;
  double* t = w.dv + n;
  run_forward(g, P, r, w, scal, true, st);
  k_decode<<<node_blocks(n), kBlock, 0, st>>>(n, P, w.H[kLayers], scal, d);
  dev::spmv(g.a, g.nSlices, d, t, st);  // t = A d
  k_residual_loss<<<kReduceBlocks, kBlock, 0, st>>>(n, r, t, w.partials);  // t = r + A d
  k_residual_loss_finish<<<1, kBlock, 0, st>>>(kReduceBlocks, w.partials, loss, scal + 3);
  dev::spmv(g.a, g.nSlices, t, d, st);  // d = A (r + A d): dL/dd / (2 / |r|^2)
  k_decode_bwd_grad<<<kGradBlocks, kBlock, 0, st>>>(n, P, w.H[kLayers], scal, d, scal + 3, w.dA, w.gradPartials);
  const GraphArgs ga = args(g, w);
  const size_t smem = sizeof(float) * kWarps * kLayerSize;
  check(cudaFuncSetAttribute(k_layer_bwd_a, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem),
        "k_layer_bwd_a shared memory");
  check(cudaFuncSetAttribute(k_layer_bwd_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, kBwdSmem),
        "k_layer_bwd_tc shared memory");
  for (int l = kLayers - 1; l >= 0; l--) {
    const int off = kLayer0 + l * kLayerSize;
    if (w.tensorCores)
      k_layer_bwd_tc<<<kGradBlocks, kTcThreads, kBwdSmem, st>>>(n, P + off, w.H[l], w.H[l + 1], w.M[l], w.dA, w.dS,
                                                                 w.dB, w.gradPartials, off, w.status);
    else
      k_layer_bwd_a<<<kGradBlocks, kBlock, smem, st>>>(n, P + off, w.H[l], w.H[l + 1], w.M[l], w.dA, w.dS, w.dB,
                                                       w.gradPartials, off);
    check(cudaGetLastError(), "layer backward launch");
    k_layer_bwd_b<<<node_blocks(n), kBlock, 0, st>>>(n, ga, w.dS, w.dB, w.dA);
  }
  k_encode_bwd<<<kGradBlocks, kBlock, 0, st>>>(n, w.u, w.H[0], w.dA, w.gradPartials);
  k_grad_reduce<<<ceil_div(kParams, kBlock), kBlock, 0, st>>>(kGradBlocks, w.gradPartials, grad);
}

int tc_wait_probe(unsigned limit) {
  int* status = nullptr;
  check(cudaMalloc(&status, sizeof(int)), "cudaMalloc");
  int h = 0;
  cudaError_t e = cudaMemset(status, 0, sizeof(int));
  if (e == cudaSuccess) {
    k_tc_wait_probe<<<1, 64>>>(limit, status);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaMemcpy(&h, status, sizeof(int), cudaMemcpyDeviceToHost);
  cudaFree(status);
  check(e, "tensor-core wait probe");
  return h;
}

void adam_step(float* params, const float* grad, float* m, float* v, float lr, int t, cudaStream_t st) {
  const float c1 = 1.f - std::pow(0.9f, (float)t);
  const float c2 = 1.f - std::pow(0.999f, (float)t);
  k_adam<<<ceil_div(kParams, kBlock), kBlock, 0, st>>>(params, grad, m, v, lr, c1, c2);
}

std::vector<float> initial_parameters(uint64_t seed) {
  // splitmix64 -> uniform(-a, a), a = sqrt(6 / fan_in)
  uint64_t x = seed * 0x9E3779B97F4A7C15ull + 0x1234567ull;
  auto next = [&]() {
    uint64_t z = (x += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    z ^= z >> 31;
    return (double)(z >> 11) / (double)(1ull << 53);
  };
  auto uni = [&](double a) { return (float)((2.0 * next() - 1.0) * a); };
  std::vector<float> p(kParams, 0.f);
  for (int c = 0; c < 32; c++) p[kEncW + c] = uni(std::sqrt(6.0));
  for (int c = 0; c < 32; c++) p[kEncB + c] = 0.1f;
  for (int l = 0; l < kLayers; l++) {
    const int o = kLayer0 + l * kLayerSize;
    for (int t = 0; t < 2048; t++) p[o + t] = uni(std::sqrt(6.0 / 64.0));
    for (int c = 0; c < 32; c++) p[o + 2048 + c] = 0.0f;
  }
  for (int c = 0; c < 32; c++) p[kDecW + c] = uni(std::sqrt(3.0 / 32.0));
  p[kDecB] = 0.f;
  return p;
}

}  // namespace nn
}  // namespace fvm

// ---------------------------------------------------------------------------
// flexible step of the solve
namespace fvm {
namespace nn {
namespace {

__global__ void k_step_alpha(const double* rq, const double* qq, double* alpha) {
  alpha[0] = qq[0] > 0.0 ? -rq[0] / qq[0] : 0.0;
}

__global__ void k_step_trial(int n, const double* __restrict__ r, const double* __restrict__ q,
                             const double* __restrict__ alpha, double* __restrict__ rt, double* partials) {
  const double a = alpha[0];
  double s = 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const double v = r[i] + a * q[i];
    rt[i] = v;
    s += fabs(v);
  }
  s = block_sum(s);
  if (threadIdx.x == 0) partials[blockIdx.x] = s;
}

__global__ void k_step_accept(int n, double* __restrict__ x, const double* __restrict__ d, double* __restrict__ r,
                              const double* __restrict__ rt, const double* __restrict__ alpha,
                              const double* __restrict__ norm, const double* __restrict__ trial,
                              double acceptFactor) {
  if (!(trial[0] < acceptFactor * norm[0])) return;
  const double a = alpha[0];
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    x[i] += a * d[i];
    r[i] = rt[i];
  }
}

__global__ void k_step_finish(double* norm, const double* trial, double* accepted, double* steps,
                              double* useful, double usefulFactor, double acceptFactor) {
  if (trial[0] < usefulFactor * norm[0]) useful[0] += 1.0;
  if (trial[0] < acceptFactor * norm[0]) {
    norm[0] = trial[0];
    accepted[0] += 1.0;
  }
  steps[0] += 1.0;
}

}  // namespace

void step_alpha(const double* rq, const double* qq, double* alpha, cudaStream_t st) {
  k_step_alpha<<<1, 1, 0, st>>>(rq, qq, alpha);
}
void step_trial(int n, const double* r, const double* q, const double* alpha, double* rt, double* partials,
                cudaStream_t st) {
  k_step_trial<<<dev::vec_blocks(n), kBlock, 0, st>>>(n, r, q, alpha, rt, partials);
}
void step_accept(int n, double* x, const double* d, double* r, const double* rt, const double* alpha,
                 const double* norm, const double* trialNorm, double acceptFactor, cudaStream_t st) {
  k_step_accept<<<dev::vec_blocks(n), kBlock, 0, st>>>(n, x, d, r, rt, alpha, norm, trialNorm, acceptFactor);
}
void step_finish(double* norm, const double* trialNorm, double* accepted, double* steps, double* useful,
                 double usefulFactor, double acceptFactor, cudaStream_t st) {
  k_step_finish<<<1, 1, 0, st>>>(norm, trialNorm, accepted, steps, useful, usefulFactor, acceptFactor);
}

}  // namespace nn

// ---------------------------------------------------------------------------
LearnedCorrection::LearnedCorrection(uint64_t seed) {
  nn::check(cudaMalloc(&dParams_, sizeof(float) * nn::kParams), "cudaMalloc");
  nn::check(cudaMalloc(&dGrad_, sizeof(float) * nn::kParams), "cudaMalloc");
  nn::check(cudaMalloc(&dM_, sizeof(float) * nn::kParams), "cudaMalloc");
  nn::check(cudaMalloc(&dV_, sizeof(float) * nn::kParams), "cudaMalloc");
  nn::check(cudaMalloc(&dScal_, sizeof(double) * 16), "cudaMalloc");
  nn::check(cudaMemset(dM_, 0, sizeof(float) * nn::kParams), "cudaMemset");
  nn::check(cudaMemset(dV_, 0, sizeof(float) * nn::kParams), "cudaMemset");
  setParams(nn::initial_parameters(seed));
}

LearnedCorrection::~LearnedCorrection() {
  for (Instance& k : inst_) {
    for (auto& pr : k.pairs) {
      cudaFree(pr.first);
      cudaFree(pr.second);
    }
    cudaFree(k.storage);
  }
  cudaFree(dParams_);
  cudaFree(dGrad_);
  cudaFree(dM_);
  cudaFree(dV_);
  cudaFree(dScal_);
}

std::vector<float> LearnedCorrection::params() const {
  std::vector<float> p(nn::kParams);
  nn::check(cudaMemcpy(p.data(), dParams_, sizeof(float) * nn::kParams, cudaMemcpyDeviceToHost), "cudaMemcpy");
  return p;
}

void LearnedCorrection::setParams(const std::vector<float>& p) {
  FVM_REQUIRE((int)p.size() == nn::kParams, kBadArgument, "learned correction: wrong parameter count");
  nn::check(cudaMemcpy(dParams_, p.data(), sizeof(float) * nn::kParams, cudaMemcpyHostToDevice), "cudaMemcpy");
  nn::check(cudaMemset(dM_, 0, sizeof(float) * nn::kParams), "cudaMemset");
  nn::check(cudaMemset(dV_, 0, sizeof(float) * nn::kParams), "cudaMemset");
  adamT_ = 0;
}

int LearnedCorrection::addInstance(const nn::Graph& g, int nEntries, cudaStream_t st) {
  Instance k;
  k.n = g.a.n;
  const size_t bCols = sizeof(int) * (size_t)nEntries, bVals = sizeof(double) * (size_t)nEntries;
  const size_t bDiag = sizeof(double) * (size_t)k.n, bMeta = sizeof(int4) * (size_t)g.nSlices;
  const size_t bRs = sizeof(int) * (size_t)k.n;
  auto al = [](size_t b) { return (b + 255) & ~size_t(255); };
  char* p = nullptr;
  nn::check(cudaMalloc((void**)&p, al(bCols) + al(bVals) + al(bDiag) + al(bMeta) + al(bRs)), "cudaMalloc");
  k.storage = p;
  int* cols = (int*)p;
  double* vals = (double*)(p + al(bCols));
  double* diag = (double*)(p + al(bCols) + al(bVals));
  int4* meta = (int4*)(p + al(bCols) + al(bVals) + al(bDiag));
  int* rs = (int*)(p + al(bCols) + al(bVals) + al(bDiag) + al(bMeta));
  nn::check(cudaMemcpyAsync(cols, g.a.cols, bCols, cudaMemcpyDeviceToDevice, st), "cudaMemcpy");
  nn::check(cudaMemcpyAsync(vals, g.a.vals, bVals, cudaMemcpyDeviceToDevice, st), "cudaMemcpy");
  nn::check(cudaMemcpyAsync(diag, g.a.diag, bDiag, cudaMemcpyDeviceToDevice, st), "cudaMemcpy");
  nn::check(cudaMemcpyAsync(meta, g.a.meta, bMeta, cudaMemcpyDeviceToDevice, st), "cudaMemcpy");
  nn::check(cudaMemcpyAsync(rs, g.rowSlice, bRs, cudaMemcpyDeviceToDevice, st), "cudaMemcpy");
  k.g = g;
  k.g.entries = nEntries;
  k.g.a.cols = cols;
  k.g.a.vals = vals;
  k.g.a.diag = diag;
  k.g.a.meta = meta;
  k.g.rowSlice = rs;
  // slice-row arrays are not used by the network kernels
  k.g.a.sliceRow = k.g.a.sliceRows = k.g.a.sliceOff = nullptr;
  inst_.push_back(k);
  return (int)inst_.size() - 1;
}

void LearnedCorrection::addPair(int k, const double* r, const double* e, cudaStream_t st) {
  FVM_REQUIRE(k >= 0 && k < (int)inst_.size(), kBadArgument, "learned correction: no such instance");
  Instance& in = inst_[k];
  const size_t b = sizeof(double) * (size_t)in.n;
  double *pr = nullptr, *pe = nullptr;
  nn::check(cudaMalloc(&pr, b), "cudaMalloc");
  nn::check(cudaMalloc(&pe, b), "cudaMalloc");
  nn::check(cudaMemcpyAsync(pr, r, b, cudaMemcpyDeviceToDevice, st), "cudaMemcpy");
  nn::check(cudaMemcpyAsync(pe, e, b, cudaMemcpyDeviceToDevice, st), "cudaMemcpy");
  in.pairs.push_back({pr, pe});
}

int LearnedCorrection::numPairs() const {
  int c = 0;
  for (const Instance& k : inst_) c += (int)k.pairs.size();
  return c;
}

void LearnedCorrection::train(int steps, float lr, uint64_t seed, double* losses, cudaStream_t st) {
  residualFactor_ = -1.0;
  const int np = numPairs();
  FVM_REQUIRE(np > 0, kBadArgument, "learned correction: no training pairs (harvest first)");
  FVM_REQUIRE(steps >= 0 && lr > 0.f, kBadArgument, "learned correction: bad training settings");
  int maxN = 0;
  std::vector<std::pair<int, int>> index;
  for (int k = 0; k < (int)inst_.size(); k++) {
    maxN = std::max(maxN, inst_[k].n);
    for (int q = 0; q < (int)inst_[k].pairs.size(); q++) index.push_back({k, q});
  }
  trainWs_.allocate(maxN, true, maxEntries());
  trainWs_.tensorCores = tensorCores_;
  double* dLoss = nullptr;
  nn::check(cudaMalloc(&dLoss, sizeof(double) * (size_t)std::max(steps, 1)), "cudaMalloc");
  uint64_t x = seed * 0x9E3779B97F4A7C15ull + 0x51ull;
  auto next = [&]() {
    uint64_t z = (x += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
  };
  for (int t = 0; t < steps; t++) {
    const auto& ix = index[next() % index.size()];
    Instance& in = inst_[ix.first];
    trainWs_.allocate(in.n, true, in.g.entries);
    if (objective_ == 1)
      nn::forward_backward_residual(in.g, dParams_, in.pairs[ix.second].first, dGrad_, dLoss + t, trainWs_, dScal_,
                                    st);
    else
      nn::forward_backward(in.g, dParams_, in.pairs[ix.second].first, in.pairs[ix.second].second, dGrad_,
                           dLoss + t, trainWs_, dScal_, st);
    nn::adam_step(dParams_, dGrad_, dM_, dV_, lr, ++adamT_, st);
  }
  if (losses && steps > 0)
    nn::check(cudaMemcpyAsync(losses, dLoss, sizeof(double) * steps, cudaMemcpyDeviceToHost, st), "cudaMemcpy");
  nn::check(cudaStreamSynchronize(st), "training");
  cudaFree(dLoss);
  trainWs_.checkStatus();
}

double LearnedCorrection::evaluate(cudaStream_t st) {
  const int np = numPairs();
  FVM_REQUIRE(np > 0, kBadArgument, "learned correction: no pairs to evaluate");
  int maxN = 0;
  for (const Instance& k : inst_) maxN = std::max(maxN, k.n);
  trainWs_.allocate(maxN, true, maxEntries());
  trainWs_.tensorCores = tensorCores_;
  double* dLoss = nullptr;
  nn::check(cudaMalloc(&dLoss, sizeof(double) * (size_t)np), "cudaMalloc");
  int q = 0;
  for (Instance& in : inst_)
    for (auto& pr : in.pairs) {
      trainWs_.allocate(in.n, true, in.g.entries);
      if (objective_ == 1)
        nn::forward_backward_residual(in.g, dParams_, pr.first, dGrad_, dLoss + q++, trainWs_, dScal_, st);
      else
        nn::forward_backward(in.g, dParams_, pr.first, pr.second, dGrad_, dLoss + q++, trainWs_, dScal_, st);
    }
  std::vector<double> l(np);
  nn::check(cudaMemcpyAsync(l.data(), dLoss, sizeof(double) * np, cudaMemcpyDeviceToHost, st), "cudaMemcpy");
  nn::check(cudaStreamSynchronize(st), "evaluation");
  cudaFree(dLoss);
  trainWs_.checkStatus();
  double s = 0.0;
  for (double v : l) s += v;
  if (objective_ == 1) residualFactor_ = std::sqrt(s / np);
  return s / np;
}

long long LearnedCorrection::maxEntries() const {
  long long e = 0;
  for (const Instance& k : inst_) e = std::max(e, k.g.entries);
  return e;
}

void LearnedCorrection::prepare(int n, long long entries) {
  applyWs_.allocate(n, false, entries);
  applyWs_.tensorCores = tensorCores_;
}

void LearnedCorrection::setUsefulFactor(double f) {
  FVM_REQUIRE(f > 0.0 && f <= 1.0, kBadArgument, "learned correction: useful factor must be in (0, 1]");
  usefulFactor_ = f;
}

void LearnedCorrection::setObjective(int o) {
  FVM_REQUIRE(o == 0 || o == 1, kBadArgument, "learned correction: objective must be 0 or 1");
  if (o != objective_) residualFactor_ = -1.0;
  objective_ = o;
}

void LearnedCorrection::setTensorCores(bool on) {
  tensorCores_ = on;
  applyWs_.tensorCores = trainWs_.tensorCores = on;
}

void LearnedCorrection::apply(const nn::Graph& g, const double* r, double* out, double* scal, cudaStream_t st) {
  FVM_REQUIRE(g.a.n <= applyWs_.cap && g.entries <= applyWs_.wcap, kBadArgument,
              "learned correction: prepare() was not called for this size");
  applyWs_.n = g.a.n;
  nn::forward(g, dParams_, r, out, applyWs_, scal, st);
}

}  // namespace fvm
