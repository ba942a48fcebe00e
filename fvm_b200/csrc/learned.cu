// Kernels of the learned correction (learned.hpp): forward, backward and
// Adam, all FP32 with fixed reduction orders (deterministic).
//
// Layout: activations node-major, h[i * 32 + c]; one warp per node, lane =
// channel, so a neighbour's activations are one coalesced 128-byte load.
// The graph is the finest level's SELL-32 matrix (neighbours j of row i:
// its stored columns, padding entries carry a zero coupling).
#include <cmath>
#include <stdexcept>

#include "common.hpp"
#include "learned.hpp"

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
};

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
    const int base = m.z + (i - m.x);
    const double di = fabs(g.diag[i]);
    float msg = 0.f;
    for (int k = 0; k < m.w; k++) {
      const int e = base + (k << 5);
      const int j = g.cols[e];
      const float w = (float)(fabs(g.vals[e]) / di);
      msg = __fmaf_rn(w, Hin[(size_t)j * 32 + lane], msg);
    }
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
    const int base = m.z + (i - m.x);
    float acc = dS[(size_t)i * 32 + lane];
    for (int k = 0; k < m.w; k++) {
      const int e = base + (k << 5);
      const int j = g.cols[e];
      const float w = (float)(fabs(g.vals[e]) / fabs(g.diag[j]));
      acc = __fmaf_rn(w, dM[(size_t)j * 32 + lane], acc);
    }
    dHin[(size_t)i * 32 + lane] = acc;
  }
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

GraphArgs args(const Graph& g) { return {g.a.cols, g.a.vals, g.a.diag, g.a.meta, g.rowSlice}; }

void check(cudaError_t e, const char* what) {
  if (e != cudaSuccess) throw Error(kDeviceError, std::string(what) + ": " + cudaGetErrorString(e));
}

constexpr int kReduceBlocks = 592;

void run_forward(const Graph& g, const float* P, const double* r, Workspace& w, double* scal, bool keepMessages,
                 cudaStream_t st) {
  const int n = w.n;
  k_scale_partials<<<kReduceBlocks, kBlock, 0, st>>>(n, r, g.a.diag, w.partials);
  dev::sum_partials(kReduceBlocks, w.partials, scal + 1, st);
  k_input<<<ceil_div(n, kBlock), kBlock, 0, st>>>(n, r, g.a.diag, scal + 1, w.u, scal);
  k_encode<<<ceil_div((long long)n * 32, kBlock), kBlock, 0, st>>>(n, w.u, P, w.H[0]);
  const GraphArgs ga = args(g);
  for (int l = 0; l < kLayers; l++)
    k_layer<<<node_blocks(n), kBlock, 0, st>>>(n, ga, P + kLayer0 + l * kLayerSize, w.H[l], w.H[l + 1],
                                               keepMessages ? w.M[l] : nullptr);
}

}  // namespace

void Workspace::allocate(int n_, bool training) {
  if (n_ <= cap && (!training || M[0])) {
    n = n_;
    return;
  }
  release();
  n = cap = n_;
  const size_t hb = sizeof(float) * (size_t)n * 32;
  check(cudaMalloc(&u, sizeof(float) * (size_t)n), "cudaMalloc");
  for (int l = 0; l <= kLayers; l++) check(cudaMalloc(&H[l], hb), "cudaMalloc");
  check(cudaMalloc(&partials, sizeof(double) * (kReduceBlocks + 8)), "cudaMalloc");
  if (training) {
    for (int l = 0; l < kLayers; l++) check(cudaMalloc(&M[l], hb), "cudaMalloc");
    check(cudaMalloc(&dA, hb), "cudaMalloc");
    check(cudaMalloc(&dB, hb), "cudaMalloc");
    check(cudaMalloc(&dS, hb), "cudaMalloc");
    gradBlocks = kGradBlocks;
    check(cudaMalloc(&gradPartials, sizeof(float) * (size_t)kGradBlocks * kParams), "cudaMalloc");
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
  u = dA = dB = dS = gradPartials = nullptr;
  partials = nullptr;
  for (auto& h : H) h = nullptr;
  for (auto& m : M) m = nullptr;
  n = cap = 0;
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
  const GraphArgs ga = args(g);
  const size_t smem = sizeof(float) * kWarps * kLayerSize;
  cudaFuncSetAttribute(k_layer_bwd_a, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  for (int l = kLayers - 1; l >= 0; l--) {
    const int off = kLayer0 + l * kLayerSize;
    k_layer_bwd_a<<<kGradBlocks, kBlock, smem, st>>>(n, P + off, w.H[l], w.H[l + 1], w.M[l], w.dA, w.dS, w.dB,
                                                     w.gradPartials, off);
    k_layer_bwd_b<<<node_blocks(n), kBlock, 0, st>>>(n, ga, w.dS, w.dB, w.dA);
  }
  k_encode_bwd<<<kGradBlocks, kBlock, 0, st>>>(n, w.u, w.H[0], w.dA, w.gradPartials);
  k_grad_reduce<<<ceil_div(kParams, kBlock), kBlock, 0, st>>>(kGradBlocks, w.gradPartials, grad);
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
                              const double* __restrict__ norm, const double* __restrict__ trial) {
  if (!(trial[0] < norm[0])) return;
  const double a = alpha[0];
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    x[i] += a * d[i];
    r[i] = rt[i];
  }
}

__global__ void k_step_finish(double* norm, const double* trial, double* accepted, double* steps,
                              double* useful, double usefulFactor) {
  if (trial[0] < usefulFactor * norm[0]) useful[0] += 1.0;
  if (trial[0] < norm[0]) {
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
                 const double* norm, const double* trialNorm, cudaStream_t st) {
  k_step_accept<<<dev::vec_blocks(n), kBlock, 0, st>>>(n, x, d, r, rt, alpha, norm, trialNorm);
}
void step_finish(double* norm, const double* trialNorm, double* accepted, double* steps, double* useful,
                 double usefulFactor, cudaStream_t st) {
  k_step_finish<<<1, 1, 0, st>>>(norm, trialNorm, accepted, steps, useful, usefulFactor);
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
  const int np = numPairs();
  FVM_REQUIRE(np > 0, kBadArgument, "learned correction: no training pairs (harvest first)");
  FVM_REQUIRE(steps >= 0 && lr > 0.f, kBadArgument, "learned correction: bad training settings");
  int maxN = 0;
  std::vector<std::pair<int, int>> index;
  for (int k = 0; k < (int)inst_.size(); k++) {
    maxN = std::max(maxN, inst_[k].n);
    for (int q = 0; q < (int)inst_[k].pairs.size(); q++) index.push_back({k, q});
  }
  trainWs_.allocate(maxN, true);
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
    trainWs_.allocate(in.n, true);
    nn::forward_backward(in.g, dParams_, in.pairs[ix.second].first, in.pairs[ix.second].second, dGrad_,
                         dLoss + t, trainWs_, dScal_, st);
    nn::adam_step(dParams_, dGrad_, dM_, dV_, lr, ++adamT_, st);
  }
  if (losses && steps > 0)
    nn::check(cudaMemcpyAsync(losses, dLoss, sizeof(double) * steps, cudaMemcpyDeviceToHost, st), "cudaMemcpy");
  nn::check(cudaStreamSynchronize(st), "training");
  cudaFree(dLoss);
}

double LearnedCorrection::evaluate(cudaStream_t st) {
  const int np = numPairs();
  FVM_REQUIRE(np > 0, kBadArgument, "learned correction: no pairs to evaluate");
  int maxN = 0;
  for (const Instance& k : inst_) maxN = std::max(maxN, k.n);
  trainWs_.allocate(maxN, true);
  double* dLoss = nullptr;
  nn::check(cudaMalloc(&dLoss, sizeof(double) * (size_t)np), "cudaMalloc");
  int q = 0;
  for (Instance& in : inst_)
    for (auto& pr : in.pairs) {
      trainWs_.allocate(in.n, true);
      nn::forward_backward(in.g, dParams_, pr.first, pr.second, dGrad_, dLoss + q++, trainWs_, dScal_, st);
    }
  std::vector<double> l(np);
  nn::check(cudaMemcpyAsync(l.data(), dLoss, sizeof(double) * np, cudaMemcpyDeviceToHost, st), "cudaMemcpy");
  nn::check(cudaStreamSynchronize(st), "evaluation");
  cudaFree(dLoss);
  double s = 0.0;
  for (double v : l) s += v;
  return s / np;
}

void LearnedCorrection::prepare(int n) { applyWs_.allocate(n, false); }

void LearnedCorrection::apply(const nn::Graph& g, const double* r, double* out, double* scal, cudaStream_t st) {
  FVM_REQUIRE(g.a.n <= applyWs_.cap, kBadArgument, "learned correction: prepare() was not called for this size");
  applyWs_.n = g.a.n;
  nn::forward(g, dParams_, r, out, applyWs_, scal, st);
}

}  // namespace fvm
