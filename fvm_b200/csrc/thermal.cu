// ThermalModel on the GPU.
#include "thermal.hpp"

#include <atomic>

#include <algorithm>
#include <chrono>
#include <functional>
#include <cmath>
#include <cstdio>

namespace fvm {

#define CUDA_OK(call)                                                                       \
  do {                                                                                      \
    cudaError_t e_ = (call);                                                                \
    if (e_ != cudaSuccess)                                                                  \
      throw ::fvm::Error(::fvm::kDeviceError, std::string(#call ": ") + cudaGetErrorString(e_)); \
  } while (0)

ThermalModel::ThermalModel(std::shared_ptr<HostMesh> mesh) : mesh_(std::move(mesh)) {
  // ThermalModel_impl.h:41-82: wall/symmetry -> SpecifiedHeatFlux,
  // velocity-inlet/pressure-outlet -> SpecifiedTemperature
  for (size_t g = 1; g < mesh_->groups.size(); g++) {
    const FaceGroup& fg = mesh_->groups[g];
    GroupBC bc;
    bc.id = fg.id;
    if (fg.type == "wall" || fg.type == "symmetry")
      bc.type = kBcSpecifiedHeatFlux;
    else if (fg.type == "velocity-inlet" || fg.type == "pressure-outlet")
      bc.type = kBcSpecifiedTemperature;
    else
      throw Error(kBadArgument, "ThermalModel: unknown face group type " + fg.type);
    bcs_.push_back(bc);
  }
}

ThermalModel::~ThermalModel() {
  releaseAdvanceGraph();
  releaseAcceleration();
  if (dOuter_) cudaFree(dOuter_);
  if (hOuter_) cudaFreeHost(hOuter_);
  solver_.reset();
  hier_.release();
  freeDevice();
  if (hPinned_) cudaFreeHost(hPinned_);
  if (dSegOff_) cudaFree(dSegOff_);
  if (dSegNorm_) cudaFree(dSegNorm_);
}

void ThermalModel::freeDevice() {
  releaseAdvanceGraph();
  arena_.release();
  dPerm_ = nullptr;  // lives in the hierarchy's arena
  if (stream_) cudaStreamDestroy(stream_);
  stream_ = nullptr;
  deviceReady_ = false;
}

GroupBC& ThermalModel::bc(int groupId) {
  for (GroupBC& b : bcs_)
    if (b.id == groupId) return b;
  throw Error(kBadArgument, "no boundary face group with id " + std::to_string(groupId));
}

namespace {
__global__ void k_fill_value(int n, double* x, double v) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) x[i] = v;
}
}  // namespace

void ThermalModel::init() {
  const int nAll = mesh_->nTotalCells();
  for (HostField* f : {&T_, &k_, &src_, &rc_, &TN1_})
    if ((int)f->size() != nAll) f->resize(nAll);
  // every field starts uniform: nothing is written on the host here
  uniform_.fill(true);
  uniformValue_[kFieldTemperature] = opt_.initialTemperature;
  uniformValue_[kFieldConductivity] = opt_.thermalConductivity;
  uniformValue_[kFieldSource] = 0.0;
  uniformValue_[kFieldSpecificHeat] = opt_.density * opt_.specificHeat;
  uniformValue_[kFieldTemperatureN1] = opt_.initialTemperature;
  tDirty_ = kDirty_ = srcDirty_ = rcDirty_ = tn1Dirty_ = true;
  matrixDirty_ = hierarchyDirty_ = true;
  initialNorm_ = -1;
  niters_ = 0;
  history_.clear();
  segFirst_.assign(numSegments(), -1.0);
  segLast_.assign(numSegments(), -1.0);
  segConvergedAt_.assign(numSegments(), -1);
  initialized_ = true;
}

void ThermalModel::setSegments(const std::vector<int>& offsets) {
  if (dSegOff_) cudaFree(dSegOff_);
  if (dSegNorm_) cudaFree(dSegNorm_);
  dSegOff_ = nullptr;
  dSegNorm_ = nullptr;
  segOff_.clear();
  if (!offsets.empty()) {
    FVM_REQUIRE(offsets.size() >= 2 && offsets.front() == 0 && offsets.back() == mesh_->nCells, kBadArgument,
                "segments: offsets must start at 0 and end at the number of cells");
    for (size_t s = 0; s + 1 < offsets.size(); s++)
      FVM_REQUIRE(offsets[s + 1] > offsets[s], kBadArgument, "segments: offsets must increase");
    segOff_ = offsets;
    CUDA_OK(cudaMalloc(&dSegOff_, sizeof(int) * segOff_.size()));
    CUDA_OK(cudaMemcpy(dSegOff_, segOff_.data(), sizeof(int) * segOff_.size(), cudaMemcpyHostToDevice));
    CUDA_OK(cudaMalloc(&dSegNorm_, sizeof(double) * (segOff_.size() - 1)));
  }
  segFirst_.assign(numSegments(), -1.0);
  segLast_.assign(numSegments(), -1.0);
  segConvergedAt_.assign(numSegments(), -1);
}

void ThermalModel::segmentStatus(std::vector<double>& first, std::vector<double>& last,
                                 std::vector<int>& convergedAt) const {
  first = segFirst_;
  last = segLast_;
  convergedAt = segConvergedAt_;
}

namespace {
// L1 norm of b over each block of cells (reference order; b is in the
// solver's permuted order), one CUDA block per segment, fixed summation order
__global__ void k_segment_l1(const int* __restrict__ off, const int* __restrict__ perm, const double* __restrict__ b,
                             double* out) {
  __shared__ double red[256];
  const int s = blockIdx.x;
  double acc = 0.0;
  for (int i = off[s] + threadIdx.x; i < off[s + 1]; i += blockDim.x) acc += fabs(b[perm[i]]);
  red[threadIdx.x] = acc;
  __syncthreads();
  for (int o = blockDim.x >> 1; o > 0; o >>= 1) {
    if ((int)threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) out[s] = red[0];
}

// Outer-loop state of advance() on the device; the outer norms follow it at
// kOuterHead bytes.
struct OuterState {
  double initialNorm;    // in: the model's first outer norm (< 0: none yet); out: as updated
  double absTol, relTol; // in: the outer tolerances
  int niter;             // in: outer iterations allowed
  int iterations;        // out: outer iterations completed
  int linearIterations;  // out: CG iterations over them
  int status;            // out: 0 running, 1 converged, 3 niter reached, 2 initial residual
                         // non-finite, 4 residual became non-finite
};
constexpr size_t kOuterHead = 64;
constexpr int kOuterHistory = 4096;  // outer norms a graph records before a longer call rebuilds it
static_assert(sizeof(OuterState) <= kOuterHead, "outer state header");

__global__ void k_outer_init(OuterState* s, cudaGraphConditionalHandle hOuter) {
  s->iterations = 0;
  s->linearIterations = 0;
  s->status = 0;
  cudaGraphSetConditional(hOuter, s->niter > 0 ? 1u : 0u);
}

// The test of the host loop of advance() on this outer iteration's linear
// system: rNorm is the L1 norm of its right-hand side (the CG's initial
// norm). A non-finite solve ends the loop before the update, as the host
// loop's exception does.
__global__ void k_outer_check(OuterState* s, double* hist, const double* cgInitialNorm, const int* cgLoop,
                              cudaGraphConditionalHandle hOuter, cudaGraphConditionalHandle hUpdate) {
  const double rNorm = cgInitialNorm[0];
  int status = 0;
  if (!isfinite(rNorm)) {
    status = 2;
  } else if (cgLoop[1] == 2) {
    status = 4;
  } else {
    const int it = s->iterations;
    hist[it] = rNorm;
    s->iterations = it + 1;
    s->linearIterations += cgLoop[0];
    if (s->initialNorm < 0) s->initialNorm = rNorm;
    const double ratio = s->initialNorm > 0 ? rNorm / s->initialNorm : 0.0;
    if (rNorm < s->absTol || ratio < s->relTol)
      status = 1;
    else if (it + 1 >= s->niter)
      status = 3;
  }
  s->status = status;
  cudaGraphSetConditional(hUpdate, status == 2 || status == 4 ? 0u : 1u);
  cudaGraphSetConditional(hOuter, status == 0 ? 1u : 0u);
}
}  // namespace

namespace {
// Anderson acceleration (type II, depth m <= kAAMax) of the outer
// fixed-point iteration x -> G(x), G = linearize at x, solve, update: with
// f_i = G(x_i) - x_i and the last mk + 1 pairs (G_i, f_i) held,
// gamma = argmin |f_k - dF gamma|_2 and x_{k+1} = G(x_k) - dG gamma, where
// the columns of dF and dG are differences of consecutive f_i and G_i
// (Walker & Ni, SIAM J. Numer. Anal. 49, 2011). x is the whole temperature
// vector, ghost cells included: a ghost's update is affine in its cell's
// (CRMatrix::solveBoundary), and the weights of the combination sum to 1.
// Three kernels: the pair store with the normal equations' partial sums,
// a one-block solve, the update. Sums in a fixed order: bitwise
// reproducible. Each returns at once when *stop is set (the outer loop has
// ended: the last plain update stays).
constexpr int kAAMax = 5;
constexpr int kAAQ = kAAMax * (kAAMax + 1) / 2 + kAAMax;  // Gram upper triangle + right-hand side
constexpr int kAABlock = 256;

struct AAState {
  int head;   // slot of the next pair
  int count;  // pairs held before this iteration's
  int cur;    // slot of this iteration's pair
  int mk;     // columns used this iteration
  double gamma[kAAMax];
};

struct AAVectors {
  double* F[kAAMax + 1];
  double* G[kAAMax + 1];
};

template <int M>
constexpr int aa_nq() {
  return M * (M + 1) / 2 + M;  // Gram upper triangle, then the right-hand side
}

// sums of acc[0..NQ) over the block in a fixed order (each warp's by
// shuffles, then the warps' sums in warp order), written to out[0..NQ) by
// threads 0..NQ-1
template <int NQ>
__device__ __forceinline__ void aa_block_sums(double (&acc)[NQ], double (*red)[NQ], double* out) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
  for (int q = 0; q < NQ; q++) {
    double v = acc[q];
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if (lane == 0) red[w][q] = v;
  }
  __syncthreads();
  if ((int)threadIdx.x < NQ) {
    double s = 0.0;
    for (int k = 0; k < kAABlock / 32; k++) s += red[k][threadIdx.x];
    out[threadIdx.x] = s;
  }
}

template <int M>
__global__ void __launch_bounds__(kAABlock) k_aa_dots(int n, const double* __restrict__ x, const double* __restrict__ xs,
                                                      AAVectors v, const AAState* st, const int* stop,
                                                      double* partials) {
  if (stop && *stop != 0) return;
  constexpr int NQ = aa_nq<M>();
  __shared__ double red[kAABlock / 32][NQ];
  const int head = st->head, mk = min(st->count, M), slots = M + 1;
  // the held pairs' f vectors, oldest first (the slot table is indexed
  // once per thread, the vectors with unrolled indices)
  const double* Fq[M + 1];
#pragma unroll
  for (int j = 0; j <= M; j++) Fq[j] = v.F[((head - mk + j) % slots + slots) % slots];
  double* const Gn = v.G[head];
  double* const Fn = v.F[head];
  double acc[NQ];
#pragma unroll
  for (int k = 0; k < NQ; k++) acc[k] = 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const double g = x[i], f = g - xs[i];
    Gn[i] = g;
    Fn[i] = f;
    double d[M];
    double prev = mk > 0 ? Fq[0][i] : 0.0;
#pragma unroll
    for (int j = 1; j <= M; j++) {
      if (j <= mk) {
        const double c = j == mk ? f : Fq[j][i];
        d[j - 1] = c - prev;
        prev = c;
      } else {
        d[j - 1] = 0.0;
      }
    }
    int k = 0;
#pragma unroll
    for (int a = 0; a < M; a++)
#pragma unroll
      for (int b = a; b < M; b++) acc[k++] += d[a] * d[b];
#pragma unroll
    for (int a = 0; a < M; a++) acc[k++] += d[a] * f;
  }
  aa_block_sums<NQ>(acc, red, partials + (size_t)blockIdx.x * NQ);
}

// Normal equations (dF^T dF) gamma = dF^T f by Cholesky; a pivot below
// 1e-12 of its diagonal entry (columns nearly dependent) restarts the
// history: this iteration takes the plain step and keeps only its own pair.
// The blocks' partials are summed by one warp per quantity, lanes striding
// over the blocks, then by shuffles: a fixed order.
template <int M>
__global__ void __launch_bounds__(kAABlock) k_aa_solve(int nb, const double* __restrict__ partials, AAState* st,
                                                       const int* stop) {
  if (stop && *stop != 0) return;
  constexpr int NQ = aa_nq<M>();
  __shared__ double tot[NQ];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  for (int q = w; q < NQ; q += kAABlock / 32) {
    double s = 0.0;
    for (int b = lane; b < nb; b += 32) s += partials[(size_t)b * NQ + q];
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    if (lane == 0) tot[q] = s;
  }
  __syncthreads();
  if (threadIdx.x != 0) return;
  const int mk = min(st->count, M);
  double H[M][M], r[M], L[M][M];
  int k = 0;
  for (int a = 0; a < M; a++)
    for (int b = a; b < M; b++) {
      H[a][b] = tot[k];
      H[b][a] = tot[k];
      k++;
    }
  for (int a = 0; a < M; a++) r[a] = tot[k++];
  bool ok = true;
  for (int a = 0; a < mk && ok; a++) {
    for (int b = 0; b <= a; b++) {
      double s = H[a][b];
      for (int c = 0; c < b; c++) s -= L[a][c] * L[b][c];
      if (a == b) {
        if (!(s > 1e-12 * H[a][a])) {
          ok = false;
          break;
        }
        L[a][a] = sqrt(s);
      } else {
        L[a][b] = s / L[b][b];
      }
    }
  }
  double y[M], gam[M];
  int used = 0;
  if (ok && mk > 0) {
    for (int a = 0; a < mk; a++) {
      double s = r[a];
      for (int c = 0; c < a; c++) s -= L[a][c] * y[c];
      y[a] = s / L[a][a];
    }
    for (int a = mk - 1; a >= 0; a--) {
      double s = y[a];
      for (int c = a + 1; c < mk; c++) s -= L[c][a] * gam[c];
      gam[a] = s / L[a][a];
    }
    used = mk;
    for (int a = 0; a < mk; a++) ok = ok && isfinite(gam[a]);
    if (!ok) used = 0;
  }
  for (int a = 0; a < kAAMax; a++) st->gamma[a] = a < used ? gam[a] : 0.0;
  st->cur = st->head;
  st->mk = used;
  st->head = (st->head + 1) % (M + 1);
  st->count = used == mk ? min(st->count + 1, M + 1) : 1;
}

template <int M>
__global__ void __launch_bounds__(kAABlock) k_aa_update(int n, double* __restrict__ x, double* __restrict__ xs,
                                                        AAVectors v, const AAState* st, const int* stop) {
  if (stop && *stop != 0) return;
  const int cur = st->cur, mk = st->mk, slots = M + 1;
  const double* Gq[M + 1];
  double gam[M];
#pragma unroll
  for (int j = 0; j <= M; j++) Gq[j] = v.G[((cur - mk + j) % slots + slots) % slots];
#pragma unroll
  for (int j = 0; j < M; j++) gam[j] = st->gamma[j];
  const double* const Gc = v.G[cur];
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const double g = Gc[i];
    double s = 0.0;
    double prev = mk > 0 ? Gq[0][i] : 0.0;
#pragma unroll
    for (int j = 1; j <= M; j++) {
      if (j <= mk) {
        const double c = j == mk ? g : Gq[j][i];
        s += gam[j - 1] * (c - prev);
        prev = c;
      }
    }
    const double xn = g - s;
    x[i] = xn;
    xs[i] = xn;
  }
}

template <int M>
void aa_step(int n, int nb, double* x, double* xs, const AAVectors& v, AAState* s, const int* stop, double* partials,
             cudaStream_t st) {
  k_aa_dots<M><<<nb, kAABlock, 0, st>>>(n, x, xs, v, s, stop, partials);
  k_aa_solve<M><<<1, kAABlock, 0, st>>>(nb, partials, s, stop);
  k_aa_update<M><<<nb, kAABlock, 0, st>>>(n, x, xs, v, s, stop);
}

__global__ void k_aa_reset(AAState* st) {
  st->head = 0;
  st->count = 0;
  st->cur = 0;
  st->mk = 0;
}

int aa_blocks(int n) {
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  return std::max(1, std::min((n + kAABlock - 1) / kAABlock, 4 * sms));
}
}  // namespace

// Buffers of the outer acceleration of depth m: (m + 1) pairs of
// temperature-sized vectors, the previous iterate, the partial sums and
// the state; allocated on first use, kept while m and the mesh stay.
void ThermalModel::ensureAcceleration(int m) {
  const int nAll = mesh_->nTotalCells();
  if (aaDepth_ == m && aaCells_ == nAll) return;
  releaseAcceleration();
  const int nb = aa_blocks(nAll);
  const size_t vec = sizeof(double) * (size_t)nAll;
  const size_t bytes = vec * (size_t)(2 * (m + 1) + 1) + sizeof(double) * (size_t)nb * kAAQ + 256;
  CUDA_OK(cudaMalloc(&dAA_, bytes));
  aaDepth_ = m;
  aaCells_ = nAll;
  aaBlocks_ = nb;
  aaGen_++;
}

void ThermalModel::releaseAcceleration() {
  if (dAA_) cudaFree(dAA_);
  dAA_ = nullptr;
  aaDepth_ = 0;
  aaCells_ = 0;
}

void ThermalModel::accelerationStart(cudaStream_t st) {
  const size_t vec = sizeof(double) * (size_t)aaCells_;
  double* xs = (double*)dAA_;
  AAState* s = (AAState*)((char*)dAA_ + vec * (size_t)(2 * (aaDepth_ + 1) + 1) +
                          sizeof(double) * (size_t)aaBlocks_ * kAAQ);
  k_aa_reset<<<1, 1, 0, st>>>(s);
  CUDA_OK(cudaGetLastError());
  CUDA_OK(cudaMemcpyAsync(xs, dT_, vec, cudaMemcpyDeviceToDevice, st));
}

void ThermalModel::accelerationStep(cudaStream_t st, const int* stop) {
  const int m = aaDepth_, n = aaCells_;
  const size_t vec = sizeof(double) * (size_t)n;
  double* base = (double*)dAA_;
  double* xs = base;
  AAVectors v{};
  for (int j = 0; j <= m; j++) {
    v.F[j] = base + (size_t)(1 + j) * n;
    v.G[j] = base + (size_t)(2 + m + j) * n;
  }
  double* partials = (double*)((char*)dAA_ + vec * (size_t)(2 * (m + 1) + 1));
  AAState* s = (AAState*)((char*)partials + sizeof(double) * (size_t)aaBlocks_ * kAAQ);
  switch (m) {
    case 1: aa_step<1>(n, aaBlocks_, dT_, xs, v, s, stop, partials, st); break;
    case 2: aa_step<2>(n, aaBlocks_, dT_, xs, v, s, stop, partials, st); break;
    case 3: aa_step<3>(n, aaBlocks_, dT_, xs, v, s, stop, partials, st); break;
    case 4: aa_step<4>(n, aaBlocks_, dT_, xs, v, s, stop, partials, st); break;
    default: aa_step<5>(n, aaBlocks_, dT_, xs, v, s, stop, partials, st); break;
  }
  CUDA_OK(cudaGetLastError());
}

void ThermalModel::releaseAdvanceGraph() {
  if (gAdvance_) cudaGraphExecDestroy(gAdvance_);
  gAdvance_ = nullptr;
}

bool ThermalModel::buildAdvanceGraph(int historyCap) {
  const auto t0 = std::chrono::steady_clock::now();
  releaseAdvanceGraph();
  if (historyCap > advHistoryCap_) {
    if (dOuter_) cudaFree(dOuter_);
    if (hOuter_) cudaFreeHost(hOuter_);
    dOuter_ = hOuter_ = nullptr;
    advHistoryCap_ = 0;
    const size_t bytes = kOuterHead + sizeof(double) * (size_t)historyCap;
    CUDA_OK(cudaMalloc(&dOuter_, bytes));
    CUDA_OK(cudaMallocHost(&hOuter_, bytes));
    advHistoryCap_ = historyCap;
  }
  OuterState* state = (OuterState*)dOuter_;
  double* hist = (double*)((char*)dOuter_ + kOuterHead);
  const dev::BoundaryData bd = boundaryData();
  const int nCells = mesh_->nCells;
  const cudaStreamCaptureMode mode = cudaStreamCaptureModeThreadLocal;
  // fn's launches on stream_ go into gr after its current leaves
  auto capture = [&](cudaGraph_t gr, const std::function<void()>& fn) {
    std::vector<cudaGraphNode_t> leaves;
    if (!graph_leaves(gr, leaves)) return false;
    if (cudaStreamBeginCaptureToGraph(stream_, gr, leaves.empty() ? nullptr : leaves.data(), nullptr, leaves.size(),
                                      mode) != cudaSuccess)
      return false;
    bool ok = true;
    try {
      fn();
    } catch (const Error&) {
      ok = false;
    }
    cudaGraph_t out = nullptr;
    return cudaStreamEndCapture(stream_, &out) == cudaSuccess && ok;
  };
  // a conditional node after gr's leaves; its body graph in *bodyOut
  auto conditional = [&](cudaGraph_t gr, cudaGraphConditionalHandle h, cudaGraphConditionalNodeType type,
                         cudaGraph_t* bodyOut) {
    std::vector<cudaGraphNode_t> leaves;
    if (!graph_leaves(gr, leaves) || leaves.empty()) return false;
    cudaGraphNodeParams cp = {};
    cp.type = cudaGraphNodeTypeConditional;
    cp.conditional.handle = h;
    cp.conditional.type = type;
    cp.conditional.size = 1;
    cudaGraphNode_t node = nullptr;
    if (cudaGraphAddNode(&node, gr, leaves.data(), leaves.size(), &cp) != cudaSuccess) return false;
    *bodyOut = cp.conditional.phGraph_out[0];
    return true;
  };
  cudaGraph_t g = nullptr, body = nullptr, upd = nullptr;
  cudaGraphConditionalHandle hOuter = 0, hUpdate = 0;
  bool ok = cudaGraphCreate(&g, 0) == cudaSuccess &&
            cudaGraphConditionalHandleCreate(&hOuter, g, 0, cudaGraphCondAssignDefault) == cudaSuccess;
  const int aaM = opt_.linear.outerAcceleration;
  if (aaM > 0) ensureAcceleration(aaM);
  ok = ok && capture(g, [&] {
    k_outer_init<<<1, 1, 0, stream_>>>(state, hOuter);
    CUDA_OK(cudaGetLastError());
    if (aaM > 0) accelerationStart(stream_);
  });
  if (ok) {
    size_t np = 0;
    cudaGraphGetNodes(g, nullptr, &np);
    advPrologueNodes_ = (long long)np;
  }
  ok = ok && conditional(g, hOuter, cudaGraphCondTypeWhile, &body);
  ok = ok && cudaGraphConditionalHandleCreate(&hUpdate, body, 0, cudaGraphCondAssignDefault) == cudaSuccess;
  ok = ok && capture(body, [&] { linearize(); });
  ok = ok && solver_->appendDeviceSolve(body, stream_);
  ok = ok && capture(body, [&] {
    k_outer_check<<<1, 1, 0, stream_>>>(state, hist, solver_->deviceInitialNorm(), solver_->deviceLoopState(),
                                        hOuter, hUpdate);
    CUDA_OK(cudaGetLastError());
  });
  ok = ok && conditional(body, hUpdate, cudaGraphCondTypeIf, &upd);
  ok = ok && capture(upd, [&] {
    dev::update_solution(nCells, dPerm_, hier_.level(0).x, bd, dFaceCells_, dCoeff_, dT_, stream_);
    // skipped on the device once the loop has ended (converged or out of
    // iterations), as the host loop skips it
    if (aaM > 0) accelerationStep(stream_, &state->status);
  });
  if (ok) {
    size_t nb = 0, nu = 0;
    cudaGraphGetNodes(body, nullptr, &nb);
    cudaGraphGetNodes(upd, nullptr, &nu);
    advOuterNodes_ = (long long)nb - 2 + (long long)nu;  // the while and if nodes launch nothing themselves
  }
  const auto t1 = std::chrono::steady_clock::now();
  ok = ok && cudaGraphInstantiate(&gAdvance_, g, 0) == cudaSuccess;
  if (getenv("FVM_TRACE")) {
    const auto t2 = std::chrono::steady_clock::now();
    fprintf(stderr, "[fvm advance] outer-loop graph: captured in %.2f ms, instantiated in %.2f ms (%s)\n",
            std::chrono::duration<double, std::milli>(t1 - t0).count(),
            std::chrono::duration<double, std::milli>(t2 - t1).count(), ok ? "ok" : "failed");
  }
  if (g) cudaGraphDestroy(g);
  if (!ok) {
    releaseAdvanceGraph();
    cudaGetLastError();
    return false;
  }
  advSolverGen_ = solverGen_;
  advKey_ = solver_->loopKey();
  advAADepth_ = aaM;
  advAAGen_ = aaGen_;
  return true;
}

bool ThermalModel::outerGraphUsable() const {
  return !advanceFailed_ && opt_.linear.outerOnDevice && !matrixDependsOnT_ && !dSegNorm_ &&
         opt_.linear.verbosity <= 0 && solver_ && solver_->deviceSolvable();
}

bool ThermalModel::advanceOnDevice(int niter, AdvanceReport& rep) {
  if (!outerGraphUsable()) return false;
  const int cap = std::max(std::max(niter, kOuterHistory), advHistoryCap_);
  const int aaM = opt_.linear.outerAcceleration;
  if (aaM > 0) ensureAcceleration(aaM);
  if (!gAdvance_ || advSolverGen_ != solverGen_ || !(advKey_ == solver_->loopKey()) || niter > advHistoryCap_ ||
      advAADepth_ != aaM || (aaM > 0 && advAAGen_ != aaGen_)) {
    if (!buildAdvanceGraph(cap)) {
      advanceFailed_ = true;
      if (getenv("FVM_TRACE")) fprintf(stderr, "[fvm advance] the outer-loop graph failed to build: host loop\n");
      return false;
    }
  }
  OuterState* hs = (OuterState*)hOuter_;
  hs->initialNorm = initialNorm_;
  hs->absTol = opt_.absoluteTolerance;
  hs->relTol = opt_.relativeTolerance;
  hs->niter = niter;
  hs->iterations = hs->linearIterations = hs->status = 0;
  CUDA_OK(cudaMemcpyAsync(dOuter_, hOuter_, sizeof(OuterState), cudaMemcpyHostToDevice, stream_));
  CUDA_OK(cudaGraphLaunch(gAdvance_, stream_));
  CUDA_OK(cudaMemcpyAsync(hOuter_, dOuter_, kOuterHead + sizeof(double) * (size_t)std::max(niter, 0),
                          cudaMemcpyDeviceToHost, stream_));
  CUDA_OK(cudaStreamSynchronize(stream_));
  const OuterState s = *hs;
  const double* hist = (const double*)((const char*)hOuter_ + kOuterHead);
  for (int i = 0; i < s.iterations; i++) history_.push_back(hist[i]);
  niters_ += s.iterations;
  initialNorm_ = s.initialNorm;
  rep.iterations += s.iterations;
  rep.linearIterations += s.linearIterations;
  if (s.iterations > 0) rep.lastNorm = hist[s.iterations - 1];
  rep.launches += advPrologueNodes_ + (long long)s.iterations * advOuterNodes_ +
                 (long long)s.linearIterations * solver_->loopBodyNodes();
  if (s.status == 2) throw Error(kNaN, "initial residual is not finite");
  if (s.status == 4) throw Error(kNaN, "residual became non-finite");
  rep.converged = s.status == 1;
  rep.outerOnDevice = true;
  return true;
}

// Per-block outer test on the L1 norm of this iteration's linear system
// (b, the residual of the delta form at delta = 0).
bool ThermalModel::segmentsConverged() {
  const int ns = numSegments();
  std::vector<double> v(ns);
  CUDA_OK(cudaMemcpyAsync(v.data(), dSegNorm_, sizeof(double) * ns, cudaMemcpyDeviceToHost, stream_));
  CUDA_OK(cudaStreamSynchronize(stream_));
  bool all = true;
  for (int s = 0; s < ns; s++) {
    if (segFirst_[s] < 0) segFirst_[s] = v[s];
    segLast_[s] = v[s];
    const double ratio = segFirst_[s] > 0 ? v[s] / segFirst_[s] : 0.0;
    const bool ok = v[s] < opt_.absoluteTolerance || ratio < opt_.relativeTolerance;
    if (ok && segConvergedAt_[s] < 0) segConvergedAt_[s] = niters_ - 1;
    all = all && ok;
  }
  return all;
}

HostField& ThermalModel::field(int f) {
  switch (f) {
    case kFieldTemperature:
      return T_;
    case kFieldConductivity:
      return k_;
    case kFieldSource:
      return src_;
    case kFieldSpecificHeat:
      return rc_;
    case kFieldTemperatureN1:
      return TN1_;
  }
  throw Error(kBadArgument, "unknown cell field");
}

void ThermalModel::materialize(int f) {
  HostField& v = field(f);
  if (uniform_[f]) std::fill(v.begin(), v.end(), uniformValue_[f]);
  uniform_[f] = false;
}

void ThermalModel::setCellField(int field, const double* values, int count) {
  FVM_REQUIRE(initialized_, kBadArgument, "ThermalModel.init() must be called before setting fields");
  const int n = mesh_->nCells, nAll = mesh_->nTotalCells();
  FVM_REQUIRE(count == nAll || count == n, kBadArgument,
              "cell field length must be nCells or nCells + ghost cells");
  if (field == kFieldTemperature && count == n) {
    // keep the ghost values the device (or the uniform start) holds when
    // only self cells are given
    if (deviceReady_ && !tDirty_) {
      CUDA_OK(cudaMemcpy(T_.data(), dT_, sizeof(double) * nAll, cudaMemcpyDeviceToHost));
      uniform_[kFieldTemperature] = false;
    } else {
      materialize(kFieldTemperature);
    }
  }
  HostField& f = this->field(field);
  // large fields are copied by all host cores (one core moves ~5-10 GB/s)
  parallel_chunks(count, [&](int b, int e) { std::copy(values + b, values + e, f.begin() + b); }, 1 << 20);
  uniform_[field] = false;
  if (count == n && field != kFieldTemperature) {
    // ghost cells take the value of their interior neighbour
    const HostMesh& m = *mesh_;
    for (size_t g = 1; g < m.groups.size(); g++)
      for (int fc = m.groups[g].offset; fc < m.groups[g].offset + m.groups[g].size; fc++)
        f[m.faceCells[2 * fc + 1]] = f[m.faceCells[2 * fc]];
  }
  switch (field) {
    case kFieldTemperature:
      tDirty_ = true;
      break;
    case kFieldConductivity:
      kDirty_ = true;
      matrixDirty_ = true;
      break;
    case kFieldSource:
      srcDirty_ = true;
      break;
    case kFieldSpecificHeat:
      rcDirty_ = true;
      matrixDirty_ = true;
      break;
    case kFieldTemperatureN1:
      tn1Dirty_ = true;
      break;
  }
}

void ThermalModel::getCellField(int field, double* out, int count) {
  FVM_REQUIRE(initialized_, kBadArgument, "ThermalModel.init() must be called first");
  const int nAll = mesh_->nTotalCells();
  FVM_REQUIRE(count == nAll || count == mesh_->nCells, kBadArgument, "bad cell field length");
  if (deviceReady_) {
    if (field == kFieldTemperature && !tDirty_)
      CUDA_OK(cudaMemcpy(T_.data(), dT_, sizeof(double) * nAll, cudaMemcpyDeviceToHost));
    if (field == kFieldTemperatureN1 && !tn1Dirty_)
      CUDA_OK(cudaMemcpy(TN1_.data(), dTN1_, sizeof(double) * nAll, cudaMemcpyDeviceToHost));
  }
  if ((field == kFieldTemperature && deviceReady_ && !tDirty_) ||
      (field == kFieldTemperatureN1 && deviceReady_ && !tn1Dirty_))
    uniform_[field] = false;  // the device copy just came back
  if (uniform_[field]) {
    std::fill(out, out + count, uniformValue_[field]);
    return;
  }
  HostField& f = this->field(field);
  parallel_chunks(count, [&](int b, int e) { std::copy(f.begin() + b, f.begin() + e, out + b); }, 1 << 20);
}

void ThermalModel::ensureDevice() {
  if (deviceReady_) return;
  HostMesh& m = *mesh_;
  CUDA_OK(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking));
  const int n = m.nCells, nAll = m.nTotalCells(), F = m.nFaces;
  // boundary faces in face order and the per-cell lists
  boundaryFaces_.clear();
  std::vector<int> bIndexOfFace(F, -1);
  for (size_t g = 1; g < m.groups.size(); g++)
    for (int f = m.groups[g].offset; f < m.groups[g].offset + m.groups[g].size; f++) {
      bIndexOfFace[f] = (int)boundaryFaces_.size();
      boundaryFaces_.push_back(f);
    }
  // per self cell: its faces ascending; its boundary faces ascending (the
  // order BCs are applied in) and the same faces by ghost index (the order
  // eliminateBoundaryEquations visits the ghost rows in)
  std::vector<int> cfRow(n + 1), cfCol, bRow(n + 1, 0), bCol, bColG;
  for (int i = 0; i < n; i++) {
    cfRow[i] = (int)cfCol.size();
    bRow[i] = (int)bCol.size();
    for (int k = m.cellFaces.row[i]; k < m.cellFaces.row[i + 1]; k++) {
      const int f = m.cellFaces.col[k];
      cfCol.push_back(f);
      if (bIndexOfFace[f] >= 0) bCol.push_back(f);
    }
    std::vector<int> g(bCol.begin() + bRow[i], bCol.end());
    std::sort(g.begin(), g.end(), [&](int a, int b) { return m.faceCells[2 * a + 1] < m.faceCells[2 * b + 1]; });
    bColG.insert(bColG.end(), g.begin(), g.end());
  }
  cfRow[n] = (int)cfCol.size();
  bRow[n] = (int)bCol.size();
  // self-row/self-column part of cellCells and the face behind each entry
  std::vector<int> fullEntryFace(m.cellCells.nnz(), -1);
  for (int f = 0; f < F; f++) {
    fullEntryFace[m.pairToCol[2 * f]] = f;
    fullEntryFace[m.pairToCol[2 * f + 1]] = f;
  }
  interiorConn_.nRows = n;
  interiorConn_.row.assign(n + 1, 0);
  interiorConn_.col.clear();
  entryFace_.clear();
  for (int i = 0; i < n; i++) {
    for (int k = m.cellCells.row[i]; k < m.cellCells.row[i + 1]; k++) {
      const int j = m.cellCells.col[k];
      if (j < n) {
        interiorConn_.col.push_back(j);
        entryFace_.push_back(fullEntryFace[k]);
      }
    }
    interiorConn_.row[i + 1] = (int)interiorConn_.col.size();
  }
  std::vector<int> ccRow(m.cellCells.row.begin(), m.cellCells.row.begin() + n + 1);
  dFaceCells_ = arena_.upload(m.faceCells);
  dCcRow_ = arena_.upload(ccRow);
  dCcCol_ = arena_.upload(m.cellCells.col);
  dGradW_ = arena_.upload(m.gradCoeff);
  dArea_ = arena_.upload(m.faceArea);
  dAreaMag_ = arena_.upload(m.faceAreaMag);
  dCentroid_ = arena_.upload(m.cellCentroid);
  dVol_ = arena_.upload(m.cellVolume);
  dCfRow_ = arena_.upload(cfRow);
  dCfCol_ = arena_.upload(cfCol);
  dBRow_ = arena_.upload(bRow);
  dBCol_ = arena_.upload(bCol);
  dBColG_ = arena_.upload(bColG);
  dBFace_ = arena_.upload(boundaryFaces_);
  dBIndexOfFace_ = arena_.upload(bIndexOfFace);
  const int nB = (int)boundaryFaces_.size();
  dBKind_ = (int*)arena_.alloc(sizeof(int) * (nB + 1));
  dBValue_ = (double*)arena_.alloc(sizeof(double) * (nB + 1));
  dBGhost_ = (double*)arena_.alloc(sizeof(double) * (nB + 1));
  dBParam_ = (double*)arena_.alloc(sizeof(double) * 3 * (nB + 1));
  dBGhostDiag_ = (double*)arena_.alloc(sizeof(double) * (nB + 1));
  dHf_ = (double*)arena_.alloc(sizeof(double) * 4 * (nB + 1));
  dHeatFlux_ = (double*)arena_.alloc(sizeof(double) * (nB + 1));
  CUDA_OK(cudaMemset(dHeatFlux_, 0, sizeof(double) * (nB + 1)));
  const size_t cb = sizeof(double) * (size_t)nAll;
  dT_ = (double*)arena_.alloc(cb);
  dK_ = (double*)arena_.alloc(cb);
  dSrc_ = (double*)arena_.alloc(cb);
  dRc_ = (double*)arena_.alloc(cb);
  dTN1_ = (double*)arena_.alloc(cb);
  dRhoVdt_ = (double*)arena_.alloc(cb);
  dGrad_ = (double*)arena_.alloc(4 * cb);  // 32-byte record per cell
  dDiagOrig_ = (double*)arena_.alloc(cb);
  dFlux_ = (double*)arena_.alloc(sizeof(double) * (size_t)F);
  dCoeff_ = (double*)arena_.alloc(sizeof(double) * (size_t)F);
  dSec_ = (double*)arena_.alloc(4 * sizeof(double) * (size_t)F);  // 32-byte record per face
  CUDA_OK(cudaMemset(dGrad_, 0, 4 * cb));
  {
    // identifies this model's level-0 pattern (interiorConn_, entryFace_)
    static std::atomic<unsigned long long> nextKey{1};
    patternKey_ = nextKey++;
  }
  deviceReady_ = true;
  tDirty_ = kDirty_ = srcDirty_ = rcDirty_ = tn1Dirty_ = true;
  matrixDirty_ = true;
}

void ThermalModel::uploadFields() {
  const size_t cb = sizeof(double) * (size_t)mesh_->nTotalCells();
  const int nAll = mesh_->nTotalCells();
  // a uniform field is filled on the device; the others are copied from
  // the pinned host arrays
  auto up = [&](int f, double* d) {
    if (uniform_[f])
      k_fill_value<<<(nAll + 255) / 256, 256, 0, stream_>>>(nAll, d, uniformValue_[f]);
    else
      CUDA_OK(cudaMemcpyAsync(d, field(f).data(), cb, cudaMemcpyHostToDevice, stream_));
  };
  if (tDirty_) up(kFieldTemperature, dT_);
  if (kDirty_) up(kFieldConductivity, dK_);
  if (srcDirty_) up(kFieldSource, dSrc_);
  // rho c and the previous step's T enter only the transient term: a steady
  // model leaves them on the host (still dirty) until it becomes transient
  const bool transient = opt_.transient;
  if (rcDirty_ && transient) up(kFieldSpecificHeat, dRc_);
  if (tn1Dirty_ && transient) up(kFieldTemperatureN1, dTN1_);
  CUDA_OK(cudaStreamSynchronize(stream_));
  tDirty_ = kDirty_ = srcDirty_ = false;
  if (transient) rcDirty_ = tn1Dirty_ = false;
  // boundary kinds and values (cheap; a change of kind or of a value the
  // matrix depends on changes the matrix)
  const int nB = (int)boundaryFaces_.size();
  std::vector<int> kind(nB + 1, 0);
  std::vector<double> val(nB + 1, 0.0), par(3 * (nB + 1), 0.0);
  int t = 0;
  matrixDependsOnT_ = false;
  for (size_t g = 1; g < mesh_->groups.size(); g++) {
    const FaceGroup& fg = mesh_->groups[g];
    const GroupBC& b = bc(fg.id);
    int k;
    double v = 0.0;
    switch (b.type) {
      case kBcSpecifiedTemperature:
        k = dev::kBkDirichlet;
        v = b.values[0];
        break;
      case kBcSpecifiedHeatFlux:
        k = dev::kBkFlux;
        v = b.values[1];
        break;
      case kBcSymmetry:
        k = dev::kBkFlux;
        break;
      case kBcConvective:
        k = dev::kBkConvective;
        break;
      case kBcRadiative:
        k = dev::kBkRadiative;
        matrixDependsOnT_ = true;
        break;
      case kBcMixed:
        k = dev::kBkMixed;
        matrixDependsOnT_ = true;
        break;
      default:
        throw Error(kUnsupported, "unknown boundary condition type");
    }
    for (int f = 0; f < fg.size; f++, t++) {
      kind[t] = k;
      val[t] = v;
      par[3 * t] = b.values[2];      // convectiveCoefficient
      par[3 * t + 1] = b.values[3];  // farFieldTemperature
      par[3 * t + 2] = b.values[4];  // surfaceEmissivity
    }
  }
  CUDA_OK(cudaMemcpy(dBKind_, kind.data(), sizeof(int) * (nB + 1), cudaMemcpyHostToDevice));
  CUDA_OK(cudaMemcpy(dBValue_, val.data(), sizeof(double) * (nB + 1), cudaMemcpyHostToDevice));
  CUDA_OK(cudaMemcpy(dBParam_, par.data(), sizeof(double) * 3 * (nB + 1), cudaMemcpyHostToDevice));
  if (par != bParamHost_) {
    bParamHost_ = par;
    matrixDirty_ = true;
  }
  if (kind != bKindHost_) {
    bKindHost_ = kind;
    matrixDirty_ = true;
  }
}

void ThermalModel::ensureMatrix() {
  // a matrix that depends on T (radiative / mixed conditions) is rebuilt
  // for every linearization
  if (!matrixDirty_ && !hierarchyDirty_ && !matrixDependsOnT_) return;
  const bool trace = getenv("FVM_TRACE") != nullptr;
  auto t0 = std::chrono::steady_clock::now();
  auto lap = [&](const char* what) {
    if (!trace) return;
    const auto t1 = std::chrono::steady_clock::now();
    fprintf(stderr, "[fvm matrix] %-26s %8.1f ms\n", what, std::chrono::duration<double, std::milli>(t1 - t0).count());
    t0 = t1;
  };
  HostMesh& m = *mesh_;
  const int n = m.nCells, F = m.nFaces;
  dev::FaceGeom g{F, n, dFaceCells_, dArea_, dAreaMag_, dCentroid_, dVol_};
  dev::face_coefficients(g, dK_, dCoeff_, dSec_, stream_);
  const double* rhoVdt = nullptr;
  if (opt_.transient) {
    FVM_REQUIRE(opt_.timeDiscretizationOrder == 1, kUnsupported,
                "only first-order time discretization is available on the GPU path");
    dev::transient_coeff(n, dRc_, dVol_, opt_.timeStep, dRhoVdt_, stream_);
    rhoVdt = dRhoVdt_;
  }
  dev::CellFaceView cf{dCfRow_, dCfCol_, dBRow_, dBCol_, dBColG_};
  const dev::BoundaryData bd = boundaryData();
  dev::assemble_matrix(n, cf, dFaceCells_, dCoeff_, dAreaMag_, rhoVdt, bd, dBIndexOfFace_, dT_, dDiagOrig_, stream_);
  if (opt_.linear.setupOnDevice && !opt_.linear.finestOnly()) {
    // the whole hierarchy is built on the GPU from the assembled face
    // coefficients and diagonal: nothing comes back to the host
    lap("assembly");
    solver_.reset();
    hier_.release();
    FinestDevice in;
    in.conn = &interiorConn_;
    in.entrySrc = &entryFace_;
    in.offSrc = dCoeff_;
    in.diag = dDiagOrig_;
    in.key = patternKey_;
    in.symmetricPattern = true;
    in.segments = segOff_;
    in.ccRow = dCcRow_;
    in.ccCol = dCcCol_;
    in.cfRow = dCfRow_;
    in.cfCol = dCfCol_;
    in.faceCells = dFaceCells_;
    CUDA_OK(cudaStreamSynchronize(stream_));
    hier_.buildDevice(in, opt_.linear, true);
    lap("hierarchy on the device");
    dPerm_ = const_cast<int*>(hier_.finestPermDevice());
    solver_.reset(new LinearSolve(hier_));
    solverGen_++;
    solver_->setLearned(learned_);
    // the solve's graphs are built while the GPU computes the coarsest
    // inverse, the build's last step
    try {
      if (outerGraphUsable()) {
        if (!buildAdvanceGraph(std::max(kOuterHistory, advHistoryCap_))) advanceFailed_ = true;
      } else {
        solver_->prebuild(stream_);
      }
      hier_.finishBuild();
    } catch (...) {
      releaseAdvanceGraph();
      solver_.reset();
      hier_.release();
      throw;
    }
    lap("solver workspace and graphs");
    matrixDirty_ = hierarchyDirty_ = false;
    return;
  }
  // face coefficients and diagonal come back through pinned buffers kept
  // for the model's lifetime
  const size_t pinBytes = sizeof(double) * ((size_t)F + (size_t)n);
  if (pinBytes > hPinnedBytes_) {
    if (hPinned_) cudaFreeHost(hPinned_);
    hPinned_ = nullptr;
    hPinnedBytes_ = 0;
    CUDA_OK(cudaMallocHost(&hPinned_, pinBytes));
    hPinnedBytes_ = pinBytes;
  }
  const double* coeff = hPinned_;
  double* hDiag = hPinned_ + F;
  CUDA_OK(cudaMemcpyAsync(hPinned_, dCoeff_, sizeof(double) * F, cudaMemcpyDeviceToHost, stream_));
  CUDA_OK(cudaMemcpyAsync(hDiag, dDiagOrig_, sizeof(double) * n, cudaMemcpyDeviceToHost, stream_));
  CUDA_OK(cudaStreamSynchronize(stream_));
  lap("assembly + copy to host");
  // the previous hierarchy's host buffers are refilled, not reallocated
  solver_.reset();
  hier_.release();
  lap("previous solver released");
  std::vector<RefLevel> levels(1);
  levels[0] = hier_.spareLevel(0);
  RefLevel& l0 = levels[0];
  l0.n = n;
  // the spare level 0 of this model's previous build already holds the
  // (fixed) connectivity of its mesh
  if (l0.conn.nRows != interiorConn_.nRows || l0.conn.col.size() != interiorConn_.col.size())
    l0.conn = interiorConn_;
  l0.symmetricPattern = true;  // cellCells restricted to self rows
  l0.segments = segOff_;       // a batch: its meshes aggregate in parallel
  l0.coarseIndex.clear();
  l0.nCoarse = 0;
  l0.diag.assign(hDiag, hDiag + n);
  l0.off.resize(entryFace_.size());
  parallel_chunks((int)entryFace_.size(), [&](int b, int e) {
    for (int k = b; k < e; k++) l0.off[k] = coeff[entryFace_[k]];
  }, 1 << 18);
  lap("finest level on host");
  hier_.build(levels, m.nTotalCells(), opt_.linear);
  lap("hierarchy");
  dPerm_ = (int*)hier_.scratch(sizeof(int) * (size_t)n);
  CUDA_OK(cudaMemcpyAsync(dPerm_, hier_.packed(0).perm.data(), sizeof(int) * (size_t)n, cudaMemcpyHostToDevice,
                          stream_));
  solver_.reset(new LinearSolve(hier_));
  solverGen_++;
  solver_->setLearned(learned_);
  lap("solver workspace");
  matrixDirty_ = hierarchyDirty_ = false;
}

void ThermalModel::linearize() {
  HostMesh& m = *mesh_;
  const int n = m.nCells, F = m.nFaces;
  dev::gradient(n, dCcRow_, dCcCol_, dGradW_, dT_, dGrad_, stream_);
  dev::ghost_gradient((int)boundaryFaces_.size(), dBFace_, dFaceCells_, dGrad_, stream_);
  dev::FaceGeom g{F, n, dFaceCells_, dArea_, dAreaMag_, dCentroid_, dVol_};
  dev::face_flux(g, dCoeff_, dSec_, dGrad_, dT_, dFlux_, stream_);
  dev::CellFaceView cf{dCfRow_, dCfCol_, dBRow_, dBCol_, dBColG_};
  const dev::BoundaryData bd = boundaryData();
  dev::assemble_rhs(n, cf, dFaceCells_, dFlux_, dCoeff_, dAreaMag_, dVol_, dSrc_,
                    opt_.transient ? dRhoVdt_ : nullptr, dTN1_, bd, dBIndexOfFace_, dT_,
                    dPerm_, hier_.level(0).b, stream_);
}

void ThermalModel::advance(int niter, AdvanceReport& rep) {
  FVM_REQUIRE(initialized_, kBadArgument, "ThermalModel.init() must be called before advance()");
  TraceRange traceAdvance("ThermalModel::advance");
  rep = AdvanceReport();
  ensureDevice();
  cudaEvent_t e0, e1, e2;
  CUDA_OK(cudaEventCreate(&e0));
  CUDA_OK(cudaEventCreate(&e1));
  CUDA_OK(cudaEventCreate(&e2));
  // the cell fields set on the host since the last call go to the device
  // first; the timed region (rep.seconds) starts with them resident
  uploadFields();
  CUDA_OK(cudaEventRecord(e0, stream_));
  const auto s0 = std::chrono::steady_clock::now();
  {
    TraceRange traceSetup("setup (matrix, AMG hierarchy)");
    ensureMatrix();
  }
  const auto s1 = std::chrono::steady_clock::now();
  rep.setupSeconds = std::chrono::duration<double>(s1 - s0).count();
  CUDA_OK(cudaEventRecord(e1, stream_));
  const long long launches0 = solver_->launches;
  HostMesh& m = *mesh_;
  const dev::BoundaryData bd = boundaryData();
  TraceRange traceOuter("outer iterations");
  const bool onDevice = advanceOnDevice(niter, rep);
  const int aaM = opt_.linear.outerAcceleration;
  if (!onDevice && aaM > 0 && niter > 0) {
    ensureAcceleration(aaM);
    accelerationStart(stream_);
    rep.launches += 2;
  }
  for (int it = 0; !onDevice && it < niter; it++) {
    if (matrixDependsOnT_ && it > 0) {
      // radiative / mixed conditions: the ghost diagonals follow T, so the
      // matrix and its AMG levels are rebuilt every outer iteration, as the
      // reference rebuilds them
      const auto s2 = std::chrono::steady_clock::now();
      ensureMatrix();
      rep.setupSeconds += std::chrono::duration<double>(std::chrono::steady_clock::now() - s2).count();
    }
    {
      TraceRange traceLin("linearize");
      linearize();
    }
    rep.launches += 4;
    if (dSegNorm_) {
      k_segment_l1<<<numSegments(), 256, 0, stream_>>>(dSegOff_, dPerm_, hier_.level(0).b, dSegNorm_);
      rep.launches += 1;
    }
    SolveReport sr;
    {
      TraceRange traceSolve("linear solve");
      sr = solver_->solve(stream_);
    }
    const double rNorm = sr.initialNorm;
    if (initialNorm_ < 0) initialNorm_ = rNorm;
    dev::update_solution(m.nCells, dPerm_, hier_.level(0).x, bd, dFaceCells_, dCoeff_, dT_,
                         stream_);
    rep.launches += 2;
    niters_++;
    history_.push_back(rNorm);
    rep.iterations++;
    rep.linearIterations += sr.iterations;
    rep.learnedSteps += sr.learnedSteps;
    rep.learnedAccepted += sr.learnedAccepted;
    rep.lastNorm = rNorm;
    if (opt_.linear.verbosity >= 0 && opt_.linear.verbosity > 0) printf("%d: %g\n", niters_ - 1, rNorm);
    const double ratio = initialNorm_ > 0 ? rNorm / initialNorm_ : 0.0;
    const bool done = dSegNorm_ ? segmentsConverged()
                                : (rNorm < opt_.absoluteTolerance || ratio < opt_.relativeTolerance);
    if (done) {
      rep.converged = true;
      break;
    }
    if (aaM > 0 && it + 1 < niter) {
      accelerationStep(stream_, nullptr);
      rep.launches += 3;
    }
  }
  CUDA_OK(cudaEventRecord(e2, stream_));
  CUDA_OK(cudaEventSynchronize(e2));
  float ms = 0;
  CUDA_OK(cudaEventElapsedTime(&ms, e0, e2));
  rep.seconds = ms * 1e-3;
  rep.initialNorm = initialNorm_;
  rep.launches += solver_->launches - launches0;
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaEventDestroy(e2);
  CUDA_OK(cudaGetLastError());
}

dev::BoundaryData ThermalModel::boundaryData() const {
  dev::BoundaryData bd;
  bd.nBFaces = (int)boundaryFaces_.size();
  bd.bFace = dBFace_;
  bd.kind = dBKind_;
  bd.value = dBValue_;
  bd.param = dBParam_;
  bd.ghostRhs = dBGhost_;
  bd.ghostDiag = dBGhostDiag_;
  bd.hf = dHf_;
  bd.heatFlux = dHeatFlux_;
  return bd;
}

double ThermalModel::heatFluxIntegral(int groupId) {
  FVM_REQUIRE(initialized_, kBadArgument, "ThermalModel.init() must be called first");
  const HostMesh& m = *mesh_;
  int t = 0;
  for (size_t g = 1; g < m.groups.size(); g++) {
    const FaceGroup& fg = m.groups[g];
    if (fg.id == groupId) {
      std::vector<double> q(fg.size, 0.0);
      if (deviceReady_ && fg.size > 0)
        CUDA_OK(cudaMemcpy(q.data(), dHeatFlux_ + t, sizeof(double) * fg.size, cudaMemcpyDeviceToHost));
      double r = 0.0;
      for (int f = 0; f < fg.size; f++) r += q[f];
      return r;
    }
    t += fg.size;
  }
  throw Error(kBadArgument, "getHeatFluxIntegral: invalid faceGroupID");
}

void ThermalModel::setLearned(LearnedCorrection* lc) {
  learned_ = lc;
  if (solver_) solver_->setLearned(lc);
}

namespace {
__global__ void k_error(int n, const double* __restrict__ xs, const double* __restrict__ x, double* e) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) e[i] = xs[i] - x[i];
}
}  // namespace

int ThermalModel::harvest(LearnedCorrection& lc, int nOuter, int perSolve, double relTol, int maxCycles) {
  FVM_REQUIRE(initialized_, kBadArgument, "ThermalModel.init() must be called first");
  FVM_REQUIRE(nOuter > 0 && perSolve > 0 && maxCycles > 1 && relTol > 0.0, kBadArgument,
              "harvest: nOuter, perSolve > 0, maxCycles > 1, relTol > 0");
  FVM_REQUIRE(opt_.linear.solver == kSolverAMG, kUnsupported, "harvest: the model's linear solver must be AMG");
  ensureDevice();
  uploadFields();
  FVM_REQUIRE(!matrixDependsOnT_, kUnsupported,
              "harvest: radiative / mixed conditions make the matrix change every iteration");
  ensureMatrix();
  HostMesh& m = *mesh_;
  const int n = m.nCells;
  DevLevel& d0 = hier_.level(0);
  const nn::Graph g{d0.view64(), d0.rowSlice, d0.nSlices, (long long)d0.entries};
  const int inst = lc.addInstance(g, (int)d0.entries, stream_);
  std::vector<double*> rs(perSolve), xs(perSolve);
  double* e = nullptr;
  DeviceArena tmp;
  for (int q = 0; q < perSolve; q++) {
    rs[q] = (double*)tmp.alloc(sizeof(double) * (size_t)n);
    xs[q] = (double*)tmp.alloc(sizeof(double) * (size_t)n);
  }
  e = (double*)tmp.alloc(sizeof(double) * (size_t)n);
  const dev::BoundaryData bd = boundaryData();
  int pairs = 0;
  for (int it = 0; it < nOuter; it++) {
    linearize();
    SolveReport sr;
    const int rec = solver_->solveRecording(stream_, relTol, maxCycles, perSolve, rs, xs, sr);
    for (int q = 0; q < rec; q++) {
      k_error<<<(n + 255) / 256, 256, 0, stream_>>>(n, d0.x, xs[q], e);
      lc.addPair(inst, rs[q], e, stream_);
      pairs++;
    }
    const double rNorm = sr.initialNorm;
    if (initialNorm_ < 0) initialNorm_ = rNorm;
    dev::update_solution(n, dPerm_, d0.x, bd, dFaceCells_, dCoeff_, dT_, stream_);
    niters_++;
    history_.push_back(rNorm);
    const double ratio = initialNorm_ > 0 ? rNorm / initialNorm_ : 0.0;
    if (rNorm < opt_.absoluteTolerance || ratio < opt_.relativeTolerance) break;
  }
  CUDA_OK(cudaStreamSynchronize(stream_));
  tDirty_ = false;
  return pairs;
}

void ThermalModel::updateTime() {
  FVM_REQUIRE(initialized_, kBadArgument, "ThermalModel.init() must be called first");
  if (!deviceReady_ || tDirty_) {
    if (uniform_[kFieldTemperature]) {
      uniform_[kFieldTemperatureN1] = true;
      uniformValue_[kFieldTemperatureN1] = uniformValue_[kFieldTemperature];
    } else {
      TN1_ = T_;
      uniform_[kFieldTemperatureN1] = false;
    }
    tn1Dirty_ = true;
    return;
  }
  CUDA_OK(cudaMemcpyAsync(dTN1_, dT_, sizeof(double) * (size_t)mesh_->nTotalCells(),
                          cudaMemcpyDeviceToDevice, stream_));
  CUDA_OK(cudaStreamSynchronize(stream_));
  tn1Dirty_ = false;
}

void ThermalModel::linearizeOnly(std::vector<double>& diag, std::vector<double>& off,
                                 std::vector<double>& b) {
  FVM_REQUIRE(initialized_, kBadArgument, "ThermalModel.init() must be called first");
  ensureDevice();
  uploadFields();
  ensureMatrix();
  linearize();
  const int n = mesh_->nCells;
  std::vector<double> bp(n);
  CUDA_OK(cudaMemcpyAsync(bp.data(), hier_.level(0).b, sizeof(double) * n, cudaMemcpyDeviceToHost,
                          stream_));
  CUDA_OK(cudaStreamSynchronize(stream_));
  const PackedLevel& p0 = hier_.packed(0);
  b.resize(n);
  for (int i = 0; i < n; i++) b[i] = bp[p0.perm[i]];
  diag = hier_.refLevels()[0].diag;
  off = hier_.refLevels()[0].off;
}

void ThermalModel::profile(int reps, double* out) {
  FVM_REQUIRE(initialized_, kBadArgument, "ThermalModel.init() must be called first");
  FVM_REQUIRE(reps > 0, kBadArgument, "reps must be positive");
  ensureDevice();
  uploadFields();
  ensureMatrix();
  linearize();
  const size_t flushBytes = 512u << 20;  // > 126 MB L2
  void* flush = nullptr;
  CUDA_OK(cudaMalloc(&flush, flushBytes));
  cudaEvent_t a, b;
  CUDA_OK(cudaEventCreate(&a));
  CUDA_OK(cudaEventCreate(&b));
  DevLevel& d = hier_.level(0);
  const bool mixed = opt_.linear.precision == kMixed;
  auto timed = [&](const std::function<void()>& body) {
    double total = 0;
    for (int r = 0; r < reps; r++) {
      CUDA_OK(cudaMemsetAsync(flush, r & 0xff, flushBytes, stream_));
      CUDA_OK(cudaEventRecord(a, stream_));
      body();
      CUDA_OK(cudaEventRecord(b, stream_));
      CUDA_OK(cudaEventSynchronize(b));
      float ms = 0;
      CUDA_OK(cudaEventElapsedTime(&ms, a, b));
      total += ms;
    }
    return total / reps;
  };
  if (mixed) dev::convert_d2f(d.n, d.b, d.bF, stream_);
  out[0] = timed([&] {
    if (mixed) {
      for (int c = 0; c < d.nColors; c++)
        dev::gs_color<float>(d.view32(), d.colorSliceStart[c], d.colorSliceStart[c + 1], d.xF, d.bF, stream_,
                             d.plan);
    } else {
      for (int c = 0; c < d.nColors; c++)
        dev::gs_color<double>(d.view64(), d.colorSliceStart[c], d.colorSliceStart[c + 1], d.x, d.b, stream_,
                              d.plan);
    }
  });
  out[1] = hier_.fineSweepBytes();
  out[2] = timed([&] { dev::residual<double>(d.view64(), d.nSlices, d.x, d.b, d.r, d.partials, stream_); });
  out[3] = d.n * 32.0 + d.entries * 12.0;
  out[4] = timed([&] {
    // as the solvers run it: the FP32 preconditioner cycle starts from
    // x = 0; the FP64 AMG iteration from the current iterate
    if (mixed) {
      dev::zero<float>(d.n, d.xF, stream_);
      hier_.cycle<float>(opt_.linear.cycleType, 0, stream_, true);
    } else {
      hier_.cycle<double>(opt_.linear.cycleType, 0, stream_);
    }
  });
  out[5] = hier_.cycleBytes();
  out[6] = hier_.numLevels();
  out[7] = d.n;
  out[8] = (double)d.entries;
  out[9] = hier_.kernelsPerCycle();
  out[10] = d.nColors;
  {
    // the face loop of the linearization (k_face_flux), compulsory bytes:
    // per face cells (int2), c_f, the secondary coefficient (3 doubles) and
    // the flux written; per cell (self + ghost) its volume, gradient (3
    // doubles) and value
    HostMesh& m = *mesh_;
    dev::FaceGeom g{m.nFaces, m.nCells, dFaceCells_, dArea_, dAreaMag_, dCentroid_, dVol_};
    out[11] = timed([&] { dev::face_flux(g, dCoeff_, dSec_, dGrad_, dT_, dFlux_, stream_); });
    out[12] = 48.0 * m.nFaces + 40.0 * m.nTotalCells();
  }
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  cudaFree(flush);
  CUDA_OK(cudaMemsetAsync(d.x, 0, sizeof(double) * d.n, stream_));
  if (d.xF) CUDA_OK(cudaMemsetAsync(d.xF, 0, sizeof(float) * d.n, stream_));
  CUDA_OK(cudaStreamSynchronize(stream_));
}

void ThermalModel::profileLevels(int reps, std::vector<double>& out) {
  FVM_REQUIRE(initialized_, kBadArgument, "ThermalModel.init() must be called first");
  FVM_REQUIRE(reps > 0, kBadArgument, "reps must be positive");
  ensureDevice();
  uploadFields();
  ensureMatrix();
  linearize();
  DevLevel& d = hier_.level(0);
  if (opt_.linear.precision == kMixed) dev::convert_d2f(d.n, d.b, d.bF, stream_);
  const size_t flushBytes = 512u << 20;  // > 126 MB L2
  void* flush = nullptr;
  CUDA_OK(cudaMalloc(&flush, flushBytes));
  try {
    hier_.profileLevels(reps, flush, flushBytes, stream_, out);
  } catch (...) {
    cudaFree(flush);
    throw;
  }
  cudaFree(flush);
}

const AmgHierarchy& ThermalModel::hierarchy() {
  FVM_REQUIRE(initialized_, kBadArgument, "ThermalModel.init() must be called first");
  ensureDevice();
  uploadFields();
  ensureMatrix();
  return hier_;
}

}  // namespace fvm
