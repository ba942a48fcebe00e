// Learned error correction for the AMG-preconditioned solve: a small
// message-passing network on the cell graph of the finest level (cells as
// nodes, matrix couplings as edges) that maps the FP64 residual to a
// correction of the solution.
//
// Network (width 32, three message-passing layers):
//   u_i   = r_i / (|a_ii| s),  s = mean_i |r_i| / |a_ii|        (input scaling)
//   h0_i  = relu(we u_i + be)                                    (encoder, 1 -> 32)
//   m_i   = sum_j w_ij h_j,  w_ij = |a_ij| / |a_ii|              (message)
//   h'_i  = relu(Ws h_i + Wm m_i + b)                            (3 layers, 64 -> 32)
//   d_i   = s (wd . h3_i + bd)                                   (decoder, 32 -> 1)
// Parameters are FP32 (6337 of them). Training minimises the relative
// squared error sum_i (d_i - e_i)^2 / sum_i e_i^2 against the error e of
// the plain solver's iterates, with hand-written forward and backward
// kernels and Adam, on the GPU. In the solve the correction is a
// flexible step x += alpha d, alpha minimising ||r + alpha A d||_2, kept
// only when it lowers the FP64 L1 residual norm (otherwise the plain AMG
// step stands).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <vector>

#include "kernels.cuh"

namespace fvm {

namespace nn {
constexpr int kWidth = 32;
constexpr int kLayers = 3;
constexpr int kEncW = 0;
constexpr int kEncB = 32;
constexpr int kLayer0 = 64;
constexpr int kLayerSize = 2 * 32 * 32 + 32;  // Ws (32x32, row = output), Wm, b
constexpr int kDecW = kLayer0 + kLayers * kLayerSize;
constexpr int kDecB = kDecW + 32;
constexpr int kParams = kDecB + 1;

// The finest level's graph in the solver's (colour-permuted) numbering.
struct Graph {
  dev::SellView<double> a;
  const int* rowSlice = nullptr;
  int nSlices = 0;
  long long entries = 0;  // stored entries (cols / vals length)
};

// Device workspace for one graph size.
struct Workspace {
  int n = 0;    // nodes of the current graph
  int cap = 0;  // nodes the buffers hold
  float* u = nullptr;            // n
  float* H[kLayers + 1] = {};    // n x 32 each
  float* M[kLayers] = {};        // n x 32 each (training only)
  float* dA = nullptr;           // n x 32 (gradient buffers)
  float* dB = nullptr;           // n x 32
  float* dS = nullptr;           // n x 32
  double* partials = nullptr;    // reductions
  float* gradPartials = nullptr; // blocks x kParams
  int gradBlocks = 0;
  int* status = nullptr;         // device flag: 1 if a tensor-core completion wait ran out
  bool tensorCores = true;       // dense layers on tcgen05 (TF32 inputs) instead of FP32 CUDA cores
  double* dv = nullptr;          // n x 2 (training with the residual objective: d, then r + A d / A(r + A d))
  float* wf = nullptr;           // per-entry message weights (forward / transpose)
  float* wb = nullptr;
  long long wcap = 0;            // entries the weight buffers hold
  void allocate(int n, bool training, long long entries);
  void release();
  // throws (and clears the flag) if a tensor-core wait ran out; synchronises
  void checkStatus();
  ~Workspace() { release(); }
};

// Runs the tensor-core layers' bounded completion wait on an mbarrier that
// no MMA signals, with `limit` tries; returns the status flag the kernel
// set (1: the wait ran out, TMEM released, the kernel returned).
int tc_wait_probe(unsigned limit);

// Forward pass: out_i = d_i (FP64, may alias nothing). sOut (device) gets
// the input scale s.
void forward(const Graph& g, const float* params, const double* r, double* out, Workspace& w,
             double* sScalar, cudaStream_t st);

// One training pass on a (residual, error) pair: forward, loss, backward;
// gradients summed into grad (kParams floats, overwritten); loss (device
// double) = relative squared error of the pair.
void forward_backward(const Graph& g, const float* params, const double* r, const double* e, float* grad,
                      double* loss, Workspace& w, double* scal, cudaStream_t st);

// The same with the residual objective: loss = |r + A d|^2 / |r|^2 for the
// network's correction d of residual r on graph g (A = g's matrix,
// symmetric), gradient 2 A (r + A d) / |r|^2 through the network. Needs
// only the residual of each pair.
void forward_backward_residual(const Graph& g, const float* params, const double* r, float* grad, double* loss,
                               Workspace& w, double* scal, cudaStream_t st);

// Adam step on the parameters (t = step number from 1).
void adam_step(float* params, const float* grad, float* m, float* v, float lr, int t, cudaStream_t st);

// Deterministic initial parameters (He-style uniform, seeded).
std::vector<float> initial_parameters(uint64_t seed);

// ---- the flexible step inside the solve (all device scalars, capturable) ----
// alpha = -(r.q)/(q.q) (0 if q.q = 0)
void step_alpha(const double* rq, const double* qq, double* alpha, cudaStream_t st);
// rt = r + alpha q, with per-block L1 partials of rt (vec_blocks(n) of them)
void step_trial(int n, const double* r, const double* q, const double* alpha, double* rt, double* partials,
                cudaStream_t st);
// if trialNorm < acceptFactor * norm: x += alpha d, r = rt
void step_accept(int n, double* x, const double* d, double* r, const double* rt, const double* alpha,
                 const double* norm, const double* trialNorm, double acceptFactor, cudaStream_t st);
// if trialNorm < acceptFactor * norm: norm = trialNorm, accepted += 1; if
// trialNorm < usefulFactor * norm: useful += 1; steps += 1
void step_finish(double* norm, const double* trialNorm, double* accepted, double* steps, double* useful,
                 double usefulFactor, double acceptFactor, cudaStream_t st);
}  // namespace nn

// A trained (or training) learned correction: parameters, Adam state and
// the training set. A training instance is one linear system's graph
// (copied, so it outlives the model it came from) with its (residual,
// error) pairs.
class LearnedCorrection {
 public:
  explicit LearnedCorrection(uint64_t seed);
  ~LearnedCorrection();
  LearnedCorrection(const LearnedCorrection&) = delete;
  LearnedCorrection& operator=(const LearnedCorrection&) = delete;

  std::vector<float> params() const;
  void setParams(const std::vector<float>& p);
  const float* deviceParams() const { return dParams_; }

  // a new instance with a copy of the graph; returns its index
  int addInstance(const nn::Graph& g, int nEntries, cudaStream_t st);
  // copies one (residual, error) pair (n doubles each, device) into instance k
  void addPair(int k, const double* r, const double* e, cudaStream_t st);
  int numPairs() const;
  int numInstances() const { return (int)inst_.size(); }

  // Adam on randomly drawn pairs; losses (optional, steps entries) gets the
  // relative squared error of each step's pair before its update.
  void train(int steps, float lr, uint64_t seed, double* losses, cudaStream_t st);
  // mean relative squared error over all pairs (no update)
  double evaluate(cudaStream_t st);

  // correction for residual r on graph g (call prepare(n) first: apply
  // allocates nothing, so it can run inside a captured graph)
  void prepare(int n, long long entries);
  void apply(const nn::Graph& g, const double* r, double* out, double* scal, cudaStream_t st);
  // largest entry count of the training instances' graphs
  long long maxEntries() const;
  // throws if a tensor-core kernel of apply() gave up waiting (synchronises)
  void checkApplyStatus() { applyWs_.checkStatus(); }

  // training objective: 0 = relative squared error of the predicted error
  // (default), 1 = residual left by the correction, |r + A d|^2 / |r|^2
  void setObjective(int o);
  int objective() const { return objective_; }
  // In the solve the step is retired after a few tries if fewer than a
  // quarter of them cut the residual below this fraction of its value
  // (default 0.5: what pays for the step's cost); 1 keeps every step that
  // lowers the residual at all.
  void setUsefulFactor(double f);
  double usefulFactor() const { return usefulFactor_; }
  // With the residual objective, evaluate() also records the residual
  // reduction the network achieves on the training pairs, sqrt(mean
  // |r + A d|^2 / |r|^2) (-1 before that). A solve does not use a network
  // whose recorded reduction is above its useful factor: the step could
  // not pay for itself.
  double residualFactor() const { return residualFactor_; }

  // dense layers on the tensor cores (default) or in FP32 on the CUDA cores
  void setTensorCores(bool on);
  bool tensorCores() const { return tensorCores_; }

 private:
  struct Instance {
    int n = 0;
    nn::Graph g;
    void* storage = nullptr;  // owns the graph copy
    std::vector<std::pair<double*, double*>> pairs;
  };
  std::vector<Instance> inst_;
  float* dParams_ = nullptr;
  float* dGrad_ = nullptr;
  float* dM_ = nullptr;
  float* dV_ = nullptr;
  double* dScal_ = nullptr;
  int adamT_ = 0;
  bool tensorCores_ = true;
  int objective_ = 0;
  double usefulFactor_ = 0.5;
  double residualFactor_ = -1.0;
  nn::Workspace trainWs_;
  nn::Workspace applyWs_;
};

}  // namespace fvm
