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
};

// Device workspace for one graph size.
struct Workspace {
  int n = 0;
  float* u = nullptr;            // n
  float* H[kLayers + 1] = {};    // n x 32 each
  float* M[kLayers] = {};        // n x 32 each (training only)
  float* dA = nullptr;           // n x 32 (gradient buffers)
  float* dB = nullptr;           // n x 32
  float* dS = nullptr;           // n x 32
  double* partials = nullptr;    // reductions
  float* gradPartials = nullptr; // blocks x kParams
  int gradBlocks = 0;
  void allocate(int n, bool training);
  void release();
  ~Workspace() { release(); }
};

// Forward pass: out_i = d_i (FP64, may alias nothing). sOut (device) gets
// the input scale s.
void forward(const Graph& g, const float* params, const double* r, double* out, Workspace& w,
             double* sScalar, cudaStream_t st);

// One training pass on a (residual, error) pair: forward, loss, backward;
// gradients summed into grad (kParams floats, overwritten); loss (device
// double) = relative squared error of the pair.
void forward_backward(const Graph& g, const float* params, const double* r, const double* e, float* grad,
                      double* loss, Workspace& w, double* scal, cudaStream_t st);

// Adam step on the parameters (t = step number from 1).
void adam_step(float* params, const float* grad, float* m, float* v, float lr, int t, cudaStream_t st);

// Deterministic initial parameters (He-style uniform, seeded).
std::vector<float> initial_parameters(uint64_t seed);
}  // namespace nn

}  // namespace fvm
