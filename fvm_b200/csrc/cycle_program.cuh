// One AMG cycle as a single persistent, cooperatively launched kernel.
//
// The host flattens a cycle (V/W/F, any sweep counts) into a list of
// phases -- one Gauss-Seidel colour pass, one Jacobi pass, one fused
// residual+restriction, one prolongation, the coarsest dense solve -- and
// the kernel walks that list, every block taking a grid-stride share of
// each phase and meeting the others at a grid barrier before the next.
// This replaces one kernel launch per phase (hundreds per cycle, most of
// them on coarse levels of a few thousand rows, where launch latency and
// the ramp of a short grid dominate) by one launch per cycle.
//
// The grid barrier spins with an iteration limit: on expiry it sets an
// error flag and the kernel returns, so a barrier can never hang the GPU;
// the host reads the flag after the cycle. The cooperative launch
// guarantees that all blocks are co-resident, so in correct operation the
// limit is never reached.
#pragma once

#include <cuda_runtime.h>

namespace fvm {
namespace dev {

enum PhaseOp : int {
  kPhaseGS = 0,        // Gauss-Seidel over slices [a, b) of `level`
  kPhaseJacobi = 1,    // Jacobi over all rows; a = 0: x -> tmp, a = 1: tmp -> x
  kPhaseRestrict = 2,  // coarse b = restricted fine residual, coarse x = 0
  kPhaseProlong = 3,   // fine x += coarse x
  kPhaseDense = 4,     // coarsest x = -Ainv b
};

struct Phase {
  int op;
  int level;
  int a;
  int b;
};

// Level descriptor for the program kernel (values of precision T).
template <class T>
struct ProgLevel {
  int n;
  int nSlices;
  int nCoarse;
  const int* sliceRow;
  const int* sliceRows;
  const int* sliceOff;
  const int* cols;
  const int* rowSlice;
  const T* vals;
  const T* diag;
  T* x;
  T* b;
  T* tmp;
  const int* ci;
  const int* c2fRow;
  const int* c2fCol;
};

struct BarrierState {
  unsigned int count;
  unsigned int generation;
  int error;  // 1: a barrier wait exceeded its iteration limit
  int pad;
};

// Launches the program (cooperatively). grid = 0 picks the co-resident
// maximum. Returns the cudaError of the launch.
template <class T>
cudaError_t run_cycle_program(const Phase* phases, int nPhases, const ProgLevel<T>* levels,
                              const double* coarseInv, int coarseN, BarrierState* barrier,
                              int grid, cudaStream_t st);

// co-resident blocks for the program kernel (blocks per SM x SMs)
template <class T>
int cycle_program_max_grid();

constexpr int kProgramBlock = 512;
constexpr int kClusterBlock = 1024;

// The phase list run by a single thread-block cluster of clusterSize CTAs
// (hardware cluster barrier between phases). coarseInvF, when set, is the
// FP32 copy of the coarsest inverse used by dense phases.
template <class T>
cudaError_t run_cluster_program(const Phase* phases, int nPhases, const ProgLevel<T>* levels,
                                const double* coarseInv, const float* coarseInvF, int coarseN, int clusterSize,
                                cudaStream_t st);
// largest usable cluster size (16 or 8), 0 if none
template <class T>
int cluster_program_size();

}  // namespace dev
}  // namespace fvm
