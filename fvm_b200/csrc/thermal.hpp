// ThermalModel<double> on the GPU: the reference's init / advance /
// updateTime semantics (ThermalModel_impl.h:84-173, 424-456, 472-495) with
// the linearization and the linear solve running as sm_100a kernels.
#pragma once

#include <cuda_runtime.h>

#include <array>
#include <cstdlib>
#include <new>
#include <memory>
#include <string>
#include <vector>

#include "mesh.hpp"
#include "solver.hpp"

namespace fvm {

// Page-locked host memory for the cell fields that cross to the device on
// every solve, so their copies run at the link's full rate; plain heap
// memory where no device is present (the host-only tests).
template <class T>
struct PinnedAllocator {
  using value_type = T;
  PinnedAllocator() = default;
  template <class U>
  PinnedAllocator(const PinnedAllocator<U>&) {}
  T* allocate(size_t n) {
    void* p = nullptr;
    if (n == 0) n = 1;
    if (cudaMallocHost(&p, n * sizeof(T)) == cudaSuccess) return static_cast<T*>(p);
    cudaGetLastError();
    p = std::malloc(n * sizeof(T));
    if (!p) throw std::bad_alloc();
    return static_cast<T*>(p);
  }
  void deallocate(T* p, size_t) {
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) == cudaSuccess && a.type == cudaMemoryTypeHost) {
      cudaFreeHost(p);
    } else {
      cudaGetLastError();
      std::free(p);
    }
  }
  template <class U>
  bool operator==(const PinnedAllocator<U>&) const { return true; }
  template <class U>
  bool operator!=(const PinnedAllocator<U>&) const { return false; }
};
using HostField = std::vector<double, PinnedAllocator<double>>;

enum BcType {
  kBcSpecifiedTemperature = 0,
  kBcSpecifiedHeatFlux = 1,
  kBcSymmetry = 2,
  kBcConvective = 3,
  kBcRadiative = 4,
  kBcMixed = 5,
};

enum CellField {
  kFieldTemperature = 0,
  kFieldConductivity = 1,
  kFieldSource = 2,
  kFieldSpecificHeat = 3,  // rho * cp
  kFieldTemperatureN1 = 4,
};

struct ThermalOptions {
  double relativeTolerance = 1e-8;   // ThermalBC.h:42
  double absoluteTolerance = 1e-16;
  bool transient = false;
  int timeDiscretizationOrder = 1;
  double initialTemperature = 300.0;
  double timeStep = 1e-7;
  // volume-condition constants (ThermalVC)
  double thermalConductivity = 1.0;
  double density = 1.0;
  double specificHeat = 1.0;
  SolverOptions linear;
  ThermalOptions() {
    // ThermalModelOptions::getLinearSolver default: AMG, relTol 0.1, 20 iterations
    linear.relativeTolerance = 1e-1;
    linear.nMaxIterations = 20;
  }
};

struct GroupBC {
  int id = 0;
  BcType type = kBcSpecifiedHeatFlux;
  // specifiedTemperature, specifiedHeatFlux, convectiveCoefficient,
  // farFieldTemperature, surfaceEmissivity (ThermalBC defaults)
  std::array<double, 5> values{{300.0, 0.0, 0.0, 300.0, 1.0}};
};

struct AdvanceReport {
  int iterations = 0;
  int linearIterations = 0;
  double initialNorm = 0;  // of the model's first linear system
  double lastNorm = 0;
  bool converged = false;
  double seconds = 0;      // device time (CUDA events) of the advance call, after the field uploads
  double setupSeconds = 0; // part spent rebuilding matrix + hierarchy
  long long launches = 0;
  int learnedSteps = 0;    // learned corrections tried / kept (all outer iterations)
  int learnedAccepted = 0;
  bool outerOnDevice = false;  // the outer iterations ran as one CUDA graph
};

class ThermalModel {
 public:
  explicit ThermalModel(std::shared_ptr<HostMesh> mesh);
  ~ThermalModel();

  HostMesh& mesh() { return *mesh_; }
  std::vector<GroupBC>& bcs() { return bcs_; }
  GroupBC& bc(int groupId);
  ThermalOptions& options() { return opt_; }
  void optionsChanged() { matrixDirty_ = true; hierarchyDirty_ = true; }
  void bcChanged() { matrixDirty_ = true; hierarchyDirty_ = true; }

  void init();
  void setCellField(int field, const double* values, int count);
  void getCellField(int field, double* out, int count);
  void advance(int niter, AdvanceReport& rep);
  void updateTime();

  // parity hooks: the current linearization (matrix in reference order and
  // rhs) and the AMG hierarchy built from it
  void linearizeOnly(std::vector<double>& diag, std::vector<double>& off,
                     std::vector<double>& b);
  const AmgHierarchy& hierarchy();
  // CUDA-event timings (ms per launch) with an L2 flush before each timed
  // launch: [0] one Gauss-Seidel pass over all colours of level 0 in the
  // configured V-cycle precision, [1] its algorithmic bytes, [2] FP64
  // residual of level 0, [3] its bytes, [4] one full cycle, [5] its bytes,
  // [6] levels, [7] rows of level 0, [8] stored entries of level 0,
  // [9] kernels per cycle, [10] colours of level 0, [11] the face loop of
  // the linearization (k_face_flux), [12] its bytes
  void profile(int reps, double* out);
  // per-level kernel timings of the cycle (AmgHierarchy::profileLevels)
  void profileLevels(int reps, std::vector<double>& out);
  const std::vector<double>& history() const { return history_; }
  // ThermalModel::getHeatFluxIntegral (ThermalModel_impl.h:400-422): sum of
  // the boundary heat flux over a face group, as the last advance() left it
  double heatFluxIntegral(int groupId);
  cudaStream_t stream() const { return stream_; }

  // Independent blocks of self cells (a batch of meshes packed into one
  // model, offsets in cell order, nSeg + 1 entries; empty = one block): the
  // outer loop of advance() then runs until every block meets the
  // tolerances on its own L1 residual norm, relative to its own first one.
  void setSegments(const std::vector<int>& offsets);
  int numSegments() const { return segOff_.empty() ? 0 : (int)segOff_.size() - 1; }
  // per block: first and last outer L1 norm, outer iteration (from 0) at
  // which it first met the tolerances (-1: not yet)
  void segmentStatus(std::vector<double>& first, std::vector<double>& last, std::vector<int>& convergedAt) const;

  // Learned correction used by the AMG solve of advance() (null disables;
  // not owned).
  void setLearned(LearnedCorrection* lc);
  // Runs up to nOuter outer iterations like advance(), each linear system
  // solved to relTol (at most maxCycles cycles) with the configured AMG,
  // and adds this linear system's graph as a training instance of lc with
  // the pairs (residual, error) of the first perSolve iterates of every
  // solve (error = final iterate - iterate). Returns the pairs added.
  int harvest(LearnedCorrection& lc, int nOuter, int perSolve, double relTol, int maxCycles);

 private:
  void ensureDevice();
  void uploadFields();
  void ensureMatrix();
  void linearize();
  void freeDevice();
  // The outer loop of advance() on the device: one CUDA graph whose
  // conditional while node runs linearize, the CG solve (its own while
  // node), the convergence test and, under a conditional if node, the
  // solution update. False (nothing ran) when the graph cannot be built.
  bool advanceOnDevice(int niter, AdvanceReport& rep);
  bool outerGraphUsable() const;
  bool buildAdvanceGraph(int historyCap);
  void releaseAdvanceGraph();
  cudaGraphExec_t gAdvance_ = nullptr;
  bool advanceFailed_ = false;
  // the solver (counted by its builds) and settings the graph was built for
  unsigned long long solverGen_ = 0, advSolverGen_ = 0;
  LinearSolve::LoopKey advKey_{};
  int advHistoryCap_ = 0;
  long long advOuterNodes_ = 0;  // graph nodes per outer iteration besides the CG iterations
  void* dOuter_ = nullptr;       // device: outer-loop state, then the outer norms
  void* hOuter_ = nullptr;       // pinned copy of the same
  long long advPrologueNodes_ = 0;
  // Anderson acceleration of the outer iteration (linear options'
  // outerAcceleration = depth m, 0 off): buffers, the start of a call (state
  // reset, previous iterate = T) and one step after an update (returns at
  // once on the device when *stop is non-zero)
  void ensureAcceleration(int m);
  void releaseAcceleration();
  void accelerationStart(cudaStream_t st);
  void accelerationStep(cudaStream_t st, const int* stop);
  void* dAA_ = nullptr;
  int aaDepth_ = 0, aaCells_ = 0, aaBlocks_ = 0;
  unsigned long long aaGen_ = 0, advAAGen_ = 0;
  int advAADepth_ = 0;

  std::shared_ptr<HostMesh> mesh_;
  std::vector<GroupBC> bcs_;
  ThermalOptions opt_;
  bool initialized_ = false;
  // host fields, self + ghost cells
  HostField T_, k_, src_, rc_, TN1_;
  // a field still holding the uniform value init() gave it is not written
  // on the host: it is filled where it is needed (on the device by a
  // kernel, on the host when only part of it is set or it is read back)
  std::array<bool, 5> uniform_{};
  std::array<double, 5> uniformValue_{};
  HostField& field(int f);
  void materialize(int f);
  bool tDirty_ = true, kDirty_ = true, srcDirty_ = true, rcDirty_ = true, tn1Dirty_ = true;
  bool matrixDirty_ = true, hierarchyDirty_ = true;
  double initialNorm_ = -1;
  int niters_ = 0;
  std::vector<double> history_;

  // device state
  cudaStream_t stream_ = nullptr;
  bool deviceReady_ = false;
  DeviceArena arena_;
  int *dFaceCells_ = nullptr, *dCcRow_ = nullptr, *dCcCol_ = nullptr;
  int *dCfRow_ = nullptr, *dCfCol_ = nullptr, *dBRow_ = nullptr, *dBCol_ = nullptr, *dBColG_ = nullptr;
  int *dBFace_ = nullptr, *dBKind_ = nullptr, *dBIndexOfFace_ = nullptr, *dPerm_ = nullptr;
  double* hPinned_ = nullptr;  // pinned host staging of the face coefficients and diagonal
  size_t hPinnedBytes_ = 0;
  double *dArea_ = nullptr, *dAreaMag_ = nullptr, *dCentroid_ = nullptr, *dVol_ = nullptr;
  double *dGradW_ = nullptr, *dGrad_ = nullptr, *dFlux_ = nullptr, *dCoeff_ = nullptr, *dSec_ = nullptr;
  double *dT_ = nullptr, *dK_ = nullptr, *dSrc_ = nullptr, *dRc_ = nullptr, *dTN1_ = nullptr;
  double *dRhoVdt_ = nullptr, *dBValue_ = nullptr, *dBGhost_ = nullptr, *dDiagOrig_ = nullptr;
  double *dBParam_ = nullptr, *dBGhostDiag_ = nullptr, *dHf_ = nullptr, *dHeatFlux_ = nullptr;
  bool matrixDependsOnT_ = false;  // radiative / mixed conditions: the matrix follows T
  dev::BoundaryData boundaryData() const;
  std::vector<int> boundaryFaces_;       // boundary faces in face order
  std::vector<int> bKindHost_;           // boundary kinds last uploaded
  std::vector<double> bParamHost_;       // and their h / far-field / emissivity
  std::vector<int> entryFace_;           // interior-only CSR entry -> face
  CSR interiorConn_;                     // cellCells restricted to self rows / self columns
  unsigned long long patternKey_ = 0;    // names interiorConn_ for the device-built hierarchy
  AmgHierarchy hier_;
  LearnedCorrection* learned_ = nullptr;
  // blocks of cells with their own convergence test
  std::vector<int> segOff_;
  int* dSegOff_ = nullptr;
  double* dSegNorm_ = nullptr;
  std::vector<double> segFirst_, segLast_;
  std::vector<int> segConvergedAt_;
  bool segmentsConverged();
  std::unique_ptr<LinearSolve> solver_;
};

}  // namespace fvm
