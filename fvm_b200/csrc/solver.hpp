// GPU AMG hierarchy and linear solvers (AMG standalone, CG and BiCGStab
// with an AMG preconditioner), FP64 or with an FP32 V-cycle under FP64
// iterative refinement. Mirrors the reference's LinearSolver / AMG / CG /
// BCGStab semantics: delta form r = b + A x, L1 residual norms over self
// rows, stop when |r| < absTol or |r|/|r0| < relTol.
#pragma once

#include <cuda_runtime.h>

#include <functional>
#include <map>
#include <mutex>
#include <memory>
#include <vector>

#include "amg_setup.hpp"
#include "kernels.cuh"
#include "learned.hpp"

namespace fvm {

enum CycleType { kVCycle = 0, kWCycle = 1, kFCycle = 2 };
enum SmootherType { kGaussSeidel = 0, kJacobi = 1 };
enum CoarseSolver { kCoarseSmooth = 0, kCoarseDirect = 1 };
enum Precision { kFP64 = 0, kMixed = 1 };
enum SolverKind { kSolverAMG = 0, kSolverCG = 1, kSolverBCGStab = 2, kSolverJacobi = 3 };
enum PreconditionerKind { kPrecAMG = 0, kPrecJacobi = 1 };

struct SolverOptions {
  SolverKind solver = kSolverAMG;
  int nMaxIterations = 100;
  double relativeTolerance = 1e-8;
  double absoluteTolerance = 1e-16;
  int verbosity = 0;
  // AMG knobs (reference AMG.h:74-81 and defaults AMG.cpp:15-22)
  int maxCoarseLevels = 30;
  int nPreSweeps = 0;
  int nPostSweeps = 1;
  int coarseGroupSize = 2;
  double weightRatioThreshold = 0.65;
  CycleType cycleType = kVCycle;
  SmootherType smootherType = kGaussSeidel;
  bool scaleCorrections = true;  // only acts on symmetric systems (never flagged here)
  // additions of this implementation
  SmootherOrdering ordering = kMulticolor;
  int coarsestSize = 0;
  CoarseSolver coarseSolver = kCoarseSmooth;
  Precision precision = kFP64;
  bool useGraphs = true;
  // multicolour Gauss-Seidel levels below the finest with at most this many
  // rows smooth with damped Jacobi (weight jacobiWeight) instead; 0 = never
  int coarseJacobiRows = 0;
  double jacobiWeight = 2.0 / 3.0;
  // preconditioner of CG / BCGStab: one AMG cycle, or two Jacobi sweeps
  // (JacobiSolver::smooth, fvmbase/JacobiSolver.cpp:27-100)
  PreconditionerKind preconditioner = kPrecAMG;
  // smoother launch plans of the SELL-32 levels: autotuned at setup, or one
  // plan forced on every level (planTpr != 0)
  bool autotune = true;
  int planTpr = 0;
  int planBlock = 0;
  // rows per thread of the Gauss-Seidel pass on ELL-32 levels (1 or 2;
  // 0: autotuned)
  int planEllRows = 0;
  // > 0: the finest level smooths with a Chebyshev polynomial of this
  // degree in D^-1 A per sweep (one launch per degree) instead of
  // multicolour Gauss-Seidel; its interval is [fraction * b, b], b the
  // Gershgorin bound of the spectrum
  int chebyshevDegree = 0;
  double chebyshevFraction = 0.3;
  // a multicolour Gauss-Seidel sweep is forward + reverse over the colours
  // (the reference's sweep, AMG.cpp:57-61); false: forward only (C colour
  // passes instead of 2C - 1; a nonsymmetric preconditioner, for flexible CG)
  bool gsReverse = true;
  // Build the coarse levels on the GPU (parallel pairwise matching and
  // Galerkin kernels) instead of the reference's sequential greedy walk on
  // the host; coarse levels then smooth with damped Jacobi. The hierarchy is
  // not the reference's: for the mixed-precision path, whose result is
  // judged by the converged field only.
  bool setupOnDevice = false;
  int matchRounds = 4;          // handshake rounds per level
  double matchBeta = 0.25;      // candidate when strength >= beta * the row's strongest
  int matchPasses = 1;          // matchings per level: 2 pairs the pairs (aggregates of about 4 rows)
  // post-smoothing sweeps on the levels below the finest (-1: nPostSweeps)
  int coarsePostSweeps = -1;
  // GPU-built hierarchies: colour and pack level 0 on the device when the
  // pattern is there (the same colouring and packing as on the host)
  bool patternOnDevice = true;
  // a zero-guess cycle without pre-smoothing folds each prolongation into
  // the level's first post-smoothing pass (bitwise the same result)
  bool fuseProlongation = true;
  // a thermal model's advance() runs all its outer iterations as one CUDA
  // graph when the solve needs no host step (deviceSolvable)
  bool outerOnDevice = true;
  // Anderson acceleration of a thermal model's outer iteration: the depth
  // (pairs of iterates mixed, 1-5); 0 = off, the reference's plain loop
  int outerAcceleration = 0;
  int postSweeps(int l) const { return l > 0 && coarsePostSweeps >= 0 ? coarsePostSweeps : nPostSweeps; }
  // only the finest level is needed (Jacobi solver or preconditioner)
  bool finestOnly() const { return solver == kSolverJacobi || preconditioner == kPrecJacobi; }
};

struct SolveReport {
  double initialNorm = 0;
  double finalNorm = 0;
  int iterations = 0;
  bool converged = false;
  std::vector<double> history;  // L1 norm after each iteration (index 0 = initial)
  int learnedSteps = 0;         // learned corrections tried / kept /
  int learnedAccepted = 0;      // kept with a residual cut that pays for the step
  int learnedUseful = 0;
};

// Device copy of one level.
struct DevLevel {
  int n = 0, nColors = 0, nSlices = 0, nCoarse = 0, maxWidth = 0;
  std::vector<int> colorSliceStart;  // host copy, launch bounds
  int *sliceRow = nullptr, *sliceRows = nullptr, *sliceOff = nullptr, *cols = nullptr;
  int* rowSlice = nullptr;
  double *vals = nullptr, *diag = nullptr;
  float *valsF = nullptr, *diagF = nullptr;
  int *ci = nullptr, *c2fRow = nullptr, *c2fCol = nullptr;
  double *x = nullptr, *b = nullptr, *r = nullptr, *tmp = nullptr;
  float *xF = nullptr, *bF = nullptr, *rF = nullptr, *tmpF = nullptr;
  double* partials = nullptr;
  int nPartials = 0;
  int4* meta = nullptr;  // per slice: first row, rows, entry offset, width
  dev::RowPlan plan;     // launch plan of this level's smoother (SELL-32 levels)
  bool splitRestrict = false;  // residual pass + gather instead of the fused restriction
  int ellWidth = 0;  // > 0: ELL-32 layout (colorSliceStart then holds rows)
  dev::SellView<double> view64() const {
    return {n, sliceRow, sliceRows, sliceOff, cols, vals, diag, meta, ellWidth};
  }
  dev::SellView<float> view32() const {
    return {n, sliceRow, sliceRows, sliceOff, cols, valsF, diagF, meta, ellWidth};
  }
  size_t entries = 0;
};

// Device allocations of one owner. release() keeps the blocks for reuse by
// later alloc() calls of the same size (a rebuilt AMG hierarchy on the same
// mesh asks for the same sizes), so rebuilding does not pay cudaFree /
// cudaMalloc again; the destructor frees everything.
class DeviceArena {
 public:
  ~DeviceArena();
  void* alloc(size_t bytes);
  template <class T>
  T* upload(const std::vector<T>& v) {
    return upload(v.data(), v.size());
  }
  template <class T>
  T* upload(const T* v, size_t count) {
    T* p = (T*)alloc(count * sizeof(T));
    if (count) copy_h2d(p, v, count * sizeof(T));
    return p;
  }
  void release();
  size_t bytes() const { return bytes_; }

 private:
  void copy_h2d(void* d, const void* h, size_t n);
  std::vector<std::pair<void*, size_t>> ptrs_;
  std::multimap<size_t, void*> free_;
  size_t bytes_ = 0;
  std::mutex mu_;  // levels are uploaded from several setup threads
};

// Level-0 input of a hierarchy built on the device: the pattern on the host
// (reference row order, self rows, implicit diagonal) and its values on the
// device.
struct FinestDevice {
  const CSR* conn = nullptr;
  // CSR entry k -> index of its value in offSrc (null: k itself)
  const std::vector<int>* entrySrc = nullptr;
  const double* offSrc = nullptr;  // device
  const double* diag = nullptr;    // device, reference order
  // equal non-zero keys promise the same pattern and entrySrc: the packed
  // level-0 structure (colouring, permutation, slices) is reused
  unsigned long long key = 0;
  bool symmetricPattern = true;
  std::vector<int> segments;  // independent diagonal blocks (a batch)
  // The same pattern on the device, so that it can be coloured and packed
  // there (all null: on the host): cellCells of the self rows (ccRow n + 1
  // offsets, ccCol with ghost columns >= n), each self cell's faces
  // ascending (cfRow, cfCol) and faceCells (2 per face). conn is then the
  // self-column part of cellCells and entrySrc the face behind each entry.
  const int *ccRow = nullptr, *ccCol = nullptr, *cfRow = nullptr, *cfCol = nullptr, *faceCells = nullptr;
};

// Cached level-0 structure of device-built hierarchies (pattern only).
struct FinestPattern {
  unsigned long long key = 0;
  int ordering = 0;
  PackedLevel packed;  // colours, permutation, slices (no columns or values on the host)
  size_t entries = 0;  // packed slots
  DeviceArena arena;
  int *sliceRow = nullptr, *sliceRows = nullptr, *sliceOff = nullptr, *cols = nullptr, *rowSlice = nullptr;
  int *posSrc = nullptr, *iperm = nullptr, *perm = nullptr;
  int4* meta = nullptr;
};

class AmgHierarchy {
 public:
  // levels[0] is the finest matrix in reference order; the hierarchy
  // (reference-exact aggregation) is built, packed and uploaded.
  void build(std::vector<RefLevel>& levels, int finestLocalSize, const SolverOptions& opt);
  // The same hierarchy built on the GPU from a level 0 resident there
  // (opt.setupOnDevice): pairwise matching, Galerkin products and SELL-32
  // packing as kernels; only level 0's colouring is host work, once per
  // pattern. refLevels() is then empty and packed(l) exists for l = 0 only.
  // The coarsest inverse is the build's last GPU work; with deferCheck the
  // call returns while it runs (the host may build graphs meanwhile) and
  // finishBuild() waits for it and checks it, before any solve.
  void buildDevice(const FinestDevice& in, const SolverOptions& opt, bool deferCheck = false);
  void finishBuild();
  bool deviceBuilt() const { return deviceBuilt_; }
  // device-built: reference row -> level-0 row, on the device
  const int* finestPermDevice() const { return deviceBuilt_ && finest_ ? finest_->perm : nullptr; }
  // fine -> coarse index of level l on the host (device-built hierarchies:
  // downloaded; level 0 in reference row order, coarse levels in their own)
  std::vector<int> coarseIndexHost(int l) const;
  // level l's matrix as CSR (diagonal apart, stored zeros left out), rows
  // numbered as coarseIndexHost numbers them
  void levelCsr(int l, std::vector<int>& row, std::vector<int>& col, std::vector<double>& val,
                std::vector<double>& diag) const;
  // Drops the device state and keeps the host-side level objects of this
  // hierarchy as spares: the next build() of a similar hierarchy refills
  // their buffers instead of allocating (and page-faulting) new ones.
  void release();
  // a spare host level object for level l (empty when there is none)
  RefLevel spareLevel(int l);
  // device memory that lives until the next release() (recycled by size)
  void* scratch(size_t bytes);
  // 32 pinned host doubles owned by the hierarchy (one solver at a time)
  double* pinnedScalars();
  AmgHierarchy() = default;
  ~AmgHierarchy();
  AmgHierarchy(const AmgHierarchy&) = delete;
  AmgHierarchy& operator=(const AmgHierarchy&) = delete;

  int numLevels() const { return (int)lv_.size(); }
  const DevLevel& level(int l) const { return lv_[l]; }
  DevLevel& level(int l) { return lv_[l]; }
  const PackedLevel& packed(int l) const { return deviceBuilt_ && l == 0 ? finest_->packed : packed_[l]; }
  const std::vector<RefLevel>& refLevels() const { return ref_; }
  std::vector<int> sizes() const;

  // one cycle on level l of precision T (x, b of each level as stored);
  // xZero: level l's x is zero on entry, so without pre-smoothing its
  // residual is b and the restriction needs no pass over the matrix
  template <class T>
  void cycle(CycleType t, int l, cudaStream_t st, bool xZero = false);
  // xc, ci: the first damped-Jacobi pass takes x = xc[ci] (a prolongation
  // fused into it); x itself is not read
  template <class T>
  void sweeps(int nSweeps, int l, cudaStream_t st, const T* xc = nullptr, const int* ci = nullptr);
  // level l's prolongation (after a zero-guess visit) is fused into its
  // first post-smoothing pass: damped Jacobi, no pre-smoothing
  bool fusedProlong(int l) const;

  // one cycle of the configured type from the finest level (xZero: level
  // 0's x is zero on entry)
  template <class T>
  void runCycle(cudaStream_t st, bool xZero = false);

  // x = z <- M^-1 applied to r (FP64 in/out; runs the cycle in the
  // configured precision): b0 <- r, x0 <- 0, cycle, z <- x0
  void apply(const double* r, double* z, cudaStream_t st);
  // the same cycle, its result left in level 0's x (FP64) or xF (mixed)
  // instead of being copied to z; AMG preconditioner only
  void applyCycle(const double* r, cudaStream_t st);

  const SolverOptions& options() const { return opt_; }

  size_t deviceBytes() const { return arena_.bytes(); }
  // Per level, CUDA-event times (ms, mean of reps, L2 flushed by a write of
  // `flush` before each timed launch) of the cycle's kernels in the
  // configured precision, with their algorithmic bytes; kLevelProfile
  // doubles per level: rows, stored entries, smoother pass (one damped
  // Jacobi launch, or one Gauss-Seidel pass over all colours; the coarsest
  // level with a direct solve: the dense solve) ms and bytes, restriction
  // (as the cycle runs it) ms and bytes, prolongation ms and bytes (0 on
  // the coarsest level).
  static constexpr int kLevelProfile = 8;
  void profileLevels(int reps, void* flush, size_t flushBytes, cudaStream_t st, std::vector<double>& out);
  // algorithmic bytes moved by one cycle (for roofline reporting)
  double cycleBytes() const;
  double fineSweepBytes() const;  // one GS pass over all colours of level 0
  // colour launches of nSweeps multicolour Gauss-Seidel sweeps in a row
  int colourPasses(int colors, int nSweeps) const;
  int kernelsPerCycle() const;

 private:
  SolverOptions opt_;
  std::vector<RefLevel> ref_;
  std::vector<PackedLevel> packed_;
  std::vector<CSR> c2f_;
  // host objects of the previous build, by level, reused by the next one
  std::vector<RefLevel> spareRef_;
  std::vector<PackedLevel> sparePacked_;
  std::vector<CSR> spareC2f_;
  double* pinned_ = nullptr;
  // the coarsest inverse's status, read back into the last pinned scalar,
  // not yet checked
  bool inversePending_ = false;
  int* pendingStatus();
  std::vector<DevLevel> lv_;
  double* coarseInv_ = nullptr;  // dense inverse of the coarsest level
  float* coarseInvF_ = nullptr;  // its FP32 copy for the FP32 cycle
  DeviceArena arena_;
  // level l (of n rows) smooths with damped Jacobi (coarseJacobiRows)
  bool dampedLevel(int l, int n) const;
  // device copy of one packed level (matrix, slice metadata, vectors) and
  // of its transfer to the next coarser level
  void uploadMatrix(const PackedLevel& p, DevLevel& d, bool mixed);
  void uploadTransfer(const PackedLevel& p, DevLevel& d, int nCoarse);
  // device-built hierarchies
  bool deviceBuilt_ = false;
  std::unique_ptr<FinestPattern> finest_;
  cudaStream_t setupStream_ = nullptr;
  void prepareFinestPattern(const FinestDevice& in, int ordering);
  // the same on the device (row-order greedy colouring by fixed-point
  // sweeps, ELL-32 packing); false (nothing kept) when the level needs the
  // host path: more than five colours, no ELL-32 layout, or a mesh whose
  // entries it cannot match to faces
  bool prepareFinestPatternDevice(const FinestDevice& in);
  void allocVectors(DevLevel& d, bool mixed);
  // picks each SELL-32 level's smoother launch plan (autotune or forced)
  void tunePlans();
  // Chebyshev smoother of level 0: coefficients (c1, c2) of each step of
  // one sweep, from the Gershgorin bound of level 0's D^-1 A
  std::vector<double> chebC1_, chebC2_;
  double chebBound_ = 0.0;
  void prepareChebyshev();
  bool chebyshevLevel(int l) const { return l == 0 && !chebC1_.empty(); }
  // one smoother pass of level l with a given plan (what the tuner times)
  void smootherPass(int l, dev::RowPlan plan, cudaStream_t st);
  // level l's residual restricted to level l + 1, fused or split
  void restrictPass(int l, bool split, cudaStream_t st);
};

// nodes of g that no node depends on
bool graph_leaves(cudaGraph_t g, std::vector<cudaGraphNode_t>& leaves);

// Linear solve of the finest system held by the hierarchy: level 0's b is
// the right-hand side, level 0's x the delta (zeroed on entry).
class LinearSolve {
 public:
  explicit LinearSolve(AmgHierarchy& h);
  ~LinearSolve();
  SolveReport solve(cudaStream_t st);
  // Learned correction applied after every refinement iteration of the AMG
  // solve (null disables); not owned.
  void setLearned(LearnedCorrection* lc);
  // AMG iterations to relTol (or maxIter) recording the residual and the
  // iterate of iterations 0..record-1 into rs[q], xs[q] (device, n each);
  // returns how many were recorded. The final iterate stays in level 0's x.
  int solveRecording(cudaStream_t st, double relTol, int maxIter, int record, const std::vector<double*>& rs,
                     const std::vector<double*>& xs, SolveReport& rep);

  // The whole solve can run inside a graph with no host step: CG under the
  // AMG cycle, graphs on, no printing, no active learned step.
  bool deviceSolvable() const;
  // Appends that solve to g after its current leaves (no host copies):
  // afterwards deviceLoopState() holds {iterations, status} (status 1
  // converged, 2 non-finite, 3 iteration limit) and deviceInitialNorm()
  // the L1 norm of the right-hand side. False when a graph call failed (g
  // is then unusable).
  bool appendDeviceSolve(cudaGraph_t g, cudaStream_t st);
  // builds the graph of solveCG's device loop now (when it will be used)
  // rather than in the first solve
  void prebuild(cudaStream_t st);
  const int* deviceLoopState() const { return loopInt_; }
  const double* deviceInitialNorm() const { return history_; }
  long long loopBodyNodes() const { return loopBodyNodes_; }
  // the CG settings a graph from appendDeviceSolve bakes in
  struct LoopKey {
    bool flexible;
    int maxIt;
    double rel, abs;
    bool operator==(const LoopKey& o) const {
      return flexible == o.flexible && maxIt == o.maxIt && rel == o.rel && abs == o.abs;
    }
  };
  LoopKey loopKey() const;

 private:
  bool cgFlexible() const;
  SolveReport solveAMG(cudaStream_t st);
  SolveReport solveCG(cudaStream_t st);
  // CG with the fused iteration, every iteration of one solve inside one
  // CUDA graph (a conditional while node whose condition a device kernel
  // sets from the residual norm): one host synchronisation per solve.
  // Returns false (and is not used again) when the graph cannot be built.
  bool solveCGLoop(cudaStream_t st, bool flexible, SolveReport& rep);
  bool buildCGLoop(cudaStream_t st, bool flexible);
  // appends the CG loop (prologue, while node, epilogue) to g after its
  // current leaves; hostCopies: the epilogue also copies the final norm,
  // the initial norm and the loop state to the pinned host scalars
  bool addCGLoop(cudaGraph_t g, cudaStream_t st, bool flexible, bool hostCopies);
  int historyCap_ = 0;
  cudaGraphExec_t gLoop_ = nullptr;
  bool loopFailed_ = false;
  bool loopFlexible_ = false;
  int loopMaxIt_ = -1;
  double loopRel_ = 0.0, loopAbs_ = 0.0;
  int* loopInt_ = nullptr;       // device: iterations, status
  long long loopBodyNodes_ = 0, loopOtherNodes_ = 0;  // kernels and copies per iteration / per solve
  double* history_ = nullptr;    // device: norms of iterations 0..nMaxIterations
  SolveReport solveBCGStab(cudaStream_t st);
  SolveReport solveJacobi(cudaStream_t st);
  void norm_into(const double* v, double* scalar, cudaStream_t st);
  void dot_into(const double* a, const double* b, double* scalar, cudaStream_t st);
  double fetch(const double* scalar, cudaStream_t st);
  // Runs body on st; with graphs enabled the first call captures it and
  // later calls replay the instantiated graph.
  void run(cudaGraphExec_t& exec, cudaStream_t st, const std::function<void()>& body);
  AmgHierarchy& h_;
  int n_;
  double* work_ = nullptr;    // vectors
  double* scal_ = nullptr;    // device scalars
  double* partials_ = nullptr;
  double* partials2_ = nullptr;  // the fused CG steps' partial sums
  double* hostScal_ = nullptr;  // pinned
  cudaGraphExec_t g1_ = nullptr, g2_ = nullptr, g3_ = nullptr, g4_ = nullptr, g5_ = nullptr;
  LearnedCorrection* learned_ = nullptr;
  // the learned step stays on while it pays: after kLsProbe tries it is
  // retired if fewer than a quarter cut the FP64 L1 residual below the
  // correction's useful factor times its value (default 0.5: the step costs
  // about two V-cycles of the mixed solve: three layers over the finest
  // graph, an SpMV, two dots)
  static constexpr int kLsProbe = 3;
  bool learnedActive_ = true;
  int lsTries_ = 0, lsKept_ = 0;
  void learnedStep(cudaStream_t st, double* x, double* r, double acceptFactor);
  std::map<const void*, long long> nodeCounts_;
  bool graphsFailed_ = false;

 public:
  long long launches = 0;  // kernels + copies enqueued (graph nodes counted per replay)
};

}  // namespace fvm
