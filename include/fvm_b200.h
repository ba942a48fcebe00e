/*
 * fvm_b200: B200-native replacement for the FVM thermal diffusion + AMG
 * hot path. Plain C ABI: opaque handles, plain pointers and sizes, int
 * status codes (0 = success); the message of the last failure on the
 * calling thread is returned by fvm_last_error().
 *
 * Each entry point names the reference interface it replaces (paths are
 * inside the c-PRIMED/fvm project, src/fvm/src/modules/...).
 *
 * Ownership: input arrays are copied; the library owns device memory;
 * handles are released with the matching *_destroy call.
 * Threading: calls on one handle must be serialised; distinct handles may
 * be used from different threads (each thermal model has its own CUDA
 * stream on the device current at its first advance).
 */
#ifndef FVM_B200_H
#define FVM_B200_H

#ifdef __cplusplus
extern "C" {
#endif

/* status codes */
#define FVM_OK 0
#define FVM_ERR_BAD_ARGUMENT 1
#define FVM_ERR_BAD_MESH 2
#define FVM_ERR_NOT_CONVERGED 3
#define FVM_ERR_NAN 4
#define FVM_ERR_DEVICE 5
#define FVM_ERR_LEARNED_REJECTED 6
#define FVM_ERR_UNSUPPORTED 7
#define FVM_ERR_TOO_LARGE 8

/* boundary condition types (ThermalBC::bcType strings, fvmbase/ThermalModel_impl.h:299-383) */
#define FVM_BC_SPECIFIED_TEMPERATURE 0
#define FVM_BC_SPECIFIED_HEAT_FLUX 1
#define FVM_BC_SYMMETRY 2
#define FVM_BC_CONVECTIVE 3
#define FVM_BC_RADIATIVE 4
#define FVM_BC_MIXED 5

/* cell fields (ThermalFields, fvmbase/ThermalFields.h) */
#define FVM_FIELD_TEMPERATURE 0
#define FVM_FIELD_CONDUCTIVITY 1
#define FVM_FIELD_SOURCE 2
#define FVM_FIELD_SPECIFIC_HEAT 3 /* density * specific heat */
#define FVM_FIELD_TEMPERATURE_N1 4

typedef struct fvm_mesh fvm_mesh;
typedef struct fvm_thermal fvm_thermal;

/* Linear solver settings: LinearSolver fields (fvmbase/LinearSolver.h:19-24)
 * and AMG knobs (fvmbase/AMG.h:74-81), plus this implementation's own. */
typedef struct fvm_linear_options {
  int solver;               /* 0 AMG, 1 CG with AMG preconditioner, 2 BCGStab with AMG */
  int nMaxIterations;
  double relativeTolerance;
  double absoluteTolerance;
  int verbosity;
  int maxCoarseLevels;
  int nPreSweeps;
  int nPostSweeps;
  int coarseGroupSize;
  double weightRatioThreshold;
  int cycleType;            /* 0 V, 1 W, 2 F */
  int smootherType;         /* 0 Gauss-Seidel, 1 Jacobi */
  int scaleCorrections;
  /* additions */
  int smootherOrdering;     /* 0 multicolour (parallel), 1 sequential (reference order, parity runs) */
  int coarsestSize;         /* stop coarsening at this many rows (0: reference rule) */
  int coarseSolver;         /* 0 smooth only (reference), 1 dense FP64 direct solve */
  int precision;            /* 0 FP64, 1 FP32 V-cycle under FP64 refinement */
  int useGraphs;            /* replay each iteration as a CUDA graph */
  int coarseJacobiRows;     /* levels below the finest with at most this many rows smooth with
                               damped Jacobi instead of multicolour Gauss-Seidel (0: never) */
  double jacobiWeight;      /* damping of that Jacobi smoother (default 2/3) */
  int preconditioner;       /* of CG / BCGStab: 0 one AMG cycle, 1 two Jacobi sweeps (JacobiSolver) */
  int autotune;             /* time the smoother launch plans of each SELL-32 level at setup and keep
                               the fastest (plans never change results) */
  int planThreadsPerRow;    /* != 0: use this plan on every SELL-32 level instead (1, 2 or 4 */
  int planBlock;            /*   threads per row; 128 or 256 threads per block, 0 = 256) */
  int setupOnDevice;        /* build the coarse levels on the GPU (parallel pairwise matching and
                               Galerkin kernels) instead of the reference's sequential greedy
                               aggregation; coarse levels then smooth with damped Jacobi. Not the
                               reference's hierarchy: meant for precision = 1 */
  int matchRounds;          /* handshake rounds per level of that matching (default 4) */
  double matchBeta;         /* a neighbour is a matching candidate when its strength is at least
                               this fraction of the row's strongest (default 0.25) */
  int matchPasses;          /* matchings per level: 1 pairs rows, 2 pairs the pairs (aggregates of
                               about 4 rows, half as many levels) */
  int coarsePostSweeps;     /* post-smoothing sweeps on the levels below the finest (-1: nPostSweeps) */
  int planEllRows;          /* != 0: rows per thread (1 or 2) of the Gauss-Seidel pass on ELL-32
                               levels instead of the autotuner's choice (results never change) */
  int chebyshevDegree;      /* > 0: the finest level smooths with a Chebyshev polynomial of this
                               degree in D^-1 A per sweep (one launch per degree) instead of
                               multicolour Gauss-Seidel (0: Gauss-Seidel, the reference's smoother) */
  double chebyshevFraction; /* its interval [fraction * b, b], b the Gershgorin bound (default 0.3) */
  int gsReverse;            /* 1: a multicolour Gauss-Seidel sweep is forward + reverse over the
                               colours (the reference's sweep); 0: forward only (a nonsymmetric
                               preconditioner: for flexible CG or standalone AMG) */
  int patternOnDevice;      /* setupOnDevice: 1 colours and packs a new mesh's finest level on the
                               GPU (the same colouring and packing as the host's), 0 on the host */
  int fuseProlongation;     /* 1: a zero-guess cycle without pre-smoothing folds each prolongation
                               into the level's first post-smoothing pass (bitwise the same result),
                               0: separate prolongation launches */
  int outerOnDevice;        /* 1: a thermal model's advance() runs all its outer iterations (linearize,
                               CG solve, update, convergence test) as one CUDA graph when the solve
                               needs no host step; 0: one host round trip per outer iteration */
  int outerAcceleration;    /* Anderson acceleration of a thermal model's outer iteration, depth 1-5
                               (that many earlier iterates mixed into each new one); 0: off, the
                               reference's plain outer loop */
} fvm_linear_options;

/* ThermalModelOptions (fvmbase/ThermalBC.h:33-67) + volume-condition constants */
typedef struct fvm_thermal_options {
  double relativeTolerance;
  double absoluteTolerance;
  int transient;
  int timeDiscretizationOrder;
  double initialTemperature;
  double timeStep;
  double thermalConductivity;
  double density;
  double specificHeat;
  fvm_linear_options linear;
} fvm_thermal_options;

typedef struct fvm_report {
  int iterations;          /* outer (advance) iterations, or solver iterations */
  int linearIterations;    /* total inner iterations */
  double initialNorm;      /* L1 norm of the first linear system */
  double lastNorm;         /* L1 norm of the last linear system / final residual */
  int converged;
  double seconds;          /* device time, CUDA events from after the upload of the
                              changed cell fields to the end of the call */
  double setupSeconds;     /* host+device time rebuilding matrix and AMG levels */
  long long launches;      /* kernels and copies issued (graph nodes counted per replay) */
  int learnedSteps;        /* learned corrections tried (0 without a learned correction) */
  int learnedAccepted;     /* ... and kept because they lowered the FP64 residual */
  int outerOnDevice;       /* 1: the outer iterations ran as one CUDA graph (linear options'
                              outerOnDevice), 0: one host round trip per outer iteration */
} fvm_report;

/* Reference AMG defaults (fvmbase/AMG.cpp:15-22) and LinearSolver defaults. */
void fvm_default_linear_options(fvm_linear_options* o);
/* ThermalModelOptions defaults; linear = AMG with relTol 0.1, 20 iterations
 * (ThermalModelOptions::getLinearSolver, fvmbase/ThermalBC.h:56-67). */
void fvm_default_thermal_options(fvm_thermal_options* o);

/* Mesh(dimension, nCells, nodes, faceCells, faceNodes, faceNodeCount,
 * faceGroupSize) -- fvmbase/Mesh.cpp:132-247, Python fvmbaseExt.Mesh
 * (fvmbase/Mesh.i:95-120). xyz: 3*nNodes; faceCells: 2*nFaces; faceNodes:
 * all face nodes back to back; groupSize[0] = interior faces, then one
 * entry per boundary group (ids 1..k, type "wall"). */
int fvm_mesh_create(int dim, int nCells, int nNodes, const double* xyz, int nFaces,
                    const int* faceCells, const int* faceNodes, const int* faceNodeCount,
                    int nGroups, const int* groupSize, fvm_mesh** out);
/* FaceGroup id/type of group g (g >= 1), as imported meshes carry them
 * (fvmbase/Mesh.h FaceGroup). */
int fvm_mesh_set_group(fvm_mesh* m, int group, int id, const char* type);

/* Fluent case-file import (importers.FluentReader, the reference's
 * src/modules/importers/FluentReader.cpp: readMesh() :572-611 reads the
 * file, getMeshList() :954-1040 and createMesh :696-952 turn each cell zone
 * into a Mesh). ASCII and binary (single / double precision) sections.
 * Not covered, with FVM_ERR_UNSUPPORTED: periodic face pairs and faces
 * between two cell zones (interfaces). */
typedef struct fvm_fluent fvm_fluent;
int fvm_fluent_read(const char* path, fvm_fluent** out);
/* number of cell zones = length of getMeshList() */
int fvm_fluent_cell_zones(const fvm_fluent* r, int* n);
/* sizes of the mesh of cell zone `zone` (ascending zone id): dim, nCells,
 * nNodes, nFaces, faceNodes entries, face groups (interior + boundary zones) */
int fvm_fluent_mesh_sizes(fvm_fluent* r, int zone, int* out6);
/* its arrays, as fvm_mesh_create takes them: xyz (3 per node), faceCells
 * (2 per face; boundary faces (cell, nCells + k)), faceNodes, faceNodeCount,
 * groupSize, and groupId (Fluent zone id per group, 0 for the interior).
 * Faces: interior zones, then boundary zones, ascending zone id; nodes in
 * first-visit order over the zone's cells and their faces. Null arrays are
 * skipped. */
int fvm_fluent_mesh_arrays(fvm_fluent* r, int zone, double* xyz, int* faceCells, int* faceNodes,
                           int* faceNodeCount, int* groupSize, int* groupId);
/* type name of face group `group` ("interior", then the zones' Fluent types
 * such as "wall" or "velocity-inlet"), NUL-terminated into buf */
int fvm_fluent_group_type(fvm_fluent* r, int zone, int group, char* buf, int cap);
/* getMeshList()[zone]: the mesh, with its boundary groups' ids and types */
int fvm_fluent_mesh_create(fvm_fluent* r, int zone, fvm_mesh** out);
int fvm_fluent_destroy(fvm_fluent* r);
/* out: dim, nCells, nGhost, nNodes, nFaces, nnz(cellCells), nGroups */
int fvm_mesh_sizes(const fvm_mesh* m, int* out7);
/* Mesh::getCellCells + CRConnectivity::getPairToColMapping
 * (fvmbase/Mesh.cpp:479-492, fvmbase/CRConnectivity.cpp:730-790). */
int fvm_mesh_connectivity(const fvm_mesh* m, int* row, int* col, int* pairToCol);
/* MeshMetricsCalculator<double>::init (fvmbase/MeshMetricsCalculator_impl.h:1944-2042) */
int fvm_mesh_geometry(const fvm_mesh* m, double* faceArea, double* faceAreaMag,
                      double* faceCentroid, double* cellCentroid, double* cellVolume);
int fvm_mesh_destroy(fvm_mesh* m);

/* ThermalModel<double>(geomFields, thermalFields, meshes)
 * (fvmbase/ThermalModel.h:28-52). One mesh per model. */
int fvm_thermal_create(fvm_mesh* const* meshes, int nMesh, fvm_thermal** out);
int fvm_thermal_set_options(fvm_thermal* t, const fvm_thermal_options* o);
int fvm_thermal_get_options(const fvm_thermal* t, fvm_thermal_options* o);
/* getBCMap()[groupId]: bcType + FloatVarDict values [specifiedTemperature,
 * specifiedHeatFlux, convectiveCoefficient, farFieldTemperature,
 * surfaceEmissivity] (fvmbase/ThermalBC.h:8-20). values may be null. */
int fvm_thermal_set_bc(fvm_thermal* t, int mesh, int groupId, int bcType, const double* values5);
int fvm_thermal_get_bc(const fvm_thermal* t, int mesh, int groupId, int* bcType, double* values5);
/* ThermalModel::init (fvmbase/ThermalModel_impl.h:84-173) */
int fvm_thermal_init(fvm_thermal* t);
/* thermalFields.<field>[cells] arrays; count = nCells (ghosts take their
 * neighbour's value, temperature ghosts are kept) or nCells + nGhost. */
int fvm_thermal_set_cell_field(fvm_thermal* t, int mesh, int field, const double* values, int count);
int fvm_thermal_get_cell_field(fvm_thermal* t, int mesh, int field, double* out, int count);
/* ThermalModel::advance (fvmbase/ThermalModel_impl.h:424-456) */
int fvm_thermal_advance(fvm_thermal* t, int niter, fvm_report* rep);
/* ThermalModel::updateTime (fvmbase/ThermalModel_impl.h:472-495) */
int fvm_thermal_update_time(fvm_thermal* t);
/* ThermalModel::getHeatFluxIntegral (fvmbase/ThermalModel_impl.h:400-422):
 * sum over the boundary face group of the heat flux the last advance()
 * left (the linearization's boundary flux plus its post-solve update,
 * LinearSystem::postSolve, fvmbase/LinearSystem.cpp:250-263) */
int fvm_thermal_heat_flux_integral(fvm_thermal* t, int mesh, int groupId, double* out);
/* outer L1 norms printed by advance(), one per iteration since init() */
int fvm_thermal_history(const fvm_thermal* t, double* norms, int cap, int* n);
/* The linearization advance() solves (ThermalModel::dumpMatrix content,
 * fvmbase/ThermalModel_impl.h:499-572): diag[nCells], off[nnz of the
 * self-row/self-column cellCells pattern in reference order], b[nCells]
 * in delta form (b = -rhs of the dump). */
int fvm_thermal_linear_system(fvm_thermal* t, double* diag, double* off, double* b, int* nnz);
/* The AMG hierarchy of the current linearization (LinearSystem::createCoarse
 * per level, fvmbase/LinearSystem.cpp:67-248): number of coarse levels,
 * their sizes, and the coarseIndex of each fine level concatenated. */
int fvm_thermal_hierarchy(fvm_thermal* t, int* nLevels, int* sizes, int sizesCap,
                          int* coarseIndex, int ciCap);
/* One level of the AMG hierarchy of the current linearization (no reference
 * counterpart; for tests of the Galerkin products): its matrix as CSR with
 * the diagonal apart, rows numbered as fvm_thermal_hierarchy's coarseIndex
 * numbers them (level 0: reference cell order). Stored zeros are left out.
 * *n and *nnz are always written; the arrays (row: n + 1, the others: cap
 * entries) only when they fit. */
int fvm_thermal_level_matrix(fvm_thermal* t, int level, int* n, int* nnz, int* row, int* col, double* val,
                             double* diag, int cap);
/* Launch plans of the smoother kernels, one per level of the current setup
 * (no reference counterpart): threads per row and threads per block as the
 * autotuner (or the forced plan) chose them; ELL-32 levels report
 * threadsPerRow[l] = -(ELL width) and block[l] = -(rows per thread of
 * their Gauss-Seidel pass). */
int fvm_thermal_launch_plans(fvm_thermal* t, int* nLevels, int* threadsPerRow, int* block, int cap);
/* Measurement hook (no reference counterpart): CUDA-event timings in ms
 * per launch, each launch preceded by a write of 512 MB to flush L2.
 * out[0] one Gauss-Seidel pass over all colours of the finest level in the
 * V-cycle precision, out[1] its algorithmic bytes, out[2] the FP64 finest
 * residual, out[3] its bytes, out[4] one full cycle, out[5] its bytes,
 * out[6] levels, out[7] finest rows, out[8] finest stored entries,
 * out[9] kernels per cycle, out[10] colours of the finest level. */
int fvm_thermal_profile(fvm_thermal* t, int reps, double* out13);
/* Measurement hook (no reference counterpart): per AMG level, CUDA-event
 * times in ms (mean of reps, each launch preceded by a 512 MB write that
 * flushes L2) of the kernels one cycle runs there, in the cycle's
 * precision, with their algorithmic bytes -- 8 doubles per level: rows,
 * stored entries, smoother pass ms, bytes (one damped-Jacobi launch, or one
 * Gauss-Seidel pass over all colours; on a coarsest level with the direct
 * solve, the dense solve), restriction ms, bytes (as the cycle runs it),
 * prolongation ms, bytes. out receives 8 * nLevels doubles when cap allows. */
int fvm_thermal_profile_levels(fvm_thermal* t, int reps, int* nLevels, double* out, int cap);
int fvm_thermal_destroy(fvm_thermal* t);

/* Raw system path (testLinearSolver / MMReader + AMG::solve,
 * src/modules/importers/testLinearSolver.cpp): solves b + A x = 0 for x
 * from x = 0, A given with implicit diagonal (row, col over n rows, diag,
 * off). history receives the L1 norm after each iteration (index 0 =
 * initial), levelSizes the coarse level sizes. */
int fvm_amg_solve_csr(int n, const int* row, const int* col, const double* diag,
                      const double* off, const double* b, double* x,
                      const fvm_linear_options* o, fvm_report* rep, double* history,
                      int historyCap, int* nHistory, int* levelSizes, int levelCap,
                      int* nLevels);
/* Residual of the raw system, host buffers: r = b + A x over n rows
 * (CRMatrix::computeResidual, fvmbase/CRMatrix.h:407-426) and its L1 norm
 * (Array::getOneNorm / MultiField::getOneNorm, fvmbase/Array.h:302-311,
 * fvmbase/MultiField.cpp:216-230). r may be null. */
int fvm_csr_residual(int n, const int* row, const int* col, const double* diag, const double* off,
                     const double* x, const double* b, double* r, double* l1norm);
/* fvm_csr_residual for callers that cannot allocate device memory (no
 * counterpart in the reference, which has no device boundary): every
 * pointer is DEVICE memory owned by the caller (row, col, diag, off, x, b
 * in; r -- may be null -- and the single double *l1norm out), work is
 * enqueued on `stream` (a cudaStream_t; null = default stream) and nothing
 * is allocated: the reduction's block sums live in a fixed 512 KB device
 * array inside the library, so n is limited to 16,777,216 rows (larger n
 * returns FVM_ERR_TOO_LARGE). The first call in each CUDA context (the
 * device's primary context, or a context the caller made current) looks up
 * that array's device address; make it outside any stream capture. After
 * cudaDeviceReset the next call looks the address up again. Calls share
 * the array: calls that overlap on one device race, so serialise them. */
int fvm_csr_residual_device_noalloc(int n, const int* row, const int* col, const double* diag,
                                    const double* off, const double* x, const double* b, double* r,
                                    double* l1norm, void* stream);
/* Host-only AMG setup of the same system (no device needed): coarse sizes
 * and concatenated coarseIndex arrays (CRMatrix::createCoarsening,
 * fvmbase/CRMatrix.h:468-586), plus, when colors != null, the greedy
 * colour of every row of every level (concatenated). */
int fvm_amg_hierarchy_csr(int n, const int* row, const int* col, const double* diag,
                          const double* off, const fvm_linear_options* o, int finestLocalSize,
                          int* nLevels, int* sizes, int sizesCap, int* coarseIndex, int ciCap,
                          int* colors, int colorsCap);

/* Batches (no reference counterpart): independent meshes packed into one
 * model (their disjoint union) solve together; with nSeg blocks of self
 * cells (cellOffsets: nSeg + 1 ascending offsets from 0 to nCells) the
 * outer loop runs until EVERY block meets the tolerances on its own L1
 * residual norm relative to its own first one, instead of the combined
 * norm the reference's multi-mesh ThermalModel tests
 * (fvmbase/MultiField.cpp:216-230). nSeg = 0 restores the combined test. */
int fvm_thermal_set_segments(fvm_thermal* t, int nSeg, const int* cellOffsets);
/* per block: first and last outer L1 norms and the outer iteration (from
 * 0) at which it first met the tolerances (-1: not yet) */
int fvm_thermal_segments(const fvm_thermal* t, int cap, double* firstNorm, double* lastNorm, int* convergedAt);

/* ---- learned correction (no reference counterpart) ----------------------
 * A message-passing network on the finest level's cell graph (width 32,
 * three layers, FP32 weights) predicting the solution error from the FP64
 * residual; used as a flexible step after every AMG refinement iteration
 * of advance(), kept only when it lowers the FP64 L1 residual norm. Trained
 * on the GPU on (residual, error) pairs harvested from the plain solver. */
typedef struct fvm_learned fvm_learned;
fvm_learned* fvm_learned_create(unsigned long long seed);
int fvm_learned_destroy(fvm_learned* l);
int fvm_learned_num_params(void);
int fvm_learned_get_params(const fvm_learned* l, float* out, int cap);
int fvm_learned_set_params(fvm_learned* l, const float* p, int n);
/* runs up to nOuter outer iterations of t (as fvm_thermal_advance), each
 * linear system solved to relTol with at most maxCycles AMG cycles; adds
 * t's finest graph as a training instance with the (residual, error) pairs
 * of the first perSolve iterates of every solve; *nPairs = pairs added */
int fvm_learned_harvest(fvm_learned* l, fvm_thermal* t, int nOuter, int perSolve, double relTol,
                        int maxCycles, int* nPairs);
int fvm_learned_num_pairs(const fvm_learned* l);
/* Adam, steps updates on pairs drawn with the seed; losses (optional,
 * steps entries) gets each step's relative squared error */
int fvm_learned_train(fvm_learned* l, int steps, float lr, unsigned long long seed, double* losses);
/* mean relative squared error over all harvested pairs */
int fvm_learned_evaluate(fvm_learned* l, double* meanLoss);
/* use l in t's solves (null disables); l must outlive its use by t */
int fvm_thermal_set_learned(fvm_thermal* t, fvm_learned* l);
/* The network on a plain CSR graph (implicit diagonal, symmetric
 * couplings), host buffers: out = correction for residual r; and the
 * gradient of the relative squared error against e (grad: num_params
 * floats) with the loss. For checking the kernels against a CPU
 * restatement. */
int fvm_learned_forward_csr(fvm_learned* l, int n, const int* row, const int* col, const double* diag,
                            const double* off, const double* r, double* out);
int fvm_learned_gradient_csr(fvm_learned* l, int n, const int* row, const int* col, const double* diag,
                             const double* off, const double* r, const double* e, float* grad,
                             double* loss);

/* Dense layers of the network (the 64 -> 32 products of the forward pass
 * and of the backward pass) on the tensor cores (on != 0, the default:
 * tcgen05 MMAs reading TF32 operands, FP32 sums) or in FP32 on the CUDA
 * cores (on == 0). Applies to training, evaluation, forward/gradient and
 * the solve. No reference counterpart (the learned correction is new). */
int fvm_learned_set_tensor_cores(fvm_learned* l, int on);
/* Training objective (no reference counterpart): 0 = relative squared
 * error of the predicted error against the pair's error (default), 1 =
 * the residual the correction leaves, |r + A d|^2 / |r|^2 (needs only the
 * pair's residual; A is the instance's matrix). */
int fvm_learned_set_objective(fvm_learned* l, int objective);
/* In the solve the learned step is retired after three tries if fewer than
 * a quarter cut the FP64 residual below f times its value (default 0.5,
 * what pays for the step; 1 keeps any step that lowers it). */
int fvm_learned_set_useful_factor(fvm_learned* l, double f);
/* With the residual objective, the reduction sqrt(mean |r + A d|^2 /
 * |r|^2) the network reached on its pairs at the last evaluation (-1 when
 * not evaluated since training). A solve does not use a network whose
 * reduction is above its useful factor. */
int fvm_learned_residual_factor(const fvm_learned* l, double* factor);
int fvm_learned_tensor_cores(const fvm_learned* l, int* on);
/* Failure-path check of the tensor-core layers' bounded completion wait (no
 * reference counterpart): one CTA allocates TMEM and waits `limit` tries on
 * an mbarrier that nothing signals; *status = 1 when the wait ran out and
 * the kernel set its error flag, released TMEM and returned (the layers'
 * own path on a stuck MMA). The context stays usable. */
int fvm_learned_wait_probe(unsigned limit, int* status);

const char* fvm_last_error(void);

#ifdef __cplusplus
}
#endif

#endif /* FVM_B200_H */
