// The C ABI (include/fvm_b200.h) over the host mesh, the GPU thermal model
// and the GPU AMG solvers.
#include "../../include/fvm_b200.h"

#include <cuda_runtime.h>

#include <cstring>
#include <map>
#include <memory>
#include <string>

#include "amg_setup.hpp"
#include "mesh.hpp"
#include "learned.hpp"
#include "solver.hpp"
#include "fluent.hpp"
#include "thermal.hpp"

using namespace fvm;

struct fvm_mesh {
  std::shared_ptr<HostMesh> m;
};
struct fvm_thermal {
  std::unique_ptr<ThermalModel> model;
};

struct fvm_learned {
  std::unique_ptr<fvm::LearnedCorrection> lc;
};

namespace fvm {
namespace {
thread_local std::string g_error;
}
void set_last_error(const std::string& msg) { g_error = msg; }
const char* last_error() { return g_error.c_str(); }
}  // namespace fvm

namespace {

template <class F>
int guarded(F f) {
  try {
    f();
    return FVM_OK;
  } catch (const Error& e) {
    set_last_error(e.what());
    return e.status;
  } catch (const std::bad_alloc&) {
    set_last_error("out of host memory");
    return FVM_ERR_TOO_LARGE;
  } catch (const std::exception& e) {
    set_last_error(e.what());
    return FVM_ERR_BAD_ARGUMENT;
  } catch (...) {
    set_last_error("unknown error");
    return FVM_ERR_BAD_ARGUMENT;
  }
}

SolverOptions to_solver(const fvm_linear_options& o) {
  SolverOptions s;
  FVM_REQUIRE(o.solver >= 0 && o.solver <= 3, kBadArgument,
              "solver must be 0 (AMG), 1 (CG), 2 (BCGStab) or 3 (Jacobi)");
  FVM_REQUIRE(o.preconditioner == 0 || o.preconditioner == 1, kBadArgument,
              "preconditioner must be 0 (AMG) or 1 (Jacobi)");
  FVM_REQUIRE(o.cycleType >= 0 && o.cycleType <= 2, kBadArgument, "cycleType must be 0 (V), 1 (W) or 2 (F)");
  FVM_REQUIRE(o.smootherType == 0 || o.smootherType == 1, kBadArgument, "smootherType must be 0 or 1");
  FVM_REQUIRE(o.nMaxIterations >= 0 && o.maxCoarseLevels >= 0 && o.nPreSweeps >= 0 &&
                  o.nPostSweeps >= 0 && o.coarseGroupSize >= 1,
              kBadArgument, "negative iteration/sweep/level count");
  s.solver = (SolverKind)o.solver;
  s.nMaxIterations = o.nMaxIterations;
  s.relativeTolerance = o.relativeTolerance;
  s.absoluteTolerance = o.absoluteTolerance;
  s.verbosity = o.verbosity;
  s.maxCoarseLevels = o.maxCoarseLevels;
  s.nPreSweeps = o.nPreSweeps;
  s.nPostSweeps = o.nPostSweeps;
  s.coarseGroupSize = o.coarseGroupSize;
  s.weightRatioThreshold = o.weightRatioThreshold;
  s.cycleType = (CycleType)o.cycleType;
  s.smootherType = (SmootherType)o.smootherType;
  s.scaleCorrections = o.scaleCorrections != 0;
  s.ordering = o.smootherOrdering == 1 ? kSequential : kMulticolor;
  s.coarsestSize = o.coarsestSize;
  s.coarseSolver = o.coarseSolver == 1 ? kCoarseDirect : kCoarseSmooth;
  s.precision = o.precision == 1 ? kMixed : kFP64;
  s.useGraphs = o.useGraphs != 0;
  FVM_REQUIRE(o.coarseJacobiRows >= 0, kBadArgument, "coarseJacobiRows must be >= 0");
  FVM_REQUIRE(o.jacobiWeight > 0.0 && o.jacobiWeight <= 1.0, kBadArgument, "jacobiWeight must be in (0, 1]");
  s.coarseJacobiRows = o.coarseJacobiRows;
  s.jacobiWeight = o.jacobiWeight;
  s.preconditioner = o.preconditioner == 1 ? kPrecJacobi : kPrecAMG;
  FVM_REQUIRE(o.planThreadsPerRow == 0 || o.planThreadsPerRow == 1 || o.planThreadsPerRow == 2 ||
                  o.planThreadsPerRow == 4,
              kBadArgument, "planThreadsPerRow must be 0, 1, 2 or 4");
  FVM_REQUIRE(o.planBlock == 0 || o.planBlock == 128 || o.planBlock == 256, kBadArgument,
              "planBlock must be 0, 128 or 256");
  s.autotune = o.autotune != 0;
  s.planTpr = o.planThreadsPerRow;
  s.planBlock = o.planBlock;
  FVM_REQUIRE(o.planEllRows >= 0 && o.planEllRows <= 2, kBadArgument, "planEllRows must be 0, 1 or 2");
  s.planEllRows = o.planEllRows;
  FVM_REQUIRE(o.chebyshevDegree >= 0 && o.chebyshevDegree <= 16, kBadArgument,
              "chebyshevDegree must be in [0, 16]");
  FVM_REQUIRE(o.chebyshevFraction > 0.0 && o.chebyshevFraction < 1.0, kBadArgument,
              "chebyshevFraction must be in (0, 1)");
  s.chebyshevDegree = o.chebyshevDegree;
  s.chebyshevFraction = o.chebyshevFraction;
  s.gsReverse = o.gsReverse != 0;
  s.patternOnDevice = o.patternOnDevice != 0;
  s.fuseProlongation = o.fuseProlongation != 0;
  s.outerOnDevice = o.outerOnDevice != 0;
  FVM_REQUIRE(o.outerAcceleration >= 0 && o.outerAcceleration <= 5, kBadArgument,
              "outerAcceleration must be in [0, 5]");
  s.outerAcceleration = o.outerAcceleration;
  FVM_REQUIRE(o.matchRounds >= 1 && o.matchRounds <= 64, kBadArgument, "matchRounds must be in [1, 64]");
  FVM_REQUIRE(o.matchBeta >= 0.0 && o.matchBeta <= 1.0, kBadArgument, "matchBeta must be in [0, 1]");
  s.setupOnDevice = o.setupOnDevice != 0;
  s.matchRounds = o.matchRounds;
  s.matchBeta = o.matchBeta;
  FVM_REQUIRE(o.matchPasses == 1 || o.matchPasses == 2, kBadArgument, "matchPasses must be 1 or 2");
  FVM_REQUIRE(o.coarsePostSweeps >= -1 && o.coarsePostSweeps <= 16, kBadArgument,
              "coarsePostSweeps must be in [-1, 16]");
  s.matchPasses = o.matchPasses;
  s.coarsePostSweeps = o.coarsePostSweeps;
  return s;
}

void from_solver(const SolverOptions& s, fvm_linear_options& o) {
  o.solver = s.solver;
  o.nMaxIterations = s.nMaxIterations;
  o.relativeTolerance = s.relativeTolerance;
  o.absoluteTolerance = s.absoluteTolerance;
  o.verbosity = s.verbosity;
  o.maxCoarseLevels = s.maxCoarseLevels;
  o.nPreSweeps = s.nPreSweeps;
  o.nPostSweeps = s.nPostSweeps;
  o.coarseGroupSize = s.coarseGroupSize;
  o.weightRatioThreshold = s.weightRatioThreshold;
  o.cycleType = s.cycleType;
  o.smootherType = s.smootherType;
  o.scaleCorrections = s.scaleCorrections ? 1 : 0;
  o.smootherOrdering = s.ordering == kSequential ? 1 : 0;
  o.coarsestSize = s.coarsestSize;
  o.coarseSolver = s.coarseSolver == kCoarseDirect ? 1 : 0;
  o.precision = s.precision == kMixed ? 1 : 0;
  o.useGraphs = s.useGraphs ? 1 : 0;
  o.coarseJacobiRows = s.coarseJacobiRows;
  o.jacobiWeight = s.jacobiWeight;
  o.preconditioner = s.preconditioner;
  o.autotune = s.autotune ? 1 : 0;
  o.planThreadsPerRow = s.planTpr;
  o.planBlock = s.planBlock;
  o.setupOnDevice = s.setupOnDevice ? 1 : 0;
  o.matchRounds = s.matchRounds;
  o.matchBeta = s.matchBeta;
  o.matchPasses = s.matchPasses;
  o.coarsePostSweeps = s.coarsePostSweeps;
  o.planEllRows = s.planEllRows;
  o.chebyshevDegree = s.chebyshevDegree;
  o.chebyshevFraction = s.chebyshevFraction;
  o.gsReverse = s.gsReverse ? 1 : 0;
  o.patternOnDevice = s.patternOnDevice ? 1 : 0;
  o.fuseProlongation = s.fuseProlongation ? 1 : 0;
  o.outerOnDevice = s.outerOnDevice ? 1 : 0;
  o.outerAcceleration = s.outerAcceleration;
}

RefLevel level_from_csr(int n, const int* row, const int* col, const double* diag, const double* off) {
  FVM_REQUIRE(n > 0 && row && col && diag && off, kBadArgument, "empty or null matrix");
  FVM_REQUIRE(row[0] == 0, kBadArgument, "row[0] must be 0");
  RefLevel l;
  l.n = n;
  l.conn.nRows = n;
  l.conn.row.assign(row, row + n + 1);
  for (int i = 0; i < n; i++)
    FVM_REQUIRE(row[i + 1] >= row[i], kBadArgument, "row offsets must be non-decreasing");
  const int nnz = row[n];
  l.conn.col.assign(col, col + nnz);
  for (int k = 0; k < nnz; k++)
    FVM_REQUIRE(col[k] >= 0 && col[k] < n, kBadArgument, "column index out of range");
  l.diag.assign(diag, diag + n);
  l.off.assign(off, off + nnz);
  l.symmetricPattern = pattern_is_symmetric(l.conn);
  return l;
}

void fill_report(fvm_report* rep, const SolveReport& s) {
  if (!rep) return;
  std::memset(rep, 0, sizeof(*rep));
  rep->iterations = s.iterations;
  rep->linearIterations = s.iterations;
  rep->initialNorm = s.initialNorm;
  rep->lastNorm = s.finalNorm;
  rep->converged = s.converged ? 1 : 0;
}

}  // namespace

extern "C" {

const char* fvm_last_error(void) { return last_error(); }

void fvm_default_linear_options(fvm_linear_options* o) {
  if (!o) return;
  SolverOptions s;
  from_solver(s, *o);
}

void fvm_default_thermal_options(fvm_thermal_options* o) {
  if (!o) return;
  ThermalOptions t;
  o->relativeTolerance = t.relativeTolerance;
  o->absoluteTolerance = t.absoluteTolerance;
  o->transient = t.transient ? 1 : 0;
  o->timeDiscretizationOrder = t.timeDiscretizationOrder;
  o->initialTemperature = t.initialTemperature;
  o->timeStep = t.timeStep;
  o->thermalConductivity = t.thermalConductivity;
  o->density = t.density;
  o->specificHeat = t.specificHeat;
  from_solver(t.linear, o->linear);
}

int fvm_mesh_create(int dim, int nCells, int nNodes, const double* xyz, int nFaces,
                    const int* faceCells, const int* faceNodes, const int* faceNodeCount,
                    int nGroups, const int* groupSize, fvm_mesh** out) {
  return guarded([&] {
    FVM_REQUIRE(out, kBadArgument, "null output handle");
    *out = nullptr;
    std::shared_ptr<HostMesh> m(make_mesh(dim, nCells, nNodes, xyz, nFaces, faceCells, faceNodes,
                                          faceNodeCount, nGroups, groupSize));
    *out = new fvm_mesh{m};
  });
}

struct fvm_fluent {
  std::unique_ptr<FluentCase> file;
  std::map<int, FluentMeshArrays> meshes;
  const FluentMeshArrays& mesh(int zone) {
    auto it = meshes.find(zone);
    if (it == meshes.end()) it = meshes.emplace(zone, file->mesh(zone)).first;
    return it->second;
  }
};

int fvm_fluent_read(const char* path, fvm_fluent** out) {
  return guarded([&] {
    FVM_REQUIRE(path && out, kBadArgument, "null argument");
    *out = nullptr;
    std::unique_ptr<fvm_fluent> r(new fvm_fluent);
    r->file.reset(new FluentCase(path));
    *out = r.release();
  });
}

int fvm_fluent_cell_zones(const fvm_fluent* r, int* n) {
  return guarded([&] {
    FVM_REQUIRE(r && n, kBadArgument, "null argument");
    *n = r->file->numCellZones();
  });
}

int fvm_fluent_mesh_sizes(fvm_fluent* r, int zone, int* out) {
  return guarded([&] {
    FVM_REQUIRE(r && out, kBadArgument, "null argument");
    const FluentMeshArrays& m = r->mesh(zone);
    out[0] = m.dim;
    out[1] = m.nCells;
    out[2] = (int)(m.xyz.size() / 3);
    out[3] = (int)m.faceNodeCount.size();
    out[4] = (int)m.faceNodes.size();
    out[5] = (int)m.groupSize.size();
  });
}

int fvm_fluent_mesh_arrays(fvm_fluent* r, int zone, double* xyz, int* faceCells, int* faceNodes,
                           int* faceNodeCount, int* groupSize, int* groupId) {
  return guarded([&] {
    FVM_REQUIRE(r, kBadArgument, "null argument");
    const FluentMeshArrays& m = r->mesh(zone);
    if (xyz) std::copy(m.xyz.begin(), m.xyz.end(), xyz);
    if (faceCells) std::copy(m.faceCells.begin(), m.faceCells.end(), faceCells);
    if (faceNodes) std::copy(m.faceNodes.begin(), m.faceNodes.end(), faceNodes);
    if (faceNodeCount) std::copy(m.faceNodeCount.begin(), m.faceNodeCount.end(), faceNodeCount);
    if (groupSize) std::copy(m.groupSize.begin(), m.groupSize.end(), groupSize);
    if (groupId) std::copy(m.groupId.begin(), m.groupId.end(), groupId);
  });
}

int fvm_fluent_group_type(fvm_fluent* r, int zone, int group, char* buf, int cap) {
  return guarded([&] {
    FVM_REQUIRE(r && buf && cap > 0, kBadArgument, "null argument");
    const FluentMeshArrays& m = r->mesh(zone);
    FVM_REQUIRE(group >= 0 && group < (int)m.groupType.size(), kBadArgument, "no such face group");
    const std::string& t = m.groupType[group];
    FVM_REQUIRE((int)t.size() < cap, kBadArgument, "buffer too small for the group type");
    std::memcpy(buf, t.c_str(), t.size() + 1);
  });
}

int fvm_fluent_mesh_create(fvm_fluent* r, int zone, fvm_mesh** out) {
  return guarded([&] {
    FVM_REQUIRE(r && out, kBadArgument, "null argument");
    *out = nullptr;
    const FluentMeshArrays& m = r->mesh(zone);
    std::shared_ptr<HostMesh> hm(make_mesh(m.dim, m.nCells, (int)(m.xyz.size() / 3), m.xyz.data(),
                                           (int)m.faceNodeCount.size(), m.faceCells.data(), m.faceNodes.data(),
                                           m.faceNodeCount.data(), (int)m.groupSize.size(), m.groupSize.data()));
    bool symmetry = false;
    for (size_t g = 1; g < m.groupSize.size(); g++) {
      hm->groups[g].id = m.groupId[g];
      hm->groups[g].type = m.groupType[g];
      symmetry = symmetry || m.groupType[g] == "symmetry";
    }
    if (symmetry) hm->build();  // ghost centroids depend on the group type
    *out = new fvm_mesh{hm};
  });
}

int fvm_fluent_destroy(fvm_fluent* r) {
  delete r;
  return FVM_OK;
}

int fvm_mesh_set_group(fvm_mesh* h, int group, int id, const char* type) {
  return guarded([&] {
    FVM_REQUIRE(h && type, kBadArgument, "null argument");
    HostMesh& m = *h->m;
    FVM_REQUIRE(group >= 1 && group < (int)m.groups.size(), kBadArgument, "no such boundary group");
    const std::string t(type);
    const bool geomChange = (t == "symmetry") != (m.groups[group].type == "symmetry");
    m.groups[group].id = id;
    m.groups[group].type = t;
    if (geomChange) m.build();  // ghost centroids depend on the group type
  });
}

int fvm_mesh_sizes(const fvm_mesh* h, int* out) {
  return guarded([&] {
    FVM_REQUIRE(h && out, kBadArgument, "null argument");
    const HostMesh& m = *h->m;
    out[0] = m.dim;
    out[1] = m.nCells;
    out[2] = m.nGhost;
    out[3] = m.nNodes;
    out[4] = m.nFaces;
    out[5] = m.cellCells.nnz();
    out[6] = (int)m.groups.size();
  });
}

int fvm_mesh_connectivity(const fvm_mesh* h, int* row, int* col, int* pairToCol) {
  return guarded([&] {
    FVM_REQUIRE(h, kBadArgument, "null mesh");
    const HostMesh& m = *h->m;
    if (row) std::memcpy(row, m.cellCells.row.data(), sizeof(int) * m.cellCells.row.size());
    if (col) std::memcpy(col, m.cellCells.col.data(), sizeof(int) * m.cellCells.col.size());
    if (pairToCol) std::memcpy(pairToCol, m.pairToCol.data(), sizeof(int) * m.pairToCol.size());
  });
}

int fvm_mesh_geometry(const fvm_mesh* h, double* fa, double* fam, double* fc, double* cc, double* vol) {
  return guarded([&] {
    FVM_REQUIRE(h, kBadArgument, "null mesh");
    const HostMesh& m = *h->m;
    if (fa) std::memcpy(fa, m.faceArea.data(), sizeof(double) * m.faceArea.size());
    if (fam) std::memcpy(fam, m.faceAreaMag.data(), sizeof(double) * m.faceAreaMag.size());
    if (fc) std::memcpy(fc, m.faceCentroid.data(), sizeof(double) * m.faceCentroid.size());
    if (cc) std::memcpy(cc, m.cellCentroid.data(), sizeof(double) * m.cellCentroid.size());
    if (vol) std::memcpy(vol, m.cellVolume.data(), sizeof(double) * m.cellVolume.size());
  });
}

int fvm_mesh_destroy(fvm_mesh* h) {
  delete h;
  return FVM_OK;
}

int fvm_thermal_create(fvm_mesh* const* meshes, int nMesh, fvm_thermal** out) {
  return guarded([&] {
    FVM_REQUIRE(out && meshes, kBadArgument, "null argument");
    *out = nullptr;
    FVM_REQUIRE(nMesh == 1, kUnsupported, "one mesh per thermal model");
    FVM_REQUIRE(meshes[0], kBadArgument, "null mesh");
    std::unique_ptr<ThermalModel> t(new ThermalModel(meshes[0]->m));
    *out = new fvm_thermal{std::move(t)};
  });
}

int fvm_thermal_set_options(fvm_thermal* h, const fvm_thermal_options* o) {
  return guarded([&] {
    FVM_REQUIRE(h && o, kBadArgument, "null argument");
    ThermalOptions& t = h->model->options();
    FVM_REQUIRE(!o->transient || o->timeStep > 0, kBadArgument, "timeStep must be positive");
    t.relativeTolerance = o->relativeTolerance;
    t.absoluteTolerance = o->absoluteTolerance;
    t.transient = o->transient != 0;
    t.timeDiscretizationOrder = o->timeDiscretizationOrder;
    t.initialTemperature = o->initialTemperature;
    t.timeStep = o->timeStep;
    t.thermalConductivity = o->thermalConductivity;
    t.density = o->density;
    t.specificHeat = o->specificHeat;
    t.linear = to_solver(o->linear);
    h->model->optionsChanged();
  });
}

int fvm_thermal_get_options(const fvm_thermal* h, fvm_thermal_options* o) {
  return guarded([&] {
    FVM_REQUIRE(h && o, kBadArgument, "null argument");
    const ThermalOptions& t = h->model->options();
    o->relativeTolerance = t.relativeTolerance;
    o->absoluteTolerance = t.absoluteTolerance;
    o->transient = t.transient ? 1 : 0;
    o->timeDiscretizationOrder = t.timeDiscretizationOrder;
    o->initialTemperature = t.initialTemperature;
    o->timeStep = t.timeStep;
    o->thermalConductivity = t.thermalConductivity;
    o->density = t.density;
    o->specificHeat = t.specificHeat;
    from_solver(t.linear, o->linear);
  });
}

int fvm_thermal_set_bc(fvm_thermal* h, int mesh, int groupId, int bcType, const double* values) {
  return guarded([&] {
    FVM_REQUIRE(h, kBadArgument, "null model");
    FVM_REQUIRE(mesh == 0, kBadArgument, "mesh index out of range");
    FVM_REQUIRE(bcType >= 0 && bcType <= 5, kBadArgument, "unknown bcType");
    GroupBC& b = h->model->bc(groupId);
    if (b.type != (BcType)bcType) h->model->bcChanged();
    b.type = (BcType)bcType;
    if (values)
      for (int i = 0; i < 5; i++) b.values[i] = values[i];
  });
}

int fvm_thermal_heat_flux_integral(fvm_thermal* h, int mesh, int groupId, double* out) {
  return guarded([&] {
    FVM_REQUIRE(h && out, kBadArgument, "null argument");
    FVM_REQUIRE(mesh == 0, kBadArgument, "mesh index out of range");
    *out = h->model->heatFluxIntegral(groupId);
  });
}

int fvm_thermal_get_bc(const fvm_thermal* h, int mesh, int groupId, int* bcType, double* values) {
  return guarded([&] {
    FVM_REQUIRE(h, kBadArgument, "null model");
    FVM_REQUIRE(mesh == 0, kBadArgument, "mesh index out of range");
    const GroupBC& b = h->model->bc(groupId);
    if (bcType) *bcType = b.type;
    if (values)
      for (int i = 0; i < 5; i++) values[i] = b.values[i];
  });
}

int fvm_thermal_init(fvm_thermal* h) {
  return guarded([&] {
    FVM_REQUIRE(h, kBadArgument, "null model");
    h->model->init();
  });
}

int fvm_thermal_set_cell_field(fvm_thermal* h, int mesh, int field, const double* values, int count) {
  return guarded([&] {
    FVM_REQUIRE(h && values, kBadArgument, "null argument");
    FVM_REQUIRE(mesh == 0, kBadArgument, "mesh index out of range");
    h->model->setCellField(field, values, count);
  });
}

int fvm_thermal_get_cell_field(fvm_thermal* h, int mesh, int field, double* out, int count) {
  return guarded([&] {
    FVM_REQUIRE(h && out, kBadArgument, "null argument");
    FVM_REQUIRE(mesh == 0, kBadArgument, "mesh index out of range");
    h->model->getCellField(field, out, count);
  });
}

int fvm_thermal_advance(fvm_thermal* h, int niter, fvm_report* rep) {
  return guarded([&] {
    FVM_REQUIRE(h, kBadArgument, "null model");
    FVM_REQUIRE(niter >= 0, kBadArgument, "niter must be non-negative");
    AdvanceReport r;
    h->model->advance(niter, r);
    if (rep) {
      rep->iterations = r.iterations;
      rep->linearIterations = r.linearIterations;
      rep->initialNorm = r.initialNorm;
      rep->lastNorm = r.lastNorm;
      rep->converged = r.converged ? 1 : 0;
      rep->seconds = r.seconds;
      rep->setupSeconds = r.setupSeconds;
      rep->launches = r.launches;
      rep->learnedSteps = r.learnedSteps;
      rep->learnedAccepted = r.learnedAccepted;
      rep->outerOnDevice = r.outerOnDevice ? 1 : 0;
    }
  });
}

int fvm_thermal_update_time(fvm_thermal* h) {
  return guarded([&] {
    FVM_REQUIRE(h, kBadArgument, "null model");
    h->model->updateTime();
  });
}

int fvm_thermal_history(const fvm_thermal* h, double* norms, int cap, int* n) {
  return guarded([&] {
    FVM_REQUIRE(h && n, kBadArgument, "null argument");
    const std::vector<double>& hist = h->model->history();
    *n = (int)hist.size();
    if (norms)
      for (int i = 0; i < (int)hist.size() && i < cap; i++) norms[i] = hist[i];
  });
}

int fvm_thermal_linear_system(fvm_thermal* h, double* diag, double* off, double* b, int* nnz) {
  return guarded([&] {
    FVM_REQUIRE(h, kBadArgument, "null model");
    std::vector<double> d, o, bb;
    h->model->linearizeOnly(d, o, bb);
    if (nnz) *nnz = (int)o.size();
    if (diag) std::memcpy(diag, d.data(), sizeof(double) * d.size());
    if (off) std::memcpy(off, o.data(), sizeof(double) * o.size());
    if (b) std::memcpy(b, bb.data(), sizeof(double) * bb.size());
  });
}

static void export_hierarchy(const std::vector<RefLevel>& lv, int* nLevels, int* sizes, int sizesCap,
                             int* coarseIndex, int ciCap) {
  const int L = (int)lv.size();
  if (nLevels) *nLevels = L - 1;
  int pos = 0;
  for (int l = 1; l < L; l++) {
    if (sizes && l - 1 < sizesCap) sizes[l - 1] = lv[l].n;
    const std::vector<int>& ci = lv[l - 1].coarseIndex;
    for (size_t i = 0; i < ci.size() && coarseIndex; i++, pos++)
      if (pos < ciCap) coarseIndex[pos] = ci[i];
  }
}

int fvm_thermal_hierarchy(fvm_thermal* h, int* nLevels, int* sizes, int sizesCap, int* coarseIndex,
                          int ciCap) {
  return guarded([&] {
    FVM_REQUIRE(h, kBadArgument, "null model");
    const AmgHierarchy& hier = h->model->hierarchy();
    if (!hier.deviceBuilt()) {
      export_hierarchy(hier.refLevels(), nLevels, sizes, sizesCap, coarseIndex, ciCap);
      return;
    }
    const int L = hier.numLevels();
    if (nLevels) *nLevels = L - 1;
    int pos = 0;
    for (int l = 1; l < L; l++) {
      if (sizes && l - 1 < sizesCap) sizes[l - 1] = hier.level(l).n;
      if (!coarseIndex) continue;
      const std::vector<int> ci = hier.coarseIndexHost(l - 1);
      for (size_t i = 0; i < ci.size(); i++, pos++)
        if (pos < ciCap) coarseIndex[pos] = ci[i];
    }
  });
}

int fvm_thermal_level_matrix(fvm_thermal* h, int level, int* n, int* nnz, int* row, int* col, double* val,
                             double* diag, int cap) {
  return guarded([&] {
    FVM_REQUIRE(h && n && nnz, kBadArgument, "null argument");
    const AmgHierarchy& hier = h->model->hierarchy();
    FVM_REQUIRE(level >= 0 && level < hier.numLevels(), kBadArgument, "no such level");
    std::vector<int> r, c;
    std::vector<double> v, d;
    hier.levelCsr(level, r, c, v, d);
    *n = (int)d.size();
    *nnz = (int)c.size();
    if (row && (int)r.size() <= cap + 1) std::copy(r.begin(), r.end(), row);
    if (col && (int)c.size() <= cap) std::copy(c.begin(), c.end(), col);
    if (val && (int)v.size() <= cap) std::copy(v.begin(), v.end(), val);
    if (diag && (int)d.size() <= cap) std::copy(d.begin(), d.end(), diag);
  });
}

int fvm_thermal_launch_plans(fvm_thermal* h, int* nLevels, int* threadsPerRow, int* block, int cap) {
  return guarded([&] {
    FVM_REQUIRE(h && nLevels, kBadArgument, "null argument");
    const AmgHierarchy& hier = h->model->hierarchy();
    *nLevels = hier.numLevels();
    for (int l = 0; l < hier.numLevels() && l < cap; l++) {
      const DevLevel& d = hier.level(l);
      if (threadsPerRow) threadsPerRow[l] = d.ellWidth ? -d.ellWidth : d.plan.tpr;
      if (block) block[l] = d.ellWidth ? -d.plan.ellRows : d.plan.block;
    }
  });
}

int fvm_thermal_profile(fvm_thermal* h, int reps, double* out) {
  return guarded([&] {
    FVM_REQUIRE(h && out, kBadArgument, "null argument");
    h->model->profile(reps, out);
  });
}

int fvm_thermal_profile_levels(fvm_thermal* h, int reps, int* nLevels, double* out, int cap) {
  return guarded([&] {
    FVM_REQUIRE(h && nLevels, kBadArgument, "null argument");
    std::vector<double> v;
    h->model->profileLevels(reps, v);
    *nLevels = (int)(v.size() / AmgHierarchy::kLevelProfile);
    if (out && (int)v.size() <= cap) std::copy(v.begin(), v.end(), out);
  });
}

int fvm_thermal_destroy(fvm_thermal* h) {
  delete h;
  return FVM_OK;
}

int fvm_csr_residual(int n, const int* row, const int* col, const double* diag, const double* off,
                     const double* x, const double* b, double* r, double* l1norm) {
  return guarded([&] {
    FVM_REQUIRE(x && b && l1norm, kBadArgument, "null argument");
    RefLevel l = level_from_csr(n, row, col, diag, off);  // validates the pattern
    const int nnz = l.conn.nnz();
    const int np = dev::csr_residual_blocks(n);
    DeviceArena arena;
    int* dRow = arena.upload(l.conn.row);
    int* dCol = arena.upload(l.conn.col);
    double* dDiag = arena.upload(l.diag);
    double* dOff = arena.upload(l.off);
    std::vector<double> hx(x, x + n), hb(b, b + n);
    double* dX = arena.upload(hx);
    double* dB = arena.upload(hb);
    double* dR = (double*)arena.alloc(sizeof(double) * (size_t)n);
    double* dP = (double*)arena.alloc(sizeof(double) * (size_t)(np + 1));
    (void)nnz;
    dev::csr_residual(n, dRow, dCol, dDiag, dOff, dX, dB, dR, dP, 0);
    dev::csr_residual_finish(np, dP, dP + np, 0);
    if (cudaMemcpy(l1norm, dP + np, sizeof(double), cudaMemcpyDeviceToHost) != cudaSuccess)
      throw Error(kDeviceError, "copy of the residual norm failed");
    if (r && cudaMemcpy(r, dR, sizeof(double) * (size_t)n, cudaMemcpyDeviceToHost) != cudaSuccess)
      throw Error(kDeviceError, "copy of the residual failed");
  });
}

int fvm_amg_hierarchy_csr(int n, const int* row, const int* col, const double* diag, const double* off,
                          const fvm_linear_options* o, int finestLocalSize, int* nLevels, int* sizes,
                          int sizesCap, int* coarseIndex, int ciCap, int* colors, int colorsCap) {
  return guarded([&] {
    FVM_REQUIRE(o, kBadArgument, "null options");
    const SolverOptions s = to_solver(*o);
    std::vector<RefLevel> levels(1);
    levels[0] = level_from_csr(n, row, col, diag, off);
    HierarchyOptions ho;
    ho.maxCoarseLevels = s.maxCoarseLevels;
    ho.groupSize = s.coarseGroupSize;
    ho.weightRatioThreshold = s.weightRatioThreshold;
    ho.coarsestSize = s.coarsestSize;
    ho.finestLocalSize = finestLocalSize > 0 ? finestLocalSize : n;
    std::vector<CSR> c2f;
    build_hierarchy(levels, ho, c2f);
    export_hierarchy(levels, nLevels, sizes, sizesCap, coarseIndex, ciCap);
    if (colors) {
      int pos = 0;
      for (const RefLevel& l : levels) {
        std::vector<int> c;
        multicolor(l.conn, c, l.symmetricPattern);
        for (int v : c) {
          if (pos < colorsCap) colors[pos] = v;
          pos++;
        }
      }
    }
  });
}

int fvm_amg_solve_csr(int n, const int* row, const int* col, const double* diag, const double* off,
                      const double* b, double* x, const fvm_linear_options* o, fvm_report* rep,
                      double* history, int historyCap, int* nHistory, int* levelSizes, int levelCap,
                      int* nLevels) {
  return guarded([&] {
    FVM_REQUIRE(o && b && x, kBadArgument, "null argument");
    const SolverOptions s = to_solver(*o);
    std::vector<RefLevel> levels(1);
    levels[0] = level_from_csr(n, row, col, diag, off);
    AmgHierarchy hier;
    hier.build(levels, n, s);
    const int L = hier.numLevels();
    if (nLevels) *nLevels = L - 1;
    for (int l = 1; l < L && levelSizes; l++)
      if (l - 1 < levelCap) levelSizes[l - 1] = hier.level(l).n;
    cudaStream_t st;
    if (cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess)
      throw Error(kDeviceError, "cannot create a CUDA stream");
    SolveReport sr;
    try {
      const PackedLevel& p0 = hier.packed(0);
      std::vector<double> bp(n);
      for (int i = 0; i < n; i++) bp[p0.perm[i]] = b[i];
      DevLevel& d = hier.level(0);
      if (cudaMemcpy(d.b, bp.data(), sizeof(double) * n, cudaMemcpyHostToDevice) != cudaSuccess)
        throw Error(kDeviceError, "copy of b failed");
      cudaEvent_t e0, e1;
      cudaEventCreate(&e0);
      cudaEventCreate(&e1);
      cudaEventRecord(e0, st);
      {
        LinearSolve ls(hier);
        sr = ls.solve(st);
        if (rep) {
          fill_report(rep, sr);
          rep->launches = ls.launches;
        }
      }
      cudaEventRecord(e1, st);
      cudaEventSynchronize(e1);
      float ms = 0;
      cudaEventElapsedTime(&ms, e0, e1);
      if (rep) rep->seconds = ms * 1e-3;
      cudaEventDestroy(e0);
      cudaEventDestroy(e1);
      std::vector<double> xp(n);
      if (cudaMemcpy(xp.data(), d.x, sizeof(double) * n, cudaMemcpyDeviceToHost) != cudaSuccess)
        throw Error(kDeviceError, "copy of x failed");
      for (int i = 0; i < n; i++) x[i] = xp[p0.perm[i]];
    } catch (...) {
      cudaStreamDestroy(st);
      throw;
    }
    cudaStreamDestroy(st);
    if (nHistory) *nHistory = (int)sr.history.size();
    for (size_t i = 0; history && i < sr.history.size() && (int)i < historyCap; i++)
      history[i] = sr.history[i];
  });
}


// ---- learned correction ------------------------------------------------------
namespace {
// A CSR graph packed in natural order (one colour) and uploaded, for the
// network test hooks.
struct CsrGraph {
  fvm::DeviceArena arena;
  fvm::nn::Graph g;
  int n = 0;
  CsrGraph(int n_, const int* row, const int* col, const double* diag, const double* off) {
    using namespace fvm;
    RefLevel l = level_from_csr(n_, row, col, diag, off);
    PackedLevel p;
    pack_level(l, kSequential, p);
    n = n_;
    std::vector<int> rs(n);
    std::vector<int4> meta(p.sliceRow.size());
    for (size_t s = 0; s < p.sliceRow.size(); s++) {
      for (int k = 0; k < p.sliceRows[s]; k++) rs[p.sliceRow[s] + k] = (int)s;
      meta[s] = make_int4(p.sliceRow[s], p.sliceRows[s], p.sliceOff[s], (p.sliceOff[s + 1] - p.sliceOff[s]) / 32);
    }
    g.a.n = n;
    g.a.cols = arena.upload(p.cols);
    g.a.vals = arena.upload(p.vals);
    g.a.diag = arena.upload(p.diag);
    g.a.meta = arena.upload(meta);
    g.rowSlice = arena.upload(rs);
    g.nSlices = (int)p.sliceRow.size();
    g.entries = (long long)p.cols.size();
  }
};
}  // namespace

int fvm_thermal_set_segments(fvm_thermal* t, int nSeg, const int* cellOffsets) {
  return guarded([&] {
    FVM_REQUIRE(t, kBadArgument, "null model");
    FVM_REQUIRE(nSeg >= 0 && (nSeg == 0 || cellOffsets), kBadArgument, "segments: null offsets");
    std::vector<int> off;
    if (nSeg > 0) off.assign(cellOffsets, cellOffsets + nSeg + 1);
    t->model->setSegments(off);
  });
}

int fvm_thermal_segments(const fvm_thermal* t, int cap, double* firstNorm, double* lastNorm, int* convergedAt) {
  return guarded([&] {
    FVM_REQUIRE(t, kBadArgument, "null model");
    std::vector<double> f, l;
    std::vector<int> c;
    t->model->segmentStatus(f, l, c);
    FVM_REQUIRE(cap >= (int)f.size(), kBadArgument, "segments: capacity below the number of segments");
    for (size_t s = 0; s < f.size(); s++) {
      if (firstNorm) firstNorm[s] = f[s];
      if (lastNorm) lastNorm[s] = l[s];
      if (convergedAt) convergedAt[s] = c[s];
    }
  });
}

fvm_learned* fvm_learned_create(unsigned long long seed) {
  fvm_learned* l = nullptr;
  const int rc = guarded([&] {
    l = new fvm_learned;
    l->lc.reset(new LearnedCorrection(seed));
  });
  if (rc != 0) {
    delete l;
    return nullptr;
  }
  return l;
}

int fvm_learned_destroy(fvm_learned* l) {
  return guarded([&] { delete l; });
}

int fvm_learned_num_params(void) { return nn::kParams; }

int fvm_learned_get_params(const fvm_learned* l, float* out, int cap) {
  return guarded([&] {
    FVM_REQUIRE(l && out && cap >= nn::kParams, kBadArgument, "null argument or capacity below num_params");
    const std::vector<float> p = l->lc->params();
    std::copy(p.begin(), p.end(), out);
  });
}

int fvm_learned_set_params(fvm_learned* l, const float* p, int n) {
  return guarded([&] {
    FVM_REQUIRE(l && p && n == nn::kParams, kBadArgument, "null argument or wrong parameter count");
    l->lc->setParams(std::vector<float>(p, p + n));
  });
}

int fvm_learned_harvest(fvm_learned* l, fvm_thermal* t, int nOuter, int perSolve, double relTol, int maxCycles,
                        int* nPairs) {
  return guarded([&] {
    FVM_REQUIRE(l && t, kBadArgument, "null argument");
    const int k = t->model->harvest(*l->lc, nOuter, perSolve, relTol, maxCycles);
    if (nPairs) *nPairs = k;
  });
}

int fvm_learned_num_pairs(const fvm_learned* l) { return l ? l->lc->numPairs() : 0; }

int fvm_learned_train(fvm_learned* l, int steps, float lr, unsigned long long seed, double* losses) {
  return guarded([&] {
    FVM_REQUIRE(l, kBadArgument, "null argument");
    l->lc->train(steps, lr, seed, losses, 0);
  });
}

int fvm_learned_evaluate(fvm_learned* l, double* meanLoss) {
  return guarded([&] {
    FVM_REQUIRE(l && meanLoss, kBadArgument, "null argument");
    *meanLoss = l->lc->evaluate(0);
  });
}

int fvm_thermal_set_learned(fvm_thermal* t, fvm_learned* l) {
  return guarded([&] {
    FVM_REQUIRE(t, kBadArgument, "null model");
    t->model->setLearned(l ? l->lc.get() : nullptr);
  });
}

int fvm_learned_forward_csr(fvm_learned* l, int n, const int* row, const int* col, const double* diag,
                            const double* off, const double* r, double* out) {
  return guarded([&] {
    FVM_REQUIRE(l && r && out, kBadArgument, "null argument");
    CsrGraph cg(n, row, col, diag, off);
    DeviceArena tmp;
    double* dr = tmp.upload(std::vector<double>(r, r + n));
    double* dOut = (double*)tmp.alloc(sizeof(double) * (size_t)n);
    double* scal = (double*)tmp.alloc(sizeof(double) * 8);
    l->lc->prepare(n, cg.g.entries);
    l->lc->apply(cg.g, dr, dOut, scal, 0);
    if (cudaMemcpy(out, dOut, sizeof(double) * (size_t)n, cudaMemcpyDeviceToHost) != cudaSuccess)
      throw Error(kDeviceError, "copy of the network output failed");
    l->lc->checkApplyStatus();
  });
}

int fvm_learned_gradient_csr(fvm_learned* l, int n, const int* row, const int* col, const double* diag,
                             const double* off, const double* r, const double* e, float* grad, double* loss) {
  return guarded([&] {
    FVM_REQUIRE(l && r && e && grad && loss, kBadArgument, "null argument");
    CsrGraph cg(n, row, col, diag, off);
    DeviceArena tmp;
    double* dr = tmp.upload(std::vector<double>(r, r + n));
    double* de = tmp.upload(std::vector<double>(e, e + n));
    float* dg = (float*)tmp.alloc(sizeof(float) * nn::kParams);
    double* scal = (double*)tmp.alloc(sizeof(double) * 8);
    nn::Workspace ws;
    ws.allocate(n, true, cg.g.entries);
    ws.tensorCores = l->lc->tensorCores();
    nn::forward_backward(cg.g, l->lc->deviceParams(), dr, de, dg, scal + 4, ws, scal, 0);
    if (cudaMemcpy(grad, dg, sizeof(float) * nn::kParams, cudaMemcpyDeviceToHost) != cudaSuccess ||
        cudaMemcpy(loss, scal + 4, sizeof(double), cudaMemcpyDeviceToHost) != cudaSuccess)
      throw Error(kDeviceError, "copy of the gradient failed");
    ws.checkStatus();
  });
}

int fvm_learned_set_tensor_cores(fvm_learned* l, int on) {
  return guarded([&] {
    FVM_REQUIRE(l, kBadArgument, "null argument");
    l->lc->setTensorCores(on != 0);
  });
}

int fvm_learned_set_useful_factor(fvm_learned* l, double f) {
  return guarded([&] {
    FVM_REQUIRE(l, kBadArgument, "null argument");
    l->lc->setUsefulFactor(f);
  });
}

int fvm_learned_residual_factor(const fvm_learned* l, double* factor) {
  return guarded([&] {
    FVM_REQUIRE(l && factor, kBadArgument, "null argument");
    *factor = l->lc->residualFactor();
  });
}

int fvm_learned_set_objective(fvm_learned* l, int objective) {
  return guarded([&] {
    FVM_REQUIRE(l, kBadArgument, "null argument");
    l->lc->setObjective(objective);
  });
}

int fvm_learned_wait_probe(unsigned limit, int* status) {
  return guarded([&] {
    FVM_REQUIRE(status, kBadArgument, "null argument");
    FVM_REQUIRE(limit >= 1 && limit <= (1u << 22), kBadArgument, "limit must be in [1, 2^22]");
    *status = nn::tc_wait_probe(limit);
  });
}

int fvm_learned_tensor_cores(const fvm_learned* l, int* on) {
  return guarded([&] {
    FVM_REQUIRE(l && on, kBadArgument, "null argument");
    *on = l->lc->tensorCores() ? 1 : 0;
  });
}

}  // extern "C"
