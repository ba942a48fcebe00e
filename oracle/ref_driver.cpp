// C ABI over the reference FVM solver, compiled from the reference's own
// sources (see oracle/Makefile) into oracle/_ref/libfvmref.so.
//
// TEST INFRASTRUCTURE ONLY. This file is the harness that lets the parity
// tests and the CPU-baseline leg of bench.py drive the *unmodified*
// reference code path (Mesh 7-argument constructor, MeshMetricsCalculator,
// ThermalModel<double>::advance, AMG/CG/BCGStab) with the same arrays that
// the CUDA path receives, and read back what the reference computed. The
// product never links or loads it.
//
// Reference entry points driven here (paths inside the reference project):
//   src/fvm/src/modules/fvmbase/Mesh.cpp:132-247            Mesh(dim,nCells,...)
//   src/fvm/src/modules/fvmbase/MeshMetricsCalculator_impl.h:1944-2042 init()
//   src/fvm/src/modules/fvmbase/ThermalModel_impl.h:84-173,424-456 init/advance
//   src/fvm/src/modules/fvmbase/AMG.cpp:150-282              createCoarseLevels/solve
//   src/fvm/src/modules/fvmbase/LinearSystem.cpp:40-248      initSolve/createCoarse
//   src/fvm/src/modules/importers/MMReader.cpp:79-184        getLS()
//   src/fvm/src/modules/importers/FluentReader.cpp:954-     getMeshList()
//
// A few private members of AMG, ThermalModel and CRMatrix are reached
// through pointers-to-member formed in explicit template instantiations
// (the one context where C++ permits naming private members), so the
// reference headers are compiled exactly as the reference compiles them.

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <iostream>
#include <map>
#include <memory>
#include <set>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

#include "Mesh.h"
#include "GeomFields.h"
#include "ThermalFields.h"
#include "MeshMetricsCalculator.h"
#include "MeshMetricsCalculator_impl.h"
#include "ThermalModel.h"
#include "ThermalModel_impl.h"
#include "AMG.h"
#include "GradientModel.h"
#include "CG.h"
#include "BCGStab.h"
#include "JacobiSolver.h"
#include "LinearSystem.h"
#include "MultiFieldMatrix.h"
#include "CRMatrix.h"
#include "MMReader.h"
#include "FluentReader.h"

namespace {

// --- access to private members -------------------------------------------
template <class Tag>
struct Stolen {
  static typename Tag::type ptr;
};
template <class Tag>
typename Tag::type Stolen<Tag>::ptr;
template <class Tag, typename Tag::type P>
struct Robber {
  struct Filler {
    Filler() { Stolen<Tag>::ptr = P; }
  };
  static Filler filler;
};
template <class Tag, typename Tag::type P>
typename Robber<Tag, P>::Filler Robber<Tag, P>::filler;

typedef ThermalModel<double> TModel;
struct AmgCycle { typedef void (AMG::*type)(AMG::CycleType, int); };
struct AmgCreate { typedef void (AMG::*type)(); };
struct AmgFinest { typedef LinearSystem* AMG::*type; };
struct AmgCoarse { typedef vector<shared_ptr<LinearSystem> > AMG::*type; };
struct AmgTotal { typedef int AMG::*type; };
struct TmImpl { typedef shared_ptr<TModel::Impl> TModel::*type; };
struct ImplIters { typedef int TModel::Impl::*type; };
struct ImplInitial { typedef MFRPtr TModel::Impl::*type; };
struct CrmBoundary { typedef Array<bool> CRMatrix<double, double, double>::*type; };
template struct Robber<AmgCycle, &AMG::cycle>;
template struct Robber<AmgCreate, &AMG::createCoarseLevels>;
template struct Robber<AmgFinest, &AMG::_finestLinearSystem>;
template struct Robber<AmgCoarse, &AMG::_coarseLinearSystems>;
template struct Robber<AmgTotal, &AMG::_totalIterations>;
template struct Robber<TmImpl, &TModel::_impl>;
template struct Robber<ImplIters, &TModel::Impl::_niters>;
template struct Robber<ImplInitial, &TModel::Impl::_initialNorm>;
template struct Robber<CrmBoundary, &CRMatrix<double, double, double>::_isBoundary>;

void amgCycle(AMG& a, AMG::CycleType t, int l) { (a.*Stolen<AmgCycle>::ptr)(t, l); }
void amgCreate(AMG& a) { (a.*Stolen<AmgCreate>::ptr)(); }
LinearSystem*& amgFinest(AMG& a) { return a.*Stolen<AmgFinest>::ptr; }
vector<shared_ptr<LinearSystem> >& amgCoarse(AMG& a) { return a.*Stolen<AmgCoarse>::ptr; }
TModel::Impl& tmImpl(TModel& m) { return *(m.*Stolen<TmImpl>::ptr); }
int& implIters(TModel::Impl& i) { return i.*Stolen<ImplIters>::ptr; }
MFRPtr& implInitialNorm(TModel::Impl& i) { return i.*Stolen<ImplInitial>::ptr; }
const Array<bool>& crmBoundary(const CRMatrix<double, double, double>& m) {
  return m.*Stolen<CrmBoundary>::ptr;
}

std::string g_err;

// Silences std::cout (the reference reports progress there) for the
// lifetime of the object by setting the stream's fail state.
struct QuietCout {
  std::ios_base::iostate saved;
  QuietCout() : saved(std::cout.rdstate()) { std::cout.setstate(std::ios_base::failbit); }
  ~QuietCout() { std::cout.clear(saved); }
};

typedef CRMatrix<double, double, double> DMatrix;
typedef Vector<double, 3> VecD3;

// L1 norm of a single-field MultiField, as MultiField::getOneNorm computes it
double oneNorm(const MultiField& mf) {
  MFRPtr n = mf.getOneNorm();
  const Field& f = *mf.getArrayIndex(0).first;
  return dynamic_cast<const Array<double>&>((*n)[f])[0];
}

const DMatrix& onlyMatrix(LinearSystem& ls, MultiField::ArrayIndex& idx) {
  MultiField& b = ls.getB();
  idx = b.getArrayIndex(0);
  return dynamic_cast<const DMatrix&>(ls.getMatrix().getMatrix(idx, idx));
}

// Copies the interior block of a CRMatrix (rows < nSelf, all columns) out.
void exportCR(const DMatrix& m, int nRows, int* rowOut, int* colOut, double* diagOut,
              double* offOut) {
  const CRConnectivity& c = m.getConnectivity();
  const Array<int>& row = c.getRow();
  const Array<int>& col = c.getCol();
  const Array<double>& d = const_cast<DMatrix&>(m).getDiag();
  const Array<double>& o = const_cast<DMatrix&>(m).getOffDiag();
  if (rowOut)
    for (int i = 0; i <= nRows; i++) rowOut[i] = row[i];
  if (colOut)
    for (int k = 0; k < row[nRows]; k++) colOut[k] = col[k];
  if (offOut)
    for (int k = 0; k < row[nRows]; k++) offOut[k] = o[k];
  if (diagOut)
    for (int i = 0; i < nRows; i++) diagOut[i] = d[i];
}

struct RefModel {
  Mesh* mesh = nullptr;
  MeshList meshes;
  GeomFields geom{"geom"};
  ThermalFields tf{"therm"};
  MeshMetricsCalculator<double>* metrics = nullptr;
  ThermalModel<double>* model = nullptr;
  AMG* amg = nullptr;
  CG* cg = nullptr;
  BCGStab* bcg = nullptr;
  JacobiSolver* jac = nullptr;
  std::vector<double> history;  // outer rNorm per advance iteration
  ~RefModel() {
    // the reference caches least-squares gradient matrices in a static map
    // keyed by Mesh*; drop this mesh's entry so that a later mesh allocated
    // at the same address does not pick it up
    if (mesh) GradientModelBase::clearGradientMatrix(*mesh);
    delete model;
    delete metrics;
    delete amg;
    delete cg;
    delete bcg;
    delete jac;
    delete mesh;
  }
};

template <class F>
int guarded(F f) {
  try {
    f();
    return 0;
  } catch (CException& e) {
    g_err = e.what();
  } catch (std::exception& e) {
    g_err = e.what();
  } catch (...) {
    g_err = "unknown exception";
  }
  return 1;
}

}  // namespace

extern "C" {

const char* ref_last_error() { return g_err.c_str(); }

// ---------------------------------------------------------------------------
// MatrixMarket known-answer path (testLinearSolver.cpp): read the system with
// MMReader, export it, and run the reference AMG cycle by cycle so that the
// full-precision L1 residual after every cycle can be returned.
// ---------------------------------------------------------------------------
int ref_mm_read(const char* matFile, const char* rhsFile, int* nRows, int* nnz,
                int* rowOut, int* colOut, double* diagOut, double* offOut, double* bOut) {
  return guarded([&] {
    QuietCout quiet;
    MMReader reader(matFile, rhsFile);
    shared_ptr<LinearSystem> ls(reader.getLS());
    MultiField::ArrayIndex idx(0, 0);
    const DMatrix& m = onlyMatrix(*ls, idx);
    const int n = m.getConnectivity().getRowDim();
    *nRows = n;
    *nnz = m.getConnectivity().getRow()[n];
    exportCR(m, n, rowOut, colOut, diagOut, offOut);
    if (bOut) {
      const Array<double>& b = dynamic_cast<const Array<double>&>(ls->getB()[idx]);
      for (int i = 0; i < n; i++) bOut[i] = b[i];
    }
  });
}

// Runs the reference AMG on a CSR system given in the reference's own
// layout (implicit diagonal, delta form r = b + A x). Returns the coarse
// level sizes and the L1 residual after each cycle (hist[0] = initial).
// opts: [maxCoarseLevels, nPreSweeps, nPostSweeps, coarseGroupSize,
//        cycleType, smootherType, nMaxIterations] ; dopts: [weightRatioThreshold,
//        relativeTolerance, absoluteTolerance]
int ref_amg_csr(int n, const int* row, const int* col, const double* diag,
                const double* off, const double* b, const int* opts,
                const double* dopts, double* xOut, int* nLevels, int* levelSizes,
                double* hist, int* nHist, int* coarseIndexOut, int coarseIndexCap) {
  return guarded([&] {
    StorageSite site(n, 0);
    CRConnectivity conn(site, site);
    conn.initCount();
    for (int i = 0; i < n; i++) conn.addCount(i, row[i + 1] - row[i]);
    conn.finishCount();
    for (int i = 0; i < n; i++)
      for (int k = row[i]; k < row[i + 1]; k++) conn.add(i, col[k]);
    conn.finishAdd();
    shared_ptr<DMatrix> m(new DMatrix(conn));
    Field field("x");
    MultiField::ArrayIndex idx(&field, &site);
    shared_ptr<Array<double> > x(new Array<double>(n));
    x->zero();
    LinearSystem ls;
    ls.getX().addArray(idx, x);
    ls.getMatrix().addMatrix(idx, idx, m);
    ls.initAssembly();
    for (int i = 0; i < n; i++) m->getDiag()[i] = diag[i];
    for (int k = 0; k < row[n]; k++) m->getOffDiag()[k] = off[k];
    Array<double>& bb = dynamic_cast<Array<double>&>(ls.getB()[idx]);
    for (int i = 0; i < n; i++) bb[i] = b[i];
    ls.initSolve();

    AMG amg;
    amg.maxCoarseLevels = opts[0];
    amg.nPreSweeps = opts[1];
    amg.nPostSweeps = opts[2];
    amg.coarseGroupSize = opts[3];
    amg.cycleType = (AMG::CycleType)opts[4];
    amg.smootherType = (AMG::SmootherType)opts[5];
    amg.nMaxIterations = opts[6];
    amg.weightRatioThreshold = dopts[0];
    amg.relativeTolerance = dopts[1];
    amg.absoluteTolerance = dopts[2];
    amg.verbosity = 0;

    // AMG::solve, unrolled so that each cycle's residual is observable
    amgFinest(amg) = &ls;
    amgCreate(amg);
    *nLevels = (int)amgCoarse(amg).size();
    int ciPos = 0;
    for (int l = 0; l < *nLevels; l++) {
      LinearSystem& c = *amgCoarse(amg)[l];
      levelSizes[l] = c.getMatrix().getSize();
      LinearSystem& f = (l == 0) ? ls : *amgCoarse(amg)[l - 1];
      MultiField& ciF = f.getCoarseIndex();
      const Array<int>& ci = dynamic_cast<const Array<int>&>(ciF[ciF.getArrayIndex(0)]);
      const int nf = (l == 0) ? n : f.getMatrix().getSize();
      for (int i = 0; i < nf && coarseIndexOut && ciPos < coarseIndexCap; i++)
        coarseIndexOut[ciPos++] = ci[i];
    }
    const MultiFieldMatrix& fm = ls.getMatrix();
    fm.computeResidual(ls.getDelta(), ls.getB(), ls.getResidual());
    const double r0 = oneNorm(ls.getResidual());
    int h = 0;
    hist[h++] = r0;
    if (!(r0 < amg.absoluteTolerance)) {
      for (int i = 1; i < amg.nMaxIterations; i++) {
                amgCycle(amg, amg.cycleType, 0);
        fm.computeResidual(ls.getDelta(), ls.getB(), ls.getResidual());
        const double rn = oneNorm(ls.getResidual());
        hist[h++] = rn;
        if (rn < amg.absoluteTolerance || rn / r0 < amg.relativeTolerance) break;
      }
    }
    *nHist = h;
    if (xOut) {
      const Array<double>& d = dynamic_cast<const Array<double>&>(ls.getDelta()[idx]);
      for (int i = 0; i < n; i++) xOut[i] = d[i];
    }
  });
}

// ---------------------------------------------------------------------------
// Fluent mesh import (FluentReader): exports the first cell zone's mesh as
// the arrays the Mesh 7-argument constructor takes, plus group ids/types.
// Call once with null outputs to get sizes, then again with buffers.
// ---------------------------------------------------------------------------
int ref_fluent_read(const char* path, int* sizes /*dim,nCells,nNodes,nFaces,nFaceNodes,nGroups*/,
                    double* xyz, int* faceCells, int* faceNodes, int* faceNodeCount,
                    int* groupSize, int* groupId, char* groupTypes /*nGroups*32*/) {
  return guarded([&] {
    QuietCout quiet;
    FluentReader reader(path);
    reader.readMesh();
    MeshList ml = reader.getMeshList();
    if (ml.empty()) throw CException("no mesh");
    Mesh& mesh = *ml[0];
    const StorageSite& cells = mesh.getCells();
    const StorageSite& faces = mesh.getFaces();
    const StorageSite& nodes = mesh.getNodes();
    const CRConnectivity& fc = mesh.getAllFaceCells();
    const CRConnectivity& fn = mesh.getAllFaceNodes();
    std::vector<const FaceGroup*> groups;
    for (const FaceGroupPtr& g : mesh.getAllFaceGroups()) groups.push_back(g.get());
    sizes[0] = mesh.getDimension();
    sizes[1] = cells.getSelfCount();
    sizes[2] = nodes.getCount();
    sizes[3] = faces.getCount();
    sizes[4] = fn.getRow()[faces.getCount()];
    sizes[5] = (int)groups.size();
    if (!xyz) return;
    const Array<VecD3>& coords = mesh.getNodeCoordinates();
    for (int i = 0; i < nodes.getCount(); i++)
      for (int d = 0; d < 3; d++) xyz[3 * i + d] = coords[i][d];
    int p = 0;
    for (int f = 0; f < faces.getCount(); f++) {
      faceCells[2 * f] = fc(f, 0);
      faceCells[2 * f + 1] = fc(f, 1);
      faceNodeCount[f] = fn.getCount(f);
      for (int j = 0; j < fn.getCount(f); j++) faceNodes[p++] = fn(f, j);
    }
    for (size_t g = 0; g < groups.size(); g++) {
      groupSize[g] = groups[g]->site.getCount();
      groupId[g] = groups[g]->id;
      std::strncpy(groupTypes + 32 * g, groups[g]->groupType.c_str(), 31);
      groupTypes[32 * g + 31] = 0;
      if (g > 0 && groups[g]->site.getOffset() != groups[g - 1]->site.getOffset() + groups[g - 1]->site.getCount())
        throw CException("face groups are not contiguous");
    }
    for (Mesh* m : ml) delete m;
  });
}

// ---------------------------------------------------------------------------
// ThermalModel<double> driven through the Mesh 7-argument constructor.
// ---------------------------------------------------------------------------
void* ref_thermal_create(int dim, int nCells, int nNodes, const double* xyz, int nFaces,
                         const int* faceCells, const int* faceNodes, const int* faceNodeCount,
                         int nGroups, const int* groupSize, const int* groupId,
                         const char* groupTypes /* nGroups*32 or null */) {
  RefModel* r = new RefModel();
  int rc = guarded([&] {
    Array<VecD3> nodes(nNodes);
    for (int i = 0; i < nNodes; i++)
      for (int d = 0; d < 3; d++) nodes[i][d] = xyz[3 * i + d];
    Array<int> fcA(2 * nFaces);
    for (int i = 0; i < 2 * nFaces; i++) fcA[i] = faceCells[i];
    int nfn = 0;
    for (int f = 0; f < nFaces; f++) nfn += faceNodeCount[f];
    Array<int> fnA(nfn);
    for (int i = 0; i < nfn; i++) fnA[i] = faceNodes[i];
    Array<int> fncA(nFaces);
    for (int f = 0; f < nFaces; f++) fncA[f] = faceNodeCount[f];
    Array<int> gsA(nGroups);
    for (int g = 0; g < nGroups; g++) gsA[g] = groupSize[g];
    r->mesh = new Mesh(dim, nCells, nodes, fcA, fnA, fncA, gsA);
    // the 7-argument constructor numbers boundary groups 1..k as "wall";
    // imported meshes carry their own ids and types
    if (groupId || groupTypes) {
      int g = 1;
      for (const FaceGroupPtr& fg : r->mesh->getBoundaryFaceGroups()) {
        FaceGroup& w = const_cast<FaceGroup&>(*fg);
        if (groupId) const_cast<int&>(w.id) = groupId[g];
        if (groupTypes) w.groupType = std::string(groupTypes + 32 * g);
        g++;
      }
    }
    r->meshes.push_back(r->mesh);
    r->metrics = new MeshMetricsCalculator<double>(r->geom, r->meshes);
    r->metrics->init();
    r->model = new ThermalModel<double>(r->geom, r->tf, r->meshes);
  });
  if (rc) {
    delete r;
    return nullptr;
  }
  return r;
}

void ref_thermal_destroy(void* h) { delete (RefModel*)h; }

// bcType: 0 SpecifiedTemperature, 1 SpecifiedHeatFlux, 2 Symmetry,
//         3 Convective, 4 Radiative, 5 Mixed
// vals: [specifiedTemperature, specifiedHeatFlux, convectiveCoefficient,
//        farFieldTemperature, surfaceEmissivity]
int ref_thermal_set_bc(void* h, int groupId, int bcType, const double* vals) {
  RefModel* r = (RefModel*)h;
  return guarded([&] {
    static const char* types[] = {"SpecifiedTemperature", "SpecifiedHeatFlux", "Symmetry",
                                  "Convective", "Radiative", "Mixed"};
    auto& bcMap = r->model->getBCMap();
    if (bcMap.find(groupId) == bcMap.end()) throw CException("no such boundary group");
    ThermalBC<double>& bc = *bcMap[groupId];
    bc.bcType = types[bcType];
    static const char* names[] = {"specifiedTemperature", "specifiedHeatFlux",
                                  "convectiveCoefficient", "farFieldTemperature",
                                  "surfaceEmissivity"};
    for (int i = 0; i < 5; i++) bc.find(names[i])->second = FloatVal<double>(vals[i]);
  });
}

// Options mirror ThermalModelOptions plus the linear solver.
// iopts: [solver(0 AMG, 1 CG+AMG, 2 BCGStab+AMG, 3 JacobiSolver,
//         4 CG+JacobiSolver, 5 BCGStab+JacobiSolver), maxCoarseLevels, nPreSweeps,
//         nPostSweeps, coarseGroupSize, cycleType, smootherType,
//         nMaxIterations, transient, linearVerbosity]
// dopts: [outer relTol, outer absTol, linear relTol, linear absTol,
//         weightRatioThreshold, initialTemperature, timeStep,
//         thermalConductivity(vc), density(vc), specificHeat(vc)]
int ref_thermal_set_options(void* h, const int* iopts, const double* dopts) {
  RefModel* r = (RefModel*)h;
  return guarded([&] {
    ThermalModelOptions<double>& o = r->model->getOptions();
    delete r->amg;
    delete r->cg;
    delete r->bcg;
    delete r->jac;
    r->amg = new AMG();
    r->cg = nullptr;
    r->bcg = nullptr;
    r->jac = nullptr;
    AMG& a = *r->amg;
    a.maxCoarseLevels = iopts[1];
    a.nPreSweeps = iopts[2];
    a.nPostSweeps = iopts[3];
    a.coarseGroupSize = iopts[4];
    a.cycleType = (AMG::CycleType)iopts[5];
    a.smootherType = (AMG::SmootherType)iopts[6];
    a.weightRatioThreshold = dopts[4];
    a.verbosity = 0;
    LinearSolver* ls = r->amg;
    LinearSolver* pre = r->amg;
    if (iopts[0] >= 3) {
      r->jac = new JacobiSolver();
      r->jac->verbosity = 0;
      pre = ls = r->jac;
    }
    if (iopts[0] == 1 || iopts[0] == 4) {
      r->cg = new CG();
      r->cg->preconditioner = pre;
      ls = r->cg;
    } else if (iopts[0] == 2 || iopts[0] == 5) {
      r->bcg = new BCGStab();
      r->bcg->preconditioner = pre;
      ls = r->bcg;
    }
    ls->nMaxIterations = iopts[7];
    ls->relativeTolerance = dopts[2];
    ls->absoluteTolerance = dopts[3];
    ls->verbosity = iopts[9];
    o.linearSolver = ls;
    o.transient = iopts[8] != 0;
    o.relativeTolerance = dopts[0];
    o.absoluteTolerance = dopts[1];
    o.find("initialTemperature")->second = FloatVal<double>(dopts[5]);
    o.find("timeStep")->second = FloatVal<double>(dopts[6]);
    for (auto& vcp : r->model->getVCMap()) {
      vcp.second->find("thermalConductivity")->second = FloatVal<double>(dopts[7]);
      vcp.second->find("density")->second = FloatVal<double>(dopts[8]);
      vcp.second->find("specificHeat")->second = FloatVal<double>(dopts[9]);
    }
  });
}

int ref_thermal_init(void* h) {
  RefModel* r = (RefModel*)h;
  return guarded([&] { r->model->init(); });
}

// field: 0 temperature, 1 conductivity, 2 source, 3 specificHeat (rho*cp),
//        4 temperatureN1. Arrays cover self + ghost cells.
int ref_thermal_set_cell_field(void* h, int field, const double* vals) {
  RefModel* r = (RefModel*)h;
  return guarded([&] {
    Field* fs[] = {&r->tf.temperature, &r->tf.conductivity, &r->tf.source, &r->tf.specificHeat,
                   &r->tf.temperatureN1};
    const StorageSite& cells = r->mesh->getCells();
    Array<double>& a = dynamic_cast<Array<double>&>((*fs[field])[cells]);
    for (int i = 0; i < a.getLength(); i++) a[i] = vals[i];
  });
}

int ref_thermal_get_cell_field(void* h, int field, double* out) {
  RefModel* r = (RefModel*)h;
  return guarded([&] {
    Field* fs[] = {&r->tf.temperature, &r->tf.conductivity, &r->tf.source, &r->tf.specificHeat,
                   &r->tf.temperatureN1};
    const StorageSite& cells = r->mesh->getCells();
    const Array<double>& a = dynamic_cast<const Array<double>&>((*fs[field])[cells]);
    for (int i = 0; i < a.getLength(); i++) out[i] = a[i];
  });
}

int ref_thermal_sizes(void* h, int* out /* nSelf, nGhost, nnzAll */) {
  RefModel* r = (RefModel*)h;
  return guarded([&] {
    const StorageSite& cells = r->mesh->getCells();
    out[0] = cells.getSelfCount();
    out[1] = cells.getCount() - cells.getSelfCount();
    const CRConnectivity& cc = r->mesh->getCellCells();
    out[2] = cc.getRow()[cells.getCount()];
  });
}

// cellCells (all rows incl. ghosts) and the per-face pair->col mapping
int ref_thermal_connectivity(void* h, int* row, int* col, int* pairToCol) {
  RefModel* r = (RefModel*)h;
  return guarded([&] {
    const Mesh& mesh = *r->mesh;
    const StorageSite& cells = mesh.getCells();
    const CRConnectivity& cc = mesh.getCellCells();
    const int nr = cells.getCount();
    for (int i = 0; i <= nr; i++) row[i] = cc.getRow()[i];
    for (int k = 0; k < cc.getRow()[nr]; k++) col[k] = cc.getCol()[k];
    const CRConnectivity& fc = mesh.getAllFaceCells();
    const Array<Vector<int, 2> >& p2c = cc.getPairToColMapping(fc);
    for (int f = 0; f < mesh.getFaces().getCount(); f++) {
      pairToCol[2 * f] = p2c[f][0];
      pairToCol[2 * f + 1] = p2c[f][1];
    }
  });
}

// geometry: faceArea(3F) faceAreaMag(F) faceCentroid(3F) cellCentroid(3(N+G)) cellVolume(N+G)
int ref_thermal_geometry(void* h, double* fa, double* fam, double* fcn, double* ccn, double* vol) {
  RefModel* r = (RefModel*)h;
  return guarded([&] {
    const Mesh& mesh = *r->mesh;
    const StorageSite& faces = mesh.getFaces();
    const StorageSite& cells = mesh.getCells();
    const Array<VecD3>& a = dynamic_cast<const Array<VecD3>&>(r->geom.area[faces]);
    const Array<double>& am = dynamic_cast<const Array<double>&>(r->geom.areaMag[faces]);
    const Array<VecD3>& fc = dynamic_cast<const Array<VecD3>&>(r->geom.coordinate[faces]);
    const Array<VecD3>& cc = dynamic_cast<const Array<VecD3>&>(r->geom.coordinate[cells]);
    const Array<double>& v = dynamic_cast<const Array<double>&>(r->geom.volume[cells]);
    for (int f = 0; f < faces.getCount(); f++) {
      for (int d = 0; d < 3; d++) {
        fa[3 * f + d] = a[f][d];
        fcn[3 * f + d] = fc[f][d];
      }
      fam[f] = am[f];
    }
    for (int c = 0; c < cells.getCount(); c++) {
      for (int d = 0; d < 3; d++) ccn[3 * c + d] = cc[c][d];
      vol[c] = v[c];
    }
  });
}

// One linearization exactly as advance() performs it (initLinearization,
// initAssembly, linearize, initSolve), exporting the cell-cell matrix over
// all rows (self + ghost) and b. Temperature is left as linearize() leaves
// it (Dirichlet ghosts set to their boundary value).
int ref_thermal_linearize(void* h, double* diag, double* off, double* b, int* isBoundary) {
  RefModel* r = (RefModel*)h;
  return guarded([&] {
    auto& impl = tmImpl(*r->model);
    LinearSystem ls;
    impl.initLinearization(ls);
    ls.initAssembly();
    impl.linearize(ls);
    ls.initSolve();
    const StorageSite& cells = r->mesh->getCells();
    MultiField::ArrayIndex ti(&r->tf.temperature, &cells);
    const DMatrix& m = dynamic_cast<const DMatrix&>(ls.getMatrix().getMatrix(ti, ti));
    const int nr = cells.getCount();
    exportCR(m, nr, nullptr, nullptr, diag, off);
    const Array<double>& bb = dynamic_cast<const Array<double>&>(ls.getB()[ti]);
    for (int i = 0; i < nr; i++) b[i] = bb[i];
    if (isBoundary)
      for (int i = 0; i < nr; i++) isBoundary[i] = crmBoundary(m)[i] ? 1 : 0;
  });
}

// AMG hierarchy the reference builds for the current linearization:
// coarse sizes and, concatenated, the coarseIndex array of every fine level
// (self rows only). Matrices of each coarse level go to the optional
// buffers (rows, cols, diag, offdiag concatenated level by level).
int ref_thermal_hierarchy(void* h, int groupSize, double thr, int maxLevels, int* nLevels,
                          int* sizes, int* coarseIndex, int* coarseNnz, int* rows, int* cols,
                          double* diags, double* offs) {
  RefModel* r = (RefModel*)h;
  return guarded([&] {
    auto& impl = tmImpl(*r->model);
    LinearSystem ls;
    impl.initLinearization(ls);
    ls.initAssembly();
    impl.linearize(ls);
    ls.initSolve();
    AMG amg;
    amg.verbosity = 0;
    amg.maxCoarseLevels = maxLevels;
    amg.coarseGroupSize = groupSize;
    amg.weightRatioThreshold = thr;
    amgFinest(amg) = &ls;
    amgCreate(amg);
    const int nl = (int)amgCoarse(amg).size();
    *nLevels = nl;
    int ciPos = 0, rp = 0, cp = 0, dp = 0;
    for (int l = 0; l < nl; l++) {
      LinearSystem& c = *amgCoarse(amg)[l];
      sizes[l] = c.getMatrix().getSize();
      LinearSystem& f = (l == 0) ? ls : *amgCoarse(amg)[l - 1];
      MultiField& ciF = f.getCoarseIndex();
      MultiField::ArrayIndex ai = ciF.getArrayIndex(0);
      const Array<int>& ci = dynamic_cast<const Array<int>&>(ciF[ai]);
      const int nf = ai.second->getSelfCount();
      for (int i = 0; i < nf; i++) coarseIndex[ciPos++] = ci[i];
      MultiField::ArrayIndex cidx(0, 0);
      const DMatrix& cm = onlyMatrix(c, cidx);
      const int n = cm.getConnectivity().getRowDim();
      coarseNnz[l] = cm.getConnectivity().getRow()[n];
      if (rows) {
        exportCR(cm, n, rows + rp, cols + cp, diags + dp, offs + cp);
        rp += n + 1;
        cp += coarseNnz[l];
        dp += n;
      }
    }
  });
}

// advance(niter) as ThermalModel_impl.h:424-456 performs it, step by step
// through the reference's own Impl methods, so that the full-precision
// rNorm of each outer iteration can be returned. Returns the wall time of
// the loop in seconds.
int ref_thermal_advance(void* h, int niter, double* norms, int* nDone, double* seconds) {
  RefModel* r = (RefModel*)h;
  return guarded([&] {
    QuietCout quiet;
    TModel::Impl& impl = tmImpl(*r->model);
    ThermalModelOptions<double>& opts = impl.getOptions();
    auto t0 = std::chrono::steady_clock::now();
    int done = 0;
    for (int n = 0; n < niter; n++) {
      LinearSystem ls;
      impl.initLinearization(ls);
      ls.initAssembly();
      impl.linearize(ls);
      ls.initSolve();
      MFRPtr rNorm(opts.getLinearSolver().solve(ls));
      MFRPtr& initial = implInitialNorm(impl);
      if (!initial) initial = rNorm;
      MFRPtr normRatio((*rNorm) / (*initial));
      opts.getLinearSolver().cleanup();
      ls.postSolve();
      ls.updateSolution();
      implIters(impl)++;
      norms[done++] = dynamic_cast<const Array<double>&>((*rNorm)[r->tf.temperature])[0];
      if (*rNorm < opts.absoluteTolerance || *normRatio < opts.relativeTolerance) break;
    }
    auto t1 = std::chrono::steady_clock::now();
    *seconds = std::chrono::duration<double>(t1 - t0).count();
    *nDone = done;
  });
}

int ref_thermal_update_time(void* h) {
  RefModel* r = (RefModel*)h;
  return guarded([&] { r->model->updateTime(); });
}

int ref_thermal_heat_flux_integral(void* h, int groupId, double* out) {
  RefModel* r = (RefModel*)h;
  return guarded([&] { *out = r->model->getHeatFluxIntegral(*r->mesh, groupId); });
}

}  // extern "C"
