// GPU AMG hierarchy and the linear solvers built on it.
#include "solver.hpp"

#include <math_constants.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <cstdlib>
#include <exception>
#include <functional>
#include <thread>
#include <limits>
#include <type_traits>
#include <map>
#include <mutex>
#include <tuple>

namespace fvm {

#define CUDA_OK(call)                                                                       \
  do {                                                                                      \
    cudaError_t e_ = (call);                                                                \
    if (e_ != cudaSuccess)                                                                  \
      throw ::fvm::Error(::fvm::kDeviceError, std::string(#call ": ") + cudaGetErrorString(e_)); \
  } while (0)

// ---------------------------------------------------------------------------
DeviceArena::~DeviceArena() {
  release();
  for (auto& kv : free_) cudaFree(kv.second);
  free_.clear();
}

void* DeviceArena::alloc(size_t bytes) {
  std::lock_guard<std::mutex> lock(mu_);
  void* p = nullptr;
  if (bytes == 0) bytes = 16;
  auto it = free_.find(bytes);
  if (it != free_.end()) {
    p = it->second;
    free_.erase(it);
  } else {
    CUDA_OK(cudaMalloc(&p, bytes));
  }
  ptrs_.push_back({p, bytes});
  bytes_ += bytes;
  return p;
}

void DeviceArena::copy_h2d(void* d, const void* h, size_t n) {
  CUDA_OK(cudaMemcpy(d, h, n, cudaMemcpyHostToDevice));
}

void DeviceArena::release() {
  std::lock_guard<std::mutex> lock(mu_);
  for (auto& pb : ptrs_) free_.insert({pb.second, pb.first});
  ptrs_.clear();
  bytes_ = 0;
}

// ---------------------------------------------------------------------------
namespace {
// moves the objects of `from` into the spare slots of the same index
template <class T>
void keep_spares(std::vector<T>& from, std::vector<T>& spares) {
  if (spares.size() < from.size()) spares.resize(from.size());
  for (size_t l = 0; l < from.size(); l++) spares[l] = std::move(from[l]);
  from.clear();
}
template <class T>
T take_spare(std::vector<T>& spares, size_t l) {
  if (l < spares.size()) return std::move(spares[l]);
  return T();
}
}  // namespace

void AmgHierarchy::release() {
  // nothing of the arena may still be in use by the setup stream
  if (setupStream_) cudaStreamSynchronize(setupStream_);
  inversePending_ = false;
  deviceBuilt_ = false;
  arena_.release();
  lv_.clear();
  keep_spares(packed_, sparePacked_);
  keep_spares(ref_, spareRef_);
  keep_spares(c2f_, spareC2f_);
  coarseInv_ = nullptr;
  coarseInvF_ = nullptr;
}

RefLevel AmgHierarchy::spareLevel(int l) { return take_spare(spareRef_, (size_t)l); }

void* AmgHierarchy::scratch(size_t bytes) { return arena_.alloc(bytes); }

double* AmgHierarchy::pinnedScalars() {
  if (!pinned_) CUDA_OK(cudaMallocHost(&pinned_, sizeof(double) * 32));
  return pinned_;
}

AmgHierarchy::~AmgHierarchy() {
  if (setupStream_) cudaStreamSynchronize(setupStream_);
  if (pinned_) cudaFreeHost(pinned_);
  if (setupStream_) cudaStreamDestroy(setupStream_);
}

std::vector<int> AmgHierarchy::sizes() const {
  std::vector<int> s;
  for (const DevLevel& l : lv_) s.push_back(l.n);
  return s;
}

void AmgHierarchy::build(std::vector<RefLevel>& levels, int finestLocalSize, const SolverOptions& opt) {
  TraceRange traceRange("AMG hierarchy (reference aggregation)");
  const bool trace = getenv("FVM_TRACE") != nullptr;
  auto t0 = std::chrono::steady_clock::now();
  auto lap = [&](const char* what) {
    if (!trace) return;
    const auto t1 = std::chrono::steady_clock::now();
    fprintf(stderr, "[fvm setup] %-28s %8.1f ms\n", what, std::chrono::duration<double, std::milli>(t1 - t0).count());
    t0 = t1;
  };
  release();
  lap("previous hierarchy released");
  opt_ = opt;
  ref_ = std::move(levels);
  levels.clear();
  HierarchyOptions ho;
  ho.maxCoarseLevels = opt.finestOnly() ? 0 : opt.maxCoarseLevels;
  ho.groupSize = opt.coarseGroupSize;
  ho.weightRatioThreshold = opt.weightRatioThreshold;
  ho.coarsestSize = opt.coarsestSize;
  ho.finestLocalSize = finestLocalSize;
  const bool mixed = opt.precision == kMixed;
  // Every level is coloured, packed and uploaded on a thread of its own as
  // soon as its matrix exists: level 0 while the coarse levels are
  // aggregated, level l while levels l+1, ... are (the greedy walks are
  // sequential and leave the other cores free). ref_, packed_ and lv_ have
  // room for every level, so appending levels never moves one in use.
  const size_t maxL = (size_t)std::max(1, opt.maxCoarseLevels) + 2;
  ref_.reserve(maxL);
  packed_.resize(maxL);
  lv_.resize(maxL);
  std::vector<std::thread> th(maxL);
  std::vector<std::exception_ptr> errs(maxL);
  auto packAndUpload = [&](int l) {
    try {
      // levels smoothed by damped Jacobi need no colouring
      const SmootherOrdering ord =
          l == 0 ? (opt.finestOnly() ? kSequential : opt.ordering)
                 : (dampedLevel(l, ref_[l].n) ? kSequential : opt.ordering);
      pack_level(ref_[l], ord, packed_[l]);
      uploadMatrix(packed_[l], lv_[l], mixed);
    } catch (...) {
      errs[l] = std::current_exception();
    }
  };
  const auto tBuild = std::chrono::steady_clock::now();
  auto startLevel = [&](int l) {
    if (trace && l > 0)
      fprintf(stderr, "[fvm setup]   level %d (%d rows) ready at %8.1f ms\n", l, ref_[l].n,
              std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - tBuild).count());
    packed_[l] = take_spare(sparePacked_, (size_t)l);
    th[l] = std::thread(packAndUpload, l);
  };
  auto joinAll = [&] {
    for (auto& t : th)
      if (t.joinable()) t.join();
  };
  startLevel(0);
  std::vector<CSR>& c2f = c2f_;
  try {
    build_hierarchy(ref_, ho, c2f, &spareRef_, &spareC2f_, startLevel);
  } catch (...) {
    joinAll();
    throw;
  }
  lap("aggregation + Galerkin");
  const int L = (int)ref_.size();
  // Coarsest direct solve: as soon as the coarsest level is packed and
  // uploaded, its dense form is built on the GPU and inverted on a stream of
  // its own, overlapping the packing and uploads of the other levels.
  const bool direct = opt.coarseSolver == kCoarseDirect && !opt.finestOnly();
  cudaStream_t gjStream = nullptr;
  void* gjScratch = nullptr;
  int coarseN = 0;
  bool gjUnpivoted = false;
  auto startCoarseInverse = [&](int l) {
    const PackedLevel& c = packed_[l];
    const size_t nn = (size_t)c.n * c.n;
    coarseN = c.n;
    FVM_REQUIRE(c.n <= 4096, kTooLarge,
                "coarsest level too large for the dense direct solve (max 4096 rows); set coarsestSize");
    if (c.n <= 128) {
      std::vector<double> inv;
      dense_inverse(c, inv);
      coarseInv_ = arena_.upload(inv);
      return;
    }
    FVM_REQUIRE(lv_[l].ellWidth == 0, kUnsupported, "coarsest level in ELL-32 layout");
    // diagonally dominant rows (a diffusion operator and its Galerkin
    // levels): Gauss-Jordan needs no pivoting, and the in-place sweep runs
    // one kernel per 16 pivots; otherwise the partial-pivoting path. Rows
    // whose dominance is exact in real arithmetic (interior rows of a
    // diffusion operator) can miss it by rounding: a relative slack of 1e-8
    // accepts them and leaves the growth bound (about 2) intact.
    const RefLevel& rl = ref_[l];
    bool dominant = true;
    for (int i = 0; i < rl.n && dominant; i++) {
      double s = 0.0;
      for (int k = rl.conn.row[i]; k < rl.conn.row[i + 1]; k++) s += std::fabs(rl.off[k]);
      dominant = rl.diag[i] != 0.0 && s <= std::fabs(rl.diag[i]) * (1.0 + 1e-8);
    }
    // symmetric to a relative 1e-12 entry by entry (a diffusion operator
    // and its Galerkin levels): the symmetric sweep, half the products
    bool symmetric = dominant;
    for (int i = 0; i < rl.n && symmetric; i++)
      for (int k = rl.conn.row[i]; k < rl.conn.row[i + 1] && symmetric; k++) {
        const int j = rl.conn.col[k];
        bool found = false;
        for (int q = rl.conn.row[j]; q < rl.conn.row[j + 1]; q++)
          if (rl.conn.col[q] == i) {
            found = std::fabs(rl.off[k] - rl.off[q]) <= 1e-12 * std::max(std::fabs(rl.off[k]), std::fabs(rl.off[q]));
            break;
          }
        symmetric = found;
      }
    gjScratch = arena_.alloc(dev::gauss_jordan_scratch_bytes(c.n));
    coarseInv_ = (double*)arena_.alloc(sizeof(double) * nn);
    CUDA_OK(cudaStreamCreateWithFlags(&gjStream, cudaStreamNonBlocking));
    gjUnpivoted = dominant;
    if (dominant) {
      dev::dense_from_sell(lv_[l].view64(), lv_[l].nSlices, coarseInv_, gjStream);
      if (symmetric)
        dev::gauss_jordan_inverse_symmetric(c.n, coarseInv_, gjScratch, gjStream);
      else
        dev::gauss_jordan_inverse_dominant(c.n, coarseInv_, gjScratch, gjStream);
      return;
    }
    double* dA = (double*)arena_.alloc(sizeof(double) * nn);
    dev::dense_from_sell(lv_[l].view64(), lv_[l].nSlices, dA, gjStream);
    dev::gauss_jordan_inverse(c.n, dA, coarseInv_, gjScratch, gjStream);
  };
  if (th[L - 1].joinable()) th[L - 1].join();
  try {
    if (errs[L - 1]) std::rethrow_exception(errs[L - 1]);
    if (direct) startCoarseInverse(L - 1);
  } catch (...) {
    joinAll();
    throw;
  }
  joinAll();
  for (int l = 0; l < L; l++)
    if (errs[l]) std::rethrow_exception(errs[l]);
  packed_.resize(L);
  lv_.resize(L);
  lap("colouring + packing (+ level 0 upload)");
  {
    // transfer maps of all levels at once (level l writes only its own)
    std::vector<std::thread> tt;
    std::vector<std::exception_ptr> terr(L);
    for (int l = 0; l + 1 < L; l++)
      tt.emplace_back([&, l] {
        try {
          pack_transfer(ref_[l], c2f[l], packed_[l], packed_[l + 1]);
          uploadTransfer(packed_[l], lv_[l], packed_[l + 1].n);
        } catch (...) {
          terr[l] = std::current_exception();
        }
      });
    for (auto& t : tt) t.join();
    for (auto& e : terr)
      if (e) std::rethrow_exception(e);
  }
  lap("transfer maps + uploads");
  if (direct) {
    if (gjStream) {
      int singular = 0;
      const cudaError_t e1 = cudaMemcpyAsync(&singular, dev::gauss_jordan_status(coarseN, gjScratch), sizeof(int),
                                             cudaMemcpyDeviceToHost, gjStream);
      const cudaError_t e2 = cudaStreamSynchronize(gjStream);
      cudaStreamDestroy(gjStream);
      CUDA_OK(e1);
      CUDA_OK(e2);
      FVM_REQUIRE(singular == 0, kBadArgument, "singular coarsest-level matrix");
    }
    if (mixed) {
      const size_t nn = (size_t)coarseN * coarseN;
      coarseInvF_ = (float*)arena_.alloc(sizeof(float) * nn);
      dev::cast_d2f(nn, coarseInv_, coarseInvF_, 0);
    }
    CUDA_OK(cudaDeviceSynchronize());
    lap(gjUnpivoted ? "coarsest inverse (unpivoted)" : "coarsest inverse");
  }
  prepareChebyshev();
  tunePlans();
  lap("launch plans");
  if (trace) {
    fprintf(stderr, "[fvm setup] levels:");
    for (int l = 0; l < L; l++)
      fprintf(stderr, " %d(%dc%s)", lv_[l].n, lv_[l].nColors, lv_[l].splitRestrict ? ",split" : "");
    fprintf(stderr, "\n");
  }
}

// ---- autotuned launch plans --------------------------------------------------
namespace {
struct PlanKey {
  int n;
  size_t entries;
  int width, colors;
  bool f32, damped;
  bool operator<(const PlanKey& o) const {
    return std::tie(n, entries, width, colors, f32, damped) <
           std::tie(o.n, o.entries, o.width, o.colors, o.f32, o.damped);
  }
};
std::mutex gPlanMu;
std::map<PlanKey, dev::RowPlan> gPlanCache;  // per process: a shape is timed once
constexpr int kTuneMinRows = 4096;           // smaller levels are launch-bound: default plan
const dev::RowPlan kCandidatePlans[] = {{1, 256}, {1, 128}, {2, 256}, {2, 128}, {4, 256}, {4, 128}};
struct SplitKey {
  int n;
  size_t entries;
  int nCoarse;
  bool f32;
  bool operator<(const SplitKey& o) const {
    return std::tie(n, entries, nCoarse, f32) < std::tie(o.n, o.entries, o.nCoarse, o.f32);
  }
};
std::map<SplitKey, bool> gSplitCache;
}  // namespace

void AmgHierarchy::restrictPass(int l, bool split, cudaStream_t st) {
  DevLevel& d = lv_[l];
  DevLevel& c = lv_[l + 1];
  if (opt_.precision == kMixed)
    dev::residual_restrict<float>(d.view32(), d.nSlices, d.rowSlice, c.n, d.c2fRow, d.c2fCol, d.xF, d.bF, c.bF,
                                  c.xF, split ? d.rF : nullptr, st);
  else
    dev::residual_restrict<double>(d.view64(), d.nSlices, d.rowSlice, c.n, d.c2fRow, d.c2fCol, d.x, d.b, c.b, c.x,
                                   split ? d.r : nullptr, st);
}

void AmgHierarchy::smootherPass(int l, dev::RowPlan plan, cudaStream_t st) {
  DevLevel& d = lv_[l];
  const bool f32 = opt_.precision == kMixed;
  const bool damped = dampedLevel(l, d.n);
  auto pass = [&](auto a, auto* x, auto* t, const auto* b) {
    using T = std::remove_pointer_t<decltype(x)>;
    if (damped || opt_.smootherType != kGaussSeidel) {
      dev::jacobi_damped<T>(a, d.nSlices, x, t, b, (T)opt_.jacobiWeight, st, plan);
    } else {
      for (int c = 0; c < d.nColors; c++)
        dev::gs_color<T>(a, d.colorSliceStart[c], d.colorSliceStart[c + 1], x, b, st, plan);
    }
  };
  if (f32)
    pass(d.view32(), d.xF, d.tmpF, (const float*)d.bF);
  else
    pass(d.view64(), d.x, d.tmp, (const double*)d.b);
}

// Each SELL-32 level's smoother runs with the fastest of the candidate
// plans, timed here with CUDA events (one warm-up and five timed passes,
// median). All plans give bitwise the same result, so the choice changes
// speed only. Levels of one shape are timed once per process.
void AmgHierarchy::tunePlans() {
  const int L = (int)lv_.size();
  const bool f32 = opt_.precision == kMixed;
  const bool direct = opt_.coarseSolver == kCoarseDirect && !opt_.finestOnly();
  cudaStream_t st = nullptr;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  bool touched = false;
  // one warm-up and five timed runs, median
  auto median_ms = [&](auto&& fn) {
    fn();
    std::vector<float> t;
    for (int r = 0; r < 5; r++) {
      CUDA_OK(cudaEventRecord(e0, st));
      fn();
      CUDA_OK(cudaEventRecord(e1, st));
      CUDA_OK(cudaEventSynchronize(e1));
      float ms = 0.f;
      CUDA_OK(cudaEventElapsedTime(&ms, e0, e1));
      t.push_back(ms);
    }
    std::sort(t.begin(), t.end());
    return t[2];
  };
  for (int l = 0; l < L; l++) {
    DevLevel& d = lv_[l];
    d.plan = dev::RowPlan();
    if (d.ellWidth) {
      // ELL-32 Gauss-Seidel levels: one or two rows per thread
      if (opt_.planEllRows) {
        d.plan.ellRows = opt_.planEllRows;
        continue;
      }
      if (!opt_.autotune || d.n < kTuneMinRows || opt_.smootherType != kGaussSeidel || dampedLevel(l, d.n) ||
          opt_.ordering != kMulticolor || chebyshevLevel(l))
        continue;
      const PlanKey key{d.n, d.entries, -d.ellWidth, d.nColors, f32, false};
      {
        std::lock_guard<std::mutex> lock(gPlanMu);
        auto it = gPlanCache.find(key);
        if (it != gPlanCache.end()) {
          d.plan = it->second;
          continue;
        }
      }
      if (!st) {
        CUDA_OK(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
        CUDA_OK(cudaEventCreate(&e0));
        CUDA_OK(cudaEventCreate(&e1));
      }
      touched = true;
      dev::RowPlan two;
      two.ellRows = 2;
      const float t1 = median_ms([&] { smootherPass(l, dev::RowPlan(), st); });
      const float t2 = median_ms([&] { smootherPass(l, two, st); });
      if (t2 < t1) d.plan = two;
      std::lock_guard<std::mutex> lock(gPlanMu);
      gPlanCache[key] = d.plan;
      continue;
    }
    if (opt_.planTpr) {
      d.plan.tpr = opt_.planTpr;
      d.plan.block = opt_.planBlock ? opt_.planBlock : 256;
      continue;
    }
    if (!opt_.autotune || d.n < kTuneMinRows || (direct && l == L - 1)) continue;
    if (opt_.smootherType != kGaussSeidel && !dampedLevel(l, d.n)) continue;  // plain Jacobi: not tuned
    const PlanKey key{d.n, d.entries, d.maxWidth, d.nColors, f32, dampedLevel(l, d.n)};
    {
      std::lock_guard<std::mutex> lock(gPlanMu);
      auto it = gPlanCache.find(key);
      if (it != gPlanCache.end()) {
        d.plan = it->second;
        continue;
      }
    }
    if (!st) {
      CUDA_OK(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
      CUDA_OK(cudaEventCreate(&e0));
      CUDA_OK(cudaEventCreate(&e1));
    }
    touched = true;
    float best = std::numeric_limits<float>::max();
    dev::RowPlan bestPlan;
    for (const dev::RowPlan& p : kCandidatePlans) {
      const float t = median_ms([&] { smootherPass(l, p, st); });
      if (t < best) {
        best = t;
        bestPlan = p;
      }
    }
    d.plan = bestPlan;
    std::lock_guard<std::mutex> lock(gPlanMu);
    gPlanCache[key] = bestPlan;
  }
  // residual + restriction of each level above the coarsest: the fused
  // kernel (gathers of scattered fine rows) or the coalesced residual pass
  // followed by the gather of r, whichever is faster (same result bits)
  for (int l = 0; l + 1 < L; l++) {
    DevLevel& d = lv_[l];
    d.splitRestrict = false;
    if (!opt_.autotune || d.n < kTuneMinRows) continue;
    const SplitKey key{d.n, d.entries, lv_[l + 1].n, f32};
    {
      std::lock_guard<std::mutex> lock(gPlanMu);
      auto it = gSplitCache.find(key);
      if (it != gSplitCache.end()) {
        d.splitRestrict = it->second;
        continue;
      }
    }
    if (!st) {
      CUDA_OK(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
      CUDA_OK(cudaEventCreate(&e0));
      CUDA_OK(cudaEventCreate(&e1));
    }
    touched = true;
    const float fused = median_ms([&] { restrictPass(l, false, st); });
    const float split = median_ms([&] { restrictPass(l, true, st); });
    d.splitRestrict = split < fused;
    std::lock_guard<std::mutex> lock(gPlanMu);
    gSplitCache[key] = d.splitRestrict;
  }
  if (st) {
    CUDA_OK(cudaStreamSynchronize(st));
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaStreamDestroy(st);
  }
  if (touched) {
    // the timed passes wrote the level vectors: back to the state after upload
    for (int l = 0; l < L; l++) {
      DevLevel& d = lv_[l];
      CUDA_OK(cudaMemset(d.x, 0, sizeof(double) * d.n));
      CUDA_OK(cudaMemset(d.tmp, 0, sizeof(double) * d.n));
      if (d.xF) CUDA_OK(cudaMemset(d.xF, 0, sizeof(float) * d.n));
      if (d.tmpF) CUDA_OK(cudaMemset(d.tmpF, 0, sizeof(float) * d.n));
    }
  }
}

// Chebyshev iteration (Saad, Iterative Methods for Sparse Linear Systems,
// 2nd ed., Alg. 12.1) on D^-1 A with eigenvalues taken in [alpha, beta]:
// theta = (beta + alpha) / 2, delta = (beta - alpha) / 2, sigma = theta /
// delta; step 0: d = z / theta; step k: rho_k = 1 / (2 sigma - rho_{k-1}),
// d = rho_k rho_{k-1} d + (2 rho_k / delta) z, with z = -D^-1 (b + A x) the
// scaled residual and rho_0 = 1 / sigma. beta is the Gershgorin bound of
// level 0 (never below the spectrum), alpha = chebyshevFraction * beta: the
// polynomial damps the upper part of the spectrum, what a smoother must.
void AmgHierarchy::prepareChebyshev() {
  chebC1_.clear();
  chebC2_.clear();
  chebBound_ = 0.0;
  if (opt_.chebyshevDegree <= 0 || lv_.empty() || opt_.finestOnly()) return;
  DevLevel& d = lv_[0];
  double* dv = (double*)scratch(sizeof(double));
  dev::gershgorin_bound(d.view64(), d.nSlices, dv, nullptr);
  CUDA_OK(cudaMemcpy(&chebBound_, dv, sizeof(double), cudaMemcpyDeviceToHost));
  FVM_REQUIRE(std::isfinite(chebBound_) && chebBound_ > 0.0, kBadArgument,
              "Chebyshev smoother: no finite spectrum bound (zero diagonal?)");
  const double beta = chebBound_, alpha = opt_.chebyshevFraction * beta;
  const double theta = 0.5 * (beta + alpha), delta = 0.5 * (beta - alpha), sigma = theta / delta;
  double rho = 1.0 / sigma;
  chebC1_.push_back(0.0);
  chebC2_.push_back(1.0 / theta);
  for (int k = 1; k < opt_.chebyshevDegree; k++) {
    const double rn = 1.0 / (2.0 * sigma - rho);
    chebC1_.push_back(rn * rho);
    chebC2_.push_back(2.0 * rn / delta);
    rho = rn;
  }
}

bool AmgHierarchy::dampedLevel(int l, int n) const {
  // device-built coarse levels carry no colouring
  if (deviceBuilt_ && l > 0 && opt_.smootherType == kGaussSeidel) return true;
  return l > 0 && opt_.coarseJacobiRows > 0 && n <= opt_.coarseJacobiRows && opt_.smootherType == kGaussSeidel &&
         opt_.ordering == kMulticolor;
}

void AmgHierarchy::uploadMatrix(const PackedLevel& p, DevLevel& d, bool mixed) {
  d.n = p.n;
  d.nColors = p.nColors;
  d.nSlices = (int)p.sliceRow.size();
  d.maxWidth = p.maxWidth;
  d.ellWidth = p.ellWidth;
  d.colorSliceStart = p.colorSliceStart;
  d.entries = p.cols.size();
  d.sliceRow = arena_.upload(p.sliceRow);
  d.sliceRows = arena_.upload(p.sliceRows);
  d.sliceOff = arena_.upload(p.sliceOff);
  d.cols = arena_.upload(p.cols);
  d.vals = arena_.upload(p.vals);
  d.diag = arena_.upload(p.diag);
  std::vector<int> rs(p.n);
  std::vector<int4> meta(d.nSlices);
  for (int s = 0; s < d.nSlices; s++) {
    for (int k = 0; k < p.sliceRows[s]; k++) rs[p.sliceRow[s] + k] = s;
    meta[s] = make_int4(p.sliceRow[s], p.sliceRows[s], p.sliceOff[s], (p.sliceOff[s + 1] - p.sliceOff[s]) / 32);
  }
  d.rowSlice = arena_.upload(rs);
  d.meta = arena_.upload(meta);
  const size_t nb = (size_t)p.n * sizeof(double);
  d.x = (double*)arena_.alloc(nb);
  d.b = (double*)arena_.alloc(nb);
  d.r = (double*)arena_.alloc(nb);
  d.tmp = (double*)arena_.alloc(nb);
  CUDA_OK(cudaMemset(d.x, 0, nb));
  CUDA_OK(cudaMemset(d.b, 0, nb));
  d.nPartials = dev::residual_partials(d.nSlices, d.n, d.ellWidth);
  d.partials = (double*)arena_.alloc(sizeof(double) * (d.nPartials + 1));
  if (mixed) {
    d.valsF = (float*)arena_.alloc(sizeof(float) * p.vals.size());
    d.diagF = (float*)arena_.alloc(sizeof(float) * p.diag.size());
    dev::cast_d2f(p.vals.size(), d.vals, d.valsF, 0);
    dev::cast_d2f(p.diag.size(), d.diag, d.diagF, 0);
    const size_t fb = (size_t)p.n * sizeof(float);
    d.xF = (float*)arena_.alloc(fb);
    d.bF = (float*)arena_.alloc(fb);
    d.rF = (float*)arena_.alloc(fb);
    d.tmpF = (float*)arena_.alloc(fb);
    CUDA_OK(cudaMemset(d.xF, 0, fb));
  }
}

void AmgHierarchy::uploadTransfer(const PackedLevel& p, DevLevel& d, int nCoarse) {
  d.nCoarse = nCoarse;
  d.ci = arena_.upload(p.coarseIndex);
  d.c2fRow = arena_.upload(p.c2fRow);
  d.c2fCol = arena_.upload(p.c2fCol);
}

template <>
void AmgHierarchy::runCycle<double>(cudaStream_t st, bool xZero) {
  cycle<double>(opt_.cycleType, 0, st, xZero);
}

template <>
void AmgHierarchy::runCycle<float>(cudaStream_t st, bool xZero) {
  cycle<float>(opt_.cycleType, 0, st, xZero);
}

template <class T>
static T* vec_x(DevLevel& d);
template <>
double* vec_x<double>(DevLevel& d) { return d.x; }
template <>
float* vec_x<float>(DevLevel& d) { return d.xF; }
template <class T>
static T* vec_b(DevLevel& d);
template <>
double* vec_b<double>(DevLevel& d) { return d.b; }
template <>
float* vec_b<float>(DevLevel& d) { return d.bF; }
template <class T>
static T* vec_r(DevLevel& d);
template <>
double* vec_r<double>(DevLevel& d) { return d.r; }
template <>
float* vec_r<float>(DevLevel& d) { return d.rF; }
template <class T>
static T* vec_tmp(DevLevel& d);
template <>
double* vec_tmp<double>(DevLevel& d) { return d.tmp; }
template <>
float* vec_tmp<float>(DevLevel& d) { return d.tmpF; }
template <class T>
static dev::SellView<T> view(const DevLevel& d);
template <>
dev::SellView<double> view<double>(const DevLevel& d) { return d.view64(); }
template <>
dev::SellView<float> view<float>(const DevLevel& d) { return d.view32(); }

template <class T>
void AmgHierarchy::sweeps(int nSweeps, int l, cudaStream_t st, const T* xc, const int* ci) {
  DevLevel& d = lv_[l];
  const dev::SellView<T> a = view<T>(d);
  T* x = vec_x<T>(d);
  const T* b = vec_b<T>(d);
  const bool damped = dampedLevel(l, d.n);
  if (chebyshevLevel(l) && nSweeps > 0) {
    // x and tmp alternate as the step's input and output; the level's r
    // holds the step direction (every use of r recomputes it afterwards)
    T* bufs[2] = {x, vec_tmp<T>(d)};
    T* dv = vec_r<T>(d);
    int cur = 0;
    for (int s = 0; s < nSweeps; s++)
      for (size_t k = 0; k < chebC1_.size(); k++) {
        dev::chebyshev_step<T>(a, d.nSlices, bufs[cur], bufs[cur ^ 1], dv, b, (T)chebC1_[k], (T)chebC2_[k], k == 0,
                               st);
        cur ^= 1;
      }
    if (cur) CUDA_OK(cudaMemcpyAsync(x, bufs[1], sizeof(T) * (size_t)d.n, cudaMemcpyDeviceToDevice, st));
    return;
  }
  for (int s = 0; s < nSweeps; s++) {
    if (damped) {
      // small coarse levels: two damped Jacobi passes instead of 2C-1
      // launch-bound colour passes
      T* t = vec_tmp<T>(d);
      const T w = (T)opt_.jacobiWeight;
      // the first pass after a fused prolongation reads xc[ci] for x
      if (s == 0 && xc)
        dev::jacobi_damped<T>(a, d.nSlices, x, t, b, w, st, d.plan, xc, ci);
      else
        dev::jacobi_damped<T>(a, d.nSlices, x, t, b, w, st, d.plan);
      dev::jacobi_damped<T>(a, d.nSlices, t, x, b, w, st, d.plan);
    } else if (opt_.smootherType == kGaussSeidel) {
      if (opt_.ordering == kSequential) {
        dev::gs_sequential<T>(a, x, b, false, st);
        dev::gs_sequential<T>(a, x, b, true, st);
      } else {
        const int C = d.nColors;
        // a symmetric sweep ends with colour 0, whose rows then agree with
        // their (unchanged) neighbours: the next sweep's colour-0 pass would
        // write bitwise the same values, so it starts at colour 1
        const int c0 = (s > 0 && opt_.gsReverse) ? 1 : 0;
        // after a fused prolongation the first forward pass reads the rows
        // of colours not yet visited from xc[ci]
        const bool pro = s == 0 && xc;
        for (int c = c0; c < C; c++)
          dev::gs_color<T>(a, d.colorSliceStart[c], d.colorSliceStart[c + 1], x, b, st, d.plan, pro ? xc : nullptr,
                           pro ? ci : nullptr);
        // reverse pass; its first colour would repeat the last update exactly
        if (opt_.gsReverse)
          for (int c = C - 2; c >= 0; c--)
            dev::gs_color<T>(a, d.colorSliceStart[c], d.colorSliceStart[c + 1], x, b, st, d.plan);
      }
    } else {
      T* t = vec_tmp<T>(d);
      dev::jacobi<T>(a, d.nSlices, x, t, b, st);
      dev::jacobi<T>(a, d.nSlices, t, x, b, st);
    }
  }
}

template <class T>
void AmgHierarchy::cycle(CycleType t, int l, cudaStream_t st, bool xZero) {
  const int L = (int)lv_.size();
  DevLevel& d = lv_[l];
  const bool coarsest = (l == L - 1);
  if (coarsest && coarseInv_) {
    if constexpr (std::is_same<T, float>::value) {
      if (coarseInvF_) {
        dev::dense_solve_f32(d.n, coarseInvF_, d.bF, d.xF, st);
        return;
      }
    }
    dev::dense_solve<T>(d.n, coarseInv_, vec_b<T>(d), vec_x<T>(d), st);
    return;
  }
  // xZero: x is taken as zero. Without pre-smoothing its memory is not read
  // before the prolongation assigns it; pre-smoothing, and the smoothing of
  // a coarsest level, need it zeroed first.
  const bool rhsOnly = xZero && opt_.nPreSweeps == 0 && !coarsest;
  if (xZero && !rhsOnly) dev::zero<T>(d.n, vec_x<T>(d), st);
  sweeps<T>(opt_.nPreSweeps, l, st);
  if (!coarsest) {
    DevLevel& c = lv_[l + 1];
    if (rhsOnly)
      dev::restrict_rhs<T>(c.n, d.c2fRow, d.c2fCol, vec_b<T>(d), vec_b<T>(c), (T*)nullptr, st);
    else
      dev::residual_restrict<T>(view<T>(d), d.nSlices, d.rowSlice, c.n, d.c2fRow, d.c2fCol, vec_x<T>(d),
                                vec_b<T>(d), vec_b<T>(c), vec_x<T>(c), d.splitRestrict ? vec_r<T>(d) : nullptr, st);
    cycle<T>(t, l + 1, st, true);
    if (t == kWCycle)
      cycle<T>(kWCycle, l + 1, st);
    else if (t == kFCycle)
      cycle<T>(kVCycle, l + 1, st);
    if (rhsOnly && fusedProlong(l)) {
      // x = xc[ci] is read straight from the coarse level by the first
      // damped-Jacobi pass (bitwise the same values)
      sweeps<T>(opt_.postSweeps(l), l, st, vec_x<T>(c), d.ci);
      return;
    }
    dev::prolong<T>(d.n, d.ci, vec_x<T>(c), vec_x<T>(d), st, rhsOnly);
  }
  sweeps<T>(opt_.postSweeps(l), l, st);
}

bool AmgHierarchy::fusedProlong(int l) const {
  const int L = (int)lv_.size();
  if (!opt_.fuseProlongation || l + 1 >= L || opt_.nPreSweeps != 0 || opt_.postSweeps(l) <= 0 || chebyshevLevel(l))
    return false;
  const DevLevel& d = lv_[l];
  if (dampedLevel(l, d.n)) return true;
  // multicolour Gauss-Seidel on an ELL-32 level (the fused colour kernel)
  return opt_.smootherType == kGaussSeidel && opt_.ordering == kMulticolor && d.ellWidth > 0 && d.nColors > 0;
}

void AmgHierarchy::applyCycle(const double* r, cudaStream_t st) {
  DevLevel& d = lv_[0];
  if (opt_.precision == kMixed) {
    dev::convert_d2f(d.n, r, d.bF, st);
    runCycle<float>(st, true);
  } else {
    dev::copy_d(d.n, r, d.b, st);
    runCycle<double>(st, true);
  }
}

void AmgHierarchy::apply(const double* r, double* z, cudaStream_t st) {
  DevLevel& d = lv_[0];
  if (opt_.preconditioner == kPrecJacobi) {
    // JacobiSolver::smooth: two Jacobi sweeps from zero with b = r
    dev::zero<double>(d.n, z, st);
    dev::jacobi<double>(d.view64(), d.nSlices, z, d.tmp, r, st);
    dev::jacobi<double>(d.view64(), d.nSlices, d.tmp, z, r, st);
    return;
  }
  if (opt_.precision == kMixed) {
    dev::convert_d2f(d.n, r, d.bF, st);
    runCycle<float>(st, true);
    dev::zero<double>(d.n, z, st);
    dev::add_f2d(d.n, d.xF, z, st);
  } else {
    dev::copy_d(d.n, r, d.b, st);
    runCycle<double>(st, true);
    dev::copy_d(d.n, d.x, z, st);
  }
}

int AmgHierarchy::colourPasses(int colors, int nSweeps) const {
  if (nSweeps <= 0) return 0;
  if (!opt_.gsReverse) return nSweeps * colors;
  // forward + reverse (2C - 1 passes), later sweeps without their first pass
  return nSweeps * (2 * colors - 1) - (nSweeps - 1);
}

double AmgHierarchy::fineSweepBytes() const {
  // one pass over every row of level 0: b, diag, x (read+write) per row,
  // col + val per stored entry
  const DevLevel& d = lv_[0];
  const double vb = opt_.precision == kMixed ? 4.0 : 8.0;
  return d.n * (4.0 * vb) + d.entries * (4.0 + vb);
}

// Algorithmic bytes of one cycle from a zero guess (the preconditioner's
// use; the FP64 standalone iteration adds a residual pass on level 0), in
// the configured precision, following AmgHierarchy::cycle: per level its
// smoothing passes, the restriction (of b alone from a zero guess without
// pre-smoothing) and the prolongation; the coarsest level's dense solve.
double AmgHierarchy::cycleBytes() const {
  const double vb = opt_.precision == kMixed ? 4.0 : 8.0;
  double total = 0;
  const int L = (int)lv_.size();
  for (int l = 0; l < L; l++) {
    const DevLevel& d = lv_[l];
    const double pass = d.n * (4.0 * vb) + d.entries * (4.0 + vb);
    if (l == L - 1 && coarseInv_) {
      total += (double)d.n * d.n * (opt_.precision == kMixed && coarseInvF_ ? 4.0 : 8.0) + 2.0 * vb * d.n;
      continue;
    }
    const int sweeps = opt_.nPreSweeps + opt_.postSweeps(l);
    if (chebyshevLevel(l)) {
      // a Chebyshev step: x, b, diag, the direction (read but in the first
      // step, written) and the new x per row, col + val per entry
      const int steps = sweeps * (int)chebC1_.size();
      total += steps * (d.n * 6.0 * vb + d.entries * (4.0 + vb)) - sweeps * d.n * vb;
      if (steps & 1) total += 2.0 * vb * d.n;
    } else if (opt_.smootherType == kGaussSeidel && !dampedLevel(l, d.n) && d.nColors > 0) {
      // colour passes of the pre- and post-smoothing (C of which make one
      // pass over the level)
      total += (double)(colourPasses(d.nColors, opt_.nPreSweeps) + colourPasses(d.nColors, opt_.postSweeps(l))) /
               d.nColors * pass;
    } else {
      total += sweeps * 2.0 * pass;  // a sweep: two (damped) Jacobi passes
    }
    if (l + 1 < L) {
      const DevLevel& c = lv_[l + 1];
      if (opt_.nPreSweeps == 0)
        total += (vb + 4.0) * d.n + (4.0 + vb) * c.n;  // b restricted; x assigned below
      else
        total += 3.0 * vb * d.n + (4.0 + vb) * d.entries + (4.0 + 2.0 * vb) * c.n;
      if (fusedProlong(l))
        // the first Jacobi pass reads ci and xc instead of x: no x write
        // and read of the prolongation
        total += 4.0 * d.n + vb * c.n - vb * d.n;
      else
        total += (2.0 * vb + 4.0) * d.n + vb * c.n;
    }
  }
  return total;
}

int AmgHierarchy::kernelsPerCycle() const {
  int k = 0;
  const int L = (int)lv_.size();
  for (int l = 0; l < L; l++) {
    const DevLevel& d = lv_[l];
    if (l == L - 1 && coarseInv_) {
      k += 1;
      continue;
    }
    const int sw = opt_.nPreSweeps + opt_.postSweeps(l);
    if (chebyshevLevel(l))
      k += (int)chebC1_.size() * sw;
    else if (opt_.smootherType == kGaussSeidel && !dampedLevel(l, d.n) && opt_.ordering != kSequential)
      k += colourPasses(d.nColors, opt_.nPreSweeps) + colourPasses(d.nColors, opt_.postSweeps(l));
    else
      k += 2 * sw;
    if (l + 1 < L) k += fusedProlong(l) ? 1 : 2;  // restriction, prolongation (unless fused)
  }
  return k;
}

void AmgHierarchy::profileLevels(int reps, void* flush, size_t flushBytes, cudaStream_t st,
                                 std::vector<double>& out) {
  const int L = (int)lv_.size();
  const bool f32 = opt_.precision == kMixed;
  const double vb = f32 ? 4.0 : 8.0;
  cudaEvent_t a, b;
  CUDA_OK(cudaEventCreate(&a));
  CUDA_OK(cudaEventCreate(&b));
  auto timed = [&](const std::function<void()>& body) {
    double total = 0;
    for (int r = 0; r < reps; r++) {
      CUDA_OK(cudaMemsetAsync(flush, r & 0xff, flushBytes, st));
      CUDA_OK(cudaEventRecord(a, st));
      body();
      CUDA_OK(cudaEventRecord(b, st));
      CUDA_OK(cudaEventSynchronize(b));
      float ms = 0;
      CUDA_OK(cudaEventElapsedTime(&ms, a, b));
      total += ms;
    }
    return total / reps;
  };
  out.assign((size_t)kLevelProfile * L, 0.0);
  for (int l = 0; l < L; l++) {
    DevLevel& d = lv_[l];
    double* o = &out[(size_t)kLevelProfile * l];
    o[0] = d.n;
    o[1] = (double)d.entries;
    const double pass = d.n * 4.0 * vb + d.entries * (4.0 + vb);
    if (l == L - 1 && coarseInv_) {
      o[2] = timed([&] {
        if (f32 && coarseInvF_)
          dev::dense_solve_f32(d.n, coarseInvF_, d.bF, d.xF, st);
        else if (f32)
          dev::dense_solve<float>(d.n, coarseInv_, d.bF, d.xF, st);
        else
          dev::dense_solve<double>(d.n, coarseInv_, d.b, d.x, st);
      });
      o[3] = (double)d.n * d.n * ((f32 && coarseInvF_) ? 4.0 : 8.0) + 2.0 * vb * d.n;
      continue;
    }
    o[2] = timed([&] { smootherPass(l, d.plan, st); });
    o[3] = pass;
    if (l + 1 < L) {
      DevLevel& c = lv_[l + 1];
      const bool rhsOnly = opt_.nPreSweeps == 0 && (f32 || l > 0);  // x = 0 on entry
      o[4] = timed([&] {
        if (rhsOnly) {
          if (f32)
            dev::restrict_rhs<float>(c.n, d.c2fRow, d.c2fCol, d.bF, c.bF, c.xF, st);
          else
            dev::restrict_rhs<double>(c.n, d.c2fRow, d.c2fCol, d.b, c.b, c.x, st);
        } else {
          restrictPass(l, d.splitRestrict, st);
        }
      });
      if (rhsOnly)
        o[5] = (vb + 4.0) * d.n + (4.0 + 2.0 * vb) * c.n;
      else if (d.splitRestrict)
        o[5] = pass + (vb + 4.0) * d.n + (4.0 + 2.0 * vb) * c.n;
      else
        o[5] = 3.0 * vb * d.n + (4.0 + vb) * d.entries + (4.0 + 2.0 * vb) * c.n;
      o[6] = timed([&] {
        if (f32)
          dev::prolong<float>(d.n, d.ci, c.xF, d.xF, st);
        else
          dev::prolong<double>(d.n, d.ci, c.x, d.x, st);
      });
      o[7] = (2.0 * vb + 4.0) * d.n + vb * c.n;
    }
  }
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  // the timed passes wrote the level vectors
  for (int l = 0; l < L; l++) {
    DevLevel& d = lv_[l];
    CUDA_OK(cudaMemsetAsync(d.x, 0, sizeof(double) * d.n, st));
    if (d.xF) CUDA_OK(cudaMemsetAsync(d.xF, 0, sizeof(float) * d.n, st));
    if (d.tmpF) CUDA_OK(cudaMemsetAsync(d.tmpF, 0, sizeof(float) * d.n, st));
  }
  CUDA_OK(cudaStreamSynchronize(st));
}

void AmgHierarchy::levelCsr(int l, std::vector<int>& row, std::vector<int>& col, std::vector<double>& val,
                            std::vector<double>& diag) const {
  FVM_REQUIRE(l >= 0 && l < (int)lv_.size(), kBadArgument, "no such level");
  const DevLevel& d = lv_[l];
  const int n = d.n;
  std::vector<int> cols(d.entries);
  std::vector<double> vals(d.entries), dg(n);
  std::vector<int4> meta(d.nSlices);
  CUDA_OK(cudaMemcpy(cols.data(), d.cols, sizeof(int) * d.entries, cudaMemcpyDeviceToHost));
  CUDA_OK(cudaMemcpy(vals.data(), d.vals, sizeof(double) * d.entries, cudaMemcpyDeviceToHost));
  CUDA_OK(cudaMemcpy(dg.data(), d.diag, sizeof(double) * n, cudaMemcpyDeviceToHost));
  if (d.ellWidth) {
    for (int s = 0; s < d.nSlices; s++)
      meta[s] = make_int4(32 * s, std::min(32, n - 32 * s), 32 * s * d.ellWidth, d.ellWidth);
  } else {
    CUDA_OK(cudaMemcpy(meta.data(), d.meta, sizeof(int4) * d.nSlices, cudaMemcpyDeviceToHost));
  }
  // storage row -> row of the exported numbering
  const std::vector<int>* iperm = nullptr;
  if (deviceBuilt_) {
    if (l == 0) iperm = &finest_->packed.iperm;
  } else if (!packed_[l].iperm.empty()) {
    iperm = &packed_[l].iperm;
  }
  auto out = [&](int p) { return iperm ? (*iperm)[p] : p; };
  std::vector<std::vector<std::pair<int, double>>> rows(n);
  diag.assign(n, 0.0);
  for (int s = 0; s < d.nSlices; s++) {
    const int4 m = meta[s];
    for (int q = 0; q < m.y; q++) {
      const int p = m.x + q;
      const int i = out(p);
      diag[i] = dg[p];
      for (int k = 0; k < m.w; k++) {
        const size_t e = (size_t)m.z + 32 * (size_t)k + q;
        if (vals[e] != 0.0 && cols[e] != p) rows[i].push_back({out(cols[e]), vals[e]});
      }
    }
  }
  row.assign(n + 1, 0);
  col.clear();
  val.clear();
  for (int i = 0; i < n; i++) {
    for (const auto& cv : rows[i]) {
      col.push_back(cv.first);
      val.push_back(cv.second);
    }
    row[i + 1] = (int)col.size();
  }
}

template void AmgHierarchy::cycle<double>(CycleType, int, cudaStream_t, bool);
template void AmgHierarchy::cycle<float>(CycleType, int, cudaStream_t, bool);

// ---------------------------------------------------------------------------
namespace {
enum Scal {
  kRho = 0,
  kRhoPrev,
  kPtq,
  kAlpha,
  kBeta,
  kNorm,
  kOmega,
  kRtv,
  kTdotr,
  kTdott,
  kOmegaPrev,
  kAlphaPrev,
  kRzPrev,
  // learned step
  kLsScale = 20,  // and kLsScale + 1 (input sum)
  kLsRq = 22,
  kLsQq,
  kLsAlpha,
  kLsTrial,
  kLsAccepted,
  kLsSteps,
  kLsUseful,
  kLsBefore,  // |r + A z1|_1 before the CG post-correction
  kNumScal
};
static_assert(kNumScal <= 32, "device scalars");
constexpr int kWorkVectors = 11;

// z = d1 + alpha d (the learned post-correction added to the cycle's z)
__global__ void k_combine(int n, const double* __restrict__ d1, const double* alpha, const double* __restrict__ d,
                          double* z) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) z[i] = d1[i] + alpha[0] * d[i];
}
// y = (double) x
__global__ void k_f2d(int n, const float* __restrict__ x, double* y) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) y[i] = (double)x[i];
}
// y = a + b
__global__ void k_add_vec(int n, const double* __restrict__ a, const double* __restrict__ b, double* y) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) y[i] = a[i] + b[i];
}

// Device-side loop control of the CG graph. Status: 0 running, 1
// converged, 2 non-finite residual, 3 iteration limit.
__global__ void k_cg_loop_init(double* scal, int* loopInt, double* history, double absTol, int maxIt,
                               cudaGraphConditionalHandle h) {
  const double r0 = scal[kNorm];
  history[0] = r0;
  loopInt[0] = 0;
  const bool finite = isfinite(r0);
  const bool done = !finite || r0 < absTol || maxIt <= 0;
  loopInt[1] = !finite ? 2 : (r0 < absTol ? 1 : (maxIt <= 0 ? 3 : 0));
  scal[kRho] = CUDART_INF;  // first beta = 0
  cudaGraphSetConditional(h, done ? 0u : 1u);
}

__global__ void k_cg_loop_check(const double* scal, int* loopInt, double* history, double relTol, double absTol,
                                int maxIt, cudaGraphConditionalHandle h) {
  const double rn = scal[kNorm];
  const int i = loopInt[0] + 1;
  loopInt[0] = i;
  history[i] = rn;
  const double r0 = history[0];
  int status = 0;
  if (!isfinite(rn))
    status = 2;
  else if (rn < absTol || rn / r0 < relTol)
    status = 1;
  else if (i >= maxIt)
    status = 3;
  loopInt[1] = status;
  cudaGraphSetConditional(h, status == 0 ? 1u : 0u);
}
}  // namespace

// Device workspace comes from the hierarchy's arena (recycled by the next
// build of the same sizes, so a rebuild allocates nothing); the pinned
// scalars are the hierarchy's too.
LinearSolve::LinearSolve(AmgHierarchy& h) : h_(h), n_(h.level(0).n) {
  work_ = (double*)h.scratch(sizeof(double) * (size_t)n_ * kWorkVectors);
  scal_ = (double*)h.scratch(sizeof(double) * 32);
  CUDA_OK(cudaMemset(scal_, 0, sizeof(double) * 32));
  partials_ = (double*)h.scratch(sizeof(double) * (dev::vec_blocks(n_) + 1));
  {
    const DevLevel& d = h.level(0);
    const int np = std::max(2 * dev::vec_blocks(n_), dev::spmv_dot_blocks(d.view64(), d.nSlices));
    partials2_ = (double*)h.scratch(sizeof(double) * (np + 2));
  }
  hostScal_ = h.pinnedScalars();
}

LinearSolve::~LinearSolve() {
  if (gLoop_) cudaGraphExecDestroy(gLoop_);
  if (g1_) cudaGraphExecDestroy(g1_);
  if (g2_) cudaGraphExecDestroy(g2_);
  if (g3_) cudaGraphExecDestroy(g3_);
  if (g4_) cudaGraphExecDestroy(g4_);
  if (g5_) cudaGraphExecDestroy(g5_);
}

void LinearSolve::norm_into(const double* v, double* scalar, cudaStream_t st) {
  dev::l1_partials(n_, v, partials_, st);
  dev::sum_partials(dev::vec_blocks(n_), partials_, scalar, st);
}

void LinearSolve::dot_into(const double* a, const double* b, double* scalar, cudaStream_t st) {
  dev::dot_partials(n_, a, b, partials_, st);
  dev::sum_partials(dev::vec_blocks(n_), partials_, scalar, st);
}

double LinearSolve::fetch(const double* scalar, cudaStream_t st) {
  CUDA_OK(cudaMemcpyAsync(hostScal_, scalar, sizeof(double), cudaMemcpyDeviceToHost, st));
  CUDA_OK(cudaStreamSynchronize(st));
  return hostScal_[0];
}

void LinearSolve::run(cudaGraphExec_t& exec, cudaStream_t st, const std::function<void()>& body) {
  if (!h_.options().useGraphs) {
    body();
    return;
  }
  if (graphsFailed_) {
    body();
    return;
  }
  if (!exec) {
    cudaGraph_t g = nullptr;
    CUDA_OK(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
    try {
      body();
    } catch (const Error& e) {
      // a launch that cannot be captured (e.g. cooperative launch on an
      // older driver): drop graphs for this solver and run eagerly
      if (getenv("FVM_TRACE")) fprintf(stderr, "[fvm solve] graph capture failed, running eagerly: %s\n", e.what());
      cudaStreamEndCapture(st, &g);
      if (g) cudaGraphDestroy(g);
      cudaGetLastError();
      graphsFailed_ = true;
      body();
      return;
    }
    CUDA_OK(cudaStreamEndCapture(st, &g));
    size_t nodes = 0;
    cudaGraphGetNodes(g, nullptr, &nodes);
    CUDA_OK(cudaGraphInstantiate(&exec, g, 0));
    cudaGraphDestroy(g);
    nodeCounts_[&exec] = (long long)nodes;
  }
  CUDA_OK(cudaGraphLaunch(exec, st));
  launches += nodeCounts_[&exec];
}

SolveReport LinearSolve::solve(cudaStream_t st) {
  SolveReport r;
  switch (h_.options().solver) {
    case kSolverCG:
      r = solveCG(st);
      break;
    case kSolverBCGStab:
      r = solveBCGStab(st);
      break;
    case kSolverJacobi:
      r = solveJacobi(st);
      break;
    default:
      r = solveAMG(st);
  }
  return r;
}

static bool stop_test(double rn, double r0, const SolverOptions& o) {
  return rn < o.absoluteTolerance || rn / r0 < o.relativeTolerance;
}

// AMG::solve (AMG.cpp:220-282): r0 = |b + A x|, then cycles until the L1
// ratio drops below relTol. With mixed precision each cycle runs in FP32
// on the FP64 residual and its correction is added in FP64 (iterative
// refinement), so the stopping test is always on the FP64 residual.
SolveReport LinearSolve::solveAMG(cudaStream_t st) {
  const SolverOptions& o = h_.options();
  DevLevel& d = h_.level(0);
  SolveReport rep;
  CUDA_OK(cudaMemsetAsync(d.x, 0, sizeof(double) * (size_t)n_, st));
  if (learned_) CUDA_OK(cudaMemsetAsync(scal_ + kLsAccepted, 0, 3 * sizeof(double), st));
  dev::residual<double>(d.view64(), d.nSlices, d.x, d.b, d.r, d.partials, st);
  dev::sum_partials(d.nPartials, d.partials, scal_ + kNorm, st);
  launches += 3;
  const double r0 = fetch(scal_ + kNorm, st);
  rep.initialNorm = r0;
  rep.finalNorm = r0;
  rep.history.push_back(r0);
  if (o.verbosity > 0) printf("0: %g\n", r0);
  if (!std::isfinite(r0)) throw Error(kNaN, "initial residual is not finite");
  if (r0 < o.absoluteTolerance) {
    rep.converged = true;
    return rep;
  }
  for (int i = 1; i < o.nMaxIterations; i++) {
    const bool useLs = learned_ && learnedActive_;
    run(useLs ? g4_ : g1_, st, [&] {
      if (o.precision == kMixed) {
        dev::convert_d2f(n_, d.r, d.bF, st);
        h_.runCycle<float>(st, true);
        dev::add_f2d(n_, d.xF, d.x, st);
      } else {
        h_.runCycle<double>(st);
      }
      dev::residual<double>(d.view64(), d.nSlices, d.x, d.b, d.r, d.partials, st);
      dev::sum_partials(d.nPartials, d.partials, scal_ + kNorm, st);
      if (useLs) {
        learnedStep(st, d.x, d.r, 1.0);
        CUDA_OK(cudaMemcpyAsync(hostScal_ + 1, scal_ + kLsAccepted, sizeof(double), cudaMemcpyDeviceToHost, st));
        CUDA_OK(cudaMemcpyAsync(hostScal_ + 2, scal_ + kLsUseful, sizeof(double), cudaMemcpyDeviceToHost, st));
      }
      CUDA_OK(cudaMemcpyAsync(hostScal_, scal_ + kNorm, sizeof(double), cudaMemcpyDeviceToHost, st));
    });
    CUDA_OK(cudaStreamSynchronize(st));
    const double rn = hostScal_[0];
    if (useLs) {
      // Any step that lowers the residual is kept. The step is retired for
      // good once it has been tried kLsProbe times and fewer than a quarter
      // of the tries cut the residual by the factor that pays for its cost
      // (the correction's useful factor).
      const int kept = (int)hostScal_[1], useful = (int)hostScal_[2];
      rep.learnedSteps++;
      lsTries_++;
      lsKept_ += useful - rep.learnedUseful;
      rep.learnedAccepted = kept;
      rep.learnedUseful = useful;
      if (lsTries_ >= kLsProbe && 4 * lsKept_ < lsTries_) learnedActive_ = false;
    }
    rep.iterations = i;
    rep.finalNorm = rn;
    rep.history.push_back(rn);
    if (o.verbosity > 0) printf("%d: %g\n", i, rn);
    if (!std::isfinite(rn)) throw Error(kNaN, "residual became non-finite");
    if (stop_test(rn, r0, o)) {
      rep.converged = true;
      break;
    }
  }
  return rep;
}

// JacobiSolver::solve (fvmbase/JacobiSolver.cpp:42-80): one Jacobi sweep
// per iteration, same stopping test as the AMG solve.
SolveReport LinearSolve::solveJacobi(cudaStream_t st) {
  const SolverOptions& o = h_.options();
  DevLevel& d = h_.level(0);
  SolveReport rep;
  CUDA_OK(cudaMemsetAsync(d.x, 0, sizeof(double) * (size_t)n_, st));
  dev::residual<double>(d.view64(), d.nSlices, d.x, d.b, d.r, d.partials, st);
  dev::sum_partials(d.nPartials, d.partials, scal_ + kNorm, st);
  launches += 3;
  const double r0 = fetch(scal_ + kNorm, st);
  rep.initialNorm = rep.finalNorm = r0;
  rep.history.push_back(r0);
  if (!std::isfinite(r0)) throw Error(kNaN, "initial residual is not finite");
  if (r0 < o.absoluteTolerance) {
    rep.converged = true;
    return rep;
  }
  for (int i = 1; i < o.nMaxIterations; i++) {
    run(g5_, st, [&] {
      dev::jacobi<double>(d.view64(), d.nSlices, d.x, d.tmp, d.b, st);
      dev::copy_d(n_, d.tmp, d.x, st);
      dev::residual<double>(d.view64(), d.nSlices, d.x, d.b, d.r, d.partials, st);
      dev::sum_partials(d.nPartials, d.partials, scal_ + kNorm, st);
      CUDA_OK(cudaMemcpyAsync(hostScal_, scal_ + kNorm, sizeof(double), cudaMemcpyDeviceToHost, st));
    });
    CUDA_OK(cudaStreamSynchronize(st));
    const double rn = hostScal_[0];
    rep.iterations = i;
    rep.finalNorm = rn;
    rep.history.push_back(rn);
    if (o.verbosity > 0) printf("%d: %g\n", i, rn);
    if (!std::isfinite(rn)) throw Error(kNaN, "residual became non-finite");
    if (stop_test(rn, r0, o)) {
      rep.converged = true;
      break;
    }
  }
  return rep;
}

void LinearSolve::setLearned(LearnedCorrection* lc) {
  if (lc != learned_) {
    if (g4_) cudaGraphExecDestroy(g4_);
    g4_ = nullptr;
  }
  learned_ = lc;
  // a network whose measured residual reduction cannot pay is not tried
  learnedActive_ = !(lc && lc->residualFactor() >= 0.0 && lc->residualFactor() > lc->usefulFactor());
  lsTries_ = lsKept_ = 0;
  if (lc) lc->prepare(n_, (long long)h_.level(0).entries);
}

// Flexible learned step after an AMG refinement iteration: d = N(r),
// q = A d, alpha = -(r.q)/(q.q), kept (x += alpha d, r += alpha q) only
// when the FP64 L1 norm of r + alpha q is below acceptFactor times that of
// r. Scalars stay on the device, so the step is part of the captured
// iteration graph.
void LinearSolve::learnedStep(cudaStream_t st, double* x, double* r, double acceptFactor) {
  DevLevel& d = h_.level(0);
  double* D = work_ + 6 * (size_t)n_;
  double* Q = work_ + 7 * (size_t)n_;
  double* RT = work_ + 8 * (size_t)n_;
  const nn::Graph g{d.view64(), d.rowSlice, d.nSlices, (long long)d.entries};
  learned_->apply(g, r, D, scal_ + kLsScale, st);
  dev::spmv(d.view64(), d.nSlices, D, Q, st);
  dot_into(r, Q, scal_ + kLsRq, st);
  dot_into(Q, Q, scal_ + kLsQq, st);
  nn::step_alpha(scal_ + kLsRq, scal_ + kLsQq, scal_ + kLsAlpha, st);
  nn::step_trial(n_, r, Q, scal_ + kLsAlpha, RT, partials_, st);
  dev::sum_partials(dev::vec_blocks(n_), partials_, scal_ + kLsTrial, st);
  nn::step_accept(n_, x, D, r, RT, scal_ + kLsAlpha, scal_ + kNorm, scal_ + kLsTrial, acceptFactor, st);
  nn::step_finish(scal_ + kNorm, scal_ + kLsTrial, scal_ + kLsAccepted, scal_ + kLsSteps, scal_ + kLsUseful,
                  learned_->usefulFactor(), acceptFactor, st);
  launches += 19;
}

int LinearSolve::solveRecording(cudaStream_t st, double relTol, int maxIter, int record,
                                const std::vector<double*>& rs, const std::vector<double*>& xs, SolveReport& rep) {
  const SolverOptions& o = h_.options();
  DevLevel& d = h_.level(0);
  const size_t nb = sizeof(double) * (size_t)n_;
  rep = SolveReport();
  CUDA_OK(cudaMemsetAsync(d.x, 0, nb, st));
  dev::residual<double>(d.view64(), d.nSlices, d.x, d.b, d.r, d.partials, st);
  dev::sum_partials(d.nPartials, d.partials, scal_ + kNorm, st);
  const double r0 = fetch(scal_ + kNorm, st);
  rep.initialNorm = rep.finalNorm = r0;
  rep.history.push_back(r0);
  int recorded = 0;
  auto keep = [&]() {
    if (recorded < record) {
      CUDA_OK(cudaMemcpyAsync(rs[recorded], d.r, nb, cudaMemcpyDeviceToDevice, st));
      CUDA_OK(cudaMemcpyAsync(xs[recorded], d.x, nb, cudaMemcpyDeviceToDevice, st));
      recorded++;
    }
  };
  if (!(r0 > 0.0)) return 0;
  keep();
  for (int i = 1; i < maxIter; i++) {
    if (o.precision == kMixed) {
      dev::convert_d2f(n_, d.r, d.bF, st);
      h_.runCycle<float>(st, true);
      dev::add_f2d(n_, d.xF, d.x, st);
    } else {
      h_.runCycle<double>(st);
    }
    dev::residual<double>(d.view64(), d.nSlices, d.x, d.b, d.r, d.partials, st);
    dev::sum_partials(d.nPartials, d.partials, scal_ + kNorm, st);
    const double rn = fetch(scal_ + kNorm, st);
    rep.iterations = i;
    rep.finalNorm = rn;
    rep.history.push_back(rn);
    if (!std::isfinite(rn)) throw Error(kNaN, "residual became non-finite");
    if (rn / r0 < relTol) {
      rep.converged = true;
      break;
    }
    keep();
  }
  return recorded;
}

// CG::solve (CG.cpp:26-139) with the AMG cycle as preconditioner. The
// reference's beta = rho_k+1 / rho_k assumes a symmetric preconditioner;
// the FP32 cycle and cycles with nPreSweeps != nPostSweeps are not, so
// those use the flexible (Polak-Ribiere) beta (r_k+1, z_k+1 - z_k) / rho_k,
// equal to the reference's in exact arithmetic for a symmetric one.
SolveReport LinearSolve::solveCG(cudaStream_t st) {
  const SolverOptions& o = h_.options();
  DevLevel& d = h_.level(0);
  double* X = work_;
  double* R = work_ + (size_t)n_;
  double* Z = work_ + 2 * (size_t)n_;
  double* P = work_ + 3 * (size_t)n_;
  double* Q = work_ + 4 * (size_t)n_;
  double* B = work_ + 5 * (size_t)n_;
  const bool flexible = cgFlexible();
  SolveReport rep;
  // the whole solve on the device when nothing needs the host between
  // iterations (no learned step, no printing)
  if (o.preconditioner == kPrecAMG && o.useGraphs && o.verbosity <= 0 && !(learned_ && learnedActive_) &&
      !graphsFailed_ && solveCGLoop(st, flexible, rep))
    return rep;
  if (getenv("FVM_TRACE"))
    fprintf(stderr, "[fvm solve] CG on the host loop (learned step %s, graphs %s, loop graph %s)\n",
            learned_ && learnedActive_ ? "active" : "inactive", graphsFailed_ ? "failed" : "ok",
            loopFailed_ ? "failed" : "ok");
  CUDA_OK(cudaMemsetAsync(X, 0, sizeof(double) * (size_t)n_, st));
  CUDA_OK(cudaMemsetAsync(P, 0, sizeof(double) * (size_t)n_, st));
  CUDA_OK(cudaMemsetAsync(Z, 0, sizeof(double) * (size_t)n_, st));  // z_0 enters the first flexible beta
  dev::copy_d(n_, d.b, B, st);
  // r = b at x = 0, with its norm (the FP32 copy below, when the cycle takes it)
  dev::cg_start(n_, B, R, nullptr, partials_, st);
  dev::sum_partials(dev::vec_blocks(n_), partials_, scal_ + kNorm, st);
  {
    const double inf = std::numeric_limits<double>::infinity();
    CUDA_OK(cudaMemcpyAsync(scal_ + kRho, &inf, sizeof(double), cudaMemcpyHostToDevice, st));
  }
  const double r0 = fetch(scal_ + kNorm, st);
  rep.initialNorm = r0;
  rep.finalNorm = r0;
  rep.history.push_back(r0);
  if (o.verbosity > 0) printf("0: %g\n", r0);
  if (!std::isfinite(r0)) throw Error(kNaN, "initial residual is not finite");
  // With the AMG preconditioner the vector work of an iteration is fused:
  // z taken from the cycle with both dots, beta; p update; q = A p with
  // p.q; alpha; the x and r updates with |r|.
  const bool fused = o.preconditioner == kPrecAMG;
  const bool mixedCycle = o.precision == kMixed;
  // the FP32 cycle's right-hand side: r in FP32, written by each update
  float* rF = fused && mixedCycle ? d.bF : nullptr;
  if (rF) {
    dev::convert_d2f(n_, R, rF, st);
    launches += 1;
  }
  for (int i = 0; i < o.nMaxIterations; i++) {
    // learned post-correction of the preconditioner (flexible CG): after the
    // cycle's z1, the network corrects the residual r + A z1 that z1 leaves,
    // with the step length alpha that minimises |r + A z1 + alpha A d|_2
    const bool useLs = fused && learned_ && learnedActive_;
    if (useLs) {
      double* D1 = work_ + 6 * (size_t)n_;
      double* R1 = work_ + 7 * (size_t)n_;
      double* DN = work_ + 8 * (size_t)n_;
      double* Q2 = work_ + 9 * (size_t)n_;
      double* RT = work_ + 10 * (size_t)n_;
      run(g4_, st, [&] {
        h_.applyCycle(R, st);
        const int gb = (n_ + 255) / 256;
        if (mixedCycle)
          k_f2d<<<gb, 256, 0, st>>>(n_, d.xF, D1);
        else
          dev::copy_d(n_, d.x, D1, st);
        dev::spmv(d.view64(), d.nSlices, D1, R1, st);
        k_add_vec<<<gb, 256, 0, st>>>(n_, R, R1, R1);
        const nn::Graph g{d.view64(), d.rowSlice, d.nSlices, (long long)d.entries};
        learned_->apply(g, R1, DN, scal_ + kLsScale, st);
        dev::spmv(d.view64(), d.nSlices, DN, Q2, st);
        dot_into(R1, Q2, scal_ + kLsRq, st);
        dot_into(Q2, Q2, scal_ + kLsQq, st);
        nn::step_alpha(scal_ + kLsRq, scal_ + kLsQq, scal_ + kLsAlpha, st);
        norm_into(R1, scal_ + kLsBefore, st);
        nn::step_trial(n_, R1, Q2, scal_ + kLsAlpha, RT, partials_, st);
        dev::sum_partials(dev::vec_blocks(n_), partials_, scal_ + kLsTrial, st);
        k_combine<<<gb, 256, 0, st>>>(n_, D1, scal_ + kLsAlpha, DN, D1);
        dev::cg_take_z<double>(n_, D1, R, Z, partials2_, st);
        dev::cg_beta(dev::vec_blocks(n_), partials2_, scal_ + kRho, scal_ + kRhoPrev, scal_ + kBeta, flexible, st);
        dev::xpby_dev(n_, Z, scal_ + kBeta, P, st);
        dev::spmv_dot(d.view64(), d.nSlices, P, Q, partials2_, st);
        dev::cg_alpha(dev::spmv_dot_blocks(d.view64(), d.nSlices), partials2_, scal_ + kRho, scal_ + kAlpha, st);
        dev::cg_update(n_, scal_ + kAlpha, P, Q, X, R, partials_, st, rF);
        dev::sum_partials(dev::vec_blocks(n_), partials_, scal_ + kNorm, st);
        CUDA_OK(cudaMemcpyAsync(hostScal_, scal_ + kNorm, sizeof(double), cudaMemcpyDeviceToHost, st));
        CUDA_OK(cudaMemcpyAsync(hostScal_ + 1, scal_ + kLsBefore, sizeof(double), cudaMemcpyDeviceToHost, st));
        CUDA_OK(cudaMemcpyAsync(hostScal_ + 2, scal_ + kLsTrial, sizeof(double), cudaMemcpyDeviceToHost, st));
      });
      launches += 6;
    } else if (fused) {
      run(g1_, st, [&] {
        if (mixedCycle)
          h_.runCycle<float>(st, true);  // on rF, level 0's FP32 right-hand side
        else
          h_.applyCycle(R, st);
        if (mixedCycle)
          dev::cg_take_z<float>(n_, d.xF, R, Z, partials2_, st);
        else
          dev::cg_take_z<double>(n_, d.x, R, Z, partials2_, st);
        dev::cg_beta(dev::vec_blocks(n_), partials2_, scal_ + kRho, scal_ + kRhoPrev, scal_ + kBeta, flexible, st);
        dev::spmv_dot_pby(d.view64(), d.nSlices, Z, P, scal_ + kBeta, Q, partials2_, st);
        dev::cg_alpha(dev::spmv_dot_blocks(d.view64(), d.nSlices), partials2_, scal_ + kRho, scal_ + kAlpha, st);
        dev::cg_update_pby(n_, scal_ + kAlpha, Z, scal_ + kBeta, P, Q, X, R, partials_, st, rF);
        dev::sum_partials(dev::vec_blocks(n_), partials_, scal_ + kNorm, st);
        CUDA_OK(cudaMemcpyAsync(hostScal_, scal_ + kNorm, sizeof(double), cudaMemcpyDeviceToHost, st));
      });
    } else {
      run(g1_, st, [&] {
        if (flexible) dot_into(R, Z, scal_ + kRzPrev, st);  // (r_k+1, z_k) before z is replaced
        h_.apply(R, Z, st);
        dev::copy_d(1, scal_ + kRho, scal_ + kRhoPrev, st);
        dot_into(R, Z, scal_ + kRho, st);
        if (flexible)
          dev::scalar_flex_beta(scal_ + kRho, scal_ + kRzPrev, scal_ + kRhoPrev, scal_ + kBeta, st);
        else
          dev::scalar_div(scal_ + kRho, scal_ + kRhoPrev, scal_ + kBeta, st);  // 0 on the first pass
        dev::xpby_dev(n_, Z, scal_ + kBeta, P, st);
        dev::spmv(d.view64(), d.nSlices, P, Q, st);
        dot_into(P, Q, scal_ + kPtq, st);
        dev::scalar_div(scal_ + kRho, scal_ + kPtq, scal_ + kAlpha, st);
        dev::axpy_dev(n_, scal_ + kAlpha, -1.0, P, X, st);
        dev::axpy_dev(n_, scal_ + kAlpha, -1.0, Q, R, st);
        norm_into(R, scal_ + kNorm, st);
        CUDA_OK(cudaMemcpyAsync(hostScal_, scal_ + kNorm, sizeof(double), cudaMemcpyDeviceToHost, st));
      });
    }
    CUDA_OK(cudaStreamSynchronize(st));
    const double rn = hostScal_[0];
    if (useLs) {
      // the step pays when it cuts the residual z1 leaves by the useful factor;
      // after kLsProbe tries it is retired if fewer than a quarter did
      const double before = hostScal_[1], after = hostScal_[2];
      const bool useful = std::isfinite(after) && after < learned_->usefulFactor() * before;
      rep.learnedSteps++;
      rep.learnedAccepted += useful ? 1 : 0;
      rep.learnedUseful += useful ? 1 : 0;
      lsTries_++;
      lsKept_ += useful ? 1 : 0;
      if (lsTries_ >= kLsProbe && 4 * lsKept_ < lsTries_) learnedActive_ = false;
    }
    rep.iterations = i + 1;
    rep.finalNorm = rn;
    rep.history.push_back(rn);
    if (o.verbosity > 0) printf("%d: %g\n", i + 1, rn);
    if (!std::isfinite(rn)) throw Error(kNaN, "residual became non-finite");
    if (stop_test(rn, r0, o)) {
      rep.converged = true;
      break;
    }
  }
  // the recursively updated R can drift from b + A x: the reported final
  // norm is that of the true residual
  if (rep.iterations > 0) {
    dev::residual<double>(d.view64(), d.nSlices, X, B, R, nullptr, st);
    norm_into(R, scal_ + kNorm, st);
    rep.finalNorm = fetch(scal_ + kNorm, st);
    rep.history.back() = rep.finalNorm;
  }
  // restore the system: delta = X, b = original
  dev::copy_d(n_, X, d.x, st);
  dev::copy_d(n_, B, d.b, st);
  CUDA_OK(cudaStreamSynchronize(st));
  return rep;
}

bool graph_leaves(cudaGraph_t g, std::vector<cudaGraphNode_t>& leaves) {
  leaves.clear();
  size_t nn = 0;
  if (cudaGraphGetNodes(g, nullptr, &nn) != cudaSuccess) return false;
  std::vector<cudaGraphNode_t> nodes(nn);
  if (nn && cudaGraphGetNodes(g, nodes.data(), &nn) != cudaSuccess) return false;
  for (size_t k = 0; k < nn; k++) {
    size_t nd = 0;
    if (cudaGraphNodeGetDependentNodes(nodes[k], nullptr, &nd) != cudaSuccess) return false;
    if (nd == 0) leaves.push_back(nodes[k]);
  }
  return true;
}

bool LinearSolve::addCGLoop(cudaGraph_t g, cudaStream_t st, bool flexible, bool hostCopies) {
  const SolverOptions& o = h_.options();
  DevLevel& d = h_.level(0);
  const bool mixedCycle = o.precision == kMixed;
  // The FP32 cycle works on level 0's FP32 vectors only, so the iterate and
  // the right-hand side can be level 0's own FP64 x and b: no copy in, no
  // restore. The FP64 cycle overwrites them, so it keeps copies.
  double* X = mixedCycle ? d.x : work_;
  double* R = work_ + (size_t)n_;
  double* Z = work_ + 2 * (size_t)n_;
  double* P = work_ + 3 * (size_t)n_;
  double* Q = work_ + 4 * (size_t)n_;
  double* B = mixedCycle ? d.b : work_ + 5 * (size_t)n_;
  if (!loopInt_) loopInt_ = (int*)h_.scratch(4 * sizeof(int));
  if (!history_ || historyCap_ < o.nMaxIterations + 2) {
    history_ = (double*)h_.scratch(sizeof(double) * (size_t)(o.nMaxIterations + 2));
    historyCap_ = o.nMaxIterations + 2;
  }
  const cudaStreamCaptureMode mode = cudaStreamCaptureModeThreadLocal;
  cudaGraphConditionalHandle h = 0;
  // the loop goes after whatever g already holds
  std::vector<cudaGraphNode_t> before;
  bool ok = graph_leaves(g, before) &&
            cudaGraphConditionalHandleCreate(&h, g, 0, cudaGraphCondAssignDefault) == cudaSuccess;
  // prologue: x = 0, p = 0, z = 0, r = b, |r| (host copies of b kept in B)
  ok = ok && cudaStreamBeginCaptureToGraph(st, g, before.empty() ? nullptr : before.data(), nullptr, before.size(),
                                           mode) == cudaSuccess;
  if (ok) {
    try {
      CUDA_OK(cudaMemsetAsync(X, 0, sizeof(double) * (size_t)n_, st));
      CUDA_OK(cudaMemsetAsync(P, 0, sizeof(double) * (size_t)n_, st));
      CUDA_OK(cudaMemsetAsync(Z, 0, sizeof(double) * (size_t)n_, st));
      if (B != d.b) dev::copy_d(n_, d.b, B, st);
      // r = b at x = 0, with its norm and the FP32 cycle's right-hand side
      dev::cg_start(n_, B, R, mixedCycle ? d.bF : nullptr, partials_, st);
      dev::sum_partials(dev::vec_blocks(n_), partials_, scal_ + kNorm, st);
      k_cg_loop_init<<<1, 1, 0, st>>>(scal_, loopInt_, history_, o.absoluteTolerance, o.nMaxIterations, h);
    } catch (const Error&) {
      ok = false;
    }
    cudaGraph_t gg = nullptr;
    ok = cudaStreamEndCapture(st, &gg) == cudaSuccess && ok;
  }
  // the while node after the prologue's last node
  cudaGraphNode_t cnode = nullptr;
  cudaGraph_t body = nullptr;
  if (ok) {
    std::vector<cudaGraphNode_t> leaves;
    ok = graph_leaves(g, leaves);
    cudaGraphNodeParams cp = {};
    cp.type = cudaGraphNodeTypeConditional;
    cp.conditional.handle = h;
    cp.conditional.type = cudaGraphCondTypeWhile;
    cp.conditional.size = 1;
    ok = ok && !leaves.empty() && cudaGraphAddNode(&cnode, g, leaves.data(), leaves.size(), &cp) == cudaSuccess;
    if (ok) body = cp.conditional.phGraph_out[0];
  }
  // body: one fused iteration and the convergence check
  ok = ok && cudaStreamBeginCaptureToGraph(st, body, nullptr, nullptr, 0, mode) == cudaSuccess;
  if (ok) {
    try {
      // the FP32 cycle runs on level 0's bF, which the prologue and each
      // update write (r in FP32)
      if (mixedCycle)
        h_.runCycle<float>(st, true);
      else
        h_.applyCycle(R, st);
      if (mixedCycle)
        dev::cg_take_z<float>(n_, d.xF, R, Z, partials2_, st);
      else
        dev::cg_take_z<double>(n_, d.x, R, Z, partials2_, st);
      dev::cg_beta(dev::vec_blocks(n_), partials2_, scal_ + kRho, scal_ + kRhoPrev, scal_ + kBeta, flexible, st);
      // p = p * beta + z is formed by the SpMV where it reads p and written
      // by the update: no pass of its own
      dev::spmv_dot_pby(d.view64(), d.nSlices, Z, P, scal_ + kBeta, Q, partials2_, st);
      dev::cg_alpha(dev::spmv_dot_blocks(d.view64(), d.nSlices), partials2_, scal_ + kRho, scal_ + kAlpha, st);
      dev::cg_update_pby(n_, scal_ + kAlpha, Z, scal_ + kBeta, P, Q, X, R, partials_, st,
                         mixedCycle ? d.bF : nullptr);
      dev::sum_partials(dev::vec_blocks(n_), partials_, scal_ + kNorm, st);
      k_cg_loop_check<<<1, 1, 0, st>>>(scal_, loopInt_, history_, o.relativeTolerance, o.absoluteTolerance,
                                       o.nMaxIterations, h);
    } catch (const Error&) {
      ok = false;
    }
    cudaGraph_t bb = nullptr;
    ok = cudaStreamEndCapture(st, &bb) == cudaSuccess && ok;
    size_t nb = 0;
    if (ok) cudaGraphGetNodes(body, nullptr, &nb);
    loopBodyNodes_ = (long long)nb;
  }
  // epilogue: the system restored; with hostCopies the true residual's norm
  // and the results to the pinned host scalars (inside an outer loop nothing
  // reads that norm)
  ok = ok && cudaStreamBeginCaptureToGraph(st, g, &cnode, nullptr, 1, mode) == cudaSuccess;
  if (ok) {
    try {
      if (hostCopies) {
        dev::residual<double>(d.view64(), d.nSlices, X, B, R, nullptr, st);
        norm_into(R, scal_ + kNorm, st);
      }
      if (X != d.x) dev::copy_d(n_, X, d.x, st);
      if (B != d.b) dev::copy_d(n_, B, d.b, st);
      if (hostCopies) {
        CUDA_OK(cudaMemcpyAsync(hostScal_, scal_ + kNorm, sizeof(double), cudaMemcpyDeviceToHost, st));
        CUDA_OK(cudaMemcpyAsync(hostScal_ + 1, history_, sizeof(double), cudaMemcpyDeviceToHost, st));
        CUDA_OK(cudaMemcpyAsync(hostScal_ + 2, loopInt_, 2 * sizeof(int), cudaMemcpyDeviceToHost, st));
      }
    } catch (const Error&) {
      ok = false;
    }
    cudaGraph_t ee = nullptr;
    ok = cudaStreamEndCapture(st, &ee) == cudaSuccess && ok;
  }
  if (!ok) cudaGetLastError();
  return ok;
}

// The FP32 cycle, unequal sweeps, W cycles, one-directional or Chebyshev
// smoothing make the preconditioner non-symmetric or variable: CG then takes
// the flexible (Polak-Ribiere) beta.
bool LinearSolve::cgFlexible() const {
  const SolverOptions& o = h_.options();
  return o.preconditioner == kPrecAMG &&
         (o.precision == kMixed || o.nPreSweeps != o.nPostSweeps || o.cycleType != kVCycle || !o.gsReverse ||
          o.chebyshevDegree > 0);
}

bool LinearSolve::deviceSolvable() const {
  const SolverOptions& o = h_.options();
  return o.solver == kSolverCG && o.preconditioner == kPrecAMG && o.useGraphs && o.verbosity <= 0 &&
         !(learned_ && learnedActive_) && !graphsFailed_ && !loopFailed_;
}

LinearSolve::LoopKey LinearSolve::loopKey() const {
  const SolverOptions& o = h_.options();
  return LoopKey{cgFlexible(), o.nMaxIterations, o.relativeTolerance, o.absoluteTolerance};
}

void LinearSolve::prebuild(cudaStream_t st) {
  if (!deviceSolvable() || gLoop_) return;
  if (!buildCGLoop(st, cgFlexible())) loopFailed_ = true;
}

bool LinearSolve::appendDeviceSolve(cudaGraph_t g, cudaStream_t st) {
  return deviceSolvable() && addCGLoop(g, st, cgFlexible(), false);
}

bool LinearSolve::buildCGLoop(cudaStream_t st, bool flexible) {
  const SolverOptions& o = h_.options();
  if (gLoop_) cudaGraphExecDestroy(gLoop_);
  gLoop_ = nullptr;
  cudaGraph_t g = nullptr;
  bool ok = cudaGraphCreate(&g, 0) == cudaSuccess && addCGLoop(g, st, flexible, true);
  if (ok) {
    size_t nn = 0;
    cudaGraphGetNodes(g, nullptr, &nn);
    loopOtherNodes_ = (long long)nn - 1;  // all but the while node
  }
  ok = ok && cudaGraphInstantiate(&gLoop_, g, 0) == cudaSuccess;
  if (g) cudaGraphDestroy(g);
  if (!ok) {
    if (gLoop_) cudaGraphExecDestroy(gLoop_);
    gLoop_ = nullptr;
    cudaGetLastError();
    return false;
  }
  loopFlexible_ = flexible;
  loopMaxIt_ = o.nMaxIterations;
  loopRel_ = o.relativeTolerance;
  loopAbs_ = o.absoluteTolerance;
  return true;
}

bool LinearSolve::solveCGLoop(cudaStream_t st, bool flexible, SolveReport& rep) {
  const SolverOptions& o = h_.options();
  if (loopFailed_) return false;
  if (!gLoop_ || loopFlexible_ != flexible || loopMaxIt_ != o.nMaxIterations || loopRel_ != o.relativeTolerance ||
      loopAbs_ != o.absoluteTolerance) {
    if (!buildCGLoop(st, flexible)) {
      loopFailed_ = true;
      return false;
    }
  }
  CUDA_OK(cudaGraphLaunch(gLoop_, st));
  CUDA_OK(cudaStreamSynchronize(st));
  const double finalNorm = hostScal_[0];
  const double r0 = hostScal_[1];
  int loop[2];
  std::memcpy(loop, hostScal_ + 2, sizeof(loop));
  const int iters = loop[0], status = loop[1];
  launches += loopOtherNodes_ + (long long)iters * loopBodyNodes_;
  rep = SolveReport();
  rep.initialNorm = r0;
  rep.iterations = iters;
  rep.history.assign((size_t)iters + 1, 0.0);
  if (iters > 0)
    CUDA_OK(cudaMemcpy(rep.history.data(), history_, sizeof(double) * (iters + 1), cudaMemcpyDeviceToHost));
  else
    rep.history[0] = r0;
  if (!std::isfinite(r0)) throw Error(kNaN, "initial residual is not finite");
  if (status == 2) throw Error(kNaN, "residual became non-finite");
  rep.converged = status == 1;
  rep.finalNorm = iters > 0 ? finalNorm : r0;
  if (iters > 0) rep.history.back() = rep.finalNorm;
  return true;
}

// BCGStab::solve (BCGStab.cpp:27-170) with the AMG cycle as preconditioner.
SolveReport LinearSolve::solveBCGStab(cudaStream_t st) {
  const SolverOptions& o = h_.options();
  DevLevel& d = h_.level(0);
  double* X = work_;
  double* R = work_ + (size_t)n_;
  double* RT = work_ + 2 * (size_t)n_;
  double* P = work_ + 3 * (size_t)n_;
  double* PH = work_ + 4 * (size_t)n_;
  double* V = work_ + 5 * (size_t)n_;
  double* Tt = work_ + 6 * (size_t)n_;
  double* B = work_ + 7 * (size_t)n_;
  SolveReport rep;
  CUDA_OK(cudaMemsetAsync(X, 0, sizeof(double) * (size_t)n_, st));
  CUDA_OK(cudaMemsetAsync(P, 0, sizeof(double) * (size_t)n_, st));
  CUDA_OK(cudaMemsetAsync(V, 0, sizeof(double) * (size_t)n_, st));
  dev::copy_d(n_, d.b, B, st);
  dev::residual<double>(d.view64(), d.nSlices, X, B, R, nullptr, st);
  dev::copy_d(n_, R, RT, st);
  norm_into(R, scal_ + kNorm, st);
  {
    // first pass: beta = (rho / inf) * (alpha / omega) = 0, so p = r
    const double init[3] = {std::numeric_limits<double>::infinity(), 0.0, 1.0};
    CUDA_OK(cudaMemcpyAsync(scal_ + kRho, &init[0], sizeof(double), cudaMemcpyHostToDevice, st));
    CUDA_OK(cudaMemcpyAsync(scal_ + kAlpha, &init[1], sizeof(double), cudaMemcpyHostToDevice, st));
    CUDA_OK(cudaMemcpyAsync(scal_ + kOmega, &init[2], sizeof(double), cudaMemcpyHostToDevice, st));
  }
  const double r0 = fetch(scal_ + kNorm, st);
  rep.initialNorm = r0;
  rep.finalNorm = r0;
  rep.history.push_back(r0);
  if (o.verbosity > 0) printf("0: %g\n", r0);
  if (!std::isfinite(r0)) throw Error(kNaN, "initial residual is not finite");
  for (int i = 0; i < o.nMaxIterations; i++) {
    run(g1_, st, [&] {
      dev::copy_d(1, scal_ + kRho, scal_ + kRhoPrev, st);
      dot_into(R, RT, scal_ + kRho, st);
      dev::scalar_ratio_product(scal_ + kRho, scal_ + kRhoPrev, scal_ + kAlpha, scal_ + kOmega,
                                scal_ + kBeta, st);
      dev::bicg_p_update(n_, R, V, scal_ + kOmega, scal_ + kBeta, P, st);
      h_.apply(P, PH, st);
      dev::spmv(d.view64(), d.nSlices, PH, V, st);
      dot_into(RT, V, scal_ + kRtv, st);
      dev::scalar_div(scal_ + kRho, scal_ + kRtv, scal_ + kAlpha, st);
      dev::axpy_dev(n_, scal_ + kAlpha, -1.0, PH, X, st);
      dev::axpy_dev(n_, scal_ + kAlpha, -1.0, V, R, st);
      norm_into(R, scal_ + kNorm, st);
      CUDA_OK(cudaMemcpyAsync(hostScal_, scal_ + kNorm, sizeof(double), cudaMemcpyDeviceToHost, st));
    });
    CUDA_OK(cudaStreamSynchronize(st));
    double rn = hostScal_[0];
    rep.iterations = i + 1;
    if (!std::isfinite(rn)) throw Error(kNaN, "residual became non-finite");
    if (rn < o.absoluteTolerance) {
      rep.finalNorm = rn;
      rep.history.push_back(rn);
      rep.converged = true;
      break;
    }
    run(g2_, st, [&] {
      double* SH = PH;
      h_.apply(R, SH, st);
      dev::spmv(d.view64(), d.nSlices, SH, Tt, st);
      dot_into(Tt, R, scal_ + kTdotr, st);
      dot_into(Tt, Tt, scal_ + kTdott, st);
      dev::scalar_div(scal_ + kTdotr, scal_ + kTdott, scal_ + kOmega, st);
      dev::axpy_dev(n_, scal_ + kOmega, -1.0, SH, X, st);
      dev::axpy_dev(n_, scal_ + kOmega, -1.0, Tt, R, st);
      norm_into(R, scal_ + kNorm, st);
      CUDA_OK(cudaMemcpyAsync(hostScal_, scal_ + kNorm, sizeof(double), cudaMemcpyDeviceToHost, st));
    });
    CUDA_OK(cudaStreamSynchronize(st));
    rn = hostScal_[0];
    rep.finalNorm = rn;
    rep.history.push_back(rn);
    if (o.verbosity > 0) printf("%d: %g\n", i + 1, rn);
    if (!std::isfinite(rn)) throw Error(kNaN, "residual became non-finite");
    if (stop_test(rn, r0, o)) {
      rep.converged = true;
      break;
    }
  }
  if (rep.iterations > 0) {
    dev::residual<double>(d.view64(), d.nSlices, X, B, R, nullptr, st);
    norm_into(R, scal_ + kNorm, st);
    rep.finalNorm = fetch(scal_ + kNorm, st);
    if (!rep.history.empty()) rep.history.back() = rep.finalNorm;
  }
  dev::copy_d(n_, X, d.x, st);
  dev::copy_d(n_, B, d.b, st);
  CUDA_OK(cudaStreamSynchronize(st));
  return rep;
}

}  // namespace fvm
