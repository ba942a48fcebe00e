// Shared host-side definitions for the fvm_b200 library: error reporting,
// compressed-row (CSR) containers and CUDA call checking.
#pragma once

#include <nvtx3/nvToolsExt.h>

#include <algorithm>
#include <cstdint>
#include <stdexcept>
#include <string>
#include <thread>
#include <vector>

namespace fvm {

// An NVTX range over a scope (setup phases, outer iterations, linear
// solves): visible on a profiler's timeline, no cost without one.
struct TraceRange {
  explicit TraceRange(const char* name) { nvtxRangePushA(name); }
  ~TraceRange() { nvtxRangePop(); }
  TraceRange(const TraceRange&) = delete;
  TraceRange& operator=(const TraceRange&) = delete;
};

// Status codes returned through the C ABI (mirrored in include/fvm_b200.h).
enum Status {
  kOk = 0,
  kBadArgument = 1,
  kBadMesh = 2,
  kNotConverged = 3,
  kNaN = 4,
  kDeviceError = 5,
  kLearnedRejected = 6,
  kUnsupported = 7,
  kTooLarge = 8,
};

// An error raised anywhere below the C ABI; the ABI turns it into a status
// code plus a message readable through fvm_last_error(). This mirrors the
// reference's CException, which SWIG maps onto RuntimeError.
struct Error : std::runtime_error {
  int status;
  Error(int s, const std::string& m) : std::runtime_error(m), status(s) {}
};

void set_last_error(const std::string& msg);
const char* last_error();

#define FVM_REQUIRE(cond, status, msg)                 \
  do {                                                 \
    if (!(cond)) throw ::fvm::Error((status), (msg)); \
  } while (0)

// Compressed rows: row[i]..row[i+1] index col[] (and any value arrays kept
// alongside). Matches the reference's CRConnectivity layout.
struct CSR {
  int nRows = 0;
  std::vector<int> row;
  std::vector<int> col;
  int count(int i) const { return row[i + 1] - row[i]; }
  int nnz() const { return row.empty() ? 0 : row[nRows]; }
};

// Runs f(begin, end) over [0, n) split into contiguous chunks on the host's
// cores (at most 32 threads; one chunk when n < minItems).
// Number of chunks parallel_chunks(n, ..., minItems) splits [0, n) into.
inline int chunk_count(int n, int minItems = 20000) {
  int nt = (int)std::thread::hardware_concurrency();
  if (nt < 1) nt = 1;
  if (nt > 32) nt = 32;
  if (n < minItems || nt == 1) return 1;
  const int chunk = (n + nt - 1) / nt;
  return (n + chunk - 1) / chunk;
}

// As parallel_chunks, with f(t, begin, end) also given the chunk index t
// (0 .. chunk_count(n, minItems) - 1).
template <class F>
void parallel_chunks_indexed(int n, F f, int minItems = 20000) {
  const int nc = chunk_count(n, minItems);
  if (nc == 1) {
    f(0, 0, n);
    return;
  }
  int nt = (int)std::thread::hardware_concurrency();
  if (nt > 32) nt = 32;
  const int chunk = (n + nt - 1) / nt;
  std::vector<std::thread> th;
  for (int t = 0; t < nc; t++) {
    const int b = t * chunk, e = std::min(n, b + chunk);
    th.emplace_back([=] { f(t, b, e); });
  }
  for (auto& x : th) x.join();
}

template <class F>
void parallel_chunks(int n, F f, int minItems = 20000) {
  int nt = (int)std::thread::hardware_concurrency();
  if (nt < 1) nt = 1;
  if (nt > 32) nt = 32;
  if (n < minItems || nt == 1) {
    f(0, n);
    return;
  }
  std::vector<std::thread> th;
  const int chunk = (n + nt - 1) / nt;
  for (int t = 0; t < nt; t++) {
    const int b = t * chunk, e = std::min(n, b + chunk);
    if (b >= e) break;
    th.emplace_back([=] { f(b, e); });
  }
  for (auto& x : th) x.join();
}

}  // namespace fvm
