// fvm_csr_residual_device_noalloc: the CSR residual + L1 norm of
// fvm_csr_residual, for callers that cannot allocate device memory.
//
// Who needs it: code that runs where cudaMalloc is unavailable or not
// allowed -- inside a stream capture that must not allocate, inside a host
// callback or a real-time loop with a fixed memory budget, or in a host
// application whose own allocator owns every device byte. Such callers
// already hold their inputs and outputs in device memory; the only extra
// memory the computation needs is the per-block partial sums of the L1
// reduction, and that lives here, in a fixed file-scope device array.
//
// The array (kMaxPartials doubles, 512 KB) is part of the library image:
// every GPU that loads the library holds it until the process exits. Every
// call shares it, so calls that overlap on the GPU (different streams, or
// different host threads, on the same device) race on it; serialise them.
// Each call writes every partial it later reads, so no clearing is needed
// between calls. The array's device address is looked up once per CUDA
// context (cudaDeviceReset ends a context; the next call in the new one
// looks the address up again).
#include <cuda.h>
#include <cuda_runtime.h>

#include <map>
#include <mutex>

#include "../../include/fvm_b200.h"
#include "common.hpp"
#include "kernels.cuh"

namespace {

// one partial per 256-row block: up to 65536 blocks = 16,777,216 rows
constexpr int kMaxPartials = 65536;

__device__ __align__(256) double g_residual_scratch[kMaxPartials + 1];

typedef CUresult (*CtxGetCurrentFn)(CUcontext*);
typedef CUresult (*CtxGetIdFn)(CUcontext, unsigned long long*);

std::mutex g_setup_mutex;
// device address of the scratch array per CUDA context, keyed by the
// context's process-unique id: a context created after cudaDeviceReset, or
// a non-primary context made current by the host application, gets its own
// lookup (the array has a different address in every context)
std::map<unsigned long long, double*> g_scratch_addr;

// Unique id of the calling thread's current CUDA context (driver entry
// points obtained through the runtime, so no link-time dependency on
// libcuda). Makes the runtime initialise the device's primary context
// first when no context is current yet.
unsigned long long current_context_id() {
  static CtxGetCurrentFn getCurrent = nullptr;
  static CtxGetIdFn getId = nullptr;
  if (!getCurrent || !getId) {
    void* p0 = nullptr;
    void* p1 = nullptr;
    cudaDriverEntryPointQueryResult q0 = cudaDriverEntryPointSymbolNotFound, q1 = cudaDriverEntryPointSymbolNotFound;
    if (cudaGetDriverEntryPointByVersion("cuCtxGetCurrent", &p0, 12000, cudaEnableDefault, &q0) != cudaSuccess ||
        q0 != cudaDriverEntryPointSuccess ||
        cudaGetDriverEntryPointByVersion("cuCtxGetId", &p1, 12000, cudaEnableDefault, &q1) != cudaSuccess ||
        q1 != cudaDriverEntryPointSuccess || !p0 || !p1)
      throw fvm::Error(fvm::kDeviceError, "CUDA driver entry points cuCtxGetCurrent / cuCtxGetId unavailable");
    getCurrent = (CtxGetCurrentFn)p0;
    getId = (CtxGetIdFn)p1;
  }
  CUcontext ctx = nullptr;
  if (getCurrent(&ctx) != CUDA_SUCCESS || !ctx) {
    // no context current on this thread: cudaSetDevice binds (and
    // initialises) the current device's primary context; then ask again
    int dev = -1;
    if (cudaGetDevice(&dev) != cudaSuccess || cudaSetDevice(dev) != cudaSuccess || getCurrent(&ctx) != CUDA_SUCCESS ||
        !ctx)
      throw fvm::Error(fvm::kDeviceError, "no usable current CUDA context");
  }
  unsigned long long id = 0;
  if (getId(ctx, &id) != CUDA_SUCCESS) throw fvm::Error(fvm::kDeviceError, "cuCtxGetId failed");
  return id;
}

// Device address of the scratch array in the current context. In host code
// the symbol is only a host-side stand-in, so the address is looked up once
// per context with that context current (the first call in each context
// does this; make that first call outside any stream capture).
double* scratch_for_current_context() {
  const unsigned long long ctx = current_context_id();
  std::lock_guard<std::mutex> lock(g_setup_mutex);
  auto it = g_scratch_addr.find(ctx);
  if (it != g_scratch_addr.end()) return it->second;
  void* p = nullptr;
  const cudaError_t e = cudaGetSymbolAddress(&p, g_residual_scratch);
  if (e != cudaSuccess || !p)
    throw fvm::Error(fvm::kDeviceError,
                     std::string("cudaGetSymbolAddress of the residual scratch failed: ") + cudaGetErrorString(e));
  g_scratch_addr[ctx] = static_cast<double*>(p);
  return static_cast<double*>(p);
}

}  // namespace

extern "C" int fvm_csr_residual_device_noalloc(int n, const int* row, const int* col,
                                               const double* diag, const double* off,
                                               const double* x, const double* b, double* r,
                                               double* l1norm, void* stream) {
  try {
    FVM_REQUIRE(n > 0, fvm::kBadArgument, "n must be positive");
    FVM_REQUIRE(row && col && diag && off && x && b && l1norm, fvm::kBadArgument,
                "null device pointer");
    const int np = fvm::dev::csr_residual_blocks(n);
    FVM_REQUIRE(np <= kMaxPartials, fvm::kTooLarge,
                "fvm_csr_residual_device_noalloc handles at most 16777216 rows (its fixed "
                "scratch holds 65536 block sums); use fvm_csr_residual for larger systems");
    double* scratch = scratch_for_current_context();
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    fvm::dev::csr_residual(n, row, col, diag, off, x, b, r, scratch, st);
    fvm::dev::csr_residual_finish(np, scratch, l1norm, st);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess)
      throw fvm::Error(fvm::kDeviceError, std::string("kernel launch failed: ") + cudaGetErrorString(e));
    return FVM_OK;
  } catch (const fvm::Error& e) {
    fvm::set_last_error(e.what());
    return e.status;
  } catch (const std::exception& e) {
    fvm::set_last_error(e.what());
    return FVM_ERR_BAD_ARGUMENT;
  }
}
