// Persistent AMG cycle kernel (see cycle_program.cuh). Compiled with
// -fmad=false like the other solver kernels; vectors that change inside
// the kernel (x, b, tmp) are read with ld.global.cg so that no SM reads a
// stale L1 line written by another SM in an earlier phase.
#include <cuda_runtime.h>

#include "cycle_program.cuh"

namespace fvm {
namespace dev {

namespace {

constexpr unsigned kSpinLimit = 1u << 21;  // ~1 s of polling: far beyond any phase (<= 100 us)

__device__ __forceinline__ unsigned ld_acquire(const unsigned* p) {
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_release(unsigned* p, unsigned v) {
  asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// Grid barrier: arrive with one atomic per block, the last arrival bumps
// the generation. Waits are bounded (kSpinLimit polls); on expiry the
// error flag is raised and every block leaves the kernel.
__device__ __forceinline__ bool grid_barrier(BarrierState* bs) {
  __shared__ int s_ok;
  __syncthreads();
  if (threadIdx.x == 0) {
    const unsigned g = ld_acquire(&bs->generation);
    __threadfence();
    const unsigned arrived = atomicAdd(&bs->count, 1u) + 1u;
    int ok = 1;
    if (arrived == gridDim.x) {
      bs->count = 0u;
      __threadfence();
      st_release(&bs->generation, g + 1u);
    } else {
      unsigned spins = 0;
      while (ld_acquire(&bs->generation) == g) {
        if (++spins > kSpinLimit) {
          atomicExch(&bs->error, 1);
          ok = 0;
          break;
        }
        if ((spins & 1023u) == 0u && ld_acquire((const unsigned*)&bs->error) != 0u) {
          ok = 0;  // another block gave up: leave too
          break;
        }
        if (spins > 32) __nanosleep(40);
      }
    }
    __threadfence();
    if (ok && ld_acquire((const unsigned*)&bs->error) != 0u) ok = 0;
    s_ok = ok;
  }
  __syncthreads();
  return s_ok != 0;
}

template <class T>
__device__ __forceinline__ T ldv(const T* p) {
  return __ldcg(p);
}

// Row sum over a SELL slice in stored order; all loads of up to 16
// entries are in flight together (two dependent round trips per chunk).
template <class T>
__device__ __forceinline__ T row_sum(const ProgLevel<T>& L, int s, int lane, const T* x, T sum) {
  const int o = L.sliceOff[s];
  const int w = (L.sliceOff[s + 1] - o) >> 5;
  for (int k0 = 0; k0 < w; k0 += 16) {
    const int cnt = min(16, w - k0);
    int c[16];
    T v[16];
    T xv[16];
#pragma unroll
    for (int k = 0; k < 16; k++)
      if (k < cnt) {
        const int e = o + ((k0 + k) << 5) + lane;
        c[k] = L.cols[e];
        v[k] = L.vals[e];
      }
#pragma unroll
    for (int k = 0; k < 16; k++)
      if (k < cnt) xv[k] = ldv(x + c[k]);
#pragma unroll
    for (int k = 0; k < 16; k++)
      if (k < cnt) sum = sum + v[k] * xv[k];
  }
  return sum;
}

// Executes one phase with this thread's share (thread tid of nthreads).
template <class T>
__device__ __forceinline__ void exec_phase(const Phase ph, const ProgLevel<T>* __restrict__ levels,
                                           const double* __restrict__ coarseInv, const float* __restrict__ coarseInvF,
                                           int coarseN, int tid, int nthreads) {
  const int gwarp = tid >> 5;
  const int nwarps = nthreads >> 5;
  const int lane = threadIdx.x & 31;
  {
    const ProgLevel<T> L = levels[ph.level];
    switch (ph.op) {
      case kPhaseGS: {
        for (int s = ph.a + gwarp; s < ph.b; s += nwarps) {
          if (lane < L.sliceRows[s]) {
            const int i = L.sliceRow[s] + lane;
            const T sum = row_sum(L, s, lane, L.x, ldv(L.b + i));
            L.x[i] = -sum / L.diag[i];
          }
        }
        break;
      }
      case kPhaseJacobi: {
        const T* src = ph.a == 0 ? L.x : L.tmp;
        T* dst = ph.a == 0 ? L.tmp : L.x;
        for (int s = gwarp; s < L.nSlices; s += nwarps) {
          if (lane < L.sliceRows[s]) {
            const int i = L.sliceRow[s] + lane;
            const T sum = row_sum(L, s, lane, src, ldv(L.b + i));
            dst[i] = -sum / L.diag[i];
          }
        }
        break;
      }
      case kPhaseRestrict: {
        const ProgLevel<T> C = levels[ph.level + 1];
        for (int I = tid; I < C.n; I += nthreads) {
          T acc = T(0);
          for (int k = L.c2fRow[I]; k < L.c2fRow[I + 1]; k++) {
            const int i = L.c2fCol[k];
            const int sl = L.rowSlice[i];
            const int ln = i - L.sliceRow[sl];
            const T ri = row_sum(L, sl, ln, L.x, ldv(L.b + i) + L.diag[i] * ldv(L.x + i));
            acc = acc + ri;
          }
          C.b[I] = acc;
          C.x[I] = T(0);
        }
        break;
      }
      case kPhaseProlong: {
        const ProgLevel<T> C = levels[ph.level + 1];
        for (int i = tid; i < L.n; i += nthreads) {
          const int c = L.ci[i];
          if (c >= 0) L.x[i] = ldv(L.x + i) + ldv(C.x + c);
        }
        break;
      }
      case kPhaseDense: {
        for (int row = gwarp; row < coarseN; row += nwarps) {
          double s = 0.0;
          if (coarseInvF) {
            for (int j = lane; j < coarseN; j += 32)
              s += (double)(coarseInvF[(size_t)row * coarseN + j] * (float)ldv(L.b + j));
          } else {
            for (int j = lane; j < coarseN; j += 32) s += coarseInv[(size_t)row * coarseN + j] * (double)ldv(L.b + j);
          }
          for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
          if (lane == 0) L.x[row] = (T)(-s);
        }
        break;
      }
      default:
        break;
    }
  }
}

template <class T>
__global__ void __launch_bounds__(kProgramBlock) k_cycle_program(const Phase* __restrict__ phases, int nPhases,
                                                                  const ProgLevel<T>* __restrict__ levels,
                                                                  const double* __restrict__ coarseInv,
                                                                  int coarseN, BarrierState* bs) {
  const int tid = blockIdx.x * blockDim.x + threadIdx.x;
  const int nthreads = gridDim.x * blockDim.x;
  for (int p = 0; p < nPhases; p++) {
    exec_phase<T>(phases[p], levels, coarseInv, nullptr, coarseN, tid, nthreads);
    if (p + 1 < nPhases) {
      if (!grid_barrier(bs)) return;
    }
  }
}

// The same phase list run by ONE thread-block cluster: the CTAs of the
// cluster meet at the hardware cluster barrier (release/acquire at cluster
// scope) between phases. Meant for the small coarse levels, whose phases
// are too short to amortise a kernel launch each.
template <class T>
__global__ void __launch_bounds__(kClusterBlock, 1)
    k_cluster_program(const Phase* __restrict__ phases, int nPhases, const ProgLevel<T>* __restrict__ levels,
                      const double* __restrict__ coarseInv, const float* __restrict__ coarseInvF, int coarseN) {
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
  asm volatile("griddepcontrol.wait;" ::: "memory");
  const int tid = blockIdx.x * blockDim.x + threadIdx.x;
  const int nthreads = gridDim.x * blockDim.x;
  for (int p = 0; p < nPhases; p++) {
    exec_phase<T>(phases[p], levels, coarseInv, coarseInvF, coarseN, tid, nthreads);
    if (p + 1 < nPhases) {
      asm volatile("barrier.cluster.arrive.release.aligned;" ::: "memory");
      asm volatile("barrier.cluster.wait.acquire.aligned;" ::: "memory");
    }
  }
}

}  // namespace

template <class T>
int cycle_program_max_grid() {
  int dev = 0, sms = 0, perSM = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSM, k_cycle_program<T>, kProgramBlock, 0);
  if (perSM > 2) perSM = 2;  // fewer arrivals per barrier; 1024 threads per SM
  return perSM * sms;
}

template <class T>
cudaError_t run_cycle_program(const Phase* phases, int nPhases, const ProgLevel<T>* levels,
                              const double* coarseInv, int coarseN, BarrierState* barrier, int grid,
                              cudaStream_t st) {
  if (grid <= 0) grid = cycle_program_max_grid<T>();
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(grid);
  cfg.blockDim = dim3(kProgramBlock);
  cfg.dynamicSmemBytes = 0;
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeCooperative;
  attr[0].val.cooperative = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, k_cycle_program<T>, phases, nPhases, levels, coarseInv, coarseN, barrier);
}

template <class T>
int cluster_program_size() {
  // the largest cluster (16 non-portable, else 8) of 1024-thread CTAs the
  // device can place
  for (int cs : {16, 8}) {
    if (cs > 8 &&
        cudaFuncSetAttribute(k_cluster_program<T>, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) !=
            cudaSuccess) {
      cudaGetLastError();
      continue;
    }
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(cs);
    cfg.blockDim = dim3(kClusterBlock);
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = cs;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    int clusters = 0;
    if (cudaOccupancyMaxActiveClusters(&clusters, k_cluster_program<T>, &cfg) == cudaSuccess && clusters > 0)
      return cs;
    cudaGetLastError();
  }
  return 0;
}

template <class T>
cudaError_t run_cluster_program(const Phase* phases, int nPhases, const ProgLevel<T>* levels,
                                const double* coarseInv, const float* coarseInvF, int coarseN, int clusterSize,
                                cudaStream_t st) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(clusterSize);
  cfg.blockDim = dim3(kClusterBlock);
  cfg.dynamicSmemBytes = 0;
  cfg.stream = st;
  cudaLaunchAttribute attr[2];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = clusterSize;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  attr[1].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[1].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 2;
  return cudaLaunchKernelEx(&cfg, k_cluster_program<T>, phases, nPhases, levels, coarseInv, coarseInvF, coarseN);
}

template int cluster_program_size<double>();
template int cluster_program_size<float>();
template cudaError_t run_cluster_program<double>(const Phase*, int, const ProgLevel<double>*, const double*,
                                                 const float*, int, int, cudaStream_t);
template cudaError_t run_cluster_program<float>(const Phase*, int, const ProgLevel<float>*, const double*,
                                                const float*, int, int, cudaStream_t);
template int cycle_program_max_grid<double>();
template int cycle_program_max_grid<float>();
template cudaError_t run_cycle_program<double>(const Phase*, int, const ProgLevel<double>*, const double*, int,
                                               BarrierState*, int, cudaStream_t);
template cudaError_t run_cycle_program<float>(const Phase*, int, const ProgLevel<float>*, const double*, int,
                                              BarrierState*, int, cudaStream_t);

}  // namespace dev
}  // namespace fvm
