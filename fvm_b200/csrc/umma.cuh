// sm_100a tensor-core primitives as inline PTX: tcgen05 MMA of kind tf32
// (single CTA, both operands in shared memory, FP32 accumulator in tensor
// memory), TMEM allocation, tcgen05.ld read-back, and the shared-memory
// barrier the MMAs signal on completion. Only the forms the learned
// correction's dense layers use.
//
// Operand layout (K-major, no swizzle): a matrix of rows x K is stored as
// "core matrices" of 8 rows x 16 bytes (8 x 4 tf32 values, 128 contiguous
// bytes, row-major inside). LBO is the byte distance between core matrices
// adjacent in K, SBO the distance between adjacent 8-row groups.
#pragma once

#include <cstdint>

namespace fvm {
namespace umma {

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// Shared-memory matrix descriptor: start address [0,14), LBO [16,30), SBO
// [32,46) (all in 16-byte units), descriptor version 1 at [46,48), base
// offset 0, layout type 0 (no swizzle) at [61,64).
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
  return (uint64_t)((addr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// Instruction descriptor, kind::tf32 with FP32 accumulation, both operands
// K-major: D format F32 (1) at [4,6), A and B format TF32 (2) at [7,10) and
// [10,13), major bits 15 / 16 zero, N >> 3 at [17,23), M >> 4 at [24,29);
// dense, no negation, no shift.
__host__ __device__ constexpr uint32_t idesc_tf32(int m, int n) {
  return (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(m >> 4) << 24);
}

// D[tmem] = A * B^T (+ D if accumulate): M x N x 8, issued by one thread.
__device__ __forceinline__ void mma_tf32(uint32_t tmemD, uint64_t a, uint64_t b, uint32_t idesc, bool accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}\n"
      :
      : "r"(tmemD), "l"(a), "l"(b), "r"(idesc), "r"((uint32_t)accumulate)
      : "memory");
}

// One arrival on the barrier once every MMA this thread issued before has
// completed (its shared-memory reads and its TMEM writes).
__device__ __forceinline__ void commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_addr(bar))
               : "memory");
}

// ordering of tcgen05 operations around thread synchronisation
__device__ __forceinline__ void fence_before_sync() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after_sync() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
// this thread's ordinary shared-memory stores become visible to the tensor core
__device__ __forceinline__ void fence_smem_for_mma() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// TMEM columns for this CTA (executed by one whole warp; cols a power of
// two >= 32); the base address is written to *dst. The CTA allocates once,
// so the permit to allocate is given up right away.
__device__ __forceinline__ void tmem_alloc(uint32_t* dst, uint32_t cols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(dst)), "r"(cols)
               : "memory");
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_free(uint32_t taddr, uint32_t cols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(cols) : "memory");
}

// TMEM address of (lane, column): lane in bits [16,32), column in [0,16).
__device__ __forceinline__ uint32_t tmem_at(uint32_t base, int lane, int col) {
  return base + ((uint32_t)lane << 16) + (uint32_t)col;
}

// 32 TMEM lanes x 16 columns (whole warp): thread t gets lane (lane of
// taddr) + t, columns col .. col + 15. The wait is in the same asm
// statement, so the registers are valid when it returns.
__device__ __forceinline__ void ld16(uint32_t taddr, float (&v)[16]) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
      "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, [%16];\n\t"
      "tcgen05.wait::ld.sync.aligned;\n"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr)
      : "memory");
#pragma unroll
  for (int k = 0; k < 16; k++) v[k] = __uint_as_float(r[k]);
}

// shared-memory barrier with an expected arrival count
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// Waits for the barrier phase of the given parity to complete, trying at
// most `limit` times; false when the limit ran out.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, uint32_t limit) {
  const uint32_t a = smem_addr(bar);
  for (uint32_t it = 0; it < limit; ++it) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(done)
        : "r"(a), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}

}  // namespace umma
}  // namespace fvm
