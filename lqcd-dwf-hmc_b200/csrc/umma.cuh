// Inline-PTX wrappers for the fifth-generation tensor cores of sm_100a
// (tcgen05): tensor-memory allocation, the single-thread MMA issue with
// operands in shared memory and the accumulator in tensor memory, completion
// through an mbarrier, and the warp-wide tensor-memory load of the epilogue.
//
// Operand layout used here: K-major, no swizzle.  A "core matrix" is 8 rows
// of 16 bytes (8 BF16 along K), its rows 16 bytes apart; core matrices
// adjacent along K sit LBO bytes apart, core matrices adjacent along M (or N)
// SBO bytes apart.  One kind::f16 MMA consumes K = 16 (two core matrices
// along K) of every row.
#pragma once

#include <cstdint>

namespace b200 {

// Shared-memory matrix descriptor (64 bit): start address >> 4 in bits
// [0,14), LBO >> 4 in [16,30), SBO >> 4 in [32,46), descriptor version 1 in
// [46,48), base offset 0, layout type 0 (no swizzle) in [61,64).
__device__ __forceinline__ uint64_t umma_smem_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// Instruction descriptor of kind::f16 with BF16 A and B, FP32 accumulation,
// both operands K-major: D format in bits [4,6) (1 = F32), A and B formats
// in [7,10) and [10,13) (1 = BF16), N >> 3 in [17,23), M >> 4 in [24,29).
constexpr uint32_t umma_idesc_bf16_f32(int m, int n) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(m >> 4) << 24);
}

// Allocate ncols tensor-memory columns (a power of two >= 32) for this CTA;
// the whole warp executes it, the base address lands in shared memory.
__device__ __forceinline__ void tmem_alloc(uint32_t dst_smem, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
               :: "r"(dst_smem), "r"(ncols) : "memory");
}
__device__ __forceinline__ void tmem_relinquish() {
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" :: "r"(taddr), "r"(ncols) : "memory");
}

// Order tensor-core operations against a following / preceding thread
// synchronisation (bar.sync, mbarrier wait).
__device__ __forceinline__ void tc_fence_before_sync() {
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_after_sync() {
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}

// D (tensor memory) = A B^T (+ D when accumulate), A and B described in
// shared memory; issued by one thread, completes asynchronously.
__device__ __forceinline__ void umma_bf16_ss(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc,
                                             uint32_t idesc, bool accumulate) {
  const uint32_t mask0 = 0, mask1 = 0, mask2 = 0, mask3 = 0;   // no output lane disabled
  asm volatile(
      "{\n\t"
      ".reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t"
      "}\n"
      :: "r"(d_tmem), "l"(adesc), "l"(bdesc), "r"(idesc), "r"((uint32_t)accumulate),
         "r"(mask0), "r"(mask1), "r"(mask2), "r"(mask3)
      : "memory");
}

// Arrive once on the mbarrier when every MMA this thread issued before has
// completed.
__device__ __forceinline__ void umma_commit(uint32_t bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
               :: "r"(bar) : "memory");
}

// Warp-wide: thread t of the warp reads 16 consecutive 32-bit columns of
// tensor-memory lane (lane field of taddr) + t, and waits for the load.
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16]) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
      "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, [%16];\n\t"
      "tcgen05.wait::ld.sync.aligned;"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
        "=r"(r[14]), "=r"(r[15])
      : "r"(taddr)
      : "memory");
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

}  // namespace b200
