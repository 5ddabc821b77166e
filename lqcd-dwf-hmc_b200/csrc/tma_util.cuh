// Thin inline-PTX wrappers for the sm_90+/sm_100a bulk asynchronous copy
// engine (TMA, non-tensor "bulk" form) and shared-memory mbarriers.
//
// Only global -> own-CTA shared memory copies of this GPU's memory are used;
// no multicast form is issued anywhere in this library.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace b200 {

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}

// Make barrier initialisation visible to the asynchronous proxy.
__device__ __forceinline__ void mbar_fence_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint32_t bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint32_t bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}

// One try.  hint_ns = 0: blocks for at most a hardware-defined time slice;
// otherwise the thread may be suspended until the phase completes or at most
// hint_ns nanoseconds have passed (the PTX suspend-time hint), instead of
// re-issuing the test.
__device__ __forceinline__ bool mbar_try_wait(uint32_t bar, uint32_t parity, uint32_t hint_ns = 0) {
  uint32_t ok;
  if (hint_ns == 0) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(bar), "r"(parity)
        : "memory");
  } else {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(bar), "r"(parity), "r"(hint_ns)
        : "memory");
  }
  return ok != 0;
}

__device__ __forceinline__ uint64_t global_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// Bounded wait for the phase with the given parity: gives up after 2 s of
// global time or 2^22 tries, whichever comes first, and reports false
// instead of waiting forever.  The clock is read only after a failed try.
__device__ __forceinline__ bool mbar_wait_bounded(uint32_t bar, uint32_t parity, uint32_t hint_ns = 0) {
  if (mbar_try_wait(bar, parity, hint_ns)) return true;
  constexpr int kMaxTries = 1 << 22;
  constexpr uint64_t kMaxNs = 2000000000ull;
  const uint64_t t0 = global_ns();
  for (int i = 0; i < kMaxTries; ++i) {
    if (mbar_try_wait(bar, parity, hint_ns)) return true;
    if (global_ns() - t0 > kMaxNs) return false;
  }
  return false;
}

// The wait of the error path: copies that were issued must land before the
// CTA exits, so this bound is far longer (2^26 tries or 20 s of global time).
__device__ __forceinline__ bool mbar_wait_drain(uint32_t bar, uint32_t parity) {
  if (mbar_try_wait(bar, parity)) return true;
  constexpr int kMaxTries = 1 << 26;
  constexpr uint64_t kMaxNs = 20000000000ull;
  const uint64_t t0 = global_ns();
  for (int i = 0; i < kMaxTries; ++i) {
    if (mbar_try_wait(bar, parity)) return true;
    if (global_ns() - t0 > kMaxNs) return false;
  }
  return false;
}

// Order earlier generic-proxy accesses of shared memory before later
// asynchronous-proxy (bulk copy) writes to the same addresses.
__device__ __forceinline__ void fence_proxy_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// Bulk copy of `bytes` (multiple of 16, both addresses 16-byte aligned) from
// global memory to this CTA's shared memory, completing on `bar`.
__device__ __forceinline__ void bulk_g2s(uint32_t dst, const void* src, uint32_t bytes, uint32_t bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
      "l"(src), "r"(bytes), "r"(bar)
      : "memory");
}

}  // namespace b200
