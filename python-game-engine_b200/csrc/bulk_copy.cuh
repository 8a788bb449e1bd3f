// Bulk asynchronous global -> shared copies (the TMA engine's untiled cp.async.bulk) with
// mbarrier completion, for kernels that stream rows of a few hundred bytes into shared memory
// without spending registers or issue slots on the loads.
//
// Rules these helpers rely on: both addresses and the size of every copy are multiples of
// 16 bytes (the callers check this on the host before choosing a kernel that uses them); an
// mbarrier is initialised by one thread with an arrival count of 1 and made visible to the
// async proxy before any copy names it; the thread that arrives with expect_tx is the thread
// that issues the copies of that phase. Waits are bounded: mbar_wait gives up after
// kMbarSpinLimit polls and returns false, so a copy that never lands turns into an error
// status instead of a hung block.
#pragma once
#include <cstdint>

namespace sg {

constexpr int kMbarSpinLimit = 1 << 22;  // polls of try_wait (each may suspend ~0.1-1 us)

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}

// make initialised barriers visible to the async proxy (the bulk copies complete on them)
__device__ __forceinline__ void mbar_fence_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
               : "memory");
}

// One bulk copy of `bytes` (multiple of 16) from global src to shared dst, completing on bar.
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(smem_addr(dst)),
      "l"(src), "r"(bytes), "r"(smem_addr(bar))
      : "memory");
}

// Wait until the barrier's phase with the given parity has completed; false after the limit.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity) {
  const uint32_t a = smem_addr(bar);
  for (int it = 0; it < kMbarSpinLimit; ++it) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(a), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}

}  // namespace sg
