// tsu_bulk.cuh -- one-dimensional bulk copies from global to shared memory
// (cp.async.bulk, the TMA unit's untiled form, sm_90+) completing on a
// shared-memory mbarrier, with bounded waits.
//
// Used by the global-ring align kernels to stage a pair's packed sequences
// in shared memory.  The copies read this GPU's own memory only and carry no
// cluster multicast.  Source and destination must be 16-byte aligned and the
// size a multiple of 16 bytes (packed sequences are laid out for that:
// packed_words, tsu_common.cuh).  Every wait gives up after a fixed number
// of polls and reports it, so a copy that never completes cannot hang the
// kernel.
#pragma once

#include <cstdint>

namespace tsu {

#ifndef TSU_WARP_EMU
__device__ __forceinline__ uint32_t smem_addr(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// Initialise an mbarrier for one arriving thread, and make the initialisation
// visible to the async proxy (the bulk-copy unit).  Followed by a barrier of
// the threads that will wait on it.
__device__ __forceinline__ void mbar_init(uint64_t* mbar) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(mbar)) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// The arriving thread: expect `bytes` of transactions in the current phase.
__device__ __forceinline__ void mbar_expect(uint64_t* mbar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(mbar)), "r"(bytes)
               : "memory");
}

// Copy `bytes` from global src to shared dst, completing on mbar.
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* mbar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(smem_addr(dst)),
      "l"(src), "r"(bytes), "r"(smem_addr(mbar))
      : "memory");
}

// Wait until the phase of parity `parity` has completed; false if it has not
// after `polls` polls.
__device__ __forceinline__ bool mbar_wait(uint64_t* mbar, uint32_t parity, int polls) {
  const uint32_t a = smem_addr(mbar);
  for (int i = 0; i < polls; ++i) {
    uint32_t done;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.b32 %0, 1, 0, p;\n}"
        : "=r"(done)
        : "r"(a), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}
#endif

// Polls of a staging wait before the pair is reported as failed (each poll
// is a try_wait, which itself suspends for a short time).
constexpr int kBulkPolls = 1 << 22;

}  // namespace tsu
