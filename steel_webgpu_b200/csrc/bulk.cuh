// Global -> shared staging with the Blackwell bulk-copy engine (cp.async.bulk, no multicast),
// completing on an mbarrier.
#pragma once
#include "common.cuh"

namespace steel {

constexpr uint32_t BULK_WAIT_LIMIT = 1u << 24;  // try_wait rounds before a copy counts as lost

SD uint32_t bulk_try_wait(uint32_t bar, uint32_t rounds) {
  uint32_t done = 0u;
  for (uint32_t it = 0; it < rounds && done == 0u; it++) {
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(done) : "r"(bar), "r"(0u) : "memory");
  }
  return done;
}

// Copies `bytes` from global `src` into shared `dst`. Every thread of the block calls it (it has
// block barriers). With both addresses 16-byte aligned and `bytes` a multiple of 16, thread 0
// issues one bulk copy and the block waits on `mbar` (a fresh barrier: one use per launch) for at
// most `wait_limit` try_wait rounds; otherwise the block copies with plain loads. Returns the same
// value in every thread: false when some thread's wait ran out. Before returning false the block
// waits again, at most BULK_WAIT_LIMIT rounds, for the copy still in flight, so that no copy into
// this block's shared memory outlives the block; the caller then reports the error and skips the
// scene (dst is undefined).
SD bool stage_to_shared(float* dst, const float* src, uint32_t bytes, uint64_t* mbar, uint32_t wait_limit) {
  const bool bulk = ((reinterpret_cast<uintptr_t>(src) | reinterpret_cast<uintptr_t>(dst) | bytes) & 15u) == 0u &&
                    bytes > 0u;
  if (!bulk) {
    for (uint32_t i = threadIdx.x; i < bytes / 4u; i += blockDim.x) dst[i] = src[i];
    __syncthreads();
    return true;
  }
  const uint32_t bar = (uint32_t)__cvta_generic_to_shared(mbar);
  const uint32_t d = (uint32_t)__cvta_generic_to_shared(dst);
  if (threadIdx.x == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
                 ::"r"(d), "l"(src), "r"(bytes), "r"(bar) : "memory");
  }
  const uint32_t done = bulk_try_wait(bar, wait_limit);
  if (__syncthreads_and(done != 0u)) return true;
  // Timed out: drain the copy (bounded) before the block moves on or exits.
  if (threadIdx.x == 0) (void)bulk_try_wait(bar, BULK_WAIT_LIMIT);
  __syncthreads();
  return false;
}

}  // namespace steel
