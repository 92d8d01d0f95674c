// Global -> shared staging with the Blackwell bulk-copy engine (cp.async.bulk, no multicast),
// completing on an mbarrier.
#pragma once
#include "common.cuh"

namespace steel {

constexpr uint32_t BULK_WAIT_LIMIT = 1u << 24;  // try_wait rounds before a copy counts as lost

// Copies `bytes` from global `src` into shared `dst`. Every thread of the block calls it (it has
// block barriers). With both addresses 16-byte aligned and `bytes` a multiple of 16, thread 0
// issues one bulk copy and the block waits on `mbar` (a fresh barrier: one use per launch);
// otherwise the block copies with plain loads. Returns false when the bulk copy did not complete
// within BULK_WAIT_LIMIT waits (the caller reports the error; dst is then undefined).
SD bool stage_to_shared(float* dst, const float* src, uint32_t bytes, uint64_t* mbar) {
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
  uint32_t done = 0u;
  for (uint32_t it = 0; it < BULK_WAIT_LIMIT && done == 0u; it++) {
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(done) : "r"(bar), "r"(0u) : "memory");
  }
  __syncthreads();
  return done != 0u;
}

}  // namespace steel
