// Block-wide integer scans on warp shuffles (one block per scene).
#pragma once
#include "common.cuh"

namespace steel {

// Exclusive prefix sum of v over the block's threads, in thread order; *total gets the sum.
// tmp: shared memory of at least 33 words. All threads must call it.
SD uint32_t block_excl_scan(uint32_t v, uint32_t* tmp, uint32_t* total) {
  const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5u, nw = (blockDim.x + 31u) >> 5u;
  uint32_t x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= (uint32_t)o) x += y;
  }
  if (lane == 31u) tmp[warp] = x;
  __syncthreads();
  if (warp == 0u) {
    uint32_t w = lane < nw ? tmp[lane] : 0u;
    uint32_t s = w;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      uint32_t y = __shfl_up_sync(0xffffffffu, s, o);
      if (lane >= (uint32_t)o) s += y;
    }
    if (lane < nw) tmp[lane] = s - w;
    if (lane == nw - 1u) tmp[32] = s;
  }
  __syncthreads();
  uint32_t r = tmp[warp] + x - v;
  *total = tmp[32];
  __syncthreads();
  return r;
}

// Exclusive prefix sum of a[0..n) in place (any n), by contiguous per-thread chunks.
SD uint32_t block_scan_array(uint32_t* a, uint32_t n, uint32_t* tmp) {
  uint32_t ch = (n + blockDim.x - 1u) / blockDim.x;
  uint32_t lo = min(threadIdx.x * ch, n), hi = min(lo + ch, n);
  uint32_t s = 0u;
  for (uint32_t i = lo; i < hi; i++) s += a[i];
  uint32_t total;
  uint32_t off = block_excl_scan(s, tmp, &total);
  for (uint32_t i = lo; i < hi; i++) { uint32_t x = a[i]; a[i] = off; off += x; }
  __syncthreads();
  return total;
}

}  // namespace steel
