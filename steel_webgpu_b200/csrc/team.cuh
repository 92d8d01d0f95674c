#pragma once
// The threads that solve one scene together.
//
// Team<false> is the calling block: the batched path, one block per scene, barriers are
// __syncthreads(). Team<true> is every block of a cooperative launch working on one large scene
// (a batch of one scene, such as an 8192-body pour or a thousand articulations): loops over a
// scene's bodies, rows, units and articulations are spread over all threads of the grid, and a
// barrier is a grid barrier. The reference runs such a scene on one workgroup (sim.js:663,
// wgsl.js:2504); the work between two barriers is the same, only more threads share it, so the
// results do not change.
//
// The grid barrier: each block's thread 0 publishes the block's writes (__threadfence), adds one
// to an arrival counter that is zero when the launch starts, and polls it until every block of
// this barrier generation has arrived, then fences again before the block proceeds. The poll is
// bounded: after `limit` polls the block records ERR_TEAM_TIMEOUT, stops waiting at this and every
// later barrier, and runs to its end, so the launch always ends (its results are then void and
// the host reports the error). The launch is cooperative, so every block is resident and the
// limit is never reached in a correct run.
#include "batch.cuh"

namespace steel {

template <bool TEAM> struct Team;

template <> struct Team<false> {
  __device__ uint32_t rank() const { return threadIdx.x; }
  __device__ uint32_t size() const { return blockDim.x; }
  __device__ bool lead() const { return threadIdx.x == 0u; }
  __device__ void sync() const { __syncthreads(); }
};

__device__ __forceinline__ uint32_t ld_acquire_gpu(const uint32_t* p) {
  uint32_t v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

template <> struct Team<true> {
  uint32_t* count;  // arrival counter in global memory, zero at launch
  uint32_t* error;  // the batch's device error word
  uint32_t limit;   // polls of the counter per barrier before giving up
  uint32_t* state;  // this block's shared words: [0] barriers passed, [1] nonzero after a timeout
  __device__ uint32_t rank() const { return blockIdx.x * blockDim.x + threadIdx.x; }
  __device__ uint32_t size() const { return gridDim.x * blockDim.x; }
  __device__ bool lead() const { return blockIdx.x == 0u && threadIdx.x == 0u; }
  __device__ void sync() const {
    __syncthreads();
    if (threadIdx.x == 0u) {
      const uint32_t want = (state[0] + 1u) * gridDim.x;
      state[0] += 1u;
      if (state[1] == 0u) {
        __threadfence();
        atomicAdd(count, 1u);
        uint32_t polls = 0u;
        while (ld_acquire_gpu(count) < want) {
          if (++polls >= limit) {
            state[1] = 1u;
            atomicCAS(error, 0u, (uint32_t)ERR_TEAM_TIMEOUT);
            break;
          }
          if (polls > 32u) __nanosleep(32);
        }
        __threadfence();
      }
    }
    __syncthreads();
  }
};

}  // namespace steel
