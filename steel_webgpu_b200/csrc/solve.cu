// Solve kernel: one block per scene (body: solve_scene, solve.cuh), and the fused prepare + solve
// kernel of the frame graph: one block runs a scene's prepare and then its solve, so no block waits
// for the whole batch's prepare; blocks take scenes in B.order (longest first).
#include "prepare.cuh"
#include "solve.cuh"

namespace steel {

static_assert(PREP_THREADS == SOLVE_THREADS, "the fused kernel runs both bodies with one block size");

__global__ void __launch_bounds__(SOLVE_THREADS, 4) k_solve(BatchDev B) { solve_scene(B, blockIdx.x); }

__global__ void __launch_bounds__(SOLVE_THREADS, 4) k_prepare_solve(BatchDev B) {
  const uint32_t sc = B.order[blockIdx.x];
  prepare_scene(B, sc);
  __syncthreads();
  solve_scene(B, sc);
}

cudaError_t configure_prepare_solve(size_t smem_bytes) {
  return cudaFuncSetAttribute(k_prepare_solve, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_bytes);
}
void launch_prepare_solve(const BatchDev& b, cudaStream_t st) {
  k_prepare_solve<<<b.nscenes, SOLVE_THREADS, b.prep_smem > b.solve_smem ? b.prep_smem : b.solve_smem, st>>>(b);
}

cudaError_t configure_solve(size_t smem_bytes) {
  return cudaFuncSetAttribute(k_solve, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_bytes);
}
void launch_solve(const BatchDev& b, cudaStream_t st) { k_solve<<<b.nscenes, SOLVE_THREADS, b.solve_smem, st>>>(b); }

}  // namespace steel
