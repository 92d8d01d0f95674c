// Solve kernel: one block per scene (body: solve_scene, solve.cuh); blocks take scenes in B.order
// (longest first), so the scenes with the longest serial chains start in the first wave.
#include "solve.cuh"

namespace steel {

__global__ void __launch_bounds__(SOLVE_THREADS, 4) k_solve(BatchDev B) { solve_scene(B, B.order[blockIdx.x]); }
__global__ void __launch_bounds__(BIG_THREADS, 1) k_solve_big(BatchDev B) { solve_scene(B, B.order[blockIdx.x]); }

cudaError_t configure_solve(size_t smem_bytes) {
  cudaError_t e = cudaFuncSetAttribute(k_solve, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_bytes);
  if (e != cudaSuccess) return e;
  return cudaFuncSetAttribute(k_solve_big, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_bytes);
}
void launch_solve(const BatchDev& b, cudaStream_t st) {
  if (b.big) k_solve_big<<<b.nscenes, BIG_THREADS, b.solve_smem, st>>>(b);
  else k_solve<<<b.nscenes, SOLVE_THREADS, b.solve_smem, st>>>(b);
}

}  // namespace steel
