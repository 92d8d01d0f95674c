// Solve kernel: one block per scene (body: solve_scene, solve.cuh); blocks take scenes in B.order
// (longest first), so the scenes with the longest serial chains start in the first wave.
#include "solve.cuh"

namespace steel {

__global__ void __launch_bounds__(SOLVE_THREADS, 4) k_solve(BatchDev B) { solve_scene(B, B.order[blockIdx.x]); }

cudaError_t configure_solve(size_t smem_bytes) {
  return cudaFuncSetAttribute(k_solve, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_bytes);
}
void launch_solve(const BatchDev& b, cudaStream_t st) { k_solve<<<b.nscenes, SOLVE_THREADS, b.solve_smem, st>>>(b); }

}  // namespace steel
