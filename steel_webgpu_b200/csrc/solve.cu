// Solve kernel: one block per scene (body: solve_scene, solve.cuh), and the fused prepare + solve
// kernel of the frame graph: one block runs a scene's prepare and then its solve, so no block waits
// for the whole batch's prepare; blocks take scenes in B.order (longest first).
#include "prepare.cuh"
#include "solve.cuh"

namespace steel {

static_assert(PREP_THREADS == SOLVE_THREADS, "the fused kernel runs both bodies with one block size");

__global__ void __launch_bounds__(SOLVE_THREADS, 4) k_solve(BatchDev B) { solve_scene(B, blockIdx.x); }

// F64: as k_prepare's, the instance launched when a scene of the batch has ART_F64.
template <bool F64>
__global__ void __launch_bounds__(SOLVE_THREADS, 4) k_prepare_solve(BatchDev B) {
  const uint32_t sc = B.order[blockIdx.x];
  prepare_scene<F64>(B, sc);
  __syncthreads();
  solve_scene(B, sc);
}

cudaError_t configure_prepare_solve(size_t smem_bytes) {
  cudaError_t e =
      cudaFuncSetAttribute(k_prepare_solve<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_bytes);
  if (e != cudaSuccess) return e;
  return cudaFuncSetAttribute(k_prepare_solve<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_bytes);
}
void launch_prepare_solve(const BatchDev& b, cudaStream_t st) {
  const uint32_t smem = b.prep_smem > b.solve_smem ? b.prep_smem : b.solve_smem;
  if (b.art_f64) k_prepare_solve<true><<<b.nscenes, SOLVE_THREADS, smem, st>>>(b);
  else k_prepare_solve<false><<<b.nscenes, SOLVE_THREADS, smem, st>>>(b);
}

cudaError_t configure_solve(size_t smem_bytes) {
  return cudaFuncSetAttribute(k_solve, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_bytes);
}
void launch_solve(const BatchDev& b, cudaStream_t st) { k_solve<<<b.nscenes, SOLVE_THREADS, b.solve_smem, st>>>(b); }

}  // namespace steel
