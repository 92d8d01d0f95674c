// Solve kernel: one block per scene (body: solve_scene, solve.cuh); blocks take scenes in B.order
// (longest first), so the scenes with the longest serial chains start in the first wave.
#include "solve.cuh"

namespace steel {

// EXT: the batch has a scene with torsional/rolling friction of articulated contacts or the
// contact-then-internal row schedule; only that instance carries the 5-row angular block in its
// contact loop and the two-phase iteration.
template <bool EXT>
__global__ void __launch_bounds__(SOLVE_THREADS, 4) k_solve(BatchDev B) { solve_scene<EXT>(B, B.order[blockIdx.x]); }
template <bool EXT>
__global__ void __launch_bounds__(BIG_THREADS, 1) k_solve_big(BatchDev B) { solve_scene<EXT>(B, B.order[blockIdx.x]); }

cudaError_t configure_solve(size_t smem_bytes) {
  const void* fns[4] = {(const void*)k_solve<false>, (const void*)k_solve<true>, (const void*)k_solve_big<false>,
                        (const void*)k_solve_big<true>};
  for (const void* f : fns) {
    cudaError_t e = cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_bytes);
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}
void launch_solve(const BatchDev& b, cudaStream_t st) {
  if (b.big) {
    if (b.solve_ext) k_solve_big<true><<<b.nscenes, BIG_THREADS, b.solve_smem, st>>>(b);
    else k_solve_big<false><<<b.nscenes, BIG_THREADS, b.solve_smem, st>>>(b);
  } else {
    if (b.solve_ext) k_solve<true><<<b.nscenes, SOLVE_THREADS, b.solve_smem, st>>>(b);
    else k_solve<false><<<b.nscenes, SOLVE_THREADS, b.solve_smem, st>>>(b);
  }
}

}  // namespace steel
