// Prepare kernel: one block per scene; the body is prepare_scene (prepare.cuh).
#include "prepare.cuh"

namespace steel {

// F64: the instance with the FP64 articulated-inertia branch, launched when a scene of the batch
// has ART_F64 (scenes without it still run the FP32 branch in that instance).
template <bool F64>
__global__ void __launch_bounds__(PREP_THREADS, 4) k_prepare(BatchDev B) { prepare_scene<F64>(B, B.order[blockIdx.x]); }
template <bool F64>
__global__ void __launch_bounds__(BIG_THREADS, 1) k_prepare_big(BatchDev B) { prepare_scene<F64>(B, B.order[blockIdx.x]); }

cudaError_t configure_prepare(size_t smem_bytes) {
  const int n = (int)smem_bytes;
  const void* fns[] = {(const void*)k_prepare<false>, (const void*)k_prepare<true>, (const void*)k_prepare_big<false>,
                       (const void*)k_prepare_big<true>};
  for (const void* f : fns) {
    cudaError_t e = cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, n);
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}
void launch_prepare(const BatchDev& b, cudaStream_t st) {
  if (b.big) {
    if (b.art_f64) k_prepare_big<true><<<b.nscenes, BIG_THREADS, b.prep_smem, st>>>(b);
    else k_prepare_big<false><<<b.nscenes, BIG_THREADS, b.prep_smem, st>>>(b);
  } else {
    if (b.art_f64) k_prepare<true><<<b.nscenes, PREP_THREADS, b.prep_smem, st>>>(b);
    else k_prepare<false><<<b.nscenes, PREP_THREADS, b.prep_smem, st>>>(b);
  }
}

}  // namespace steel
