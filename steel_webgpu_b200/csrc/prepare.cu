// Prepare kernel: one block per scene; the body is prepare_scene (prepare.cuh).
#include "prepare.cuh"

namespace steel {

__global__ void __launch_bounds__(PREP_THREADS, 4) k_prepare(BatchDev B) { prepare_scene(B, blockIdx.x); }

cudaError_t configure_prepare(size_t smem_bytes) {
  return cudaFuncSetAttribute(k_prepare, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_bytes);
}
void launch_prepare(const BatchDev& b, cudaStream_t st) { k_prepare<<<b.nscenes, PREP_THREADS, b.prep_smem, st>>>(b); }

}  // namespace steel
