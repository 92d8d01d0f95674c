// Solve kernel instances for one block size: STEEL_BLOCK threads per block, set by the build
// (solve.cu is compiled once per size into solve_<N>.o). One block per scene (body: solve_scene,
// solve.cuh); blocks take scenes in B.order (longest first), so the scenes with the longest serial
// chains start in the first wave.
#include "solve.cuh"

#ifndef STEEL_BLOCK
#error "compile with -DSTEEL_BLOCK=<threads per block>"
#endif
#define STEEL_CAT2(a, b) a##b
#define STEEL_CAT(a, b) STEEL_CAT2(a, b)
#define STEEL_NS STEEL_CAT(t, STEEL_BLOCK)

namespace steel {
namespace STEEL_NS {
// EXT: the batch has a scene with torsional/rolling friction of articulated contacts or the
// contact-then-internal row schedule; only that instance carries the 5-row angular block in its
// contact loop and the two-phase iteration.
template <bool EXT>
__global__ void __launch_bounds__(STEEL_BLOCK, blocks_per_sm_of(STEEL_BLOCK)) k_solve(BatchDev B) {
  const uint32_t sc = B.order[blockIdx.x];
  const unsigned long long t0 = B.trace_solve ? trace_clock() : 0ull;
  solve_scene<EXT, false>(B, sc, Team<false>{});
  if (B.trace_solve) trace_block(B.trace_solve + 3ull * sc, t0);
}
#if STEEL_BLOCK == 512  // team launches run the 512-thread instances (one block per SM)
// A batch of one large scene: every block of this cooperative launch solves it together (team.cuh).
template <bool EXT>
__global__ void __launch_bounds__(STEEL_BLOCK, blocks_per_sm_of(STEEL_BLOCK)) k_solve_team(BatchDev B) {
  __shared__ uint32_t team_state[2];
  if (threadIdx.x == 0u) { team_state[0] = 0u; team_state[1] = 0u; }  // published by copy_scene's barrier
  const uint32_t sc = B.order[0];
  const unsigned long long t0 = B.trace_solve ? trace_clock() : 0ull;
  solve_scene<EXT, true>(B, sc, Team<true>{B.team_bar, B.error, TEAM_WAIT_LIMIT, team_state});
  if (B.trace_solve && blockIdx.x == 0u) trace_block(B.trace_solve + 3ull * sc, t0);
}
#endif
}  // namespace STEEL_NS

template <>
cudaError_t configure_solve_t<STEEL_BLOCK>(size_t smem_bytes) {
  const void* fns[] = {(const void*)STEEL_NS::k_solve<false>, (const void*)STEEL_NS::k_solve<true>,
#if STEEL_BLOCK == 512
                       (const void*)STEEL_NS::k_solve_team<false>, (const void*)STEEL_NS::k_solve_team<true>
#endif
  };
  for (const void* f : fns) {
    cudaError_t e = cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_bytes);
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}
template <>
void launch_solve_t<STEEL_BLOCK>(const BatchDev& b, cudaStream_t st) {
#if STEEL_BLOCK == 512
  if (b.team_blocks) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(b.team_blocks);
    cfg.blockDim = dim3(STEEL_BLOCK);
    cfg.dynamicSmemBytes = b.solve_smem;
    cfg.stream = st;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeCooperative;  // every block resident: the grid barrier's guarantee
    at[0].val.cooperative = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    cudaMemsetAsync(b.team_bar, 0, sizeof(uint32_t), st);
    if (b.solve_ext) cudaLaunchKernelEx(&cfg, STEEL_NS::k_solve_team<true>, b);
    else cudaLaunchKernelEx(&cfg, STEEL_NS::k_solve_team<false>, b);
    return;
  }
#endif
  if (b.solve_ext) STEEL_NS::k_solve<true><<<b.nlaunch, STEEL_BLOCK, b.solve_smem, st>>>(b);
  else STEEL_NS::k_solve<false><<<b.nlaunch, STEEL_BLOCK, b.solve_smem, st>>>(b);
}
template <>
int solve_team_blocks_per_sm_t<STEEL_BLOCK>(size_t smem_bytes) {
#if STEEL_BLOCK == 512
  int n = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, STEEL_NS::k_solve_team<true>, STEEL_BLOCK, smem_bytes) !=
      cudaSuccess)
    return 0;
  return n;
#else
  (void)smem_bytes;
  return 0;
#endif
}

}  // namespace steel
