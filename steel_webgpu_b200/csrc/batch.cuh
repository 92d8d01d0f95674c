// Batch-level device data and the kernel launchers shared by the .cu files.
#pragma once
#include "common.cuh"

namespace steel {

// All scenes of one batch, stepped together (one graph-capturable launch sequence per substep).
struct BatchDev {
  SceneDev* scenes;           // [nscenes]
  uint32_t nscenes;
  uint32_t nshapes;           // shapes over all scenes
  const uint32_t* shape_scene;  // global shape -> scene
  const uint32_t* shape_local;  // global shape -> shape index within its scene
  const uint4* tiles;         // broadphase tile jobs: (scene, tile i, tile j, 0)
  uint32_t ntiles;
  uint4* pairs;               // candidate pairs over all scenes: (scene, shape i, shape j, 0)
  uint32_t pair_cap;
  uint32_t* pair_count;       // [1]
  double* phase;              // per-scene clock (sim.js:674-678)
  unsigned long long* substep_count;  // [1]
  uint32_t* error;            // [1] first device-side error code (0 = none)
};

constexpr uint32_t BROAD_TILE = 32;
constexpr int NARROW_WARPS = 8;          // warps per narrowphase block
constexpr int SORT_THREADS = 512;
constexpr int PREP_THREADS = 512;
constexpr int SOLVE_THREADS = 256;

// Device error codes written to BatchDev::error.
enum : uint32_t { ERR_NONE = 0, ERR_SORT_CAPACITY = 1 };

void launch_params(const BatchDev& b, uint32_t substep, cudaStream_t st);
void launch_shapes(const BatchDev& b, cudaStream_t st);
void launch_broad(const BatchDev& b, cudaStream_t st);
void launch_narrow(const BatchDev& b, uint32_t narrow_blocks, cudaStream_t st);
void launch_csort(const BatchDev& b, size_t smem_keys, cudaStream_t st);
cudaError_t configure_sort(size_t smem_keys);
void launch_prepare(const BatchDev& b, cudaStream_t st);
void launch_solve(const BatchDev& b, cudaStream_t st);
void launch_frame_end(const BatchDev& b, cudaStream_t st);
// Host-I/O staging: scatter packed joint targets into each scene, gather packed body poses.
void launch_scatter_targets(const BatchDev& b, const float* packed, const uint64_t* offsets, cudaStream_t st);
void launch_gather_poses(const BatchDev& b, float* packed, const uint64_t* offsets, cudaStream_t st);

}  // namespace steel
