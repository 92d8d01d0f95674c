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
  uint32_t* pair_count;       // [2]: candidate pairs, narrowphase jobs
  uint4* jobs;                // narrowphase jobs [pair_cap][NJOB_WORDS / 4]
  double* phase;              // per-scene clock (sim.js:674-678)
  unsigned long long* substep_count;  // [nscenes] substeps each scene has run (warm-table parity)
  const uint32_t* active;     // [nscenes] nonzero: the scene steps in this frame (serving loop mask)
  const uint32_t* order;      // [nscenes] scenes in the per-scene kernels' block order (longest first)
  uint32_t nlaunch;           // blocks of the per-scene kernels (csort, prepare, solve): order[0..nlaunch) step
                              // (all scenes, or the serving loop's admitted instances)
  uint32_t* error;            // [1] first device-side error code (0 = none)
  uint32_t prep_smem;         // dynamic shared memory of k_prepare / k_solve launches (bytes)
  uint32_t solve_smem;
  uint32_t art_f64;           // some scene has ART_F64: launch the prepare instances that carry it
  uint32_t solve_ext;         // some scene has ANG_ART or CTI: launch the solve instances that carry them
  uint32_t block_threads;     // threads per prepare / solve block (one of BLOCK_SIZES)
  uint32_t wait_limit;        // try_wait rounds of a shared-memory bulk copy (BULK_WAIT_LIMIT unless a test
                              // lowers it to make the bounded wait run out)
  unsigned long long* trace_prep;   // null, or [nscenes][3]: each scene's last k_prepare block, its start and
  unsigned long long* trace_solve;  // end (%globaltimer, ns) and SM; the same for k_solve (steel_trace)
  uint32_t team_blocks;       // nonzero: the batch's one scene is prepared and solved by this many
                              // cooperating blocks (team.cuh)
  uint32_t* team_bar;         // [8]: [0] grid-barrier arrival counter of a team launch (zeroed before each
                              // launch), [4..7] counts the prepare's block 0 hands to the other blocks
};

// Block trace: the global timer (ns) and the block's record after the scene's body, written by
// thread 0 once every thread is done. Called by all threads, only when tracing is on.
__device__ __forceinline__ unsigned long long trace_clock() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}
__device__ __forceinline__ void trace_block(unsigned long long* rec, unsigned long long t0) {
  __syncthreads();
  if (threadIdx.x == 0u) {
    uint32_t sm;
    asm volatile("mov.u32 %0, %%smid;" : "=r"(sm));
    rec[0] = t0;
    rec[1] = trace_clock();
    rec[2] = sm;
  }
}

constexpr uint32_t BROAD_TILE = 32;
constexpr int NARROW_WARPS = 8;          // warps per narrowphase block
constexpr int NARROW_JOB_THREADS = 128;  // threads per block of the narrowphase job kernel
constexpr uint32_t NJOB_WORDS = 44;     // words per narrowphase job record
constexpr int SORT_THREADS = 512;
// Prepare and solve run one block per scene. Every block size below has its own kernel instances
// (prepare_<N>.o, solve_<N>.o), all at 128 registers per thread, so a size of N threads keeps
// 65536 / (128 N) blocks per SM when shared memory allows: small blocks keep more scenes resident
// and hide the latency of each scene's serial passes, large blocks give a few large scenes more
// threads for their parallel phases. Results do not depend on the block size.
constexpr uint32_t BLOCK_SIZES[] = {32u, 64u, 128u, 256u, 512u};
constexpr uint32_t DEFAULT_THREADS = 128;  // batches with more scenes than SMs
constexpr int BIG_THREADS = 512;           // batches of no more scenes than SMs: one block per SM
constexpr uint32_t blocks_per_sm_of(uint32_t threads) { return 65536u / (threads * 128u); }

// Device error codes written to BatchDev::error.
enum : uint32_t { ERR_NONE = 0, ERR_SORT_CAPACITY = 1, ERR_JOB_CAPACITY = 2, ERR_STAGE_TIMEOUT = 3, ERR_SORT_TIMEOUT = 4,
                  ERR_TEAM_TIMEOUT = 5 };

// Contact sort of scenes whose padded keys may exceed the block sort's shared array
// (next_pow2(MAXC) > SORT_SMEM_KEYS): a device-wide LSD radix sort, onesweep style (one histogram
// pass over all digits, then one launch per 8-bit digit that ranks a tile, looks back over the
// preceding tiles' bucket counts and scatters). Keys are (pair, feature, point-bit hash) with the
// raw index carried along; stable passes from the least significant digit give the lexicographic
// order of (pair, feature, hash, raw index).
constexpr uint32_t SORT_SMEM_KEYS = 8192;   // largest padded key count k_csort sorts in shared memory
constexpr uint32_t RS_THREADS = 256;
constexpr uint32_t RS_ITEMS = 16;           // keys per thread and tile
constexpr uint32_t RS_TILE = RS_THREADS * RS_ITEMS;
constexpr uint32_t RS_DIGITS = 12;          // 96 key bits, 8 per digit
constexpr uint32_t RS_SPIN_LIMIT = 1u << 22;  // polls of a preceding tile's status before giving up
constexpr uint32_t TEAM_WAIT_LIMIT = 1u << 22;  // polls of a team launch's grid barrier before giving up
// Team launches (team.cuh) on a batch of one scene: the default takes scenes of at least
// TEAM_MIN_BODIES bodies or TEAM_MIN_ARTS articulations; such a scene's per-thread scratch has
// slices for TEAM_SCRATCH_BLOCKS blocks, so the prepare's scratch passes spread over that many.
constexpr uint32_t TEAM_MIN_BODIES = 2048u, TEAM_MIN_ARTS = 64u, TEAM_SCRATCH_BLOCKS = 32u;
struct RadixDev {
  uint4* keys[2];     // ping-pong key buffers [MAXC] (x pair, y feature, z hash, w raw index)
  uint32_t* status;   // [RS_DIGITS][tiles][256] look-back words: bits 30-31 flag (1 tile count, 2 prefix)
  uint32_t* hist;     // [RS_DIGITS][256] bucket counts of all keys
  uint32_t* ctr;      // [RS_DIGITS] tile tickets
  uint32_t tiles;     // tiles of MAXC keys
  uint32_t scene;
};

// Shared-memory staging of a scene inside k_prepare / k_solve. A scene is staged when its part
// fits the cap; the launch's dynamic shared memory is the largest staged scene's need.
enum : uint32_t { STAGE_LINKS = 1u, STAGE_BODIES = 2u, STAGE_QD = 4u, STAGE_WMASK = 8u };
// Caps keep four prepare / solve blocks resident per SM.
constexpr uint32_t STAGE_LINK_CAP = 44u * 1024u;   // link blocks (NL * 1072 B)
constexpr uint32_t STAGE_BODY_CAP = 8u * 1024u;    // twists + impulses (NB * 64 B)
constexpr uint32_t STAGE_QD_CAP = 8u * 1024u;      // generalized velocities of the solve (ND * 4 B)
constexpr uint32_t STAGE_WMASK_CAP = 16u * 1024u;  // per-body color masks (NB * NCOLW words)
// Byte offsets of a scene's parts in k_prepare's dynamic shared memory: link blocks (if staged),
// color counts, color masks (if staged).
struct PrepSmem { uint32_t links, wcount, wmask, total; };
__host__ __device__ inline PrepSmem prep_smem_layout(uint32_t stage, uint32_t NL, uint32_t NB, uint32_t NCOLW,
                                                     uint32_t NCOL) {
  PrepSmem m{};
  uint32_t o = 0;
  m.links = o;
  if (stage & STAGE_LINKS) o += 4u * NL * 268u;
  m.wcount = o;
  o += 4u * (NCOL + 2u);
  m.wmask = o;
  if (stage & STAGE_WMASK) o += 4u * NB * NCOLW;
  m.total = (o + 15u) & ~15u;
  return m;
}
// Byte offsets of a scene's parts in k_solve's dynamic shared memory: [tw | imp] (if bodies
// are staged), qd (if staged), color starts, link blocks (if staged).
struct SolveSmem { uint32_t tw, imp, aqd, wcs, links, total; };
__host__ __device__ inline SolveSmem solve_smem_layout(uint32_t stage, uint32_t NB, uint32_t ND, uint32_t NCOL,
                                                       uint32_t NL) {
  SolveSmem m{};
  uint32_t o = 0;
  if (stage & STAGE_BODIES) { m.tw = 0; m.imp = 32u * NB; o = 64u * NB; }
  m.aqd = o;
  if (stage & STAGE_QD) o += 4u * ND;
  m.wcs = o;
  o += 4u * (NCOL + 2u);
  o = (o + 15u) & ~15u;
  m.links = o;
  if (stage & STAGE_LINKS) o += 4u * NL * 268u;
  m.total = o;
  return m;
}

// Copies a scene's descriptor into shared memory (all threads of the block call it; ends with a
// barrier), so the per-scene kernels read offsets and sizes at shared-memory latency.
__device__ inline void copy_scene(SceneDev& dst, const SceneDev& src) {
  static_assert(sizeof(SceneDev) % 4 == 0, "SceneDev is copied as words");
  const uint32_t* s = reinterpret_cast<const uint32_t*>(&src);
  uint32_t* d = reinterpret_cast<uint32_t*>(&dst);
  for (uint32_t i = threadIdx.x; i < sizeof(SceneDev) / 4u; i += blockDim.x) d[i] = s[i];
  __syncthreads();
}

void launch_params(const BatchDev& b, uint32_t substep, cudaStream_t st);
void launch_shapes(const BatchDev& b, cudaStream_t st);
void launch_broad(const BatchDev& b, cudaStream_t st);
void launch_narrow(const BatchDev& b, uint32_t narrow_blocks, cudaStream_t st);
int narrow_blocks_per_sm();
void launch_csort(const BatchDev& b, size_t smem_keys, const RadixDev* radix, uint32_t nradix, cudaStream_t st);
cudaError_t configure_sort(size_t smem_keys);
// One instance set per block size (template argument = threads per block).
template <int T> cudaError_t configure_prepare_t(size_t smem_bytes);
template <int T> cudaError_t configure_solve_t(size_t smem_bytes);
template <int T> void launch_prepare_t(const BatchDev& b, cudaStream_t st);
template <int T> void launch_solve_t(const BatchDev& b, cudaStream_t st);
template <int T> int solve_team_blocks_per_sm_t(size_t smem_bytes);
template <int T> int prepare_team_blocks_per_sm_t(size_t smem_bytes);
#define STEEL_DECLARE_BLOCK(N)                                                  \
  template <> cudaError_t configure_prepare_t<N>(size_t smem_bytes);            \
  template <> cudaError_t configure_solve_t<N>(size_t smem_bytes);              \
  template <> void launch_prepare_t<N>(const BatchDev& b, cudaStream_t st);     \
  template <> void launch_solve_t<N>(const BatchDev& b, cudaStream_t st);       \
  template <> int solve_team_blocks_per_sm_t<N>(size_t smem_bytes);      \
  template <> int prepare_team_blocks_per_sm_t<N>(size_t smem_bytes);
STEEL_DECLARE_BLOCK(32)
STEEL_DECLARE_BLOCK(64)
STEEL_DECLARE_BLOCK(128)
STEEL_DECLARE_BLOCK(256)
STEEL_DECLARE_BLOCK(512)
#undef STEEL_DECLARE_BLOCK
cudaError_t configure_prepare(uint32_t threads, size_t smem_bytes);
cudaError_t configure_solve(uint32_t threads, size_t smem_bytes);
void launch_prepare(const BatchDev& b, cudaStream_t st);
void launch_solve(const BatchDev& b, cudaStream_t st);
// Resident blocks per SM of the team solve kernel at this block size and dynamic shared memory.
int solve_team_blocks_per_sm(uint32_t threads, size_t smem_bytes);
int prepare_team_blocks_per_sm(uint32_t threads, size_t smem_bytes);
void launch_set_stage(const BatchDev& b, const uint32_t* stage, cudaStream_t st);
void launch_frame_end(const BatchDev& b, cudaStream_t st);
// Host-I/O staging: scatter packed joint targets into each scene, gather packed body poses.
void launch_scatter_targets(const BatchDev& b, const float* packed, const uint64_t* offsets, cudaStream_t st);
void launch_gather_poses(const BatchDev& b, float* packed, const uint64_t* offsets, cudaStream_t st);
void launch_copy_poses(const float4* pos, const float4* rot, uint32_t nb, float4* dst, cudaStream_t st);

}  // namespace steel
