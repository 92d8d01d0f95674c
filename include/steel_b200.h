/* C ABI of the B200 implementation of steel-webgpu's Sim.step hot path.
 *
 * The reference's host (packages/steel-webgpu/src/sim.js, class Sim) packs a scene into its
 * static buffers statF/statU and a constant table C (sim.js:95-477), uploads them with
 * queue.writeBuffer, and per frame dispatches seven WGSL kernels per substep
 * (sim.js:648-701). This library takes exactly that packed form (plus the initial state of
 * sim.js:486-502) and runs the substeps on one GPU as CUDA kernels. Scenes are grouped into a
 * batch that steps together; a single Sim is a batch of one.
 *
 * Every call returns 0 on success or a STEEL_E_* code; steel_last_error() then describes the
 * failure (thread-local). A batch is used by one host thread at a time.
 */
#ifndef STEEL_B200_H
#define STEEL_B200_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define STEEL_OK 0
#define STEEL_E_INVALID 1     /* bad argument or malformed scene; Sim's throw new Error(...) */
#define STEEL_E_UNSUPPORTED 2 /* reserved for a solver option outside the supported set; every option of the
                                 reference constant table (sim.js:412-477) is supported, so none returns it */
#define STEEL_E_CAPACITY 3    /* a device capacity was exceeded and work was dropped */
#define STEEL_E_CUDA 4        /* CUDA runtime error */
#define STEEL_E_NOMEM 5       /* device allocation failed */
#define STEEL_E_NODEVICE 6    /* no CUDA device; the reference's UnsupportedError (device.js:2-9) */
#define STEEL_E_TIMEOUT 7     /* a bounded device-side wait ran out (a shared-memory bulk copy, the radix
                                 sort's look-back, a team launch's grid barrier); the work that waited was
                                 skipped or is void, so reset before trusting the state */

typedef struct steel_ctx steel_ctx;
typedef struct steel_batch steel_batch;

/* One packed scene, in the reference's layout. */
typedef struct {
  const char* constants;     /* "KEY=VALUE\n" lines: the C table of sim.js:456-477 plus the
                                writeParams inputs as PARAM_fps, PARAM_substeps, PARAM_iterations,
                                PARAM_baumgarte, PARAM_gravity0..2, PARAM_warm, PARAM_reg,
                                PARAM_target_frames, PARAM_driven, PARAM_integral_count */
  const float* statF;        /* statF (sim.js:225), statF_floats = 4 * vec4 count */
  uint64_t statF_floats;
  const uint32_t* statU;     /* statU (sim.js:237) */
  uint64_t statU_words;
  const float* body_pose;    /* NB * 8: COM position, 0, quaternion (sim.js:258-281) */
  const float* body_vel;     /* NB * 8: linear, 0, angular, 0 (sim.js:490-491) */
  const float* art;          /* the art buffer's initial contents, A_* layout of C (sim.js:486-501) */
  uint64_t art_floats;
} steel_scene_desc;

/* SimStats (src/sim.d.ts:30-43, sim.js:822-834). overflow: bit 0 pairs, 1 contacts, 2 units,
   3 dense rows (the buffers that filled up and dropped work). */
typedef struct {
  uint32_t max_contacts, max_colors, max_units, max_pairs, contacts, colors, max_dense, asleep, overflow;
} steel_stats;

/* Sizes of scene s of a batch. */
typedef struct {
  uint32_t NB, NS, NA, NL, ND, NQ;
  uint32_t max_pairs, max_contacts, max_units, max_dense;
} steel_scene_info;

/* Context: one CUDA device and stream. Replaces initDevice (src/device.js:7-26). */
int steel_ctx_create(int device, steel_ctx** out);
int steel_ctx_destroy(steel_ctx* ctx);
const char* steel_last_error(void);

/* new Sim(device, scene) for n scenes at once (sim.js:63-75, 95-611). */
int steel_batch_create(steel_ctx* ctx, const steel_scene_desc* scenes, uint32_t n, steel_batch** out);
int steel_batch_destroy(steel_batch* b);                          /* Sim.destroy (sim.js:85-93) */

/* new Sim(device, scene, opts) from the scene's own files: scene.json text and scene.bin bytes as
   loadScene reads them (sim.js:40-61), packed by the library (the C++ restatement of Sim.build,
   sim.js:95-521) and created as a batch of one. opts_json: the SimOptions object (sim.d.ts:3-28:
   substeps, iterations, regularization, warmStart, colorWords, solver) or NULL, plus an optional
   "capacities" object (MAXP, MAXC, MAXU, UH, WH, MAXDENSE, AH) replacing the reference's fixed
   ones. Unsupported scenes and options fail with STEEL_E_INVALID and the reference's message
   (sim.js:73, :128, :159, :166, :376-379, :412-420). */
int steel_scene_create(steel_ctx* ctx, const char* json, uint64_t json_len, const void* bin, uint64_t bin_len,
                       const char* opts_json, steel_batch** out);
/* The same for n scenes stepped together (arrays of n; opts_json may be NULL, or hold NULLs). */
int steel_batch_create_files(steel_ctx* ctx, uint32_t n, const char* const* json, const uint64_t* json_len,
                             const void* const* bin, const uint64_t* bin_len, const char* const* opts_json,
                             steel_batch** out);
/* Convex hull of a point cloud, the hull SceneBuilder.addConvexHull stores for a hull shape
   (builder.js:61-173), in C++ (host only, no device needed): quickhull in double with the
   reference's steps and order, coplanar triangles merged into polygons. pts: n points (x, y, z).
   Caller buffers sized for n points: verts [3n] the hull's vertices in increasing order of their
   index among the distinct input points; planes [8n] per face the outward unit normal and d
   (n . x = d); face_start [2n + 1] offsets into face_verts; face_verts [6n] each face's vertices
   counter-clockwise about its normal. *nv, *nf: vertex and face counts. STEEL_E_INVALID for fewer
   than 4 distinct points, or collinear or coplanar points. */
int steel_convex_hull(const double* pts, uint32_t n, double* verts, double* planes, uint32_t* face_start,
                      uint32_t* face_verts, uint32_t* nv, uint32_t* nf);

/* Packing alone, without a device (tools and tests): the steel_scene_desc a scene's files pack to.
   The desc's pointers stay valid until steel_packed_free. */
typedef struct steel_packed steel_packed;
int steel_pack(const char* json, uint64_t json_len, const void* bin, uint64_t bin_len, const char* opts_json,
               steel_packed** out);
int steel_packed_desc(const steel_packed* p, steel_scene_desc* out);
int steel_packed_free(steel_packed* p);
int steel_scene_info_get(steel_batch* b, uint32_t scene, steel_scene_info* out);

int steel_reset(steel_batch* b);                                  /* Sim.reset (sim.js:613-623) */
int steel_step(steel_batch* b, uint32_t frames);                  /* Sim.step (sim.js:692-701), async */
int steel_sync(steel_batch* b);                                   /* queue.onSubmittedWorkDone */
/* Capture one frame's substeps into a CUDA graph and replay it (on by default). */
int steel_set_graph(steel_batch* b, int enabled);

/* Tile configuration of a batch's launches. No counterpart in the reference, whose workgroup sizes
   are fixed in the WGSL (one 256-invocation workgroup per prepare/solve, wgsl.js:1222, :2501).
   Prepare and solve run one block per scene; block_threads picks the kernel instance (32, 64, 128,
   256 or 512 threads, all at 128 registers per thread, so 65536 / (128 * block_threads) blocks fit
   an SM); smem_budget caps the dynamic shared memory a block uses to stage a scene's link blocks,
   twists, qd and color masks (0: per-part caps only); narrow_blocks_per_sm sizes the persistent
   narrowphase grid (0: as many as fit); stream_groups splits the scenes into that many contiguous
   groups of about equal size whose launch sequences run on parallel streams (branches of the frame
   graph), so one group's kernels use the SMs another group's kernel tails leave idle (0 or 1: one
   sequence; the serving loop always uses one). A batch starts at 512 threads when it has no more
   scenes than SMs (the per-thread scratch is sized for that), else at 128, which is also the
   largest block it accepts. Results are the same bits under every configuration. */
typedef struct {
  uint32_t block_threads;
  uint32_t smem_budget;
  uint32_t narrow_blocks_per_sm;
  uint32_t stream_groups;
} steel_tiles;
int steel_get_tiles(steel_batch* b, steel_tiles* out);
int steel_set_tiles(steel_batch* b, const steel_tiles* tiles);
/* Autotuner: steps the batch from its initial state under each candidate configuration (block
   sizes with staging budgets that keep 1-16 blocks resident per SM, then one narrowphase grid
   smaller than the default, then two stream groups for batches of more than twice the SM count;
   for a batch of one scene, then team sizes of the solve, see steel_set_team), times `frames`
   frames of each after two warm-up frames (CUDA events), keeps the fastest and resets the batch
   (as steel_reset). Returns the chosen tiles and their device time per frame in milliseconds
   (steel_get_team gives the chosen team). */
int steel_autotune(steel_batch* b, uint32_t frames, steel_tiles* best, float* best_ms_per_frame);

/* Team launches for a batch of one large scene. No counterpart in the reference, which prepares and
   solves a scene on one 256-invocation workgroup (wgsl.js:1222, :2501-2504, sim.js:663). The prepare
   and solve kernels are launched cooperatively with `blocks` blocks of the batch's block size that
   share the scene's bodies, contacts, rows and articulations and meet at grid barriers (bounded
   waits: STEEL_E_TIMEOUT, never a hang); the prepare's scan-based passes (contact classification,
   unit scan, sleep islands, coloring) stay on the team's first block.
   0: one block (the batched path). STEEL_TEAM_AUTO, the default: a scene of at least 2048 bodies or
   64 articulations gets one thread per body or a warp per articulation, capped by the blocks that
   fit the GPU. Other values: that many blocks (STEEL_E_INVALID if more than fit). Team launches
   run the 512-thread kernel instances (one block per SM): under tiles of another block size, and
   for batches of several scenes or scenes with Nesterov momentum, the batch runs one block per
   scene. Results are the same bits either way. steel_get_team returns the blocks in use (0: one block). */
#define STEEL_TEAM_AUTO 0xffffffffu
int steel_set_team(steel_batch* b, uint32_t blocks);
int steel_get_team(steel_batch* b, uint32_t* blocks);

/* Readback (Sim.state, sim.js:732-763; Sim.poses, sim.js:804). Caller-owned buffers. */
int steel_read_poses(steel_batch* b, uint32_t scene, float* poses /* NB*8 */);
int steel_read_state(steel_batch* b, uint32_t scene, float* poses /* NB*8 */, float* vel /* NB*8 */,
                     float* q /* NQ */, float* qd /* ND */, float* link_v /* NL*6, (w, v) at the COM */);
int steel_get_stats(steel_batch* b, uint32_t scene, steel_stats* out);  /* Sim.stats (sim.js:822-834) */
/* Sim.state() (sim.js:732-763) in Newton's layout, for scenes created from their files:
   bodyQ (body origin position, quaternion x y z w; 7 floats per body), bodyQd (COM linear and
   angular velocity, world frame; 6 per body), jointQ and jointQd in Newton's joint layout (sizes from
   steel_newton_info). Caller-owned buffers. */
typedef struct {
  uint32_t bodies, joint_coords, joint_dofs;
} steel_newton_info_t;
int steel_newton_info(steel_batch* b, uint32_t scene, steel_newton_info_t* out);
int steel_state(steel_batch* b, uint32_t scene, float* bodyQ, float* bodyQd, float* jointQ, float* jointQd);
/* The port dof of a Newton joint dof (Sim.dofMap, sim.js:716-719): the index the joint setters
   below take. STEEL_E_INVALID with the reference's message for a dof outside the articulations. */
int steel_newton_dof(steel_batch* b, uint32_t scene, uint32_t newton_dof, uint32_t* port_dof);
/* Zero-copy pose export, the role of Sim.buffers.poses with PoseBridge.copy (sim.d.ts:75,
   three/poseBridge.ts:12-45): copies scene s's body poses GPU to GPU into a caller-owned device
   buffer of NB BodyPose records (COM position vec4, then quaternion x, y, z, w vec4; 32 bytes each,
   16-byte aligned), e.g. a renderer's instance buffer mapped into CUDA. Enqueued on `stream` (a
   cudaStream_t of the batch's device; NULL: the batch's own stream) after the frames already
   queued; nothing passes through host memory and the call does not wait. */
int steel_copy_poses_device(steel_batch* b, uint32_t scene, float* dst, void* stream);

/* User control (sim.js:716-785), port dof/body indices; held until changed. */
int steel_set_joint_target(steel_batch* b, uint32_t scene, uint32_t dof, float pos, float vel);
int steel_set_joint_force(steel_batch* b, uint32_t scene, uint32_t dof, float value);
int steel_set_body_wrench(steel_batch* b, uint32_t scene, uint32_t body, const float force[3], const float torque[3]);
int steel_set_body_pose(steel_batch* b, uint32_t scene, uint32_t body, const float com[3], const float quat[4]);
int steel_set_body_twist(steel_batch* b, uint32_t scene, uint32_t body, const float twist[6]);

/* Inspection for parity checks: steel_collide runs shapes, broad, narrow and the contact sort on
   the current state (substep-0 parameters) without advancing it; the readers then copy a scene's
   candidate pairs (2 u32 each, unordered) and its sorted contact records (5 vec4 each, then the
   shape-mu vec4s) from that run. */
int steel_collide(steel_batch* b);
int steel_read_pairs(steel_batch* b, uint32_t scene, uint32_t* pairs, uint32_t cap, uint32_t* count);
int steel_read_contacts(steel_batch* b, uint32_t scene, float* records, uint32_t cap, uint32_t* count);
/* Stage-level inspection (parity checks), one substep at a time as steel_step runs them: stage 0
   writes the next substep's parameters and runs the collision kernels, 1 the prepare kernel, 2 the
   solve kernel (ending the frame after the last substep). steel_read_words copies
   `count` 4-byte words from one of a scene's device buffers ("art", "rows", "sched", "slots", "warm",
   "contacts") at a word offset; steel_layout_get returns a named offset of that layout (an A_* or
   S_* offset, or ROWS). */
int steel_debug_stage(steel_batch* b, int stage);
int steel_read_words(steel_batch* b, uint32_t scene, const char* buffer, uint64_t offset, uint64_t count, void* out);
int steel_layout_get(steel_batch* b, uint32_t scene, const char* key, uint64_t* value);
/* One control step of a whole batch through host memory (a policy loop's call): joint targets for
   every articulation dof of every scene (scene after scene, ND floats each; NULL keeps the current
   targets) are copied in, `frames` frames run, and every scene's body poses (NB * 8 floats each,
   scene after scene) are copied out. Targets given here replace a scene's recorded trajectory,
   as setJointTargets does (sim.js:716-728). Blocks until the poses are on the host. */
int steel_step_io(steel_batch* b, uint32_t frames, const float* targets, uint64_t n_targets, float* poses,
                  uint64_t n_poses);
/* Runs `frames` frames with CUDA events around every kernel launch and returns the mean device
   time per launch of each kernel, in milliseconds: [params, shapes, broad, narrow, csort,
   prepare, solve] (7 floats). */
int steel_profile_kernels(steel_batch* b, uint32_t frames, float* ms_per_launch);
/* Device time of the last steel_step_timed call's frames, in milliseconds (CUDA events). */
int steel_step_timed(steel_batch* b, uint32_t frames, float* ms);
/* Block trace of the per-scene kernels, the batched counterpart of Sim.step(frames, timestamps)'s
   pass timestamps (sim.js:606-610, 681-698): with tracing on, every prepare and solve block
   records its start and end (the GPU's global timer, ns) and its SM. Off by default; turning it
   on or off allocates or frees the record buffer and recaptures the frame graph, so call it
   outside stream capture. Results do not change. */
int steel_trace(steel_batch* b, int on);
/* The records of the last prepare and solve launches: 6 words per scene, out[3 s + k] for the
   prepare block of scene s and out[3 (n_scenes + s) + k] for its solve block, k = 0 start,
   1 end, 2 SM index; zeros for scenes that have not run since tracing was turned on. */
int steel_trace_read(steel_batch* b, uint64_t* out, uint64_t words);
/* Failure-path testing: the number of try_wait rounds the prepare and solve kernels give a
   shared-memory bulk copy before they record STEEL_E_TIMEOUT. steel_batch_create sets
   STEEL_WAIT_LIMIT_DEFAULT; 0 makes every staged scene's wait run out at once. After a timeout the
   kernel still waits, with the default limit, for its copy in flight, skips the scene and
   returns, so the context stays usable. No counterpart in the reference (WebGPU has no bounded
   waits). */
#define STEEL_WAIT_LIMIT_DEFAULT 16777216u
int steel_debug_set_wait_limit(steel_batch* b, uint32_t rounds);

/* Serving loop: continuous batching over the batch's scenes as resident instances. No direct
   counterpart in the reference; the closest is Sim.run (sim.js:705-712), which keeps up to four
   frames of one scene in flight. Requests of `frames` frames queue per instance; up to max_active
   instances are admitted at a time, first come first served (0 or a value above the scene count:
   all) and within the byte budget of steel_serve_budget. Each tick steps every admitted instance by
   one frame and waits for it (the per-scene kernels launch one block per admitted instance; the
   other instances' shape and pair work is skipped); an instance whose request is done takes its
   next queued request or makes room for the next waiting instance.
   Latency is measured from submit to the end of the request's last tick. While the loop runs,
   steel_step and steel_collide step only the admitted instances; steel_serve_end makes every
   scene step again. Scenes are independent, so an instance's result is the same alone and in any
   mix. */
int steel_serve_config(steel_batch* b, uint32_t max_active);
/* Admission by memory: the admitted instances' state (their share of the batch's device arena:
   static scene data, bodies, contacts, rows, articulation blocks, scratch) may total at most
   `bytes` (0: no limit; the head of the queue is admitted whenever nothing is). This bounds the
   working set each tick's kernels read and write, so instances of different sizes share the
   device by size rather than by count. The per-scene kernels launch one block per admitted
   instance (the others launch nothing), and ticks launch their kernels directly, without the
   frame graph, since the launch sizes change from tick to tick. */
int steel_serve_budget(steel_batch* b, uint64_t bytes);
/* Bytes of one scene's state in the batch arena (the unit of steel_serve_budget). */
int steel_scene_bytes(steel_batch* b, uint32_t scene, uint64_t* bytes);
int steel_serve_submit(steel_batch* b, uint32_t instance, uint32_t frames, uint64_t* id);
int steel_serve_tick(steel_batch* b, uint32_t* stepped /* instances stepped in this tick */);
int steel_serve_poll(steel_batch* b, uint64_t* ids, uint32_t* instances, double* latency_ms, uint32_t cap,
                     uint32_t* count /* finished requests returned (and removed) */);
int steel_serve_end(steel_batch* b);

/* Canonical contact sort that allocates no device memory. No counterpart in the reference (its
   sort runs only inside Sim.step); it exists for callers that cannot call cudaMalloc: a robot
   controller on a fixed-rate loop, where cudaMalloc/cudaFree may block and synchronise the whole
   device, or a host engine that hands all device memory out of its own pool sized at start-up.
   Sorts n raw contact records into the order steel_collide/steel_read_contacts produce. Both
   buffers are caller-owned device memory of the calling thread's current device (or mapped host
   memory), 16-byte aligned, not overlapping, 24 * n floats each, laid out as steel_read_contacts
   returns them: n records of 5 vec4, then n shape-mu vec4. `stream` is a cudaStream_t of that
   device (NULL: the default stream); the call only enqueues the work.
   The key scratch is a static device array of STEEL_NOALLOC_MAX_CONTACTS keys (1 MiB) that every
   GPU which loads this library holds until exit; n above that maximum fails with
   STEEL_E_CAPACITY before anything is launched. The first call in each CUDA context (a device's
   primary context, and again after cudaDeviceReset) looks up the array's device address (set-up)
   and caches it with the context's id; make that first call before any stream capture. Up to 2048
   padded keys sort in the kernel's static shared memory instead of the array. All calls on a device
   share the array: calls whose kernels overlap on the GPU race and corrupt each other's results,
   so order them (for example on one stream). */
#define STEEL_NOALLOC_MAX_CONTACTS 65536
int steel_sort_contacts_noalloc(const float* raw, uint32_t n, float* sorted, void* stream);

#ifdef __cplusplus
}
#endif
#endif
