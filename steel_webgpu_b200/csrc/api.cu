// Host side of the C ABI (include/steel_b200.h): batch construction from the reference's packed
// scenes, one device arena per batch, the per-substep launch sequence (captured as a CUDA graph),
// readback and user control.
#include <algorithm>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <sstream>
#include <string>
#include <vector>

#include "../../include/steel_b200.h"
#include "batch.cuh"
#include "bulk.cuh"
#include "scene.h"
#include "hull.h"

using namespace steel;

namespace {

thread_local std::string g_err;

int fail(int code, const std::string& msg) {
  g_err = msg;
  return code;
}
#define CU(x)                                                                                      \
  do {                                                                                             \
    cudaError_t e_ = (x);                                                                          \
    if (e_ != cudaSuccess) return fail(STEEL_E_CUDA, std::string(#x ": ") + cudaGetErrorString(e_)); \
  } while (0)

uint64_t next_pow2(uint64_t x) {
  uint64_t p = 1;
  while (p < x) p <<= 1;
  return p;
}

}  // namespace

namespace steel {
// Records the calling thread's error for steel_last_error(); for the entry points that live in
// other translation units.
int set_last_error(int code, const std::string& msg) { return fail(code, msg); }
}  // namespace steel

namespace {

struct Consts {
  std::map<std::string, double> kv;
  bool parse(const char* text) {
    if (!text) return false;
    std::istringstream in(text);
    std::string line;
    while (std::getline(in, line)) {
      if (line.empty()) continue;
      size_t eq = line.find('=');
      if (eq == std::string::npos) return false;
      kv[line.substr(0, eq)] = std::strtod(line.c_str() + eq + 1, nullptr);
    }
    return true;
  }
  bool has(const char* k) const { return kv.count(k) != 0; }
  double get(const char* k, double def = 0.0) const {
    auto it = kv.find(k);
    return it == kv.end() ? def : it->second;
  }
  uint32_t u(const char* k, uint32_t def = 0) const { return (uint32_t)get(k, def); }
  float f(const char* k, float def = 0.0f) const { return (float)get(k, def); }
};

// Sequential sub-allocation of one device arena (256-byte aligned pieces).
struct Layout {
  size_t bytes = 0;
  size_t take(size_t n) {
    size_t off = (bytes + 255) & ~(size_t)255;
    bytes = off + n;
    return off;
  }
};

struct SceneHost {
  Consts C;
  SceneDev d{};  // device pointers filled after allocation
  // arena offsets
  size_t o_sf, o_su, o_pos, o_rot, o_ppos, o_prot, o_lv, o_av, o_spos, o_srot, o_alo, o_ahi, o_art, o_cnt, o_stats,
      o_params, o_craw, o_con, o_ckeys, o_rows, o_slots, o_warm, o_sched, o_tw, o_imp, o_aqd, o_tscr;
  // Device-wide radix sort of a scene whose padded keys may exceed the block sort's shared array.
  bool large_sort = false;
  uint32_t sort_tiles = 0;
  size_t o_rkeys1 = 0, o_rstat = 0, o_rhist = 0, o_rctr = 0;
  size_t art_floats = 0, sched_words = 0, warm_words = 0, tscr_floats = 0;
  std::vector<float> statF;
  std::vector<uint32_t> statU;
  std::vector<float4> pos0, rot0, lv0, av0;
  std::vector<float> art0;
  uint32_t collide_pairs = 0, collide_contacts = 0;  // counts of the last steel_collide
  size_t arena_bytes = 0;                             // this scene's share of the batch arena
  // Newton index maps and scene data of a scene created from its files (steel_scene_create):
  // what Sim.state() and the Newton-indexed setters need (sim.js:716-785).
  std::shared_ptr<const scene::Packed> files;
};

}  // namespace

struct steel_packed {
  steel::scene::Packed p;
};

struct steel_ctx {
  int device = 0;
  cudaStream_t stream = nullptr;
  int sms = 148;
};

struct steel_batch {
  steel_ctx* ctx = nullptr;
  std::vector<SceneHost> sc;
  uint8_t* arena = nullptr;
  size_t arena_bytes = 0;
  BatchDev bd{};
  uint32_t substeps = 4;
  uint32_t narrow_blocks = 0;
  uint32_t debug_substep = 0;  // substep cursor of steel_debug_stage
  size_t sort_keys = 0;
  std::vector<RadixDev> radix;  // large scenes' device-wide contact sorts
  uint32_t max_threads = DEFAULT_THREADS;  // largest prepare / solve block the per-thread scratch allows
  steel_tiles tile_cfg{};                   // the launches' tile configuration (apply_tiles)
  size_t o_stage = 0;                       // staging flags of every scene (apply_tiles upload)
  bool use_graph = true;
  cudaGraphExec_t graph = nullptr;
  unsigned long long* trace = nullptr;  // steel_trace records (6 words per scene), or null
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  cudaEvent_t ev_pose = nullptr;  // orders a pose export on the caller's stream after the batch's frames
  // Scene groups: contiguous ranges of scenes whose launch sequences run on parallel streams (graph
  // branches), so one group's kernels fill the SMs the other group's kernel tails leave idle.
  struct Group {
    uint32_t lo = 0, hi = 0;                  // scene range
    size_t shape_lo = 0, tile_lo = 0, pair_lo = 0;
    BatchDev bd{};                            // the batch's view restricted to the range
    std::vector<RadixDev> radix;
    cudaStream_t st = nullptr;
    cudaEvent_t done = nullptr;
    uint8_t* mem = nullptr;                   // group-local tables (shape scenes, tiles, order, pair counters)
  };
  std::vector<Group> groups;                  // empty: one launch sequence for the whole batch
  cudaEvent_t ev_fork = nullptr;
  std::vector<uint32_t> pair_cap_of;          // MAXP of each scene (pair and job list partitions)
  size_t o_scenes, o_shape_scene, o_shape_local, o_tiles, o_pairs, o_pair_count, o_jobs, o_phase, o_ssc, o_active, o_order, o_err;
  std::vector<uint32_t> shape_scene, shape_local;
  std::vector<uint4> tiles;
  // host-I/O staging (steel_step_io): packed targets/poses on the device and their offsets
  size_t o_tgt_off, o_pose_off, o_tgt_buf, o_pose_buf;
  uint64_t n_targets = 0, n_poses = 0;
  // Serving loop (steel_serve_*): per-instance request queues, the admitted set and finished work.
  struct Req { uint64_t id; uint32_t frames_left, frames; double t_submit; };
  struct Done { uint64_t id; uint32_t instance, frames; double latency_ms; };
  std::vector<std::deque<Req>> serve_queue;
  std::deque<uint32_t> serve_waiting;          // instances with queued work, not admitted, FIFO
  std::vector<uint8_t> serve_state;            // 0 idle, 1 waiting, 2 admitted
  std::vector<uint32_t> serve_mask;            // host copy of the device activity mask
  std::vector<Done> serve_done;
  uint32_t serve_admitted = 0, serve_max_active = 0;
  uint64_t serve_budget = 0, serve_bytes = 0;  // admission budget (bytes of admitted instances' state), in use
  bool serve_dirty = false;                    // admitted set changed: upload the launch order
  std::vector<uint32_t> order_host;  // block order of the prepare and solve kernels
  uint32_t team_req = STEEL_TEAM_AUTO;  // steel_set_team request (0 off, STEEL_TEAM_AUTO, or blocks)
  size_t o_team = 0;                    // the team launches' words (BatchDev::team_bar)
  uint64_t serve_next_id = 1;
  bool serve_on = false;
};

namespace {

// threads: the largest prepare / solve block; one_scene: the batch has this scene alone (a team
// launch may run it, whose scratch passes use TEAM_SCRATCH_BLOCKS blocks' threads).
int build_scene(SceneHost& s, const steel_scene_desc& in, Layout& L, uint32_t threads, bool one_scene,
                std::string& why) {
  Consts& C = s.C;
  if (!C.parse(in.constants)) { why = "malformed constants text"; return STEEL_E_INVALID; }
  if (in.statF_floats != (uint64_t)C.u("LEN_STATF4") * 4u || in.statU_words != C.u("LEN_STATU") ||
      in.art_floats != C.u("LEN_ART")) {
    why = "statF/statU/art sizes do not match the constants";
    return STEEL_E_INVALID;
  }
  SceneDev& d = s.d;
#define K(n) d.n = C.u(#n);
  K(SF_BODY) K(SF_SHAPE) K(SF_HAABB) K(SF_VERTS) K(SF_FPLANE) K(SF_LINK) K(SF_DOF) K(SF_PATH) K(SF_LOOP)
  K(SF_MIMIC) K(SF_CTRL) K(SU_HULL) K(SU_FACE) K(SU_FV) K(SU_HEDGE) K(SU_EDGE) K(SU_ART) K(SU_ACON)
  K(SU_FILTER) K(NB) K(NS) K(NA) K(NL) K(ND) K(NDA) K(JM) K(MAXPATH) K(MAXLP) K(NLOOP) K(NMIMIC) K(PATCH)
  K(EXTRA) K(SHARED) K(FSHARED) K(REST) K(FSTART) K(TGT_HELD) K(CTRL_KIND) K(CTRL_A) K(CTRL_B) K(VLIM_FREE) K(VLIM_ON) K(ART_F64) K(SLEEP) K(NEST) K(MO) K(TORS) K(TO) K(COMPL) K(CO) K(VELITERS) K(JFL) K(DRIVE_ROWS) K(FUSE_VLIM)
  K(VEL_DRIVE_ACTIVE) K(FMODE) K(FMO) K(ANG) K(ANG_ART) K(EO) K(PYRAMID) K(CTI) K(LONGEST_FIRST)
  K(FRICTION_COMBINE) K(RESTITUTION_COMBINE) K(NCOLW) K(NCOL) K(MAXP) K(MAXC) K(MAXU) K(WH) K(AH)
  K(MAXDENSE) K(ROWS) K(PO) K(DHDR) K(DPS)
#undef K
#define F(n) d.n = C.f(#n);
  F(F_ANCHOR_BETA) F(F_CFM) F(F_OMEGA) F(F_SPEC) F(F_GAP_GATE) F(F_FGAP) F(F_FSCALE) F(F_REST_SPEED) F(F_FR_MUT)
  F(F_FR_MUR) F(F_BP_CELL) F(F_JL_GAP) F(F_JL_SPEED) F(F_VLIM_FRAC) F(F_SLEEP_LIN) F(F_SLEEP_ANG) F(F_SLEEP_TIME) F(F_CREEP)
#undef F
  if (d.NCOLW == 0u || d.NCOLW > 64u || d.NCOL != d.NCOLW * 32u) { why = "bad color table size"; return STEEL_E_INVALID; }
  if (d.MAXC == 0u || d.MAXP == 0u || d.WH == 0u || d.AH == 0u) { why = "zero capacity"; return STEEL_E_INVALID; }
  d.fps = C.get("PARAM_fps", 60.0);
  d.substeps = C.u("PARAM_substeps", 4);
  d.iterations = C.u("PARAM_iterations", 12);
  d.target_frames = C.u("PARAM_target_frames");
  d.driven = C.u("PARAM_driven");
  d.integral_count = C.u("PARAM_integral_count");
  d.user_targets = 0u;
  d.beta = (float)C.get("PARAM_baumgarte", 0.2);
  d.warm = (float)C.get("PARAM_warm", 0.0);
  d.reg = (float)C.get("PARAM_reg", 0.0);
  d.gx = (float)C.get("PARAM_gravity0", 0.0);
  d.gy = (float)C.get("PARAM_gravity1", 0.0);
  d.gz = (float)C.get("PARAM_gravity2", -9.81);
  uint32_t NB = d.NB, NS = d.NS, NA = d.NA, NL = d.NL, ND = d.ND;
  uint32_t NQ = C.u("A_QD") - C.u("A_Q");
  d.NQ = NQ;
  const uint32_t MAXC = d.MAXC;
  // Articulation buffer (sim.js:452-455 order), sized with this scene's capacities.
  {
    size_t ao = 0;
    auto put = [&](uint32_t& field, size_t n) { field = (uint32_t)ao; ao += n > 0 ? n : 1; };
    put(d.A_Q, NQ); put(d.A_QD, ND); put(d.A_QDH, ND); put(d.A_INT, ND); put(d.A_TGT, ND); put(d.A_TGTV, ND);
    put(d.A_LIM, 2 * ND); put(d.A_DRV, ND); put(d.A_JFL, ND); put(d.A_JF, ND); put(d.A_BF, NB * 8); put(d.A_SLP, (NB + NA) * 4);
    put(d.A_FRIC, ND); put(d.A_HINV, ND);
    ao = (ao + 3) & ~(size_t)3;  // link blocks start on a 16-byte boundary (bulk copies)
    put(d.A_LINK, (size_t)(NL > 0 ? NL : 1) * 268); put(d.A_SNAP, NB * 8 + ND);
    put(d.A_VLG, ND + NB * 6); put(d.A_AVL, NA); put(d.A_LG, ND); put(d.A_RL, ND); put(d.A_RLN, NA);
    put(d.A_ULOAD, d.PATCH ? (size_t)MAXC : 0); put(d.A_DENSE, (size_t)d.MAXDENSE * d.DPS);
    s.art_floats = ao;
  }
  // Scheduling arrays; unit-indexed arrays are sized by MAXC (every contact may be its own unit).
  {
    size_t so = 0;
    auto put = [&](uint32_t& field, size_t n) { field = (uint32_t)so; so += n > 0 ? n : 1; };
    put(d.S_UNITOF, MAXC); put(d.S_DSLOT, MAXC); put(d.S_CORDER, MAXC); put(d.S_UKEY, MAXC);
    put(d.S_USTART0, MAXC + 1); put(d.S_USIZE, MAXC); put(d.S_USTART, MAXC + 1); put(d.S_RK0, MAXC);
    put(d.S_RK1, MAXC); put(d.S_RK2, MAXC); put(d.S_BPC, 4 * (size_t)MAXC); put(d.S_LEAD, MAXC);
    put(d.S_KEEP, MAXC); put(d.S_SLOT, 26 * (size_t)MAXC); put(d.S_KEPT, MAXC); put(d.S_ROWOF, MAXC);
    put(d.S_RUNIT, MAXC); put(d.S_RCON, MAXC); put(d.S_PCOL, MAXC); put(d.S_PORD, MAXC);
    put(d.S_CSTART, d.NCOL + 2); put(d.S_META, 8); put(d.S_WWIN, d.WH); put(d.S_WSLOT, (size_t)MAXC + d.MAXDENSE);
    put(d.S_WMASK, (size_t)NB * d.NCOLW); put(d.S_WCOUNT, d.NCOL + 2); put(d.S_LINKHIT, NB); put(d.S_JSPLIT, NL);
    put(d.S_UF, NB + NA); put(d.S_UFF, NB + NA); put(d.S_UTP, MAXC);
    put(d.S_DSTART, NA + 1); put(d.S_DOFF, NA); put(d.S_DLIST, d.MAXDENSE);
    // parallel coloring: per-body row lists and frontiers, row keys
    put(d.S_BSTART, NB + 1); put(d.S_BPOS, NB); put(d.S_BREADY, NB); put(d.S_BLIST, 2 * (size_t)MAXC);
    put(d.S_RKEY, MAXC); put(d.S_RFLAG, MAXC); put(d.S_WL, 2 * (size_t)NB);
    s.sched_words = so;
  }
  s.warm_words = 10ull * d.WH + 30ull * d.AH;
  {
    size_t a = 2ull * d.MAXPATH + 6ull * d.MAXPATH * d.JM;
    size_t b = 6ull * d.NDA + 54ull * d.MAXLP + 8;  // dense rows: J, Y, three-way generalized solve
    s.tscr_floats = a > b ? a : b;
    d.TSCR = (uint32_t)s.tscr_floats;
  }
  // Host copies: static data and initial state (the reference's reset() contents).
  s.statF.assign(in.statF, in.statF + in.statF_floats);
  s.statU.assign(in.statU, in.statU + in.statU_words);
  s.pos0.resize(NB); s.rot0.resize(NB); s.lv0.resize(NB); s.av0.resize(NB);
  for (uint32_t b = 0; b < NB; b++) {
    const float* p = in.body_pose + b * 8;
    const float* v = in.body_vel + b * 8;
    s.pos0[b] = make_float4(p[0], p[1], p[2], p[3]);
    s.rot0[b] = make_float4(p[4], p[5], p[6], p[7]);
    s.lv0[b] = make_float4(v[0], v[1], v[2], v[3]);
    s.av0[b] = make_float4(v[4], v[5], v[6], v[7]);
  }
  s.art0.assign(s.art_floats, 0.0f);
  auto copy_block = [&](uint32_t dst, const char* src_key, uint32_t n) {
    uint32_t src = C.u(src_key);
    for (uint32_t i = 0; i < n; i++) s.art0[dst + i] = in.art[src + i];
  };
  copy_block(d.A_Q, "A_Q", NQ);
  copy_block(d.A_QD, "A_QD", ND);
  copy_block(d.A_TGT, "A_TGT", ND);
  copy_block(d.A_TGTV, "A_TGTV", ND);
  // Arena pieces.
  const size_t arena0 = L.bytes;
  s.o_sf = L.take(s.statF.size() * 4);
  s.o_su = L.take(s.statU.size() * 4);
  s.o_pos = L.take((size_t)NB * 16); s.o_rot = L.take((size_t)NB * 16);
  s.o_ppos = L.take((size_t)NB * 16); s.o_prot = L.take((size_t)NB * 16);
  s.o_lv = L.take((size_t)NB * 16); s.o_av = L.take((size_t)NB * 16);
  s.o_spos = L.take((size_t)NS * 16); s.o_srot = L.take((size_t)NS * 16);
  s.o_alo = L.take((size_t)NS * 16); s.o_ahi = L.take((size_t)NS * 16);
  s.o_art = L.take(s.art_floats * 4);
  s.o_cnt = L.take(64); s.o_stats = L.take(64); s.o_params = L.take(sizeof(Params));
  s.o_craw = L.take((size_t)MAXC * 6 * 16); s.o_con = L.take((size_t)MAXC * 6 * 16);
  s.large_sort = next_pow2(MAXC) > SORT_SMEM_KEYS;
  s.o_ckeys = L.take(s.large_sort ? (size_t)MAXC * 16 : 16);
  if (s.large_sort) {
    s.sort_tiles = (MAXC + RS_TILE - 1u) / RS_TILE;
    s.o_rkeys1 = L.take((size_t)MAXC * 16);
    s.o_rstat = L.take(4ull * RS_DIGITS * s.sort_tiles * 256u);
    s.o_rhist = L.take(4ull * RS_DIGITS * 256u);
    s.o_rctr = L.take(4ull * RS_DIGITS);
  }
  s.o_rows = L.take((size_t)MAXC * d.ROWS * 16); s.o_slots = L.take((size_t)MAXC * 2 * 16);
  s.o_warm = L.take(s.warm_words * 4);
  s.o_sched = L.take(s.sched_words * 4);
  s.o_tw = L.take((size_t)NB * 32); s.o_imp = L.take((size_t)NB * 32);
  s.o_aqd = L.take((size_t)(ND > 0 ? ND : 1) * 4);
  const bool team_sized = one_scene && (NB >= TEAM_MIN_BODIES || d.NA >= TEAM_MIN_ARTS);
  d.TSCR_T = team_sized ? threads * TEAM_SCRATCH_BLOCKS : threads;
  s.o_tscr = L.take((size_t)d.TSCR_T * s.tscr_floats * 4);
  s.arena_bytes = L.bytes - arena0;
  return STEEL_OK;
}

template <class T> T* at(uint8_t* base, size_t off) { return reinterpret_cast<T*>(base + off); }

int upload_state(steel_batch* b) {
  cudaStream_t st = b->ctx->stream;
  for (auto& s : b->sc) {
    const SceneDev& d = s.d;
    CU(cudaMemcpyAsync(d.pos, s.pos0.data(), s.pos0.size() * 16, cudaMemcpyHostToDevice, st));
    CU(cudaMemcpyAsync(d.rot, s.rot0.data(), s.rot0.size() * 16, cudaMemcpyHostToDevice, st));
    CU(cudaMemcpyAsync(d.ppos, s.pos0.data(), s.pos0.size() * 16, cudaMemcpyHostToDevice, st));
    CU(cudaMemcpyAsync(d.prot, s.rot0.data(), s.rot0.size() * 16, cudaMemcpyHostToDevice, st));
    CU(cudaMemcpyAsync(d.lv, s.lv0.data(), s.lv0.size() * 16, cudaMemcpyHostToDevice, st));
    CU(cudaMemcpyAsync(d.av, s.av0.data(), s.av0.size() * 16, cudaMemcpyHostToDevice, st));
    CU(cudaMemcpyAsync(d.art, s.art0.data(), s.art0.size() * 4, cudaMemcpyHostToDevice, st));
    CU(cudaMemsetAsync(d.warm_tab, 0, s.warm_words * 4, st));
    CU(cudaMemsetAsync(d.counters, 0, 64, st));
    CU(cudaMemsetAsync(d.stats, 0, 64, st));
  }
  CU(cudaMemsetAsync(b->bd.phase, 0, sizeof(double) * b->sc.size(), st));
  CU(cudaMemsetAsync(b->bd.substep_count, 0, sizeof(unsigned long long) * b->sc.size(), st));
  CU(cudaMemsetAsync(b->bd.error, 0, sizeof(uint32_t), st));
  return STEEL_OK;
}

void enqueue_sequence(const steel_batch* b, const BatchDev& bd, const std::vector<RadixDev>& radix, cudaStream_t st) {
  for (uint32_t s = 0; s < b->substeps; s++) {
    launch_params(bd, s, st);
    launch_shapes(bd, st);
    launch_broad(bd, st);
    launch_narrow(bd, b->narrow_blocks, st);
    launch_csort(bd, b->sort_keys, radix.data(), (uint32_t)radix.size(), st);
    launch_prepare(bd, st);
    launch_solve(bd, st);
  }
  launch_frame_end(bd, st);
}

// One frame's launches. With scene groups (not while serving, whose launch sizes change per tick),
// each group's sequence goes to its own stream, forked from and joined back into `st` by events;
// captured, they become parallel branches of the frame graph.
void enqueue_substeps(steel_batch* b, cudaStream_t st) {
  if (b->groups.empty() || b->serve_on) {
    enqueue_sequence(b, b->bd, b->radix, st);
    return;
  }
  cudaEventRecord(b->ev_fork, st);
  for (auto& g : b->groups) {
    cudaStreamWaitEvent(g.st, b->ev_fork, 0);
    enqueue_sequence(b, g.bd, g.radix, g.st);
    cudaEventRecord(g.done, g.st);
    cudaStreamWaitEvent(st, g.done, 0);
  }
}

int check_device_error(steel_batch* b) {
  uint32_t e = 0;
  CU(cudaMemcpyAsync(&e, b->bd.error, 4, cudaMemcpyDeviceToHost, b->ctx->stream));
  CU(cudaStreamSynchronize(b->ctx->stream));
  if (e == ERR_SORT_CAPACITY) return fail(STEEL_E_CAPACITY, "contact sort capacity exceeded");
  if (e == ERR_JOB_CAPACITY) return fail(STEEL_E_CAPACITY, "narrowphase job capacity exceeded");
  if (e == ERR_SORT_TIMEOUT)
    return fail(STEEL_E_TIMEOUT, "the contact radix sort's look-back gave up waiting for a preceding tile");
  if (e == ERR_STAGE_TIMEOUT)
    return fail(STEEL_E_TIMEOUT, "a shared-memory bulk copy did not complete within its wait limit; the scene's "
                                 "substep was skipped");
  if (e == ERR_TEAM_TIMEOUT)
    return fail(STEEL_E_TIMEOUT, "a block of a team launch gave up waiting at a grid barrier");
  if (e != 0) return fail(STEEL_E_CUDA, "device error " + std::to_string(e));
  return STEEL_OK;
}

void drop_graph(steel_batch* b) {
  if (b->graph) cudaGraphExecDestroy(b->graph);
  b->graph = nullptr;
}

// Shared-memory staging flags of a scene under a per-block budget of dynamic shared memory (0: the
// per-part caps alone). Link blocks first, then twists and impulses, qd, and the color masks; a part
// is staged when it is under its cap and both kernels' layouts stay within the budget.
uint32_t stage_flags(const SceneDev& d, uint32_t budget) {
  const uint64_t lim = budget ? budget : ~0ull;
  auto fits = [&](uint32_t f) {
    return prep_smem_layout(f, d.NL, d.NB, d.NCOLW, d.NCOL).total <= lim &&
           solve_smem_layout(f, d.NB, d.ND, d.NCOL, d.NL).total <= lim;
  };
  uint32_t st = 0u;
  if (d.NL > 0u && 4ull * d.NL * 268u <= STAGE_LINK_CAP && fits(st | STAGE_LINKS)) st |= STAGE_LINKS;
  if (64ull * d.NB <= STAGE_BODY_CAP && fits(st | STAGE_BODIES)) st |= STAGE_BODIES;
  if (4ull * d.ND <= STAGE_QD_CAP && fits(st | STAGE_QD)) st |= STAGE_QD;
  if (4ull * d.NB * d.NCOLW <= STAGE_WMASK_CAP && fits(st | STAGE_WMASK)) st |= STAGE_WMASK;
  return st;
}

// Blocks of the team launches of prepare and solve (team.cuh) for the batch's block size and shared
// memory: a batch of one scene without Nesterov momentum, on the 512-thread instances;
// STEEL_TEAM_AUTO takes scenes of at least TEAM_MIN_BODIES bodies or TEAM_MIN_ARTS articulations,
// with one thread per body or a warp per articulation, capped by the blocks that fit the GPU. Fewer
// than two blocks: the one-block path. `strict`: a request for more blocks than fit, or under
// smaller tiles, is an error (steel_set_team) rather than capped (a later change of tiles).
int team_blocks_for(const steel_batch* b, uint32_t req, bool strict, uint32_t* out) {
  *out = 0u;
  if (req == 0u || b->sc.size() != 1u || b->sc[0].d.NEST != 0u) return STEEL_OK;
  const SceneDev& d = b->sc[0].d;
  const uint32_t T = b->bd.block_threads;
  if (T != (uint32_t)BIG_THREADS) {  // team launches run the 512-thread instances, one block per SM
    if (strict && req != STEEL_TEAM_AUTO)
      return fail(STEEL_E_INVALID, "team launches use 512-thread blocks; the batch's tiles have " + std::to_string(T));
    return STEEL_OK;
  }
  const int per_sm = std::min(solve_team_blocks_per_sm(T, b->bd.solve_smem),
                              prepare_team_blocks_per_sm(T, b->bd.prep_smem));
  const uint32_t cap = per_sm > 0 ? (uint32_t)per_sm * (uint32_t)b->ctx->sms : 0u;
  uint32_t n = 0u;
  if (req == STEEL_TEAM_AUTO) {
    if (d.NB >= TEAM_MIN_BODIES || d.NA >= TEAM_MIN_ARTS) n = std::min((std::max(d.NB, 32u * d.NA) + T - 1u) / T, cap);
  } else {
    if (req > cap && strict)
      return fail(STEEL_E_INVALID, "at most " + std::to_string(cap) + " team blocks of " + std::to_string(T) +
                                       " threads fit this GPU");
    n = std::min(req, cap);
  }
  *out = n >= 2u ? n : 0u;
  return STEEL_OK;
}
int update_team(steel_batch* b) {
  uint32_t n = 0u;
  if (int rc = team_blocks_for(b, b->team_req, false, &n)) return rc;
  if (n != b->bd.team_blocks) {
    b->bd.team_blocks = n;
    drop_graph(b);
  }
  return STEEL_OK;
}

bool valid_block(uint32_t t) {
  for (uint32_t v : BLOCK_SIZES)
    if (v == t) return true;
  return false;
}

void free_groups(steel_batch* b) {
  for (auto& g : b->groups) {
    if (g.st) cudaStreamDestroy(g.st);
    if (g.done) cudaEventDestroy(g.done);
    if (g.mem) cudaFree(g.mem);
  }
  b->groups.clear();
}

// The group views of the batch: the batch's launch parameters (tiles, wait limit) with scene,
// shape, tile, pair and job tables restricted to each group's scene range.
void refresh_groups(steel_batch* b) {
  for (auto& g : b->groups) {
    BatchDev v = b->bd;  // pointers, tables and counters below are the group's
    const uint32_t n = g.hi - g.lo;
    v.scenes = b->bd.scenes + g.lo;
    v.nscenes = n;
    v.nlaunch = n;
    v.nshapes = g.bd.nshapes;
    v.shape_scene = g.bd.shape_scene;
    v.shape_local = b->bd.shape_local + g.shape_lo;
    v.tiles = g.bd.tiles;
    v.ntiles = g.bd.ntiles;
    v.pairs = b->bd.pairs + g.pair_lo;
    v.pair_cap = g.bd.pair_cap;
    v.pair_count = g.bd.pair_count;
    v.jobs = b->bd.jobs + g.pair_lo * (NJOB_WORDS / 4u);
    v.phase = b->bd.phase + g.lo;
    v.substep_count = b->bd.substep_count + g.lo;
    v.active = b->bd.active + g.lo;
    v.order = g.bd.order;
    v.trace_prep = b->bd.trace_prep ? b->bd.trace_prep + 3ull * g.lo : nullptr;
    v.trace_solve = b->bd.trace_solve ? b->bd.trace_solve + 3ull * g.lo : nullptr;
    g.bd = v;
  }
}

// Splits the batch into `count` groups of contiguous scenes with about equal body counts (1: one
// launch sequence for the whole batch).
int make_groups(steel_batch* b, uint32_t count) {
  CU(cudaSetDevice(b->ctx->device));
  CU(cudaStreamSynchronize(b->ctx->stream));
  free_groups(b);
  const uint32_t n = (uint32_t)b->sc.size();
  if (count <= 1u || n < 2u * count) return STEEL_OK;
  if (!b->ev_fork) CU(cudaEventCreateWithFlags(&b->ev_fork, cudaEventDisableTiming));
  uint64_t total = 0;
  for (auto& s : b->sc) total += s.d.NB + 8ull * s.d.NL;
  std::vector<uint32_t> cut{0u};
  uint64_t acc = 0;
  for (uint32_t i = 0; i < n && cut.size() < count; i++) {
    acc += b->sc[i].d.NB + 8ull * b->sc[i].d.NL;
    if (acc * count >= total * cut.size() && i + 1u < n) cut.push_back(i + 1u);
  }
  cut.push_back(n);
  size_t shape_lo = 0, tile_lo = 0, pair_lo = 0;
  uint32_t tile_i = 0;
  for (size_t k = 0; k + 1 < cut.size(); k++) {
    steel_batch::Group g;
    g.lo = cut[k];
    g.hi = cut[k + 1];
    if (g.hi <= g.lo) continue;
    std::vector<uint32_t> shape_scene, order;
    std::vector<uint4> tiles;
    uint32_t cap = 0;
    for (uint32_t s = g.lo; s < g.hi; s++) {
      for (uint32_t q = 0; q < b->sc[s].d.NS; q++) shape_scene.push_back(s - g.lo);
      cap += b->pair_cap_of[s];
    }
    while (tile_i < b->tiles.size() && b->tiles[tile_i].x < g.hi) {
      uint4 t = b->tiles[tile_i++];
      t.x -= g.lo;
      tiles.push_back(t);
    }
    for (uint32_t s : b->order_host)
      if (s >= g.lo && s < g.hi) order.push_back(s - g.lo);
    for (const RadixDev& r : b->radix)
      if (r.scene >= g.lo && r.scene < g.hi) {
        RadixDev rr = r;
        rr.scene -= g.lo;
        g.radix.push_back(rr);
      }
    g.shape_lo = shape_lo;
    g.tile_lo = tile_lo;
    g.pair_lo = pair_lo;
    shape_lo += shape_scene.size();
    tile_lo += tiles.size();
    pair_lo += cap;
    // Tables: shape scenes, tiles, order, pair counters (each 256-byte aligned).
    Layout L;
    const size_t o_ss = L.take(4 * shape_scene.size() + 4), o_t = L.take(16 * tiles.size() + 16),
                 o_o = L.take(4 * order.size() + 4), o_pc = L.take(8);
    if (cudaMalloc(&g.mem, L.bytes) != cudaSuccess) {
      free_groups(b);
      return fail(STEEL_E_NOMEM, "scene group tables");
    }
    cudaStream_t st = b->ctx->stream;
    CU(cudaMemcpyAsync(g.mem + o_ss, shape_scene.data(), 4 * shape_scene.size(), cudaMemcpyHostToDevice, st));
    CU(cudaMemcpyAsync(g.mem + o_t, tiles.data(), 16 * tiles.size(), cudaMemcpyHostToDevice, st));
    CU(cudaMemcpyAsync(g.mem + o_o, order.data(), 4 * order.size(), cudaMemcpyHostToDevice, st));
    CU(cudaMemsetAsync(g.mem + o_pc, 0, 8, st));
    CU(cudaStreamSynchronize(st));
    g.bd.nshapes = (uint32_t)shape_scene.size();
    g.bd.shape_scene = at<uint32_t>(g.mem, o_ss);
    g.bd.tiles = at<uint4>(g.mem, o_t);
    g.bd.ntiles = (uint32_t)tiles.size();
    g.bd.order = at<uint32_t>(g.mem, o_o);
    g.bd.pair_count = at<uint32_t>(g.mem, o_pc);
    g.bd.pair_cap = cap;
    CU(cudaStreamCreateWithFlags(&g.st, cudaStreamNonBlocking));
    CU(cudaEventCreateWithFlags(&g.done, cudaEventDisableTiming));
    b->groups.push_back(std::move(g));
  }
  refresh_groups(b);
  return STEEL_OK;
}

// Makes `t` the batch's tile configuration: block size of prepare and solve, each scene's
// shared-memory staging under the budget, the launches' dynamic shared memory and the
// narrowphase grid. The frame graph is captured again at the next step. Results do not depend on
// the configuration.
int apply_tiles(steel_batch* b, const steel_tiles& t) {
  if (!valid_block(t.block_threads) || t.block_threads > b->max_threads)
    return fail(STEEL_E_INVALID, "block_threads must be 32, 64, 128, 256 or 512 and at most " +
                                     std::to_string(b->max_threads) + " for this batch");
  const uint32_t narrow_max = (uint32_t)narrow_blocks_per_sm();
  if (t.narrow_blocks_per_sm > narrow_max)
    return fail(STEEL_E_INVALID, "narrow_blocks_per_sm above the " + std::to_string(narrow_max) + " that fit an SM");
  if (t.stream_groups > 8u) return fail(STEEL_E_INVALID, "at most 8 stream groups");
  const uint32_t n = (uint32_t)b->sc.size();
  std::vector<uint32_t> stages(n);
  size_t prep = 0, solve = 0;
  for (uint32_t i = 0; i < n; i++) {
    SceneDev& d = b->sc[i].d;
    d.stage = stage_flags(d, t.smem_budget);
    stages[i] = d.stage;
    prep = std::max<size_t>(prep, prep_smem_layout(d.stage, d.NL, d.NB, d.NCOLW, d.NCOL).total);
    solve = std::max<size_t>(solve, solve_smem_layout(d.stage, d.NB, d.ND, d.NCOL, d.NL).total);
  }
  CU(cudaSetDevice(b->ctx->device));
  cudaStream_t st = b->ctx->stream;
  CU(cudaStreamSynchronize(st));
  CU(configure_prepare(t.block_threads, prep));
  CU(configure_solve(t.block_threads, solve));
  CU(cudaMemcpyAsync(b->arena + b->o_stage, stages.data(), 4ull * n, cudaMemcpyHostToDevice, st));
  launch_set_stage(b->bd, reinterpret_cast<const uint32_t*>(b->arena + b->o_stage), st);
  CU(cudaGetLastError());
  CU(cudaStreamSynchronize(st));
  b->bd.prep_smem = (uint32_t)prep;
  b->bd.solve_smem = (uint32_t)solve;
  b->bd.block_threads = t.block_threads;
  b->narrow_blocks = (uint32_t)b->ctx->sms * (t.narrow_blocks_per_sm ? t.narrow_blocks_per_sm : narrow_max);
  const uint32_t want_groups = t.stream_groups > 1u ? t.stream_groups : 1u;
  const uint32_t have_groups = b->groups.empty() ? 1u : (uint32_t)b->groups.size();
  if (want_groups != have_groups || t.stream_groups != b->tile_cfg.stream_groups) {
    if (int rc = make_groups(b, want_groups)) return rc;
  }
  refresh_groups(b);
  b->tile_cfg = t;
  b->tile_cfg.stream_groups = b->groups.empty() ? 1u : (uint32_t)b->groups.size();
  drop_graph(b);
  return update_team(b);
}

SceneHost* scene_of(steel_batch* b, uint32_t s) { return (b && s < b->sc.size()) ? &b->sc[s] : nullptr; }

}  // namespace

extern "C" {

const char* steel_last_error(void) { return g_err.c_str(); }

int steel_ctx_create(int device, steel_ctx** out) {
  if (!out) return fail(STEEL_E_INVALID, "null output");
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) return fail(STEEL_E_NODEVICE, "no CUDA device");
  if (device < 0 || device >= n) return fail(STEEL_E_INVALID, "bad device index");
  CU(cudaSetDevice(device));
  auto* c = new steel_ctx();
  c->device = device;
  cudaDeviceProp prop;
  if (cudaGetDeviceProperties(&prop, device) == cudaSuccess) c->sms = prop.multiProcessorCount;
  if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess) {
    delete c;
    return fail(STEEL_E_CUDA, "stream creation failed");
  }
  *out = c;
  return STEEL_OK;
}

int steel_ctx_destroy(steel_ctx* ctx) {
  if (!ctx) return STEEL_OK;
  cudaSetDevice(ctx->device);
  if (ctx->stream) cudaStreamDestroy(ctx->stream);
  delete ctx;
  return STEEL_OK;
}

int steel_batch_create(steel_ctx* ctx, const steel_scene_desc* scenes, uint32_t n, steel_batch** out) {
  if (!ctx || !scenes || !out || n == 0) return fail(STEEL_E_INVALID, "null argument or empty batch");
  CU(cudaSetDevice(ctx->device));
  std::unique_ptr<steel_batch> b(new steel_batch());
  b->ctx = ctx;
  b->sc.resize(n);
  Layout L;
  const bool big = n <= (uint32_t)ctx->sms;
  b->max_threads = big ? BIG_THREADS : DEFAULT_THREADS;
  for (uint32_t i = 0; i < n; i++) {
    std::string why;
    int rc = build_scene(b->sc[i], scenes[i], L, b->max_threads, n == 1u, why);
    if (rc) return fail(rc, "scene " + std::to_string(i) + ": " + why);
    if (i > 0 && b->sc[i].d.substeps != b->sc[0].d.substeps)
      return fail(STEEL_E_INVALID, "scenes of one batch must share the substep count");
  }
  b->substeps = b->sc[0].d.substeps;
  // Batch-level tables.
  uint32_t pair_cap = 0;
  size_t max_c = 1;
  for (uint32_t i = 0; i < n; i++) {
    const SceneDev& d = b->sc[i].d;
    for (uint32_t s = 0; s < d.NS; s++) { b->shape_scene.push_back(i); b->shape_local.push_back(s); }
    uint32_t nt = (d.NS + BROAD_TILE - 1) / BROAD_TILE;
    for (uint32_t ti = 0; ti < nt; ti++)
      for (uint32_t tj = ti; tj < nt; tj++) b->tiles.push_back(make_uint4(i, ti, tj, 0u));
    pair_cap += d.MAXP;
    b->pair_cap_of.push_back(d.MAXP);
    max_c = std::max<size_t>(max_c, d.MAXC);
  }
  b->o_scenes = L.take(sizeof(SceneDev) * n);
  b->o_shape_scene = L.take(4 * b->shape_scene.size() + 4);
  b->o_shape_local = L.take(4 * b->shape_local.size() + 4);
  b->o_tiles = L.take(16 * b->tiles.size() + 16);
  b->o_pairs = L.take(16ull * pair_cap);
  b->o_pair_count = L.take(8);
  b->o_jobs = L.take(4ull * NJOB_WORDS * pair_cap + 16);
  b->o_phase = L.take(8ull * n);
  b->o_ssc = L.take(8ull * n);
  b->o_active = L.take(4ull * n);
  b->o_order = L.take(4ull * n);
  b->o_err = L.take(4);
  b->o_team = L.take(32);
  b->o_stage = L.take(4ull * n);
  std::vector<uint64_t> tgt_off(n), pose_off(n);
  for (uint32_t i = 0; i < n; i++) {
    tgt_off[i] = b->n_targets;
    pose_off[i] = b->n_poses;
    b->n_targets += b->sc[i].d.ND;
    b->n_poses += 8ull * b->sc[i].d.NB;
  }
  b->o_tgt_off = L.take(8ull * n);
  b->o_pose_off = L.take(8ull * n);
  b->o_tgt_buf = L.take(4ull * b->n_targets + 16);
  b->o_pose_buf = L.take(4ull * b->n_poses + 16);
  b->arena_bytes = L.bytes;
  if (cudaMalloc(&b->arena, b->arena_bytes) != cudaSuccess)
    return fail(STEEL_E_NOMEM, "device arena of " + std::to_string(b->arena_bytes) + " bytes");
  cudaStream_t st = ctx->stream;
  CU(cudaMemsetAsync(b->arena, 0, b->arena_bytes, st));
  uint8_t* A = b->arena;
  std::vector<SceneDev> dev(n);
  uint32_t art_f64 = 0, solve_ext = 0;
  for (uint32_t i = 0; i < n; i++) {
    SceneHost& s = b->sc[i];
    SceneDev& d = s.d;
    d.sf = RO<float4>{at<float4>(A, s.o_sf)};
    d.su = RO<uint32_t>{at<uint32_t>(A, s.o_su)};
    d.pos = at<float4>(A, s.o_pos); d.rot = at<float4>(A, s.o_rot);
    d.ppos = at<float4>(A, s.o_ppos); d.prot = at<float4>(A, s.o_prot);
    d.lv = at<float4>(A, s.o_lv); d.av = at<float4>(A, s.o_av);
    d.spos = at<float4>(A, s.o_spos); d.srot = at<float4>(A, s.o_srot);
    d.alo = at<float4>(A, s.o_alo); d.ahi = at<float4>(A, s.o_ahi);
    d.art = at<float>(A, s.o_art);
    d.counters = at<uint32_t>(A, s.o_cnt); d.stats = at<uint32_t>(A, s.o_stats);
    d.params = at<Params>(A, s.o_params);
    d.craw = at<float4>(A, s.o_craw); d.con = at<float4>(A, s.o_con); d.ckeys = at<uint4>(A, s.o_ckeys);
    d.rows = at<float4>(A, s.o_rows); d.slots = at<float4>(A, s.o_slots);
    d.warm_tab = at<uint32_t>(A, s.o_warm); d.sched = at<uint32_t>(A, s.o_sched);
    d.tw = at<float4>(A, s.o_tw); d.imp = at<float4>(A, s.o_imp); d.aqd = at<float>(A, s.o_aqd);
    d.tscr = at<float>(A, s.o_tscr);
    d.scene_index = i;
    if (s.large_sort) {
      RadixDev r{};
      r.keys[0] = d.ckeys;
      r.keys[1] = at<uint4>(A, s.o_rkeys1);
      r.status = at<uint32_t>(A, s.o_rstat);
      r.hist = at<uint32_t>(A, s.o_rhist);
      r.ctr = at<uint32_t>(A, s.o_rctr);
      r.tiles = s.sort_tiles;
      r.scene = i;
      b->radix.push_back(r);
    }
    d.stage = 0u;  // set by apply_tiles below
    art_f64 |= d.ART_F64;
    solve_ext |= d.ANG_ART | d.CTI;
    dev[i] = d;
    CU(cudaMemcpyAsync((void*)d.sf.p, s.statF.data(), s.statF.size() * 4, cudaMemcpyHostToDevice, st));
    CU(cudaMemcpyAsync((void*)d.su.p, s.statU.data(), s.statU.size() * 4, cudaMemcpyHostToDevice, st));
  }
  BatchDev& bd = b->bd;
  bd.scenes = at<SceneDev>(A, b->o_scenes);
  bd.nscenes = n;
  bd.nshapes = (uint32_t)b->shape_scene.size();
  bd.shape_scene = at<uint32_t>(A, b->o_shape_scene);
  bd.shape_local = at<uint32_t>(A, b->o_shape_local);
  bd.tiles = at<uint4>(A, b->o_tiles);
  bd.ntiles = (uint32_t)b->tiles.size();
  bd.pairs = at<uint4>(A, b->o_pairs);
  bd.pair_cap = pair_cap;
  bd.pair_count = at<uint32_t>(A, b->o_pair_count);
  bd.jobs = at<uint4>(A, b->o_jobs);
  bd.phase = at<double>(A, b->o_phase);
  bd.substep_count = at<unsigned long long>(A, b->o_ssc);
  bd.active = at<uint32_t>(A, b->o_active);
  bd.order = at<uint32_t>(A, b->o_order);
  bd.nlaunch = n;
  {
    // Prepare and solve blocks take the scenes longest first (chain length, then bodies), so
    // short scenes fill the end of the launch. (An order by estimated block time, 16 bodies per
    // chain link plus bodies, measured the same frame time on the uneven batch.)
    std::vector<uint32_t> order(n);
    for (uint32_t i = 0; i < n; i++) order[i] = i;
    std::stable_sort(order.begin(), order.end(), [&](uint32_t x, uint32_t y) {
      const SceneDev &a = b->sc[x].d, &c = b->sc[y].d;
      return a.MAXLP != c.MAXLP ? a.MAXLP > c.MAXLP : a.NB > c.NB;
    });
    b->order_host = order;
    CU(cudaMemcpyAsync(A + b->o_order, b->order_host.data(), 4ull * n, cudaMemcpyHostToDevice, st));
  }
  CU(cudaMemsetAsync(A + b->o_active, 1, 4ull * n, st));  // every scene steps (nonzero words)
  bd.error = at<uint32_t>(A, b->o_err);
  bd.team_bar = at<uint32_t>(A, b->o_team);
  bd.team_blocks = 0;
  bd.art_f64 = art_f64 != 0u ? 1u : 0u;
  bd.solve_ext = solve_ext != 0u ? 1u : 0u;
  bd.block_threads = b->max_threads;
  bd.wait_limit = STEEL_WAIT_LIMIT_DEFAULT;
  bd.trace_prep = nullptr;
  bd.trace_solve = nullptr;
  static_assert(STEEL_WAIT_LIMIT_DEFAULT == BULK_WAIT_LIMIT, "one default wait limit");
  CU(cudaMemcpyAsync(bd.scenes, dev.data(), sizeof(SceneDev) * n, cudaMemcpyHostToDevice, st));
  CU(cudaMemcpyAsync((void*)bd.shape_scene, b->shape_scene.data(), 4 * b->shape_scene.size(), cudaMemcpyHostToDevice, st));
  CU(cudaMemcpyAsync((void*)bd.shape_local, b->shape_local.data(), 4 * b->shape_local.size(), cudaMemcpyHostToDevice, st));
  CU(cudaMemcpyAsync((void*)bd.tiles, b->tiles.data(), 16 * b->tiles.size(), cudaMemcpyHostToDevice, st));
  CU(cudaMemcpyAsync(A + b->o_tgt_off, tgt_off.data(), 8ull * n, cudaMemcpyHostToDevice, st));
  CU(cudaMemcpyAsync(A + b->o_pose_off, pose_off.data(), 8ull * n, cudaMemcpyHostToDevice, st));
  b->sort_keys = std::min<size_t>(next_pow2(max_c), SORT_SMEM_KEYS);
  CU(configure_sort(b->sort_keys));
  {
    steel_tiles t{};
    t.block_threads = b->max_threads;  // one block per SM for few scenes, 4 per SM otherwise
    t.smem_budget = 0;                 // the per-part staging caps alone
    t.narrow_blocks_per_sm = 0;        // as many as fit
    t.stream_groups = 1;               // one launch sequence
    int rc = apply_tiles(b.get(), t);
    if (rc) return rc;
  }
  CU(cudaEventCreate(&b->ev0));
  CU(cudaEventCreate(&b->ev1));
  int rc = upload_state(b.get());
  if (rc) return rc;
  CU(cudaStreamSynchronize(st));
  *out = b.release();
  return STEEL_OK;
}

int steel_convex_hull(const double* pts, uint32_t n, double* verts, double* planes, uint32_t* face_start,
                      uint32_t* face_verts, uint32_t* nv, uint32_t* nf) {
  if (!pts || !verts || !planes || !face_start || !face_verts || !nv || !nf) return fail(STEEL_E_INVALID, "null argument");
  hull::Hull h;
  std::string err;
  if (!hull::convex_hull(pts, n, h, err)) return fail(STEEL_E_INVALID, err);
  const size_t faces = h.face_start.size() - 1u;
  // Euler's formula bounds a hull of v <= n vertices by 2v - 4 faces and 6v - 12 face corners.
  if (h.verts.size() > 3ull * n || faces > 2ull * n || h.face_verts.size() > 6ull * n)
    return fail(STEEL_E_INVALID, "hull larger than its bounds");
  std::memcpy(verts, h.verts.data(), h.verts.size() * sizeof(double));
  std::memcpy(planes, h.planes.data(), h.planes.size() * sizeof(double));
  std::memcpy(face_start, h.face_start.data(), h.face_start.size() * sizeof(uint32_t));
  std::memcpy(face_verts, h.face_verts.data(), h.face_verts.size() * sizeof(uint32_t));
  *nv = (uint32_t)(h.verts.size() / 3u);
  *nf = (uint32_t)faces;
  return STEEL_OK;
}

int steel_pack(const char* json, uint64_t json_len, const void* bin, uint64_t bin_len, const char* opts_json,
               steel_packed** out) {
  if (!json || !out || (!bin && bin_len)) return fail(STEEL_E_INVALID, "null argument");
  scene::JV js, opts;
  std::string err;
  if (!scene::parse_json(json, json_len, js, err)) return fail(STEEL_E_INVALID, "scene.json: " + err);
  if (opts_json && *opts_json && !scene::parse_json(opts_json, std::strlen(opts_json), opts, err))
    return fail(STEEL_E_INVALID, "options: " + err);
  std::unique_ptr<steel_packed> p(new steel_packed());
  if (!scene::pack(js, static_cast<const uint8_t*>(bin), bin_len, &opts, p->p, err)) return fail(STEEL_E_INVALID, err);
  *out = p.release();
  return STEEL_OK;
}

int steel_packed_desc(const steel_packed* p, steel_scene_desc* out) {
  if (!p || !out) return fail(STEEL_E_INVALID, "null argument");
  const scene::Packed& k = p->p;
  out->constants = k.constants.c_str();
  out->statF = k.statF.data();
  out->statF_floats = k.statF.size();
  out->statU = k.statU.data();
  out->statU_words = k.statU.size();
  out->body_pose = k.body_pose.data();
  out->body_vel = k.body_vel.data();
  out->art = k.art.data();
  out->art_floats = k.art.size();
  return STEEL_OK;
}

int steel_packed_free(steel_packed* p) {
  delete p;
  return STEEL_OK;
}

int steel_batch_create_files(steel_ctx* ctx, uint32_t n, const char* const* json, const uint64_t* json_len,
                             const void* const* bin, const uint64_t* bin_len, const char* const* opts_json,
                             steel_batch** out) {
  if (!ctx || !json || !json_len || !bin || !bin_len || !out || n == 0) return fail(STEEL_E_INVALID, "null argument");
  std::vector<std::shared_ptr<steel_packed>> packed(n);
  std::vector<steel_scene_desc> descs(n);
  for (uint32_t i = 0; i < n; i++) {
    steel_packed* p = nullptr;
    int rc = steel_pack(json[i], json_len[i], bin[i], bin_len[i], opts_json ? opts_json[i] : nullptr, &p);
    if (rc) return fail(rc, "scene " + std::to_string(i) + ": " + g_err);
    packed[i].reset(p);
    steel_packed_desc(p, &descs[i]);
  }
  steel_batch* b = nullptr;
  int rc = steel_batch_create(ctx, descs.data(), n, &b);
  if (rc) return rc;
  for (uint32_t i = 0; i < n; i++)
    b->sc[i].files = std::shared_ptr<const scene::Packed>(packed[i], &packed[i]->p);
  *out = b;
  return STEEL_OK;
}

int steel_scene_create(steel_ctx* ctx, const char* json, uint64_t json_len, const void* bin, uint64_t bin_len,
                       const char* opts_json, steel_batch** out) {
  return steel_batch_create_files(ctx, 1, &json, &json_len, &bin, &bin_len, &opts_json, out);
}

int steel_newton_info(steel_batch* b, uint32_t scene, steel_newton_info_t* out) {
  SceneHost* s = scene_of(b, scene);
  if (!s || !out) return fail(STEEL_E_INVALID, "bad scene index or null output");
  if (!s->files) return fail(STEEL_E_INVALID, "the scene was not created from its files (steel_scene_create)");
  const scene::Packed& k = *s->files;
  out->bodies = k.NB;
  out->joint_coords = (uint32_t)k.joint_q.size();
  out->joint_dofs = k.joint_qd_count;
  return STEEL_OK;
}

int steel_newton_dof(steel_batch* b, uint32_t scene, uint32_t newton_dof, uint32_t* port_dof) {
  SceneHost* s = scene_of(b, scene);
  if (!s || !port_dof) return fail(STEEL_E_INVALID, "bad scene index or null output");
  if (!s->files) return fail(STEEL_E_INVALID, "the scene was not created from its files (steel_scene_create)");
  auto it = s->files->dof_map.find(newton_dof);
  if (it == s->files->dof_map.end())
    return fail(STEEL_E_INVALID, "dof " + std::to_string(newton_dof) + " is not simulated as an articulation dof");
  *port_dof = it->second;
  return STEEL_OK;
}

int steel_state(steel_batch* b, uint32_t scene, float* bodyQ, float* bodyQd, float* jointQ, float* jointQd) {
  SceneHost* s = scene_of(b, scene);
  if (!s || !bodyQ || !bodyQd || !jointQ || !jointQd) return fail(STEEL_E_INVALID, "bad scene index or null buffer");
  if (!s->files) return fail(STEEL_E_INVALID, "the scene was not created from its files (steel_scene_create)");
  const scene::Packed& k = *s->files;
  const SceneDev& d = s->d;
  const uint32_t NB = d.NB;
  std::vector<float> poses(8ull * NB), vel(8ull * NB), q(std::max(d.NQ, 1u)), qd(std::max(d.ND, 1u)),
      lv(6ull * std::max(d.NL, 1u));
  int rc = steel_read_state(b, scene, poses.data(), vel.data(), q.data(), qd.data(), lv.data());
  if (rc) return rc;
  // Articulated links keep their COM twist in the link record (angular, then linear).
  for (uint32_t l = 0; l < d.NL; l++) {
    const uint32_t bd = k.link_body[l];
    const float* t = &lv[6ull * l];
    const float w[8] = {t[3], t[4], t[5], 0.0f, t[0], t[1], t[2], 0.0f};
    std::memcpy(&vel[8ull * bd], w, sizeof w);
  }
  for (uint32_t i = 0; i < NB; i++) {
    const double x = poses[8ull * i + 4], y = poses[8ull * i + 5], z = poses[8ull * i + 6], w = poses[8ull * i + 7];
    const double* c = &k.body_com[3ull * i];
    const double ux = 2 * (x * c[0] + y * c[1] + z * c[2]);
    const double s2 = w * w - (x * x + y * y + z * z);
    const double cx = y * c[2] - z * c[1], cy = z * c[0] - x * c[2], cz = x * c[1] - y * c[0];
    const double r[3] = {ux * x + s2 * c[0] + 2 * w * cx, ux * y + s2 * c[1] + 2 * w * cy, ux * z + s2 * c[2] + 2 * w * cz};
    float* bq = bodyQ + 7ull * i;
    for (int a = 0; a < 3; a++) bq[a] = (float)((double)poses[8ull * i + a] - r[a]);
    bq[3] = (float)x; bq[4] = (float)y; bq[5] = (float)z; bq[6] = (float)w;
    float* bv = bodyQd + 6ull * i;
    bv[0] = vel[8ull * i]; bv[1] = vel[8ull * i + 1]; bv[2] = vel[8ull * i + 2];
    bv[3] = vel[8ull * i + 4]; bv[4] = vel[8ull * i + 5]; bv[5] = vel[8ull * i + 6];
  }
  std::memcpy(jointQ, k.joint_q.data(), 4 * k.joint_q.size());
  std::memset(jointQd, 0, 4ull * k.joint_qd_count);
  for (auto& kv : k.q_map) jointQ[kv.first] = q[kv.second];
  for (auto& kv : k.dof_map) jointQd[kv.first] = qd[kv.second];
  for (const auto& fj : k.free_joints) {
    std::memcpy(jointQ + fj.q_start, bodyQ + 7ull * fj.body, 28);
    std::memcpy(jointQd + fj.qd_start, bodyQd + 6ull * fj.body, 24);
  }
  return STEEL_OK;
}

int steel_batch_destroy(steel_batch* b) {
  if (!b) return STEEL_OK;
  cudaSetDevice(b->ctx->device);
  cudaStreamSynchronize(b->ctx->stream);
  if (b->graph) cudaGraphExecDestroy(b->graph);
  if (b->ev0) cudaEventDestroy(b->ev0);
  if (b->ev1) cudaEventDestroy(b->ev1);
  if (b->ev_pose) cudaEventDestroy(b->ev_pose);
  free_groups(b);
  if (b->ev_fork) cudaEventDestroy(b->ev_fork);
  if (b->arena) cudaFree(b->arena);
  if (b->trace) cudaFree(b->trace);
  delete b;
  return STEEL_OK;
}

int steel_scene_info_get(steel_batch* b, uint32_t scene, steel_scene_info* out) {
  SceneHost* s = scene_of(b, scene);
  if (!s || !out) return fail(STEEL_E_INVALID, "bad scene index");
  const SceneDev& d = s->d;
  *out = steel_scene_info{d.NB, d.NS, d.NA, d.NL, d.ND, d.NQ, d.MAXP, d.MAXC, d.MAXU, d.MAXDENSE};
  return STEEL_OK;
}

int steel_reset(steel_batch* b) {
  if (!b) return fail(STEEL_E_INVALID, "null batch");
  CU(cudaSetDevice(b->ctx->device));
  int rc = upload_state(b);
  if (rc) return rc;
  CU(cudaStreamSynchronize(b->ctx->stream));
  return STEEL_OK;
}

int steel_debug_set_wait_limit(steel_batch* b, uint32_t rounds) {
  if (!b) return fail(STEEL_E_INVALID, "null batch");
  CU(cudaSetDevice(b->ctx->device));
  CU(cudaStreamSynchronize(b->ctx->stream));
  b->bd.wait_limit = rounds;
  refresh_groups(b);
  drop_graph(b);  // the limit is a launch argument: capture again
  return STEEL_OK;
}

int steel_trace(steel_batch* b, int on) {
  if (!b) return fail(STEEL_E_INVALID, "null batch");
  CU(cudaSetDevice(b->ctx->device));
  CU(cudaStreamSynchronize(b->ctx->stream));
  const size_t n = b->sc.size();
  if (on && !b->trace) {
    CU(cudaMalloc(&b->trace, 6 * n * sizeof(unsigned long long)));
    CU(cudaMemset(b->trace, 0, 6 * n * sizeof(unsigned long long)));
  } else if (!on && b->trace) {
    CU(cudaFree(b->trace));
    b->trace = nullptr;
  }
  b->bd.trace_prep = b->trace;
  b->bd.trace_solve = b->trace ? b->trace + 3 * n : nullptr;
  refresh_groups(b);
  drop_graph(b);  // the record pointers are launch arguments: capture again
  return STEEL_OK;
}

int steel_trace_read(steel_batch* b, uint64_t* out, uint64_t words) {
  if (!b || !out) return fail(STEEL_E_INVALID, "null argument");
  if (!b->trace) return fail(STEEL_E_INVALID, "tracing is off (steel_trace)");
  const size_t n = b->sc.size();
  if (words < 6 * n) return fail(STEEL_E_INVALID, "trace buffer needs 6 words per scene");
  CU(cudaSetDevice(b->ctx->device));
  CU(cudaStreamSynchronize(b->ctx->stream));
  CU(cudaMemcpy(out, b->trace, 6 * n * sizeof(unsigned long long), cudaMemcpyDeviceToHost));
  return STEEL_OK;
}

int steel_get_tiles(steel_batch* b, steel_tiles* out) {
  if (!b || !out) return fail(STEEL_E_INVALID, "null argument");
  *out = b->tile_cfg;
  return STEEL_OK;
}

int steel_set_tiles(steel_batch* b, const steel_tiles* t) {
  if (!b || !t) return fail(STEEL_E_INVALID, "null argument");
  if (b->serve_on) return fail(STEEL_E_INVALID, "end the serving loop before changing tiles");
  return apply_tiles(b, *t);
}

int steel_set_team(steel_batch* b, uint32_t blocks) {
  if (!b) return fail(STEEL_E_INVALID, "null batch");
  if (b->serve_on) return fail(STEEL_E_INVALID, "end the serving loop before changing the team");
  uint32_t n = 0u;
  if (int rc = team_blocks_for(b, blocks, true, &n)) return rc;
  CU(cudaSetDevice(b->ctx->device));
  CU(cudaStreamSynchronize(b->ctx->stream));
  b->team_req = blocks;
  return update_team(b);
}

int steel_get_team(steel_batch* b, uint32_t* blocks) {
  if (!b || !blocks) return fail(STEEL_E_INVALID, "null argument");
  *blocks = b->bd.team_blocks;
  return STEEL_OK;
}

int steel_autotune(steel_batch* b, uint32_t frames, steel_tiles* best, float* best_ms_per_frame) {
  if (!b || frames == 0) return fail(STEEL_E_INVALID, "null batch or zero frames");
  if (b->serve_on) return fail(STEEL_E_INVALID, "end the serving loop before tuning");
  // Candidates: block size with a staging budget that keeps that many blocks resident per SM
  // (228 KiB of shared memory per SM, less 1 KiB reserved and about 2 KiB of static shared memory
  // per block), and the default caps.
  auto budget_for = [](uint32_t threads) { return 233472u / blocks_per_sm_of(threads) - 3328u; };
  std::vector<steel_tiles> cands;
  if (b->max_threads == BIG_THREADS) {
    cands = {{512, 0, 0, 1}, {256, 0, 0, 1}, {256, budget_for(256), 0, 1}, {128, budget_for(128), 0, 1}};
  } else {
    cands = {{128, 0, 0, 1}, {128, budget_for(128), 0, 1}, {64, budget_for(64), 0, 1}, {64, budget_for(64) / 2u, 0, 1},
             {32, budget_for(32), 0, 1}, {32, budget_for(32) / 2u, 0, 1}};
  }
  const uint32_t narrow_max = (uint32_t)narrow_blocks_per_sm();
  if (narrow_max > 1u) cands.push_back({0u, 0u, narrow_max - 1u, 1u});  // block size filled in from the best so far
  if (b->sc.size() > 2u * (size_t)b->ctx->sms) cands.push_back({0u, 0u, 0u, 2u});  // the best so far, two groups
  CU(cudaSetDevice(b->ctx->device));
  cudaStream_t st = b->ctx->stream;
  steel_tiles won = b->tile_cfg;
  float won_ms = 1e30f;
  for (steel_tiles c : cands) {
    if (c.block_threads == 0u) {
      c.block_threads = won.block_threads;
      c.smem_budget = won.smem_budget;
      if (c.stream_groups == 2u) c.narrow_blocks_per_sm = won.narrow_blocks_per_sm;
    }
    if (int rc = apply_tiles(b, c)) return rc;
    if (int rc = upload_state(b)) return rc;
    if (int rc = steel_step(b, 2u)) return rc;  // warm-up, graph capture
    CU(cudaEventRecord(b->ev0, st));
    if (int rc = steel_step(b, frames)) return rc;
    CU(cudaEventRecord(b->ev1, st));
    CU(cudaEventSynchronize(b->ev1));
    float ms = 0.0f;
    CU(cudaEventElapsedTime(&ms, b->ev0, b->ev1));
    if (int rc = check_device_error(b)) return rc;
    ms /= (float)frames;
    if (ms < won_ms) { won_ms = ms; won = c; }
  }
  if (int rc = apply_tiles(b, won)) return rc;
  // A batch of one scene: team sizes of the solve with the fastest tiles (one block, the default
  // rule's count, half and twice that, all that fit), kept as an explicit request when one wins.
  if (b->sc.size() == 1u && b->sc[0].d.NEST == 0u) {
    const uint32_t req0 = b->team_req;
    uint32_t n_auto = 0u, n_cap = 0u;
    if (int rc = team_blocks_for(b, STEEL_TEAM_AUTO, false, &n_auto)) return rc;
    if (int rc = team_blocks_for(b, 0x7fffffffu, false, &n_cap)) return rc;
    std::vector<uint32_t> teams{b->bd.team_blocks};  // the configuration timed last (current request)
    for (uint32_t t : {0u, n_auto, n_auto / 2u, 2u * n_auto, n_cap, 4u, 16u})
      if ((t == 0u || (t >= 2u && t <= n_cap)) && std::find(teams.begin(), teams.end(), t) == teams.end())
        teams.push_back(t);
    uint32_t won_team = b->bd.team_blocks;
    for (size_t k = 1; k < teams.size(); k++) {
      b->team_req = teams[k];
      if (int rc = update_team(b)) return rc;
      if (int rc = upload_state(b)) return rc;
      if (int rc = steel_step(b, 2u)) return rc;
      CU(cudaEventRecord(b->ev0, st));
      if (int rc = steel_step(b, frames)) return rc;
      CU(cudaEventRecord(b->ev1, st));
      CU(cudaEventSynchronize(b->ev1));
      float ms = 0.0f;
      CU(cudaEventElapsedTime(&ms, b->ev0, b->ev1));
      if (int rc = check_device_error(b)) return rc;
      ms /= (float)frames;
      if (ms < won_ms) { won_ms = ms; won_team = teams[k]; }
    }
    b->team_req = won_team == teams[0] ? req0 : won_team;
    if (int rc = update_team(b)) return rc;
  }
  if (int rc = upload_state(b)) return rc;
  CU(cudaStreamSynchronize(st));
  if (best) *best = won;
  if (best_ms_per_frame) *best_ms_per_frame = won_ms;
  return STEEL_OK;
}

int steel_set_graph(steel_batch* b, int enabled) {
  if (!b) return fail(STEEL_E_INVALID, "null batch");
  b->use_graph = enabled != 0;
  return STEEL_OK;
}

int steel_step(steel_batch* b, uint32_t frames) {
  if (!b) return fail(STEEL_E_INVALID, "null batch");
  CU(cudaSetDevice(b->ctx->device));
  cudaStream_t st = b->ctx->stream;
  const bool graph = b->use_graph && !b->serve_on;  // the serving loop's launch sizes change from tick to tick
  if (graph && !b->graph) {
    cudaGraph_t g;
    CU(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
    enqueue_substeps(b, st);
    CU(cudaStreamEndCapture(st, &g));
    cudaError_t e = cudaGraphInstantiate(&b->graph, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) return fail(STEEL_E_CUDA, std::string("graph instantiate: ") + cudaGetErrorString(e));
  }
  for (uint32_t f = 0; f < frames; f++) {
    if (graph) CU(cudaGraphLaunch(b->graph, st));
    else enqueue_substeps(b, st);
  }
  CU(cudaGetLastError());
  return STEEL_OK;
}

int steel_step_timed(steel_batch* b, uint32_t frames, float* ms) {
  if (!b || !ms) return fail(STEEL_E_INVALID, "null argument");
  CU(cudaSetDevice(b->ctx->device));
  CU(cudaEventRecord(b->ev0, b->ctx->stream));
  int rc = steel_step(b, frames);
  if (rc) return rc;
  CU(cudaEventRecord(b->ev1, b->ctx->stream));
  CU(cudaEventSynchronize(b->ev1));
  CU(cudaEventElapsedTime(ms, b->ev0, b->ev1));
  return check_device_error(b);
}

int steel_step_io(steel_batch* b, uint32_t frames, const float* targets, uint64_t n_targets, float* poses,
                  uint64_t n_poses) {
  if (!b) return fail(STEEL_E_INVALID, "null batch");
  if (targets && n_targets != b->n_targets)
    return fail(STEEL_E_INVALID, "expected " + std::to_string(b->n_targets) + " targets");
  if (poses && n_poses != b->n_poses) return fail(STEEL_E_INVALID, "expected " + std::to_string(b->n_poses) + " pose floats");
  CU(cudaSetDevice(b->ctx->device));
  cudaStream_t st = b->ctx->stream;
  uint8_t* A = b->arena;
  if (targets && b->n_targets) {
    CU(cudaMemcpyAsync(A + b->o_tgt_buf, targets, 4ull * b->n_targets, cudaMemcpyHostToDevice, st));
    launch_scatter_targets(b->bd, (const float*)(A + b->o_tgt_buf), (const uint64_t*)(A + b->o_tgt_off), st);
    for (auto& s : b->sc) s.d.user_targets = s.d.ND ? 1u : s.d.user_targets;
  }
  int rc = steel_step(b, frames);
  if (rc) return rc;
  if (poses) {
    launch_gather_poses(b->bd, (float*)(A + b->o_pose_buf), (const uint64_t*)(A + b->o_pose_off), st);
    CU(cudaMemcpyAsync(poses, A + b->o_pose_buf, 4ull * b->n_poses, cudaMemcpyDeviceToHost, st));
  }
  CU(cudaGetLastError());
  return check_device_error(b);  // synchronizes; reports a capacity or wait error raised by these frames
}

int steel_profile_kernels(steel_batch* b, uint32_t frames, float* ms_per_launch) {
  if (!b || !ms_per_launch) return fail(STEEL_E_INVALID, "null argument");
  CU(cudaSetDevice(b->ctx->device));
  cudaStream_t st = b->ctx->stream;
  const int NK = 7;
  std::vector<cudaEvent_t> ev(2 * NK * b->substeps);
  for (auto& e : ev) CU(cudaEventCreate(&e));
  double acc[NK] = {0};
  for (uint32_t f = 0; f < frames; f++) {
    for (uint32_t s = 0; s < b->substeps; s++) {
      cudaEvent_t* e = ev.data() + 2 * NK * s;
      CU(cudaEventRecord(e[0], st)); launch_params(b->bd, s, st); CU(cudaEventRecord(e[1], st));
      CU(cudaEventRecord(e[2], st)); launch_shapes(b->bd, st); CU(cudaEventRecord(e[3], st));
      CU(cudaEventRecord(e[4], st)); launch_broad(b->bd, st); CU(cudaEventRecord(e[5], st));
      CU(cudaEventRecord(e[6], st)); launch_narrow(b->bd, b->narrow_blocks, st); CU(cudaEventRecord(e[7], st));
      CU(cudaEventRecord(e[8], st)); launch_csort(b->bd, b->sort_keys, b->radix.data(), (uint32_t)b->radix.size(), st); CU(cudaEventRecord(e[9], st));
      CU(cudaEventRecord(e[10], st)); launch_prepare(b->bd, st); CU(cudaEventRecord(e[11], st));
      CU(cudaEventRecord(e[12], st)); launch_solve(b->bd, st); CU(cudaEventRecord(e[13], st));
    }
    launch_frame_end(b->bd, st);
    CU(cudaStreamSynchronize(st));
    for (uint32_t s = 0; s < b->substeps; s++)
      for (int k = 0; k < NK; k++) {
        float ms = 0.0f;
        CU(cudaEventElapsedTime(&ms, ev[2 * NK * s + 2 * k], ev[2 * NK * s + 2 * k + 1]));
        acc[k] += ms;
      }
  }
  for (auto& e : ev) cudaEventDestroy(e);
  for (int k = 0; k < NK; k++) ms_per_launch[k] = (float)(acc[k] / ((double)frames * b->substeps));
  return check_device_error(b);
}

int steel_sync(steel_batch* b) {
  if (!b) return fail(STEEL_E_INVALID, "null batch");
  CU(cudaSetDevice(b->ctx->device));
  CU(cudaStreamSynchronize(b->ctx->stream));
  return check_device_error(b);
}

int steel_read_poses(steel_batch* b, uint32_t scene, float* poses) {
  SceneHost* s = scene_of(b, scene);
  if (!s || !poses) return fail(STEEL_E_INVALID, "bad scene index or null buffer");
  CU(cudaSetDevice(b->ctx->device));
  const SceneDev& d = s->d;
  std::vector<float4> p(d.NB), q(d.NB);
  cudaStream_t st = b->ctx->stream;
  CU(cudaMemcpyAsync(p.data(), d.pos, 16ull * d.NB, cudaMemcpyDeviceToHost, st));
  CU(cudaMemcpyAsync(q.data(), d.rot, 16ull * d.NB, cudaMemcpyDeviceToHost, st));
  CU(cudaStreamSynchronize(st));
  for (uint32_t i = 0; i < d.NB; i++) {
    std::memcpy(poses + i * 8, &p[i], 16);
    std::memcpy(poses + i * 8 + 4, &q[i], 16);
  }
  return STEEL_OK;
}

int steel_copy_poses_device(steel_batch* b, uint32_t scene, float* dst, void* stream) {
  SceneHost* s = scene_of(b, scene);
  if (!s || !dst) return fail(STEEL_E_INVALID, "bad scene index or null buffer");
  if (reinterpret_cast<uintptr_t>(dst) & 15u) return fail(STEEL_E_INVALID, "pose buffer must be 16-byte aligned");
  CU(cudaSetDevice(b->ctx->device));
  cudaPointerAttributes a{};
  if (cudaPointerGetAttributes(&a, dst) != cudaSuccess || !((a.type == cudaMemoryTypeDevice && a.device == b->ctx->device) ||
                                                           a.type == cudaMemoryTypeManaged)) {
    (void)cudaGetLastError();
    return fail(STEEL_E_INVALID, "pose buffer must be device memory of the batch's device");
  }
  cudaStream_t st = b->ctx->stream;
  cudaStream_t out = stream ? static_cast<cudaStream_t>(stream) : st;
  if (out != st) {
    if (!b->ev_pose) CU(cudaEventCreateWithFlags(&b->ev_pose, cudaEventDisableTiming));
    CU(cudaEventRecord(b->ev_pose, st));
    CU(cudaStreamWaitEvent(out, b->ev_pose, 0));
  }
  const SceneDev& d = s->d;
  launch_copy_poses(d.pos, d.rot, d.NB, reinterpret_cast<float4*>(dst), out);
  CU(cudaGetLastError());
  return STEEL_OK;
}

int steel_read_state(steel_batch* b, uint32_t scene, float* poses, float* vel, float* q, float* qd, float* link_v) {
  SceneHost* s = scene_of(b, scene);
  if (!s) return fail(STEEL_E_INVALID, "bad scene index");
  int rc = poses ? steel_read_poses(b, scene, poses) : STEEL_OK;
  if (rc) return rc;
  const SceneDev& d = s->d;
  cudaStream_t st = b->ctx->stream;
  if (vel) {
    std::vector<float4> v(d.NB), w(d.NB);
    CU(cudaMemcpyAsync(v.data(), d.lv, 16ull * d.NB, cudaMemcpyDeviceToHost, st));
    CU(cudaMemcpyAsync(w.data(), d.av, 16ull * d.NB, cudaMemcpyDeviceToHost, st));
    CU(cudaStreamSynchronize(st));
    for (uint32_t i = 0; i < d.NB; i++) { std::memcpy(vel + i * 8, &v[i], 16); std::memcpy(vel + i * 8 + 4, &w[i], 16); }
  }
  if (q && d.NQ) CU(cudaMemcpyAsync(q, d.art + d.A_Q, 4ull * d.NQ, cudaMemcpyDeviceToHost, st));
  if (qd && d.ND) CU(cudaMemcpyAsync(qd, d.art + d.A_QD, 4ull * d.ND, cudaMemcpyDeviceToHost, st));
  if (link_v)
    for (uint32_t l = 0; l < d.NL; l++)
      CU(cudaMemcpyAsync(link_v + l * 6, d.art + d.A_LINK + l * 268u + 147u, 24, cudaMemcpyDeviceToHost, st));
  CU(cudaStreamSynchronize(st));
  return STEEL_OK;
}

int steel_get_stats(steel_batch* b, uint32_t scene, steel_stats* out) {
  SceneHost* s = scene_of(b, scene);
  if (!s || !out) return fail(STEEL_E_INVALID, "bad scene index or null output");
  CU(cudaSetDevice(b->ctx->device));
  uint32_t w[16];
  CU(cudaMemcpyAsync(w, s->d.stats, 64, cudaMemcpyDeviceToHost, b->ctx->stream));
  CU(cudaStreamSynchronize(b->ctx->stream));
  const SceneDev& d = s->d;
  out->max_contacts = w[1]; out->max_colors = w[2]; out->max_units = w[3]; out->max_pairs = w[4];
  out->contacts = w[5]; out->colors = w[6]; out->max_dense = w[7]; out->asleep = w[8];
  out->overflow = (w[4] >= d.MAXP ? 1u : 0u) | (w[1] >= d.MAXC ? 2u : 0u) | (w[3] >= d.MAXU ? 4u : 0u) |
                  (w[7] >= d.MAXDENSE ? 8u : 0u);
  return STEEL_OK;
}

static int write_dev(steel_batch* b, void* dst, const void* src, size_t bytes) {
  CU(cudaSetDevice(b->ctx->device));
  CU(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, b->ctx->stream));
  CU(cudaStreamSynchronize(b->ctx->stream));
  return STEEL_OK;
}

int steel_set_joint_target(steel_batch* b, uint32_t scene, uint32_t dof, float pos, float vel) {
  SceneHost* s = scene_of(b, scene);
  if (!s || dof >= s->d.ND) return fail(STEEL_E_INVALID, "bad scene or dof index");
  int rc = write_dev(b, s->d.art + s->d.A_TGT + dof, &pos, 4);
  if (!rc) rc = write_dev(b, s->d.art + s->d.A_TGTV + dof, &vel, 4);
  if (!rc && !s->d.user_targets) {
    // A user target replaces the scene's recorded trajectory (sim.js:720): driven = 0 from now on.
    s->d.user_targets = 1u;
    SceneDev* dd = b->bd.scenes + scene;
    rc = write_dev(b, &dd->user_targets, &s->d.user_targets, 4);
  }
  return rc;
}
int steel_set_joint_force(steel_batch* b, uint32_t scene, uint32_t dof, float value) {
  SceneHost* s = scene_of(b, scene);
  if (!s || dof >= s->d.ND) return fail(STEEL_E_INVALID, "bad scene or dof index");
  return write_dev(b, s->d.art + s->d.A_JF + dof, &value, 4);
}
int steel_set_body_wrench(steel_batch* b, uint32_t scene, uint32_t body, const float force[3], const float torque[3]) {
  SceneHost* s = scene_of(b, scene);
  if (!s || body >= s->d.NB) return fail(STEEL_E_INVALID, "bad scene or body index");
  float w[8] = {force[0], force[1], force[2], 0.0f, torque[0], torque[1], torque[2], 0.0f};
  return write_dev(b, s->d.art + s->d.A_BF + body * 8u, w, 32);
}
int steel_set_body_pose(steel_batch* b, uint32_t scene, uint32_t body, const float com[3], const float quat[4]) {
  SceneHost* s = scene_of(b, scene);
  if (!s || body >= s->d.NB) return fail(STEEL_E_INVALID, "bad scene or body index");
  float4 p = make_float4(com[0], com[1], com[2], 0.0f), q = make_float4(quat[0], quat[1], quat[2], quat[3]);
  int rc = write_dev(b, s->d.pos + body, &p, 16);
  return rc ? rc : write_dev(b, s->d.rot + body, &q, 16);
}
int steel_set_body_twist(steel_batch* b, uint32_t scene, uint32_t body, const float twist[6]) {
  SceneHost* s = scene_of(b, scene);
  if (!s || body >= s->d.NB) return fail(STEEL_E_INVALID, "bad scene or body index");
  float4 v = make_float4(twist[0], twist[1], twist[2], 0.0f), w = make_float4(twist[3], twist[4], twist[5], 0.0f);
  int rc = write_dev(b, s->d.lv + body, &v, 16);
  return rc ? rc : write_dev(b, s->d.av + body, &w, 16);
}

int steel_collide(steel_batch* b) {
  if (!b) return fail(STEEL_E_INVALID, "null batch");
  CU(cudaSetDevice(b->ctx->device));
  cudaStream_t st = b->ctx->stream;
  for (auto& s : b->sc) CU(cudaMemsetAsync(s.d.counters, 0, 8, st));
  launch_params(b->bd, 0, st);
  launch_shapes(b->bd, st);
  launch_broad(b->bd, st);
  launch_narrow(b->bd, b->narrow_blocks, st);
  launch_csort(b->bd, b->sort_keys, b->radix.data(), (uint32_t)b->radix.size(), st);
  CU(cudaGetLastError());
  int rc = steel_sync(b);
  if (rc) return rc;
  // Keep the counts for the readers and leave the counters as a finished substep leaves them.
  for (auto& s : b->sc) {
    uint32_t c[2];
    CU(cudaMemcpy(c, s.d.counters, 8, cudaMemcpyDeviceToHost));
    s.collide_pairs = c[0];
    s.collide_contacts = c[1];
    CU(cudaMemset(s.d.counters, 0, 8));
  }
  return STEEL_OK;
}

int steel_debug_stage(steel_batch* b, int stage) {
  if (!b) return fail(STEEL_E_INVALID, "null batch");
  CU(cudaSetDevice(b->ctx->device));
  cudaStream_t st = b->ctx->stream;
  if (stage == 0) {
    launch_params(b->bd, b->debug_substep, st);
    launch_shapes(b->bd, st);
    launch_broad(b->bd, st);
    launch_narrow(b->bd, b->narrow_blocks, st);
    launch_csort(b->bd, b->sort_keys, b->radix.data(), (uint32_t)b->radix.size(), st);
  } else if (stage == 1) {
    launch_prepare(b->bd, st);
  } else if (stage == 2) {
    launch_solve(b->bd, st);
    if (++b->debug_substep == b->substeps) { launch_frame_end(b->bd, st); b->debug_substep = 0; }
  } else {
    return fail(STEEL_E_INVALID, "bad stage");
  }
  CU(cudaGetLastError());
  return steel_sync(b);
}

int steel_read_words(steel_batch* b, uint32_t scene, const char* buffer, uint64_t offset, uint64_t count, void* out) {
  SceneHost* s = scene_of(b, scene);
  if (!s || !buffer || !out) return fail(STEEL_E_INVALID, "bad scene index or null argument");
  const SceneDev& d = s->d;
  std::string n(buffer);
  const void* base = nullptr;
  uint64_t words = 0;
  if (n == "art") { base = d.art; words = s->art_floats; }
  else if (n == "rows") { base = d.rows; words = (uint64_t)d.MAXC * d.ROWS * 4; }
  else if (n == "sched") { base = d.sched; words = s->sched_words; }
  else if (n == "slots") { base = d.slots; words = (uint64_t)d.MAXC * 8; }
  else if (n == "warm") { base = d.warm_tab; words = s->warm_words; }
  else if (n == "contacts") { base = d.con; words = (uint64_t)d.MAXC * 24; }
  else return fail(STEEL_E_INVALID, "unknown buffer " + n);
  if (offset + count > words) return fail(STEEL_E_INVALID, "read past the end of " + n);
  CU(cudaSetDevice(b->ctx->device));
  CU(cudaMemcpy(out, (const uint32_t*)base + offset, count * 4, cudaMemcpyDeviceToHost));
  return STEEL_OK;
}

int steel_layout_get(steel_batch* b, uint32_t scene, const char* key, uint64_t* value) {
  SceneHost* s = scene_of(b, scene);
  if (!s || !key || !value) return fail(STEEL_E_INVALID, "bad scene index or null argument");
  const SceneDev& d = s->d;
#define L1(k) if (!std::strcmp(key, #k)) { *value = d.k; return STEEL_OK; }
  L1(A_Q) L1(A_QD) L1(A_QDH) L1(A_INT) L1(A_TGT) L1(A_TGTV) L1(A_LIM) L1(A_DRV) L1(A_JF) L1(A_BF) L1(A_FRIC)
  L1(A_HINV) L1(A_LINK) L1(A_VLG) L1(A_LG) L1(A_RL) L1(A_RLN) L1(A_ULOAD) L1(A_DENSE) L1(A_SLP) L1(A_AVL) L1(ROWS) L1(PO)
  L1(S_UKEY) L1(S_USIZE) L1(S_USTART) L1(S_RUNIT) L1(S_RCON) L1(S_PCOL) L1(S_PORD) L1(S_CSTART) L1(S_META)
  L1(S_KEEP) L1(S_CORDER) L1(S_KEPT)
#undef L1
  return fail(STEEL_E_INVALID, std::string("unknown layout key ") + key);
}

int steel_read_pairs(steel_batch* b, uint32_t scene, uint32_t* pairs, uint32_t cap, uint32_t* count) {
  SceneHost* s = scene_of(b, scene);
  if (!s || !count) return fail(STEEL_E_INVALID, "bad scene index or null output");
  CU(cudaSetDevice(b->ctx->device));
  uint32_t total = 0;
  CU(cudaMemcpy(&total, b->bd.pair_count, 4, cudaMemcpyDeviceToHost));
  std::vector<uint4> all(total);
  if (total) CU(cudaMemcpy(all.data(), b->bd.pairs, 16ull * total, cudaMemcpyDeviceToHost));
  uint32_t n = 0;
  for (auto& p : all) {
    if (p.x != scene) continue;
    if (pairs && n < cap) { pairs[2 * n] = p.y; pairs[2 * n + 1] = p.z; }
    n++;
  }
  *count = n;
  return STEEL_OK;
}


// --- Serving loop -----------------------------------------------------------------------------
// Continuous batching over the batch's scenes as resident instances. Requests (instance, frames)
// queue per instance; up to max_active instances are admitted at a time (FIFO), each tick steps
// every admitted instance by one frame (the other scenes' blocks return at once), and an instance
// whose request is done takes its next queued request or leaves the admitted set, which admits the
// next waiting instance. Scenes are independent, so an instance's result does not depend on what
// else is admitted.
static double now_ms() {
  using namespace std::chrono;
  return duration<double, std::milli>(steady_clock::now().time_since_epoch()).count();
}
static int serve_begin(steel_batch* b) {
  if (b->serve_on) return STEEL_OK;
  const uint32_t n = (uint32_t)b->sc.size();
  b->serve_queue.assign(n, {});
  b->serve_state.assign(n, 0);
  b->serve_mask.assign(n, 0u);
  b->serve_waiting.clear();
  b->serve_done.clear();
  b->serve_admitted = 0;
  b->serve_bytes = 0;
  if (b->serve_max_active == 0 || b->serve_max_active > n) b->serve_max_active = n;
  CU(cudaSetDevice(b->ctx->device));
  CU(cudaMemcpyAsync(b->arena + b->o_active, b->serve_mask.data(), 4ull * n, cudaMemcpyHostToDevice, b->ctx->stream));
  b->serve_on = true;
  b->serve_dirty = true;
  return STEEL_OK;
}

// The per-scene kernels launch one block per admitted instance: the admitted instances, in the
// batch's longest-first order, go to the front of the launch order.
static int serve_upload_order(steel_batch* b) {
  std::vector<uint32_t> order;
  order.reserve(b->serve_admitted);
  for (uint32_t i : b->order_host)
    if (b->serve_state[i] == 2) order.push_back(i);
  cudaStream_t st = b->ctx->stream;
  CU(cudaMemcpyAsync(b->arena + b->o_active, b->serve_mask.data(), 4ull * b->sc.size(), cudaMemcpyHostToDevice, st));
  if (!order.empty()) CU(cudaMemcpyAsync(b->arena + b->o_order, order.data(), 4ull * order.size(), cudaMemcpyHostToDevice, st));
  // The host copy must outlive the copy: wait for it (the tick synchronizes anyway).
  CU(cudaStreamSynchronize(st));
  b->bd.nlaunch = (uint32_t)order.size();
  b->serve_dirty = false;
  return STEEL_OK;
}

int steel_serve_config(steel_batch* b, uint32_t max_active) {
  if (!b) return fail(STEEL_E_INVALID, "null batch");
  b->serve_max_active = max_active;
  return STEEL_OK;
}

int steel_serve_budget(steel_batch* b, uint64_t bytes) {
  if (!b) return fail(STEEL_E_INVALID, "null batch");
  b->serve_budget = bytes;
  return STEEL_OK;
}

int steel_scene_bytes(steel_batch* b, uint32_t scene, uint64_t* bytes) {
  SceneHost* s = scene_of(b, scene);
  if (!s || !bytes) return fail(STEEL_E_INVALID, "bad scene index or null output");
  *bytes = s->arena_bytes;
  return STEEL_OK;
}

int steel_serve_submit(steel_batch* b, uint32_t instance, uint32_t frames, uint64_t* id) {
  if (!b || !id) return fail(STEEL_E_INVALID, "null argument");
  if (instance >= b->sc.size()) return fail(STEEL_E_INVALID, "bad instance index");
  if (frames == 0) return fail(STEEL_E_INVALID, "a request needs at least one frame");
  if (int rc = serve_begin(b)) return rc;
  *id = b->serve_next_id++;
  b->serve_queue[instance].push_back({*id, frames, frames, now_ms()});
  if (b->serve_state[instance] == 0) {
    b->serve_state[instance] = 1;
    b->serve_waiting.push_back(instance);
  }
  return STEEL_OK;
}

int steel_serve_tick(steel_batch* b, uint32_t* stepped) {
  if (!b) return fail(STEEL_E_INVALID, "null batch");
  if (int rc = serve_begin(b)) return rc;
  CU(cudaSetDevice(b->ctx->device));
  cudaStream_t st = b->ctx->stream;
  // Admission, first come first served, within max_active instances and the byte budget of their
  // state (the head of the queue is always admitted when nothing is).
  while (b->serve_admitted < b->serve_max_active && !b->serve_waiting.empty()) {
    uint32_t i = b->serve_waiting.front();
    const uint64_t bytes = b->sc[i].arena_bytes;
    if (b->serve_budget && b->serve_admitted > 0 && b->serve_bytes + bytes > b->serve_budget) break;
    b->serve_waiting.pop_front();
    b->serve_state[i] = 2;
    b->serve_mask[i] = 1u;
    b->serve_admitted++;
    b->serve_bytes += bytes;
    b->serve_dirty = true;
  }
  if (stepped) *stepped = b->serve_admitted;
  if (b->serve_admitted == 0) return STEEL_OK;
  if (b->serve_dirty)
    if (int rc = serve_upload_order(b)) return rc;
  if (int rc = steel_step(b, 1)) return rc;
  CU(cudaStreamSynchronize(st));
  const double t = now_ms();
  for (uint32_t i = 0; i < (uint32_t)b->sc.size(); i++) {
    if (b->serve_state[i] != 2) continue;
    auto& q = b->serve_queue[i];
    steel_batch::Req& r = q.front();
    if (--r.frames_left > 0) continue;
    b->serve_done.push_back({r.id, i, r.frames, t - r.t_submit});
    q.pop_front();
    if (q.empty()) {
      b->serve_state[i] = 0;
      b->serve_mask[i] = 0u;
      b->serve_admitted--;
      b->serve_bytes -= b->sc[i].arena_bytes;
      b->serve_dirty = true;
    }
  }
  return check_device_error(b);
}

int steel_serve_poll(steel_batch* b, uint64_t* ids, uint32_t* instances, double* latency_ms, uint32_t cap,
                     uint32_t* count) {
  if (!b || !count) return fail(STEEL_E_INVALID, "null argument");
  uint32_t n = (uint32_t)std::min<size_t>(cap, b->serve_done.size());
  for (uint32_t k = 0; k < n; k++) {
    if (ids) ids[k] = b->serve_done[k].id;
    if (instances) instances[k] = b->serve_done[k].instance;
    if (latency_ms) latency_ms[k] = b->serve_done[k].latency_ms;
  }
  b->serve_done.erase(b->serve_done.begin(), b->serve_done.begin() + n);
  *count = n;
  return STEEL_OK;
}

int steel_serve_end(steel_batch* b) {
  if (!b) return fail(STEEL_E_INVALID, "null batch");
  if (!b->serve_on) return STEEL_OK;
  CU(cudaSetDevice(b->ctx->device));
  cudaStream_t st = b->ctx->stream;
  CU(cudaMemsetAsync(b->arena + b->o_active, 1, 4ull * b->sc.size(), st));
  CU(cudaMemcpyAsync(b->arena + b->o_order, b->order_host.data(), 4ull * b->order_host.size(), cudaMemcpyHostToDevice, st));
  CU(cudaStreamSynchronize(st));
  b->bd.nlaunch = (uint32_t)b->sc.size();
  b->serve_on = false;
  return STEEL_OK;
}

int steel_read_contacts(steel_batch* b, uint32_t scene, float* records, uint32_t cap, uint32_t* count) {
  SceneHost* s = scene_of(b, scene);
  if (!s || !count) return fail(STEEL_E_INVALID, "bad scene index or null output");
  CU(cudaSetDevice(b->ctx->device));
  const SceneDev& d = s->d;
  uint32_t nc = std::min(s->collide_contacts, d.MAXC);
  *count = nc;
  if (!records) return STEEL_OK;
  uint32_t n = std::min(nc, cap);
  if (n) {
    CU(cudaMemcpy(records, d.con, 80ull * n, cudaMemcpyDeviceToHost));
    CU(cudaMemcpy(records + 20ull * n, d.con + (size_t)d.MAXC * 5, 16ull * n, cudaMemcpyDeviceToHost));
  }
  return STEEL_OK;
}

}  // extern "C"
