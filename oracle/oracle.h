// Test infrastructure: the CPU oracle of steel-webgpu's Sim.step hot path.
//
// ORACLE ONLY: used by tests/, __graft_entry__.smoke() and bench.py's CPU
// baseline as the checker. The product never includes, links or runs it.
//
// A sequential restatement, in operation order, of the reference's WGSL
// kernels (packages/steel-webgpu/src/wgsl.js, artwgsl.js) over the reference's
// own buffer layout (statF/statU/poses/vel/counters/pairs/contacts/sched/rows/
// warm/art/stats, sim.js:503-519) and its compile-time constants C
// (sim.js:456-477). Each workgroup phase becomes a loop over its invocations in
// index order; barriers become phase boundaries. Subgroup min/max reductions are
// lane-major scans (the lowest lane wins ties, as the reference's no-subgroup
// fallback does); the subgroup sums of the dense-row solve (SG = 1) are
// per-lane partial sums in dof order combined by a fixed xor butterfly.
//
// Parity unpinned: the reference ships no golden vectors or known-answer tests for
// this path and cannot run here (WGSL needs a WebGPU adapter and a JS runtime), so
// this restatement is checked by construction, by physical known answers and by its
// own committed fixtures (tests/golden), not against the reference's outputs.
#pragma once
#include <cstdint>
#include <map>
#include <string>
#include <vector>

#include "omath.h"

namespace orc {

// u32 constants of C (sim.js:456-477) the oracle reads.
#define ORC_U32_CONSTS(X)                                                                                 \
  X(TGT_HELD) X(NEST) X(MO) X(NB) X(NBP) X(NCOLW) X(NCOL) X(NS) X(NA) X(NL) X(ND) X(NLOOP) X(NMIMIC)    \
  X(CTRL_KIND) X(CTRL_A) X(CTRL_B) X(NDA) X(JDIM) X(MAXDENSE) X(DHDR) X(DPS) X(MAXP) X(MAXC) X(MAXU) X(UH) \
  X(WH) X(ROWS) X(PO) X(FMO) X(FMODE) X(PATCH) X(EXTRA) X(SHARED) X(FSHARED) X(REST) X(CTI) X(SLEEP)      \
  X(DRIVE_ROWS) X(VEL_DRIVE_ACTIVE) X(FUSE_VLIM) X(VLIM_ON) X(FSTART) X(VELITERS) X(AH) X(ANG) X(ANG_ART)  \
  X(JFL) X(TORS) X(TO) X(EO) X(PYRAMID) X(CO) X(COMPL) X(LONGEST_FIRST) X(VLIM_FREE) X(FRICTION_COMBINE)             \
  X(RESTITUTION_COMBINE) X(JM) X(MAXPATH) X(MAXLP) X(ART_F64)                                                        \
  X(SF_BODY) X(SF_SHAPE) X(SF_HAABB) X(SF_VERTS) X(SF_FPLANE) X(SF_LINK) X(SF_DOF) X(SF_PATH) X(SF_LOOP)  \
  X(SF_MIMIC) X(SF_CTRL) X(SU_HULL) X(SU_FACE) X(SU_FV) X(SU_HEDGE) X(SU_EDGE) X(SU_ART) X(SU_ACON)        \
  X(SU_FILTER) X(P_BODY) X(P_SHAPE) X(P_AABB) X(P_PREV)                                                   \
  X(S_HKEY) X(S_HCNT) X(S_SLOT2U) X(S_CSLOT) X(S_CLOCAL) X(S_USIZE_TMP) X(S_UKEY) X(S_USIZE) X(S_USTART)  \
  X(S_CSTART) X(S_META) X(S_CORDER) X(S_RK0) X(S_RK1) X(S_RK2) X(S_KEPT) X(S_OSTART) X(S_LEAD) X(S_SLOT)  \
  X(S_ROWOF) X(S_RUNIT) X(S_PCOL) X(S_PORD) X(S_UTC) X(S_UTP) X(S_UF) X(S_UFF) X(S_RCON) X(S_WWIN)        \
  X(S_UWOFF) X(S_WALK) X(S_WSLOT)                                                                         \
  X(A_Q) X(A_QD) X(A_QDH) X(A_INT) X(A_TGT) X(A_TGTV) X(A_LIM) X(A_DRV) X(A_JFL) X(A_JF) X(A_BF) X(A_SLP)  \
  X(A_FRIC) X(A_HINV) X(A_LINK) X(A_SNAP) X(A_VLG) X(A_AVL) X(A_LG) X(A_RL) X(A_RLN) X(A_ULOAD) X(A_DENSE) \
  X(LEN_STATF4) X(LEN_STATU) X(LEN_SCHED) X(LEN_ART)

#define ORC_F32_CONSTS(X)                                                                                 \
  X(F_ANCHOR_BETA) X(F_CFM) X(F_OMEGA) X(F_SPEC) X(F_GAP_GATE) X(F_FGAP) X(F_FSCALE) X(F_REST_SPEED)      \
  X(F_FR_MUT) X(F_FR_MUR) X(F_BP_CELL) X(F_VLIM_FRAC) X(F_JL_GAP) X(F_JL_SPEED) X(F_SLEEP_LIN) X(F_SLEEP_ANG) \
  X(F_SLEEP_TIME) X(F_CREEP)

struct Consts {
#define X(n) uint32_t n = 0;
  ORC_U32_CONSTS(X)
#undef X
#define X(n) float n = 0.0f;
  ORC_F32_CONSTS(X)
#undef X
  // writeParams inputs (sim.js:625-639)
  double fps = 60, baumgarte = 0.2, warm = 0, reg = 0;
  double gravity[3] = {0, 0, -9.81};
  uint32_t substeps = 4, iterations = 12, target_frames = 0, driven = 0, integral_count = 0;
};

// The Params uniform (wgsl.js:34-45).
struct Params {
  float dt; uint32_t substep, parity, iterations;
  float phase, frame_dt, beta, max_depen;
  v4 gravity;
  float pad0, warm_scale; uint32_t path_frames, driven;
  uint32_t integral_count; float reg; uint32_t pad1, pad2;
  v4 pick_local, pick_target;
};

struct FaceQ { float sep; uint32_t face; };
struct EdgeQ { float sep; v3 axis, a0, a1, b0, b1; uint32_t id; };
struct SegQ { float d2; v3 ps, ph; uint32_t face, kind; };
struct Geo { uint32_t t; v3 s; uint32_t h; };
struct SV { v3 a, l; };

struct Oracle {
  Consts C;
  Params P{};
  std::vector<v4> statF;
  std::vector<uint32_t> statU;
  std::vector<v4> poses, vel;
  uint32_t counters[16] = {0};
  std::vector<uint32_t> pairs;        // 2 per pair
  std::vector<v4> contacts, craw;     // MAXC*5 records + MAXC shape-mu entries
  std::vector<uint32_t> sched;
  std::vector<v4> rows;
  std::vector<uint32_t> warm;
  std::vector<float> art;
  uint32_t stats[16] = {0};
  std::vector<u4> scratch;
  // initial state for reset()
  std::vector<v4> init_poses, init_vel;
  std::vector<float> init_art;
  // host clock (sim.js:621, 674-678)
  double phase = 0.0, time = 0.0;
  uint64_t frame = 0, substep_count = 0;
  bool user_targets = false;
  uint32_t debug_substep = 0;
  uint32_t collide_counts[2] = {0, 0};  // counts of the last oracle_collide
  std::string error;

  // --- setup / driver ---
  bool init(const char* constants, const f32_t* statF_, size_t nF, const uint32_t* statU_, size_t nU,
            const f32_t* body_pose, const f32_t* body_vel, const f32_t* art_init, size_t nArt);
  void reset();
  void write_params(uint32_t substep);
  void step(uint32_t frames);
  void substep_kernels();

  // --- kernels (wgsl.js) ---
  void k_shapes();
  void k_broad();
  void k_narrow();
  void k_csort();
  void k_prepare();
  void k_solve();

  // --- body helpers (wgsl.js:69-105) ---
  float body_inv_mass(int b) const { return statF[C.SF_BODY + (uint32_t)b * 8u].x; }
  uint32_t body_kind(int b) const { return f2u(statF[C.SF_BODY + (uint32_t)b * 8u].y); }
  int body_art(int b) const { return f2i(statF[C.SF_BODY + (uint32_t)b * 8u].z); }
  int body_link(int b) const { return f2i(statF[C.SF_BODY + (uint32_t)b * 8u].w); }
  v3 body_com_local(int b) const { return xyz(statF[C.SF_BODY + (uint32_t)b * 8u + 1u]); }
  bool same_art(int a, int b) const {
    return a >= 0 && b >= 0 && body_kind(a) == 2u && body_kind(b) == 2u && body_art(a) == body_art(b);
  }
  float body_mass(int b) const { return statF[C.SF_BODY + (uint32_t)b * 8u + 1u].w; }
  v4 body_limits(int b) const {
    uint32_t o = C.SF_BODY + (uint32_t)b * 8u;
    return mk4(statF[o + 3].w, statF[o + 4].w, statF[o + 5].w, statF[o + 6].w);
  }
  float depen_cap(int a, int b) const;
  uint32_t body_flags(int b) const { return b < 0 ? 0u : f2u(statF[C.SF_BODY + (uint32_t)b * 8u + 7u].w); }
  float body_radius(int b) const { return b < 0 ? 1e30f : statF[C.SF_BODY + (uint32_t)b * 8u + 2u].w; }
  m3 body_inertia(int b) const;
  m3 body_inv_inertia(int b) const;
  uint32_t AK() const { return 10u * C.WH; }
  uint32_t AV() const { return 10u * C.WH + 2u * C.AH; }

  // --- narrowphase (wgsl.js:185-1214) ---
  v3 hv(uint32_t h, uint32_t i) const { return xyz(statF[C.SF_VERTS + statU[C.SU_HULL + h * 4u] + i]); }
  uint32_t hnv(uint32_t h) const { return statU[C.SU_HULL + h * 4u + 1u]; }
  uint32_t hfo(uint32_t h) const { return statU[C.SU_HULL + h * 4u + 2u]; }
  uint32_t hnf(uint32_t h) const { return statU[C.SU_HULL + h * 4u + 3u]; }
  v4 fplane(uint32_t f) const { return statF[C.SF_FPLANE + f]; }
  uint32_t fstart(uint32_t f) const { return statU[C.SU_FACE + f * 2u]; }
  uint32_t fcount(uint32_t f) const { return statU[C.SU_FACE + f * 2u + 1u]; }
  uint32_t fvert(uint32_t k) const { return statU[C.SU_FV + k]; }
  uint32_t hne(uint32_t h) const { return statU[C.SU_HEDGE + h * 2u + 1u]; }
  u4 hedge(uint32_t h, uint32_t k) const {
    uint32_t o = C.SU_EDGE + (statU[C.SU_HEDGE + h * 2u] + k) * 4u;
    return {statU[o], statU[o + 1], statU[o + 2], statU[o + 3]};
  }
  FaceQ face_query(uint32_t ha, uint32_t hb, v4 rq, v3 t, uint32_t lane) const;
  float support_min(uint32_t h, v3 n) const;
  float support_max(uint32_t h, v3 n) const;
  EdgeQ edge_query(uint32_t ha, uint32_t hb, v4 rq, v3 t, uint32_t lane) const;
  void emit(uint32_t sa, uint32_t sb, v3 p, v3 n, float phi, uint32_t key);
  v3 sup_lane(uint32_t h, v3 d) const;
  v3 sup_md(uint32_t ha, uint32_t hb, v4 rq, v3 t, float r, v3 d) const;
  v4 mpr(uint32_t ha, uint32_t hb, v4 rq, v3 t, float r) const;
  v4 shape_prim(uint32_t s) const { return statF[C.SF_SHAPE + s * 7u + 3u]; }
  void prim_prim(uint32_t sa, uint32_t sb, v3 pa, v4 qa, v3 pb, v4 qb, float thresh);
  void plane_contacts(uint32_t pl, uint32_t os, v3 pp, v4 pq, v3 op, v4 oq, float thresh, bool flip);
  FaceQ face_query_seg(uint32_t h, v3 e0, v3 e1, float r, uint32_t lane) const;
  bool seg_hits_hull(uint32_t h, v3 e0, v3 e1) const;
  SegQ seg_hull_query(uint32_t h, v3 e0, v3 e1, uint32_t lane) const;
  void seg_on_face(uint32_t hs, uint32_t ps, uint32_t h, uint32_t f, v3 e0, v3 e1, float r, v3 wp, v4 wq,
                   float thresh, bool flip);
  uint32_t geo_type(uint32_t s) const { return f2u(statF[C.SF_SHAPE + s * 7u + 6u].x); }
  Geo geo(uint32_t s) const;
  v3 gsup(const Geo& g, v3 d) const;
  v3 fsup(const Geo& g, v3 d, v3 n) const;
  bool plane_supporting(const Geo& g, v3 dir, float d) const;
  void gen_run(uint32_t sa, uint32_t sb, const Geo& ga, const Geo& gb, v3 pa, v4 qa, v4 rq, v3 rt, v3 wa, v3 wb,
               v3 n, float thresh);
  float hull_out(uint32_t h, v3 x) const;
  v3 ray_face(uint32_t h, v3 o, v3 n, v3 s) const;
  void sup_witness(const Geo& ga, const Geo& gb, v4 rq, v3 rt, v3 n, bool refA, v3 out[2]) const;
  void sat_generic(uint32_t sa, uint32_t sb, uint32_t ha, uint32_t hb, v3 pa, v4 qa, v4 rBA, v3 tBA, float thresh,
                   FaceQ fa, FaceQ fb, const EdgeQ& eq);
  void plane_convex(uint32_t sa, uint32_t sb, v3 pa, v4 qa, v3 pb, v4 qb, float thresh);
  void capsule_generic(uint32_t c, uint32_t h, v3 pc, v4 qc, v3 wp, v4 wq, v3 wc, v3 wh, v3 nh, float thresh);
  void mpr_generic(uint32_t sa, uint32_t sb, uint32_t ha, uint32_t hb, v3 pa, v4 qa, v4 rBA, v3 tBA, float thresh,
                   v3 n);
  void narrow_pair(uint32_t pi);
  // gen_emit queues the generic manifold; the kernel runs it after narrow_pair (wgsl.js:941-947, 1063-1070).
  struct GenJob { bool on; uint32_t sa, sb; Geo ga, gb; v3 pa; v4 qa, rq; v3 rt, wa, wb, n; float thresh; } job{};
  void gen_emit(uint32_t sa, uint32_t sb, const Geo& ga, const Geo& gb, v3 pa, v4 qa, v4 rq, v3 rt, v3 wa, v3 wb,
                v3 n, float thresh) {
    job = GenJob{true, sa, sb, ga, gb, pa, qa, rq, rt, wa, wb, n, thresh};
  }

  // --- articulation library (artwgsl.js) ---
  uint32_t link_type(uint32_t l) const { return f2u(statF[C.SF_LINK + l * 6u].x); }
  int link_parent(uint32_t l) const { return f2i(statF[C.SF_LINK + l * 6u].y); }
  uint32_t link_dof(uint32_t l) const { return f2u(statF[C.SF_LINK + l * 6u].z); }
  int link_body(uint32_t l) const { return f2i(statF[C.SF_LINK + l * 6u].w); }
  uint32_t link_ndof(uint32_t l) const { return f2u(statF[C.SF_LINK + l * 6u + 1u].w); }
  uint32_t link_qs(uint32_t l) const { return f2u(statF[C.SF_LINK + l * 6u + 3u].w); }
  v4 dof_drive(uint32_t d) const { return statF[C.SF_DOF + d * 5u]; }
  v4 dof_limit(uint32_t d) const { return statF[C.SF_DOF + d * 5u + 1u]; }
  v4 dof_passive(uint32_t d) const { return statF[C.SF_DOF + d * 5u + 2u]; }
  v3 dof_axis(uint32_t d) const { return xyz(statF[C.SF_DOF + d * 5u + 3u]); }
  bool scalar_dof(uint32_t d) const { return statF[C.SF_DOF + d * 5u + 2u].w > 0.5f; }
  v2 dof_spring(uint32_t d) const { v4 s = statF[C.SF_DOF + d * 5u + 4u]; return mk2(s.x, s.y); }
  bool fused_dof(uint32_t d) const {
    v4 dr = dof_drive(d);
    return C.DRIVE_ROWS == 1u && C.FUSE_VLIM == 1u && (dr.y > 0.0f || dr.z > 0.0f);
  }
  u4 art_info(uint32_t a) const {
    return {statU[C.SU_ART + a * 4u], statU[C.SU_ART + a * 4u + 1u], statU[C.SU_ART + a * 4u + 2u],
            statU[C.SU_ART + a * 4u + 3u]};
  }
  int body_node(int b) const;
  bool node_asleep(int n) const { return C.SLEEP == 1u && n >= 0 && art[C.A_SLP + (uint32_t)n * 4u + 1u] > 0.5f; }
  // pair_asleep (wgsl.js:1732-1736): both sides asleep or static.
  bool pair_asleep(int a, int b) const {
    if (C.SLEEP == 0u) return false;
    int na = body_node(a), nb = body_node(b);
    return (na < 0 || node_asleep(na)) && (nb < 0 || node_asleep(nb));
  }
  uint32_t lo(uint32_t l) const { return C.A_LINK + l * 268u; }
  v3 ld3(uint32_t o) const { return mk3(art[o], art[o + 1], art[o + 2]); }
  void st3(uint32_t o, v3 v) { art[o] = v.x; art[o + 1] = v.y; art[o + 2] = v.z; }
  SV ldsv(uint32_t o) const { return SV{ld3(o), ld3(o + 3u)}; }
  void stsv(uint32_t o, SV s) { st3(o, s.a); st3(o + 3u, s.l); }
  m3 ldm(uint32_t o) const { return mcols(ld3(o), ld3(o + 3u), ld3(o + 6u)); }
  void stm(uint32_t o, const m3& m) { st3(o, m.c[0]); st3(o + 3u, m.c[1]); st3(o + 6u, m.c[2]); }
  SV imul(uint32_t o, SV m) const;
  SV ldS(uint32_t l, uint32_t k) const { return ldsv(lo(l) + 0u + k * 6u); }
  SV ldU(uint32_t l, uint32_t k) const { return ldsv(lo(l) + 36u + k * 6u); }
  float ldDI(uint32_t l, uint32_t r, uint32_t c) const { return art[lo(l) + 72u + r * C.JM + c]; }
  v3 link_r(uint32_t l) const;
  void add_shifted_inertia(uint32_t o, const m3& A, const m3& B, const m3& Cm, v3 r);
  void art_fk(uint32_t a);
  v4 link_rot(uint32_t l) const { return mk4(ld3(lo(l) + 216u), art[lo(l) + 216u + 3u]); }
  void art_factor(uint32_t a);
  void sleep_islands();
  void build_torsion(uint32_t sp);
  template <class T>
  float dof_tau(uint32_t l, uint32_t r, T& Drr) const;
  void art_back_f64(uint32_t l);
  uint32_t link_path(uint32_t l0, uint32_t* path) const;
  float dof_hinv(uint32_t l, uint32_t r) const;
  void link_response(uint32_t l, const uint32_t* split_count);
  void add_gen_jac(uint32_t x, v3 p, float sgn, v3 d0, v3 d1, v3 d2, uint32_t ds, float* J) const;
  void add_gen_ang(uint32_t x, float sgn, v3 d0, v3 d1, uint32_t ds, float* J) const;
  void art_solve_gen(uint32_t a, const float* tau, float* out) const;
  bool art_has_constraint(uint32_t a) const { return statU[C.SU_ACON + a] != 0u; }

  // --- prepare (wgsl.js:1222-2494) ---
  std::vector<uint32_t> wkey, wcol, wmask, wcount, wlinkhit, wjsplit;
  uint32_t first_free_color(int a, int b);
  uint32_t row_count(uint32_t row) const;
  void body_response(int b, v3 f, v3 t, v3 out[2]) const;
  void body_response_unsplit(int b, v3 f, v3 t, v3 out[2]) const;
  bool restitution_fires(float e, float phi, float vn) const;
  void pre_twist(int b, v3 out[2]) const;
  void put_bilateral(uint32_t o, uint32_t art_id, const float* J, uint32_t nb, v3 rhs);
  float row_weight(float phi) const { return (phi > 0.0f || P.reg <= 0.0f) ? 1.0f : 1.0f / (1.0f + P.reg); }
  uint32_t unit_of(uint32_t p, uint32_t nu) const;
  void build_patch(uint32_t sp);
  uint32_t contact_pair(uint32_t c) const {
    v4 m = contacts[c * 5u + 2u];
    return (uint32_t)(f2i(m.x) + 1) | ((uint32_t)(f2i(m.y) + 1) << 16u);
  }
  v2 contact_shape_mu(uint32_t c) const { v4 m = contacts[C.MAXC * 5u + c]; return mk2(m.x, m.y); }

  // --- solve (wgsl.js:2501-3891) ---
  std::vector<v4> tw, imp;
  std::vector<float> aqd;
  uint32_t wn_x = 0, wn_y = 0;
  std::vector<uint32_t> wcs;
  v3 twv(int b) const { return xyz(tw[(uint32_t)b * 2u]); }
  void load_tw(int b, v3 out[2]) const;
  void add_imp(int b, v3 f, v3 t);
  v3 fixed_normal_pair(v2 ut0, v4 g1, float mu, v3 lam) const;
  v3 contact_block(uint32_t mode, float un, v2 ut0, v4 g0, v4 g1, float vtarget0, float mu, v3 lam) const;
  v2 friction_pair_solve(float a0, float c0, float d0, float r0, float r1, float old0, float old1, float radius,
                         float omega) const;
  void solve_slot(uint32_t u, uint32_t mode, uint32_t it);
  void solve_unit(uint32_t us, uint32_t row, int a, int b, uint32_t s0, uint32_t s1, uint32_t mode, uint32_t it);
  void set_link_twist(uint32_t l, SV v);
  void art_twists(uint32_t a);
  void art_apply(uint32_t a);
  bool art_dense(uint32_t a, uint32_t mode, uint32_t it, uint32_t ph);
  void dense_phase(uint32_t mode, uint32_t it, uint32_t ph);
  void art_contact_impulses(uint32_t a);
  void momentum_unit(uint32_t us, uint32_t row, float beta, bool init);
  void momentum_step(uint32_t ncol, uint32_t it);
  float wmom_k = 0.0f, wmom_beta = 0.0f;  // the solve's momentum state (k, beta)
  bool vpass = false;  // velocity pass (wgsl.js:2928): rows without position bias or regularization
  void snap_tw(int b, v3 out[2]) const;
  void art_dof_impulse(uint32_t a, uint32_t l, uint32_t r, float dl);
  void art_propagate(uint32_t a, bool vlim, bool rowsOn);
  void art_dof_rows(uint32_t a, uint32_t l, uint32_t r, uint32_t d, bool vlim, bool rowsOn);
  v3 body_motion(int b, v3 x) const;
  void sweep(uint32_t mode, uint32_t ncol0, uint32_t it, uint32_t ph);
  v4 warm_row_value(uint32_t i, uint32_t nc) const;
  uint32_t warm_row_rank(uint32_t i, uint32_t nc) const;
  uint32_t warm_row_key(uint32_t i, uint32_t nc) const;
  m3 gyro_inverse3(const m3& m) const;
  v3 gyroscopic_velocity(const m3& inertia, v3 u0, float dt) const;
};

}  // namespace orc
