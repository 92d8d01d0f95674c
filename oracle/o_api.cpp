// Test infrastructure (oracle): setup, the host step driver and a C API for the Python test harness.
// Restates Sim.reset (sim.js:613-623), writeParams (sim.js:625-639) and step/encodeFrame (sim.js:681-701).
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <sstream>

#include "o_cone5.h"
#include "oracle.h"
#include "smath_o.h"

namespace orc {

static bool parse_consts(const char* text, std::map<std::string, double>& kv) {
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

// The buffer boundary: binary32 words in and out. The float instance copies them; the all-FP64
// instance (o_f64.h) converts each word to and from double.
static void f32_in(float* dst, const f32_t* src, size_t n) {
#ifndef ORC_F64
  std::memcpy(dst, src, n * 4);
#else
  for (size_t i = 0; i < n; i++) dst[i] = (double)src[i];
#endif
}
static void f32_out(f32_t* dst, const float* src, size_t n) {
#ifndef ORC_F64
  std::memcpy(dst, src, n * 4);
#else
  for (size_t i = 0; i < n; i++) dst[i] = (f32_t)src[i];
#endif
}

bool Oracle::init(const char* constants, const f32_t* statF_, size_t nF, const uint32_t* statU_, size_t nU,
                  const f32_t* body_pose, const f32_t* body_vel, const f32_t* art_init, size_t nArt) {
  std::map<std::string, double> kv;
  if (!parse_consts(constants, kv)) { error = "bad constants text"; return false; }
  auto get = [&](const char* k, double def) { auto it = kv.find(k); return it == kv.end() ? def : it->second; };
#define X(n) C.n = (uint32_t)get(#n, 0);
  ORC_U32_CONSTS(X)
#undef X
#define X(n) C.n = (float)get(#n, 0);
  ORC_F32_CONSTS(X)
#undef X
  C.fps = get("PARAM_fps", 60);
  C.substeps = (uint32_t)get("PARAM_substeps", 4);
  C.iterations = (uint32_t)get("PARAM_iterations", 12);
  C.baumgarte = get("PARAM_baumgarte", 0.2);
  C.gravity[0] = get("PARAM_gravity0", 0); C.gravity[1] = get("PARAM_gravity1", 0); C.gravity[2] = get("PARAM_gravity2", -9.81);
  C.warm = get("PARAM_warm", 0);
  C.target_frames = (uint32_t)get("PARAM_target_frames", 0);
  C.driven = (uint32_t)get("PARAM_driven", 0);
  C.integral_count = (uint32_t)get("PARAM_integral_count", 0);
  C.reg = get("PARAM_reg", 0);
  // The oracle restates every solver option of the path.
  if (nF != (size_t)C.LEN_STATF4 * 4u || nU != C.LEN_STATU || nArt != C.LEN_ART) { error = "buffer size mismatch"; return false; }
  statF.resize(C.LEN_STATF4);
  f32_in(&statF.data()->x, statF_, nF);
  statU.assign(statU_, statU_ + nU);
  init_poses.assign(C.NB * 4u + C.NS * 4u, mk4(0, 0, 0, 0));
  f32_in(&init_poses.data()->x, body_pose, C.NB * 8u);
  init_vel.assign(C.NB * 2u, mk4(0, 0, 0, 0));
  f32_in(&init_vel.data()->x, body_vel, C.NB * 8u);
  init_art.assign(nArt, 0.0f);
  f32_in(init_art.data(), art_init, nArt);
  pairs.assign(C.MAXP * 2u, 0u);
  contacts.assign(C.MAXC * 6u, mk4(0, 0, 0, 0));
  craw.assign(C.MAXC * 6u, mk4(0, 0, 0, 0));
  sched.assign(C.LEN_SCHED, 0u);
  rows.assign(C.MAXC * (C.ROWS + 2u), mk4(0, 0, 0, 0));
  warm.assign(10u * C.WH + 30u * C.AH, 0u);
  scratch.assign(C.MAXC, u4{0, 0, 0, 0});
  wkey.assign(C.MAXU, 0u);
  wcol.assign(C.MAXU, 0u);
  wmask.assign(C.NBP * C.NCOLW, 0u);
  wcount.assign(C.NCOL + 2u, 0u);
  wlinkhit.assign(C.NBP, 0u);
  wjsplit.assign(C.NL > 0 ? C.NL : 1u, 0u);
  tw.assign(C.NBP * 2u, mk4(0, 0, 0, 0));
  imp.assign(C.NBP * 2u, mk4(0, 0, 0, 0));
  aqd.assign(C.ND > 0 ? C.ND : 1u, 0.0f);
  wcs.assign(C.NCOL + 2u, 0u);
  reset();
  return true;
}

void Oracle::reset() {
  poses = init_poses;
  std::fill(poses.begin() + C.NB * 2u, poses.end(), mk4(0, 0, 0, 0));
  vel = init_vel;
  art = init_art;
  std::fill(warm.begin(), warm.end(), 0u);
  std::memset(counters, 0, sizeof(counters));
  std::memset(stats, 0, sizeof(stats));
  phase = 0.0; time = 0.0; frame = 0; substep_count = 0;
}

void Oracle::write_params(uint32_t substep) {
  double dt = 1.0 / C.fps / C.substeps;
  P = Params{};
  P.dt = (float)dt;
  P.substep = substep;
  P.parity = (uint32_t)(substep_count % 2u);
  P.iterations = C.iterations;
  P.phase = (float)phase;
  P.frame_dt = (float)(1.0 / C.fps);
  P.beta = (float)C.baumgarte;
  P.max_depen = 2.0f;
  P.gravity = mk4((float)C.gravity[0], (float)C.gravity[1], (float)C.gravity[2], 0.0f);
  P.warm_scale = (float)C.warm;
  P.path_frames = C.target_frames;
  P.driven = user_targets ? 0u : C.driven;
  P.integral_count = C.integral_count;
  P.reg = (float)C.reg;
}

void Oracle::substep_kernels() {
  k_shapes();
  k_broad();
  k_narrow();
  k_csort();
  k_prepare();
  k_solve();
}

void Oracle::step(uint32_t frames) {
  for (uint32_t f = 0; f < frames; f++) {
    for (uint32_t s = 0; s < C.substeps; s++) {
      write_params(s);
      substep_count++;
      substep_kernels();
    }
    frame++;
    time += 1.0 / C.fps;
    phase += 1.0 / C.fps;
  }
}

}  // namespace orc

using orc::Oracle;

extern "C" {

// One visit of the articulated angular friction block (o_cone5.h ell_block5), for the cone tests:
// H 25 floats (row-major 5x5 response), g, mu, lam 5 floats each, the normal load, pyramidal or
// elliptic, creep speed and relaxation; out gets the block's new impulses.
void oracle_cone5(const float* H, const float* g, const float* mu, const float* lam, float load, int pyr, float creep,
                  float omega, float* out) {
  orc::ell_block5(H, g, mu, lam, load, pyr != 0, creep, omega, out);
}


// The oracle's float sin / cos / atan2 (smath_o.h), for accuracy tests.
void oracle_trig(const float* x, float* s, float* c, size_t n) {
  for (size_t i = 0; i < n; i++) { s[i] = orc::sin_o(x[i]); c[i] = orc::cos_o(x[i]); }
}
void oracle_atan2(const float* y, const float* x, float* out, size_t n) {
  for (size_t i = 0; i < n; i++) out[i] = orc::atan2_o(y[i], x[i]);
}

void* oracle_create(const char* constants, const f32_t* statF, size_t nF, const uint32_t* statU, size_t nU,
                    const f32_t* poses, const f32_t* vel, const f32_t* art, size_t nArt, char* err, size_t errlen) {
  Oracle* o = new Oracle();
  if (!o->init(constants, statF, nF, statU, nU, poses, vel, art, nArt)) {
    if (err && errlen) { std::strncpy(err, o->error.c_str(), errlen - 1); err[errlen - 1] = 0; }
    delete o;
    return nullptr;
  }
  return o;
}
void oracle_destroy(void* h) { delete (Oracle*)h; }
void oracle_reset(void* h) { ((Oracle*)h)->reset(); }
void oracle_step(void* h, uint32_t frames) { ((Oracle*)h)->step(frames); }
void oracle_set_user_targets(void* h, int on) { ((Oracle*)h)->user_targets = on != 0; }

// Runs shapes, broad, narrow and csort for the current state (substep 0 parameters) and leaves
// pairs/contacts in place; the state is not advanced. Used for the pair-set and sort parity tests.
void oracle_collide(void* h) {
  Oracle* o = (Oracle*)h;
  o->counters[0] = o->counters[1] = 0u;
  o->write_params(0);
  o->k_shapes();
  o->k_broad();
  o->k_narrow();
  o->k_csort();
  // Keep the counts for the readers and leave the counters as a finished substep leaves them.
  o->collide_counts[0] = o->counters[0];
  o->collide_counts[1] = o->counters[1];
  o->counters[0] = o->counters[1] = 0u;
}
// The canonical contact sort alone over the raw records craw[0, n) as they stand (a test hook: a
// permuted raw buffer must sort to the same records, W:3895-3898).
void oracle_sort_raw(void* h, uint32_t n) {
  Oracle* o = (Oracle*)h;
  o->counters[1] = n;
  o->k_csort();
  o->counters[1] = 0u;
}
// One substep in stages, as step() runs it: stage 0 writes the substep's parameters and runs the
// collision kernels, 1 prepare, 2 solve (ending the frame after the last substep).
void oracle_stage(void* h, int stage) {
  Oracle* o = (Oracle*)h;
  if (stage == 0) {
    o->write_params(o->debug_substep);
    o->substep_count++;
    o->k_shapes(); o->k_broad(); o->k_narrow(); o->k_csort();
  } else if (stage == 1) {
    o->k_prepare();
  } else if (stage == 2) {
    o->k_solve();
    if (++o->debug_substep == o->C.substeps) {
      o->debug_substep = 0;
      o->frame++; o->time += 1.0 / o->C.fps; o->phase += 1.0 / o->C.fps;
    }
  }
}

// Buffer access by name, in 4-byte words (binary32 for the float buffers); returns the words copied.
size_t oracle_read(void* h, const char* name, void* out, size_t max_words) {
  Oracle* o = (Oracle*)h;
  const float* fsrc = nullptr;
  const uint32_t* usrc = nullptr;
  size_t n = 0;
  std::string s(name);
  if (s == "poses") { fsrc = &o->poses.data()->x; n = o->poses.size() * 4; }
  else if (s == "vel") { fsrc = &o->vel.data()->x; n = o->vel.size() * 4; }
  else if (s == "art") { fsrc = o->art.data(); n = o->art.size(); }
  else if (s == "contacts") { fsrc = &o->contacts.data()->x; n = o->contacts.size() * 4; }
  else if (s == "craw") { fsrc = &o->craw.data()->x; n = o->craw.size() * 4; }
  else if (s == "pairs") { usrc = o->pairs.data(); n = o->pairs.size(); }
  else if (s == "sched") { usrc = o->sched.data(); n = o->sched.size(); }
  else if (s == "rows") { fsrc = &o->rows.data()->x; n = o->rows.size() * 4; }
  else if (s == "warm") { usrc = o->warm.data(); n = o->warm.size(); }
  else if (s == "counters") { usrc = o->counters; n = 16; }
  else if (s == "collide_counts") { usrc = o->collide_counts; n = 2; }
  else if (s == "stats") { usrc = o->stats; n = 16; }
  else return 0;
  if (n > max_words) n = max_words;
  if (fsrc) orc::f32_out((f32_t*)out, fsrc, n);
  else std::memcpy(out, usrc, n * 4);
  return n;
}
// Write words into a named state buffer at a word offset (the Sim setters, sim.js:716-785).
int oracle_write(void* h, const char* name, size_t offset, const void* data, size_t words) {
  Oracle* o = (Oracle*)h;
  std::string s(name);
  float* dst = nullptr;
  size_t n = 0;
  if (s == "poses") { dst = &o->poses.data()->x; n = o->poses.size() * 4; }
  else if (s == "vel") { dst = &o->vel.data()->x; n = o->vel.size() * 4; }
  else if (s == "art") { dst = o->art.data(); n = o->art.size(); }
  else if (s == "craw") { dst = &o->craw.data()->x; n = o->craw.size() * 4; }
  else return -1;
  if (offset + words > n) return -1;
  orc::f32_in(dst + offset, (const f32_t*)data, words);
  return 0;
}
}
