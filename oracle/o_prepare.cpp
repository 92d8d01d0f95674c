// Test infrastructure (oracle): the prepare kernel, wgsl.js:1222-2494 restated.
// One workgroup's phases run as sequential loops in invocation order; atomics become plain updates.
#include <algorithm>
#include <cmath>

#include "oracle.h"
#include "smath_o.h"

namespace orc {

enum : uint32_t { L_V = 147, L_W = 153, L_POS = 213, L_COM = 220, L_W2 = 232 };
static const uint32_t UNIT_HEAD = 1u;
static const uint32_t AVN = 14u;

static const v3 BP_BINS[20] = {
    {-0.57095543f, 0.75026579f, 0.33333337f}, {-0.64404845f, 0.17218052f, 0.74535593f},
    {-0.86918069f, -0.36525859f, 0.33333330f}, {-0.93522697f, -0.11932883f, -0.33333339f},
    {-0.75091368f, 0.57010308f, -0.33333336f}, {0.36427171f, 0.86959472f, -0.33333337f},
    {-0.17291149f, 0.64385240f, -0.74535609f}, {0.47113684f, 0.47167205f, 0.74535599f},
    {0.11826704f, 0.93536185f, 0.33333335f}, {0.17291155f, -0.64385245f, 0.74535603f},
    {0.0f, 0.0f, 1.0f}, {-0.11826707f, -0.93536184f, -0.33333335f},
    {-0.36427169f, -0.86959473f, 0.33333337f}, {0.0f, 0.0f, -1.0f},
    {-0.47113677f, -0.47167196f, -0.74535609f}, {0.93522695f, 0.11932898f, 0.33333339f},
    {0.75091367f, -0.57010306f, 0.33333340f}, {0.57095545f, -0.75026579f, -0.33333334f},
    {0.64404840f, -0.17218051f, -0.74535597f}, {0.86918063f, 0.36525872f, -0.33333332f}};

m3 Oracle::body_inertia(int b) const {
  uint32_t o = C.SF_BODY + (uint32_t)b * 8u;
  return transpose(mcols(xyz(statF[o + 2u]), xyz(statF[o + 3u]), xyz(statF[o + 4u])));
}
m3 Oracle::body_inv_inertia(int b) const {
  uint32_t o = C.SF_BODY + (uint32_t)b * 8u;
  return transpose(mcols(xyz(statF[o + 5u]), xyz(statF[o + 6u]), xyz(statF[o + 7u])));
}
float Oracle::depen_cap(int a, int b) const {
  float m = 1e20f;
  if (a >= 0) { float l = body_limits(a).w; if (l > 0.0f) m = fminf_(m, l); }
  if (b >= 0) { float l = body_limits(b).w; if (l > 0.0f) m = fminf_(m, l); }
  return m;
}

// first_free_color (wgsl.js:1233-1246)
uint32_t Oracle::first_free_color(int a, int b) {
  for (uint32_t w = 0; w < C.NCOLW; w++) {
    uint32_t used = 0u;
    if (a >= 0) used |= wmask[(uint32_t)a * C.NCOLW + w];
    if (b >= 0) used |= wmask[(uint32_t)b * C.NCOLW + w];
    if (used != 0xffffffffu) {
      uint32_t k = (uint32_t)__builtin_ctz(~used);
      if (a >= 0) wmask[(uint32_t)a * C.NCOLW + w] |= 1u << k;
      if (b >= 0) wmask[(uint32_t)b * C.NCOLW + w] |= 1u << k;
      return w * 32u + k;
    }
  }
  return C.NCOL;
}

// body_response / body_response_unsplit (wgsl.js:1299-1328)
void Oracle::body_response(int b, v3 f, v3 t, v3 out[2]) const {
  if (b < 0) { out[0] = splat3(0.0f); out[1] = splat3(0.0f); return; }
  if (body_kind(b) == 1u) {
    v4 q = poses[C.P_BODY + (uint32_t)b * 2u + 1u];
    m3 R = qmat(q);
    out[0] = f * body_inv_mass(b);
    out[1] = mul(R, mul(body_inv_inertia(b), mul(transpose(R), t)));
    return;
  }
  uint32_t wo = lo((uint32_t)body_link(b)) + L_W;
  float x[6] = {f.x, f.y, f.z, t.x, t.y, t.z}, o[6];
  for (uint32_t r = 0; r < 6u; r++) {
    float s = 0.0f;
    for (uint32_t c = 0; c < 6u; c++) s += art[wo + r * 6u + c] * x[c];
    o[r] = s;
  }
  out[0] = mk3(o[0], o[1], o[2]);
  out[1] = mk3(o[3], o[4], o[5]);
}
void Oracle::body_response_unsplit(int b, v3 f, v3 t, v3 out[2]) const {
  if (b < 0 || body_kind(b) != 2u) { body_response(b, f, t, out); return; }
  uint32_t wo = lo((uint32_t)body_link(b)) + L_W2;
  float x[6] = {f.x, f.y, f.z, t.x, t.y, t.z}, o[6];
  for (uint32_t r = 0; r < 6u; r++) {
    float s = 0.0f;
    for (uint32_t c = 0; c < 6u; c++) s += art[wo + r * 6u + c] * x[c];
    o[r] = s;
  }
  out[0] = mk3(o[0], o[1], o[2]);
  out[1] = mk3(o[3], o[4], o[5]);
}
bool Oracle::restitution_fires(float e, float phi, float vn) const {
  if (C.REST == 0u || e <= 0.0f || vn >= -C.F_REST_SPEED) return false;
  return phi <= 1e-6f || phi + P.dt * vn <= 1e-6f;
}
void Oracle::pre_twist(int b, v3 out[2]) const {
  out[0] = splat3(0.0f); out[1] = splat3(0.0f);
  if (b < 0) return;
  if (body_kind(b) == 1u) { out[0] = xyz(vel[(uint32_t)b * 2u]); out[1] = xyz(vel[(uint32_t)b * 2u + 1u]); return; }
  if (body_kind(b) == 2u) {
    uint32_t o = lo((uint32_t)body_link(b)) + L_V;
    out[0] = ld3(o + 3u); out[1] = ld3(o);
  }
}
// put_bilateral (wgsl.js:1351-1369)
void Oracle::put_bilateral(uint32_t o, uint32_t art_id, const float* J, uint32_t nb, v3 rhs) {
  u4 ai = art_info(art_id);
  std::vector<float> tau(C.NDA), y(C.NDA);
  for (uint32_t r = 0; r < nb; r++) {
    for (uint32_t k = 0; k < C.NDA; k++) { tau[k] = k < ai.w ? J[r * C.NDA + k] : 0.0f; y[k] = 0.0f; }
    art_solve_gen(art_id, tau.data(), y.data());
    float kk = 0.0f;
    for (uint32_t k = 0; k < ai.w; k++) {
      art[o + C.DHDR + r * C.NDA + k] = J[r * C.NDA + k];
      art[o + C.DHDR + 3u * C.NDA + r * C.NDA + k] = y[k];
      kk += J[r * C.NDA + k] * y[k];
    }
    art[o + 5u + r] = kk > 1e-12f ? 1.0f / kk : 0.0f;
  }
  art[o] = (float)art_id; art[o + 1u] = 0.0f; art[o + 2u] = 0.0f;
  art[o + 4u] = rhs.x; art[o + 22u] = rhs.y; art[o + 23u] = rhs.z;
  art[o + 9u] = 0.0f; art[o + 10u] = 0.0f; art[o + 11u] = 0.0f;
  art[o + 21u] = (float)nb;
}

// Body-pair contact reduction keys (wgsl.js:1471-1503)
struct BPC { uint32_t k[3]; v2 pos; float gap; uint32_t pk; };
static inline uint32_t fflip(float f) {
  uint32_t i = fbits(f);
  return i ^ (((i >> 31u) != 0u ? 0xffffffffu : 0u) | 0x80000000u);
}
static BPC bp_contact(const Oracle& O, uint32_t c) {
  const auto& C = O.C;
  v4 c0 = O.contacts[c * 5u], c1 = O.contacts[c * 5u + 1u], cm = O.contacts[c * 5u + 2u], c4 = O.contacts[c * 5u + 4u];
  int a = f2i(cm.x), b = f2i(cm.y);
  uint32_t ga = f2u(c4.z), gb = f2u(c4.w);
  v3 ng = gb < ga ? -xyz(c1) : xyz(c1);
  int rb = a >= 0 ? a : b;
  v3 org = splat3(0.0f);
  if (rb >= 0) {
    v4 q = O.poses[C.P_BODY + (uint32_t)rb * 2u + 1u];
    org = xyz(O.poses[C.P_BODY + (uint32_t)rb * 2u]) - qrot(q, O.body_com_local(rb));
  }
  uint32_t bin = 0u;
  float bd = -2.0f;
  for (uint32_t i = 0; i < 20u; i++) { float d = dot(ng, BP_BINS[i]); if (d > bd) { bd = d; bin = i; } }
  v3 fn_ = BP_BINS[bin];
  v3 rv = std::fabs(fn_.y) < 0.9f ? mk3(0.0f, 1.0f, 0.0f) : mk3(1.0f, 0.0f, 0.0f);
  v3 u = normalize(rv - dot(rv, fn_) * fn_);
  v3 v = cross(fn_, u);
  v3 x = xyz(c0) - org;
  v2 pos = mk2(dot(x, u), dot(x, v));
  uint32_t cx = (uint32_t)(f2i(clampf(std::floor(pos.x / C.F_BP_CELL + 0.5f), -31.0f, 31.0f)) + 31);
  uint32_t cy = (uint32_t)(f2i(clampf(std::floor(pos.y / C.F_BP_CELL + 0.5f), -31.0f, 31.0f)) + 31);
  uint32_t qx = (uint32_t)(f2i(clampf(std::floor(pos.x * 2000.0f), -32768.0f, 32767.0f)) + 32768);
  uint32_t qy = (uint32_t)(f2i(clampf(std::floor(pos.y * 2000.0f), -8192.0f, 8191.0f)) + 8192);
  BPC r;
  r.k[0] = std::min(ga, gb); r.k[1] = std::max(ga, gb); r.k[2] = bin | (cx << 5u) | (cy << 11u);
  r.pos = pos; r.gap = c0.w; r.pk = (qx << 15u) | (qy << 1u) | 1u;
  return r;
}
static void bp_value(const BPC& g, uint32_t q, uint32_t out[2]) {
  if (q == 6u) { out[0] = fflip(-g.gap); out[1] = g.pk; return; }
  if (q > 6u && g.gap > 0.0f) { out[0] = 0u; out[1] = 0u; return; }
  float ang = (float)(q > 6u ? q - 7u : q) * 1.0471975511965976f;
  out[0] = fflip(dot(g.pos, mk2(cos_o(ang), sin_o(ang))));
  out[1] = g.pk;
}

// row_count (wgsl.js:1507-1514): the rows a contact point solves (normal, a friction pair unless it
// is a patch member, the angular three), for the longest-first color order.
uint32_t Oracle::row_count(uint32_t row) const {
  const uint32_t o = row * C.ROWS;
  uint32_t n = 1u;
  const bool member = C.EXTRA == 1u && rows[o + C.PO].w == 0.0f;
  if (rows[o + 2u].w > 0.0f && !member) n += 2u;
  if (C.ANG == 1u && (rows[o + 19u].x > 0.0f || rows[o + 19u].y > 0.0f)) n += 3u;
  return std::min(n, 7u);
}
uint32_t Oracle::unit_of(uint32_t p, uint32_t nu) const {
  uint32_t lo_ = 0u, hi = nu;
  for (uint32_t it = 0; it < 32u && hi - lo_ > 1u; it++) {
    uint32_t mid = (lo_ + hi) / 2u;
    if (sched[C.S_USTART + mid] <= p) lo_ = mid; else hi = mid;
  }
  return lo_;
}

static inline uint32_t anchor_hash(uint32_t pair, uint32_t k) { return std::max(hash_u32(pair * 2u + k), 1u); }

// build_torsion (wgsl.js:1526-1557): contact torsion (min_torsional_patch_radius), one spin row
// per articulated unit about the normal of its touching coplanar cluster. The cluster is the
// unit's rows within 0.995 of the deepest row's normal and 2 mm of its plane; its radius is the
// members' largest torsion radius. The header lives in the unit's first row: (Ma lin, mu),
// (Ma ang, 1/K), (Mb lin, spin impulse), (Mb ang, r), (n, member).
void Oracle::build_torsion(uint32_t sp) {
  const uint32_t* sc = sched.data();
  const uint32_t ROWS = C.ROWS, TO = C.TO;
  uint32_t st = sc[C.S_USTART + sp];
  uint32_t n = std::min(sc[C.S_USIZE + sp], C.MAXC - std::min(st, C.MAXC));
  if (n == 0u) return;
  uint32_t pair = sc[C.S_UKEY + sp];
  int a = (int)(pair & 0xffffu) - 1, b = (int)(pair >> 16u) - 1;
  uint32_t L = st * ROWS;
  bool art_u = (a >= 0 && body_kind(a) >= 2u) || (b >= 0 && body_kind(b) >= 2u);
  uint32_t seed = st;
  for (uint32_t i = st; i < st + n; i++)
    if (rows[i * ROWS + 1u].w < rows[seed * ROWS + 1u].w) seed = i;
  v3 ns = xyz(rows[seed * ROWS]), ps = xyz(rows[seed * ROWS + TO + 4u]);
  float r = 0.0f;
  for (uint32_t i = st; i < st + n; i++) {
    uint32_t o = i * ROWS;
    bool member = art_u && rows[o + 6u].w <= 0.0f && dot(xyz(rows[o]), ns) >= 0.995f &&
                  std::fabs(dot(xyz(rows[o + TO + 4u]) - ps, ns)) <= 0.002f;
    if (member) r = fmaxf_(r, rows[o + TO + 3u].w);
    rows[o + TO + 4u].w = member ? 1.0f : 0.0f;
  }
  float mu = rows[seed * ROWS + 2u].w;
  if (r <= 0.0f || mu <= 0.0f) { rows[L + TO] = mk4(0.0f, 0.0f, 0.0f, 0.0f); return; }
  v3 Ma[2], Mb[2];
  body_response(a, splat3(0.0f), -ns, Ma);
  body_response(b, splat3(0.0f), ns, Mb);
  float k = dot(-ns, Ma[1]) + dot(ns, Mb[1]);
  float lead = rows[L + TO + 4u].w;
  rows[L + TO] = mk4(Ma[0], mu);
  rows[L + TO + 1u] = mk4(Ma[1], k > 1e-12f ? 1.0f / (k + C.F_CFM) : 0.0f);
  rows[L + TO + 2u] = mk4(Mb[0], 0.0f);
  rows[L + TO + 3u] = mk4(Mb[1], r);
  rows[L + TO + 4u] = mk4(ns, lead);
}

// build_patch (wgsl.js:1562-1725)
void Oracle::build_patch(uint32_t sp) {
  const uint32_t ROWS = C.ROWS, PO = C.PO;
  uint32_t st = sched[C.S_USTART + sp];
  uint32_t n = std::min(sched[C.S_USIZE + sp], C.MAXC - std::min(st, C.MAXC));
  if (n == 0u) return;
  uint32_t pair = sched[C.S_UKEY + sp];
  int a = (int)(pair & 0xffffu) - 1, b = (int)(pair >> 16u) - 1;
  v3 ca = splat3(0.0f), cb = splat3(0.0f);
  v4 qa = mk4(0, 0, 0, 1);
  if (a >= 0) { ca = xyz(poses[C.P_BODY + (uint32_t)a * 2u]); qa = poses[C.P_BODY + (uint32_t)a * 2u + 1u]; }
  if (b >= 0) cb = xyz(poses[C.P_BODY + (uint32_t)b * 2u]);
  float r = fmaxf_(fminf_(body_radius(a), body_radius(b)), 1e-4f);
  uint32_t seed = st;
  for (uint32_t i = st; i < st + n; i++) if (rows[i * ROWS + 1u].w < rows[seed * ROWS + 1u].w) seed = i;
  v3 ns = xyz(rows[seed * ROWS]);
  uint32_t kept = C.S_KEPT + sched[C.S_OSTART + sp] - st;
  v2 mu_seed = contact_shape_mu(sched[kept + seed]);
  uint32_t first = seed;
  for (uint32_t i = st; i < st + n; i++) {
    uint32_t o = i * ROWS;
    v3 dseed = xyz(rows[o + PO + 2u]) - xyz(rows[seed * ROWS + PO + 2u]);
    v2 mu_i = contact_shape_mu(sched[kept + i]);
    if (dot(xyz(rows[o]), ns) < 0.995f || mu_i.x != mu_seed.x || mu_i.y != mu_seed.y ||
        std::fabs(dot(dseed, ns)) > 0.02f * r || length(dseed) > 2.0f * r)
      continue;
    rows[o + PO].w = 0.0f;
    v3 p = xyz(rows[o + PO + 2u]), pf = xyz(rows[first * ROWS + PO + 2u]);
    if (p.x < pf.x || (p.x == pf.x && (p.y < pf.y || (p.y == pf.y && p.z < pf.z)))) first = i;
  }
  v3 pf = xyz(rows[first * ROWS + PO + 2u]);
  uint32_t second = first;
  float far = (1e-8f * r) * r;
  for (uint32_t i = st; i < st + n; i++) {
    if (rows[i * ROWS + PO].w != 0.0f) continue;
    v3 d = xyz(rows[i * ROWS + PO + 2u]) - pf;
    if (dot(d, d) > far) { far = dot(d, d); second = i; }
  }
  uint32_t na = second != first ? 2u : 1u;
  v3 loc0 = xyz(rows[first * ROWS + PO + 2u]), loc1 = xyz(rows[second * ROWS + PO + 2u]);
  if (na == 2u) {
    v3 t0 = cross(ns, mk3(1.0f, 0.0f, 0.0f));
    if (dot(t0, t0) < 1e-6f) t0 = cross(ns, mk3(0.0f, 1.0f, 0.0f));
    t0 = normalize(t0);
    v3 t1 = normalize(cross(ns, t0));
    float sx = 0, sy = 0, sxx = 0, sxy = 0, syy = 0, cnt = 0;
    v3 cen = splat3(0.0f);
    for (uint32_t i = st; i < st + n; i++) {
      if (rows[i * ROWS + PO].w != 0.0f) continue;
      v3 pc = xyz(rows[i * ROWS + PO + 2u]), d = pc - pf;
      float x = dot(d, t0), y = dot(d, t1);
      sx += x; sy += y; sxx += x * x; sxy += x * y; syy += y * y; cen += pc; cnt += 1.0f;
    }
    float xx = sxx - (sx * sx) / cnt, xy = sxy - (sx * sy) / cnt, yy = syy - (sy * sy) / cnt;
    float spread = std::sqrt((xx - yy) * (xx - yy) + (4.0f * xy) * xy);
    if (spread > 1e-6f * (xx + yy)) {
      float big = 0.5f * ((xx + yy) + spread);
      v2 a2 = mk2(xy, big - xx);
      if (xx >= yy) a2 = mk2(big - yy, xy);
      a2 = normalize(a2);
      v3 ax = a2.x * t0 + a2.y * t1;
      float lo_ = 1e30f, hi = -1e30f;
      for (uint32_t i = st; i < st + n; i++) {
        if (rows[i * ROWS + PO].w != 0.0f) continue;
        float pr = dot(xyz(rows[i * ROWS + PO + 2u]) - pf, ax);
        if (pr < lo_) { lo_ = pr; first = i; }
        if (pr > hi) { hi = pr; second = i; }
      }
      v3 centroid = cen / cnt;
      loc0 = centroid + dot(xyz(rows[first * ROWS + PO + 2u]) - centroid, ax) * ax;
      loc1 = centroid + dot(xyz(rows[second * ROWS + PO + 2u]) - centroid, ax) * ax;
      v3 across = normalize(cross(ns, ax));
      float tol = fmaxf_(1e-5f * r, 0.05f * (hi - lo_));
      v3 e0 = splat3(0.0f), e1 = splat3(0.0f);
      float c0 = 0.0f, c1 = 0.0f;
      for (uint32_t i = st; i < st + n; i++) {
        if (rows[i * ROWS + PO].w != 0.0f) continue;
        v3 pc = xyz(rows[i * ROWS + PO + 2u]);
        float pr = dot(pc - pf, ax);
        if (pr <= lo_ + tol) { e0 += pc; c0 += 1.0f; }
        if (pr >= hi - tol) { e1 += pc; c1 += 1.0f; }
      }
      e0 /= fmaxf_(c0, 1.0f);
      e1 /= fmaxf_(c1, 1.0f);
      loc0 += dot(e0 - centroid, across) * across + dot(e0 - centroid, ns) * ns;
      loc1 += dot(e1 - centroid, across) * across + dot(e1 - centroid, ns) * ns;
    }
  }
  float load = 0.0f;
  for (uint32_t i = st; i < st + n; i++) {
    if (rows[i * ROWS + PO].w != 0.0f) continue;
    load += rows[i * ROWS + 6u].x;
    if (i != first && !(na == 2u && i == second)) {
      v4 r6 = rows[i * ROWS + 6u];
      rows[i * ROWS + 6u] = mk4(r6.x, 0.0f, 0.0f, r6.w);
    }
  }
  uint32_t rbase = AK() + P.parity * C.AH;
  for (uint32_t k = 0; k < na; k++) {
    uint32_t i = k == 1u ? second : first;
    uint32_t o = i * ROWS;
    v3 loc = k == 1u ? loc1 : loc0;
    v3 nn = xyz(rows[o]), t1 = xyz(rows[o + 1u]), t2 = xyz(rows[o + 2u]);
    v3 fra = loc - ca, frb = loc - cb;
    v3 Ma[2][2], Mb[2][2];
    v3 dirs[2] = {t1, t2};
    for (uint32_t q = 0; q < 2u; q++) {
      body_response(a, -dirs[q], -cross(fra, dirs[q]), Ma[q]);
      body_response(b, dirs[q], cross(frb, dirs[q]), Mb[q]);
      rows[o + 11u + q * 4u] = mk4(Ma[q][0], 0.0f);
      rows[o + 12u + q * 4u] = mk4(Ma[q][1], 0.0f);
      rows[o + 13u + q * 4u] = mk4(Mb[q][0], 0.0f);
      rows[o + 14u + q * 4u] = mk4(Mb[q][1], 0.0f);
    }
    float K[4];
    for (uint32_t x = 0; x < 2u; x++)
      for (uint32_t y = 0; y < 2u; y++) {
        v3 d = dirs[x];
        K[x * 2u + y] = ((dot(-d, Ma[y][0]) + dot(-cross(fra, d), Ma[y][1])) + dot(d, Mb[y][0])) +
                        dot(cross(frb, d), Mb[y][1]);
      }
    float ks = fmaxf_(K[0] + K[3], 1e-30f);
    float k00 = K[0] + 1e-6f * ks, k01 = 0.5f * (K[1] + K[2]), k11 = K[3] + 1e-6f * ks;
    float det = k00 * k11 - k01 * k01;
    rows[o + 5u] = mk4(k11 / det, -k01 / det, k00 / det, rows[o + 5u].w);
    rows[o + 2u] = mk4(t2, rows[o + 2u].w / (float)na);
    v3 e = splat3(0.0f), imp_ = splat3(0.0f);
    bool carried = false;
    float best = (4.0f * r) * r;
    for (uint32_t kk = 0; kk < 2u; kk++) {
      uint32_t h = anchor_hash(pair, kk) % C.AH;
      for (uint32_t probe = 0; probe < 32u; probe++) {
        uint32_t key = warm[rbase + h];
        if (key == 0u) break;
        uint32_t vo = AV() + (P.parity * C.AH + h) * AVN;
        if (key == anchor_hash(pair, kk) && warm[vo] == pair && warm[vo + 1u] == kk) {
          v3 ll = mk3(bitsf(warm[vo + 2u]), bitsf(warm[vo + 3u]), bitsf(warm[vo + 4u]));
          v3 el = mk3(bitsf(warm[vo + 5u]), bitsf(warm[vo + 6u]), bitsf(warm[vo + 7u]));
          v3 prev = ca + qrot(qa, ll);
          v3 dl = prev - loc;
          if (dot(dl, dl) <= best && std::fabs(dot(dl, nn)) <= 0.05f * r) {
            v3 ew = qrot(qa, el);
            v3 on = qrot(qa, mk3(bitsf(warm[vo + 11u]), bitsf(warm[vo + 12u]), bitsf(warm[vo + 13u])));
            float cs = dot(on, nn);
            if (cs > 0.0f) {
              v3 ax = cross(on, nn), ce = cross(ax, ew);
              ew += ce + cross(ax, ce) / (1.0f + cs);
            }
            ew -= nn * dot(nn, ew);
            if (dot(ew, ew) <= (0.01f * r) * r) {
              e = ew; best = dot(dl, dl); carried = true;
              imp_ = qrot(qa, mk3(bitsf(warm[vo + 8u]), bitsf(warm[vo + 9u]), bitsf(warm[vo + 10u])));
            }
          }
          break;
        }
        h = (h + 1u) % C.AH;
      }
    }
    if (P.warm_scale > 0.0f) {
      v4 r6 = rows[o + 6u];
      v2 lw = mk2(r6.y, r6.z);
      if (carried) lw = mk2(dot(imp_, t1), dot(imp_, t2)) * P.warm_scale;
      float rad = fmaxf_(rows[o + 2u].w * load, 0.0f);
      if (length(lw) > rad) lw = lw * (rad / length(lw));
      rows[o + 6u] = mk4(r6.x, lw.x, lw.y, r6.w);
    }
    rows[o + PO] = mk4(fra, 2.0f);
    rows[o + PO + 1u] = mk4(frb, (float)k);
    rows[o + PO + 2u] = mk4(e, 0.0f);
    rows[o + PO + 3u] = mk4(qinvrot(qa, fra), bitsf(pair));
  }
}

// sleep_islands (wgsl.js:1371-1457): islands are nodes (free bodies, articulations) joined by
// contacts. The reference's parallel union-find hooks the larger root under the smaller until no
// contact joins two islands, so every node ends pointing at its island's lowest node; a sequential
// union-find that links the larger root under the smaller, then compresses, gives that same
// state. Island flags OR onto the root: 1 supported (touches static geometry, or a fixed-base
// articulation), 2 vetoed (moving, driven, loop or mimic owner; picking is not carried), 4 some
// member younger than the quiet time.
void Oracle::sleep_islands() {
  uint32_t* sc = sched.data();
  const uint32_t NN = C.NB + C.NA;
  uint32_t* uf = sc + C.S_UF;
  uint32_t* uff = sc + C.S_UFF;
  for (uint32_t n = 0; n < NN; n++) { uf[n] = n; uff[n] = 0u; }
  sc[C.S_META + 5u] = 0u;
  const uint32_t nc = std::min(counters[1], C.MAXC);
  for (uint32_t c = 0; c < nc; c++) {
    v4 m = contacts[c * 5u + 2u];
    int na = body_node(f2i(m.x)), nb = body_node(f2i(m.y));
    if ((na < 0 || nb < 0) && std::max(na, nb) >= 0 && contacts[c * 5u].w <= 1e-5f)
      uff[(uint32_t)std::max(na, nb)] |= 1u;
  }
  auto find = [&](uint32_t n) {
    uint32_t r = n;
    for (uint32_t k = 0; k < NN && uf[r] != r; k++) r = uf[r];
    return r;
  };
  for (uint32_t c = 0; c < nc; c++) {
    v4 m = contacts[c * 5u + 2u];
    int na = body_node(f2i(m.x)), nb = body_node(f2i(m.y));
    if (na < 0 || nb < 0) continue;
    uint32_t ra = find((uint32_t)na), rb = find((uint32_t)nb);
    if (ra != rb) uf[std::max(ra, rb)] = std::min(ra, rb);
  }
  for (uint32_t n = 0; n < NN; n++) uf[n] = find(n);
  for (uint32_t n = 0; n < NN; n++) {
    bool moving = false, fixed = false, veto = false;
    if (n < C.NB) {
      if (body_kind((int)n) != 1u) continue;
      if (art[C.A_SLP + n * 4u + 1u] < 0.5f)
        moving = length(xyz(vel[n * 2u])) > C.F_SLEEP_LIN || length(xyz(vel[n * 2u + 1u])) > C.F_SLEEP_ANG;
    } else {
      u4 ai = art_info(n - C.NB);
      fixed = link_type(ai.x) != 4u;
      for (uint32_t k = 0; k < ai.y; k++) {
        SV v = ldsv(lo(ai.x + k) + L_V);
        if (art[C.A_SLP + n * 4u + 1u] < 0.5f && (length(v.l) > C.F_SLEEP_LIN || length(v.a) > C.F_SLEEP_ANG))
          moving = true;
      }
      for (uint32_t d = ai.z; d < ai.z + ai.w; d++) {
        v4 dr = dof_drive(d);
        if (dr.y > 0.0f || dr.z > 0.0f) veto = true;
      }
      if (art_has_constraint(n - C.NB)) veto = true;
    }
    uint32_t f = (fixed ? 1u : 0u) | ((moving || veto) ? 2u : 0u) | (uff[n] & 1u);
    uff[uf[n]] |= f;
  }
  for (uint32_t n = 0; n < NN; n++) {
    if (n < C.NB && body_kind((int)n) != 1u) continue;
    uint32_t r = uf[n], f = uff[r];
    float age = art[C.A_SLP + n * 4u];
    if ((f & 2u) != 0u || (f & 1u) == 0u) age = 0.0f;
    else age = fminf_(age + P.dt, C.F_SLEEP_TIME);
    art[C.A_SLP + n * 4u] = age;
    if (age < C.F_SLEEP_TIME) uff[r] |= 4u;
  }
  for (uint32_t n = 0; n < NN; n++) {
    if (n < C.NB && body_kind((int)n) != 1u) continue;
    bool s = (uff[uf[n]] & 4u) == 0u;
    art[C.A_SLP + n * 4u + 1u] = s ? 1.0f : 0.0f;
    if (s) sc[C.S_META + 5u]++;
  }
}

// The prepare kernel (wgsl.js:1788-2494) on the default flag set.
void Oracle::k_prepare() {
  const uint32_t ROWS = C.ROWS, PO = C.PO, WH = C.WH, NCOL = C.NCOL, MAXC = C.MAXC;
  uint32_t* sc = sched.data();
  // Phase 0: clears, drive targets.
  for (uint32_t i = 0; i < C.UH; i++) { sc[C.S_HKEY + i] = 0u; sc[C.S_HCNT + i] = 0u; }
  uint32_t wbase = (1u - P.parity) * WH;
  for (uint32_t i = 0; i < WH; i++) { warm[wbase + i] = 0u; sc[C.S_WWIN + i] = 0u; }
  if (C.PATCH == 1u) for (uint32_t i = 0; i < C.AH; i++) warm[AK() + (1u - P.parity) * C.AH + i] = 0u;
  std::fill(wlinkhit.begin(), wlinkhit.end(), 0u);
  std::fill(wmask.begin(), wmask.end(), 0u);
  std::fill(wcount.begin(), wcount.end(), 0u);
  sc[C.S_META + 3u] = 0u;
  if (C.SLEEP == 1u) sleep_islands();
  for (uint32_t tid = 0; tid < P.driven; tid++) {
    float ramp = ((P.phase + ((float)P.substep + 0.5f) * P.dt) * 60.0f) - 0.5f;
    float frame = clampf(C.TGT_HELD == 1u ? P.phase * 60.0f : ramp, 0.0f, (float)(P.path_frames - 1u));
    uint32_t a = f2u(frame);
    uint32_t b = std::min(a + 1u, P.path_frames - 1u);
    auto pathv = [&](uint32_t i) { v4 v = statF[C.SF_PATH + i / 4u]; uint32_t k = i % 4u; return k == 0 ? v.x : k == 1 ? v.y : k == 2 ? v.z : v.w; };
    float pa = pathv(a * P.driven + tid), pb = pathv(b * P.driven + tid);
    float value = mixf(pa, pb, frame - (float)a);
    if (tid < P.integral_count) {
      if (P.substep == 0u) {
        float err = clampf(value - art[C.A_Q + tid], -0.08f, 0.08f);
        art[C.A_INT + tid] = clampf(art[C.A_INT + tid] + (3.0f * P.frame_dt) * err, -0.12f, 0.12f);
      }
      value += art[C.A_INT + tid];
    }
    art[C.A_TGT + tid] = value;
  }
  if (C.CTRL_KIND == 1u) {
    v4 c = statF[C.SF_CTRL];
    art[C.A_TGTV + C.CTRL_B] = c.y * clampf(art[C.A_Q + C.CTRL_A] / c.x, 0.0f, 1.0f);
  }
  std::fill(wjsplit.begin(), wjsplit.end(), 0u);
  for (uint32_t tid = 0; tid < C.NA; tid++) {
    u4 ai = art_info(tid);
    // Joint velocity limits (wgsl.js:1829-1854): scale the articulation's scalar dof speeds so the
    // most exceeded limit is met, then mark the dofs near their limit (rows exist only there).
    if (C.VLIM_ON == 1u) {
      auto fused = [&](uint32_t d) {
        v4 dr = dof_drive(d);
        return C.DRIVE_ROWS == 1u && C.FUSE_VLIM == 1u && (dr.y > 0.0f || dr.z > 0.0f);
      };
      float ratio = 1.0f;
      for (uint32_t k = 0; k < ai.w; k++) {
        uint32_t d = ai.z + k;
        float vl = dof_passive(d).z;
        if (vl < 0.0f || fused(d)) continue;
        float sp = std::fabs(art[C.A_QD + d]);
        if (sp > vl) ratio = fminf_(ratio, vl / sp);
      }
      if (ratio < 1.0f)
        for (uint32_t k = 0; k < ai.w; k++) {
          uint32_t d = ai.z + k;
          if (scalar_dof(d) && !fused(d)) art[C.A_QD + d] *= ratio;
        }
      bool any = false;
      for (uint32_t k = 0; k < ai.w; k++) {
        uint32_t d = ai.z + k;
        bool on = std::fabs(art[C.A_QD + d]) >= C.F_VLIM_FRAC * dof_passive(d).z;
        art[C.A_VLG + d] = on ? 1.0f : 0.0f;
        any = any || (on && dof_passive(d).z >= 0.0f && scalar_dof(d));
      }
      art[C.A_AVL + tid] = any ? 1.0f : 0.0f;
    }
    uint32_t n = 0u;
    for (uint32_t k = 0; k < ai.w; k++) {
      uint32_t d = ai.z + k;
      v4 lim = dof_limit(d);
      bool on = false;
      if (lim.z > 0.5f) {
        uint32_t l = f2u(lim.w);
        float q = art[C.A_Q + link_qs(l) + d - link_dof(l)];
        float g = C.F_JL_GAP + (C.F_JL_SPEED * P.dt) * std::fabs(art[C.A_QD + d]);
        on = q <= lim.x + g || q >= lim.y - g;
      }
      art[C.A_LG + d] = on ? 1.0f : 0.0f;
      v4 dr = dof_drive(d);
      bool row = on || dof_passive(d).y > 0.0f || C.JFL == 1u || (C.DRIVE_ROWS == 1u && (dr.y > 0.0f || dr.z > 0.0f));
      if (row && scalar_dof(d)) { art[C.A_RL + ai.z + n] = (float)d; n++; }
    }
    art[C.A_RLN + tid] = (float)n;
    art_fk(tid);
    art_factor(tid);
  }
  // Phase 1: group contacts into body-pair runs.
  uint32_t nc = std::min(counters[1], MAXC);
  uint32_t ndc = 0u;
  {
    uint32_t prev = 0xffffffffu;
    for (uint32_t c = 0; c < nc; c++) {
      v4 m = contacts[c * 5u + 2u];
      int a = f2i(m.x), b = f2i(m.y);
      uint32_t pk = (uint32_t)(a + 1) | ((uint32_t)(b + 1) << 16u);
      uint32_t cls = 0xfffffffeu;
      if (!pair_asleep(a, b)) {
        if (same_art(a, b)) {
          cls = 0xffffffffu;
          bool rows = !node_asleep(body_node(a));
          if (rows) ndc++;
          sc[C.S_CLOCAL + c] = rows ? 1u : 0u;
        } else {
          cls = (c == 0u || prev != pk) ? UNIT_HEAD : 0u;
        }
      }
      sc[C.S_CSLOT + c] = cls;
      prev = pk;
    }
    uint32_t unit = 0u, run0 = 0u;
    for (uint32_t c = 0; c < nc; c++) {
      uint32_t cls = sc[C.S_CSLOT + c];
      if (cls >= 0xfffffffeu) continue;
      v4 cmeta = contacts[c * 5u + 2u];
      int a = f2i(cmeta.x), b = f2i(cmeta.y);
      if (cls == UNIT_HEAD) { unit++; run0 = c; }
      uint32_t h = unit - 1u;
      if (h >= C.UH) { sc[C.S_CSLOT + c] = 0xfffffffeu; continue; }
      if (c == run0) sc[C.S_HKEY + h] = contact_pair(c);
      sc[C.S_HCNT + h]++;
      sc[C.S_CSLOT + c] = h;
      sc[C.S_CLOCAL + c] = c - run0;
      if (a >= 0 && body_kind(a) == 2u) wlinkhit[(uint32_t)a] = 1u;
      if (b >= 0 && body_kind(b) == 2u) wlinkhit[(uint32_t)b] = 1u;
    }
  }
  // Phase 2: compact occupied slots into units, joint split, link responses.
  uint32_t u = 0u, woff = 0u;
  for (uint32_t h = 0; h < C.UH; h++) {
    uint32_t key = sc[C.S_HKEY + h];
    if (key != 0u) {
      if (u < C.MAXU) { wkey[u] = key; sc[C.S_USIZE_TMP + u] = sc[C.S_HCNT + h]; }
      sc[C.S_SLOT2U + h] = u;
      sc[C.S_UWOFF + h] = woff;
      woff += sc[C.S_HCNT + h];
      u++;
    }
  }
  uint32_t wnu = std::min(u, C.MAXU), wnwalk = woff;
  for (uint32_t l = 0; l < C.NL; l++) {
    if (wlinkhit[(uint32_t)link_body(l)] == 0u) continue;
    int j = (int)l;
    while (j >= 0) { wjsplit[(uint32_t)j]++; j = link_parent((uint32_t)j); }
  }
  {
    std::vector<uint32_t> path(C.MAXPATH), cnt(C.MAXPATH);
    for (uint32_t l = 0; l < C.NL; l++) {
      if (wlinkhit[(uint32_t)link_body(l)] == 0u) continue;
      uint32_t np = link_path(l, path.data());
      for (uint32_t i = 0; i < np; i++) cnt[i] = wjsplit[path[i]];
      link_response(l, cnt.data());
    }
  }
  for (uint32_t d = 0; d < C.ND; d++) {
    v4 lim = dof_limit(d);
    v4 dr = dof_drive(d);
    if (lim.z > 0.5f || dof_passive(d).y > 0.0f || dof_passive(d).z >= 0.0f || statF[C.SF_DOF + d * 5u + 3u].w > 0.0f ||
        (C.DRIVE_ROWS == 1u && (dr.y > 0.0f || dr.z > 0.0f))) {
      uint32_t l = f2u(lim.w);
      art[C.A_HINV + d] = dof_hinv(l, d - link_dof(l));
    }
  }
  for (uint32_t c = 0; c < nc; c++) {
    uint32_t h = sc[C.S_CSLOT + c];
    if (h >= C.UH) continue;
    uint32_t u0 = sc[C.S_SLOT2U + h];
    sc[C.S_WALK + sc[C.S_UWOFF + h] + sc[C.S_CLOCAL + c]] = u0 >= C.MAXU ? 0xffffffffu : c;
  }
  uint32_t nu = wnu;
  sc[C.S_META + 0u] = nu;
  sc[C.S_META + 2u] = nc;
  for (uint32_t i = 0; i < nu; i++) {
    sc[C.S_UKEY + i] = wkey[i];
    sc[C.S_USIZE + i] = sc[C.S_USIZE_TMP + i];
    wcol[i] = i;
  }
  auto prefix_ustart = [&]() {
    uint32_t off = 0u;
    for (uint32_t i = 0; i < nu; i++) { sc[C.S_USTART + i] = off; off += sc[C.S_USIZE + i]; }
    sc[C.S_USTART + nu] = off;
  };
  prefix_ustart();
  // Phase 5: list each unit's contacts and reduce them by group.
  for (uint32_t c = 0; c < nc; c++) {
    uint32_t slot = sc[C.S_CSLOT + c];
    if (slot >= 0xfffffffeu) continue;
    uint32_t u0 = sc[C.S_SLOT2U + slot];
    if (u0 >= C.MAXU) continue;
    sc[C.S_CORDER + sc[C.S_USTART + wcol[u0]] + sc[C.S_CLOCAL + c]] = c;
  }
  uint32_t nl = std::min(sc[C.S_USTART + nu], MAXC);
  std::vector<BPC> bpc(nl);
  for (uint32_t p = 0; p < nl; p++) {
    bpc[p] = bp_contact(*this, sc[C.S_CORDER + p]);
    sc[C.S_RK0 + p] = bpc[p].k[0]; sc[C.S_RK1 + p] = bpc[p].k[1]; sc[C.S_RK2 + p] = bpc[p].k[2];
  }
  for (uint32_t sp = 0; sp < nu; sp++) sc[C.S_OSTART + sp] = sc[C.S_USTART + sp];
  for (uint32_t p = 0; p < nl; p++) {
    uint32_t st = sc[C.S_USTART + unit_of(p, nu)];
    uint32_t k0 = sc[C.S_RK0 + p], k1 = sc[C.S_RK1 + p], k2 = sc[C.S_RK2 + p];
    uint32_t lead = p;
    for (uint32_t m = st; m < p; m++)
      if (sc[C.S_RK2 + m] == k2 && sc[C.S_RK0 + m] == k0 && sc[C.S_RK1 + m] == k1) { lead = m; break; }
    sc[C.S_LEAD + p] = lead;
    for (uint32_t q = 0; q < 26u; q++) sc[C.S_SLOT + p * 26u + q] = 0u;
  }
  uint32_t v[2];
  for (uint32_t p = 0; p < nl; p++) {
    uint32_t sl = C.S_SLOT + sc[C.S_LEAD + p] * 26u;
    for (uint32_t q = 0; q < 13u; q++) { bp_value(bpc[p], q, v); if (v[1] != 0u) sc[sl + q * 2u] = std::max(sc[sl + q * 2u], v[0]); }
  }
  for (uint32_t p = 0; p < nl; p++) {
    uint32_t sl = C.S_SLOT + sc[C.S_LEAD + p] * 26u;
    for (uint32_t q = 0; q < 13u; q++) {
      bp_value(bpc[p], q, v);
      if (v[1] != 0u && v[0] == sc[sl + q * 2u]) sc[sl + q * 2u + 1u] = std::max(sc[sl + q * 2u + 1u], v[1]);
    }
  }
  for (uint32_t p = 0; p < nl; p++) {
    uint32_t sl = C.S_SLOT + sc[C.S_LEAD + p] * 26u;
    bool win = false;
    for (uint32_t q = 0; q < 13u; q++) {
      bp_value(bpc[p], q, v);
      if (v[1] != 0u && v[0] == sc[sl + q * 2u] && v[1] == sc[sl + q * 2u + 1u]) win = true;
    }
    sc[C.S_LEAD + p] = (win || C.COMPL == 1u) ? 1u : 0u;
  }
  for (uint32_t sp = 0; sp < nu; sp++) {
    uint32_t n = sc[C.S_USIZE + sp], st = sc[C.S_USTART + sp], kept = 0u;
    for (uint32_t j = 0; j < n; j++) {
      if (st + j >= MAXC) break;
      if (sc[C.S_LEAD + st + j] != 0u) { sc[C.S_KEPT + st + kept] = sc[C.S_CORDER + st + j]; kept++; }
    }
    sc[C.S_USIZE + sp] = kept;
  }
  prefix_ustart();
  // Phase 6: build rows.
  uint32_t rbase = P.parity * WH;
  uint32_t total = std::min(sc[C.S_USTART + nu], MAXC);
  for (uint32_t idx = 0; idx < total; idx++) {
    uint32_t sp = unit_of(idx, nu);
    uint32_t c = sc[C.S_KEPT + sc[C.S_OSTART + sp] + idx - sc[C.S_USTART + sp]];
    v4 c0 = contacts[c * 5u], c1 = contacts[c * 5u + 1u], cmeta = contacts[c * 5u + 2u];
    int a = f2i(cmeta.x), b = f2i(cmeta.y);
    uint32_t key = std::max(f2u(cmeta.z) | (f2u(cmeta.w) << 16u), 1u);
    v3 p = xyz(c0), n = xyz(c1);
    float phi = c0.w;
    float mu = phi <= C.F_FGAP ? c1.w * C.F_FSCALE : 0.0f;
    v3 t1 = cross(n, mk3(1.0f, 0.0f, 0.0f));
    if (dot(t1, t1) < 0.1f) t1 = cross(n, mk3(0.0f, 1.0f, 0.0f));
    t1 = normalize(t1);
    v3 t2 = cross(n, t1);
    v3 ca = splat3(0.0f), cb = splat3(0.0f);
    if (a >= 0) ca = xyz(poses[C.P_BODY + (uint32_t)a * 2u]);
    if (b >= 0) cb = xyz(poses[C.P_BODY + (uint32_t)b * 2u]);
    float half = C.SHARED == 1u ? 0.0f : 0.5f * phi;
    v3 ra = (p - n * half) - ca, rb = (p + n * half) - cb;
    v3 fa = ra, fb = rb;
    if (C.FSHARED == 1u) { fa = p - ca; fb = p - cb; }
    uint32_t o = idx * ROWS;
    v3 dirs[3] = {n, t1, t2};
    v3 Ma[3][2], Mb[3][2];
    for (uint32_t r = 0; r < 3u; r++) {
      v3 d = dirs[r];
      v3 aa = r == 0u ? ra : fa, ab = r == 0u ? rb : fb;
      body_response(a, -d, -cross(aa, d), Ma[r]);
      body_response(b, d, cross(ab, d), Mb[r]);
      rows[o + 7u + r * 4u] = mk4(Ma[r][0], 0.0f);
      rows[o + 8u + r * 4u] = mk4(Ma[r][1], 0.0f);
      rows[o + 9u + r * 4u] = mk4(Mb[r][0], 0.0f);
      rows[o + 10u + r * 4u] = mk4(Mb[r][1], 0.0f);
    }
    float K[9];
    for (uint32_t r = 0; r < 3u; r++)
      for (uint32_t s = 0; s < 3u; s++) {
        v3 d = dirs[r];
        v3 aa = r == 0u ? ra : fa, ab = r == 0u ? rb : fb;
        K[r * 3u + s] = ((dot(-d, Ma[s][0]) + dot(-cross(aa, d), Ma[s][1])) + dot(d, Mb[s][0])) + dot(cross(ab, d), Mb[s][1]);
      }
    if (C.EXTRA == 1u) {
      rows[o + PO] = mk4(fa, 1.0f);
      rows[o + PO + 1u] = mk4(fb, 0.0f);
      rows[o + PO + 2u] = mk4(p, 0.0f);
    }
    if (C.TORS == 1u) {
      rows[o + C.TO + 3u] = mk4(0.0f, 0.0f, 0.0f, contacts[c * 5u + 3u].w);
      rows[o + C.TO + 4u] = mk4(p, 0.0f);
    }
    if (C.FMODE > 0u) {
      rows[o + C.FMO] = mk4(K[0], 0.5f * (K[1] + K[3]), 0.5f * (K[2] + K[6]), 0.0f);
      rows[o + C.FMO + 1u] = mk4(K[4], 0.5f * (K[5] + K[7]), K[8], 0.0f);
    }
    float kscale = fmaxf_((K[0] + K[4]) + K[8], 1e-30f);
    float effn = 0.0f;
    if (K[0] > 1e-6f * kscale && K[0] > 1e-12f) effn = 1.0f / (K[0] + C.F_CFM);
    float k00 = (K[4] + 1e-6f * kscale) + C.F_CFM, k01 = 0.5f * (K[5] + K[7]), k11 = (K[8] + 1e-6f * kscale) + C.F_CFM;
    float det = k00 * k11 - k01 * k01;
    float rhs = 0.0f;
    if (phi < 0.0f) rhs = fmaxf_((P.beta * phi) / P.dt, -depen_cap(a, b));
    else rhs = (C.F_SPEC * phi) / P.dt;
    float e = contacts[c * 5u + 3u].x;
    bool bounce = false;
    if (e > 0.0f) {
      v3 ta0[2], tb0[2];
      pre_twist(a, ta0);
      pre_twist(b, tb0);
      float vn0 = dot(n, (tb0[0] + cross(tb0[1], rb)) - (ta0[0] + cross(ta0[1], ra)));
      bounce = restitution_fires(e, phi, vn0);
      if (bounce) rhs = e * vn0;
    }
    float ln = 0.0f;
    v3 lf = splat3(0.0f);
    uint32_t h = key % WH;
    for (uint32_t probe = 0; probe < 32u; probe++) {
      uint32_t k = warm[rbase + h];
      if (k == 0u) break;
      if (k == key) {
        uint32_t vo = 2u * WH + (rbase + h) * 4u;
        ln = bitsf(warm[vo]) * P.warm_scale;
        lf = mk3(bitsf(warm[vo + 1u]), bitsf(warm[vo + 2u]), bitsf(warm[vo + 3u])) * P.warm_scale;
        break;
      }
      h = (h + 1u) % WH;
    }
    v2 lt = mk2(dot(lf, t1), dot(lf, t2));
    float lim = mu * ln;
    float lm = length(lt);
    if (lm > lim) lt = lt * (lim / fmaxf_(lm, 1e-12f));
    float effc = effn, rhsc = rhs;
    if (C.COMPL == 1u) {
      // contact_compliance (wgsl.js:2194-2206): a spring-damper normal row; the pair's series
      // stiffness and summed damping are split over the unit's kept points.
      v4 kc4 = contacts[c * 5u + 4u];
      float nk = (float)std::max(sc[C.S_USIZE + sp], 1u);
      v2 kc = mk2(kc4.x / nk, kc4.y / nk);
      float gam = 0.0f;
      if (kc.x > 0.0f) {
        float ce = phi <= 0.0f ? kc.y : 0.0f;
        float den = P.dt * kc.x + ce;
        gam = 1.0f / (P.dt * den);
        rhsc = (kc.x * phi) / den;
        if (effn > 0.0f) effc = 1.0f / (1.0f / effn + gam);
      }
      rows[o + C.CO] = mk4(gam, 0.0f, 0.0f, 0.0f);
    }
    rows[o + 0u] = mk4(n, effc);
    rows[o + 1u] = mk4(t1, rhsc);
    rows[o + 2u] = mk4(t2, mu);
    rows[o + 3u] = mk4(ra, (float)(key & 0xffffu));
    rows[o + 4u] = mk4(rb, (float)(key >> 16u));
    float wrow = row_weight(phi);
    if (wrow < 1.0f && ((a >= 0 && body_kind(a) == 2u) || (b >= 0 && body_kind(b) == 2u))) {
      v3 ua[2], ub[2];
      body_response_unsplit(a, -n, -cross(ra, n), ua);
      body_response_unsplit(b, n, cross(rb, n), ub);
      float du = ((dot(-n, ua[0]) + dot(-cross(ra, n), ua[1])) + dot(n, ub[0])) + dot(cross(rb, n), ub[1]);
      if (du > 0.0f && K[0] != du) wrow = (wrow * K[0]) / (wrow * K[0] + (1.0f - wrow) * du);
    }
    rows[o + 5u] = mk4(k11 / det, -k01 / det, k00 / det, bounce ? 1.0f : wrow);
    rows[o + 6u] = mk4(ln, lt.x, lt.y, bounce ? 1e30f : phi);
    if (C.ANG == 1u) {
      // Torsional (about n) and rolling (about t1, t2) rows of free bodies (wgsl.js:2223-2243):
      // angular-only Jacobians, the spin row's 1 / K and the rolling pair's inverse 2x2 block.
      const v4 mat = contacts[c * 5u + 3u];
      v3 MA[3][2], MB[3][2];
      for (uint32_t r = 0; r < 3u; r++) {
        const v3 d = dirs[r];
        body_response(a, splat3(0.0f), -d, MA[r]);
        body_response(b, splat3(0.0f), d, MB[r]);
        rows[o + 22u + r * 4u] = mk4(MA[r][0], 0.0f);
        rows[o + 23u + r * 4u] = mk4(MA[r][1], 0.0f);
        rows[o + 24u + r * 4u] = mk4(MB[r][0], 0.0f);
        rows[o + 25u + r * 4u] = mk4(MB[r][1], 0.0f);
      }
      float KA[9];
      for (uint32_t r = 0; r < 3u; r++)
        for (uint32_t s3 = 0; s3 < 3u; s3++) KA[r * 3u + s3] = dot(-dirs[r], MA[s3][1]) + dot(dirs[r], MB[s3][1]);
      const float ks = fmaxf_(KA[0], 1e-12f);
      const float r00 = KA[4] + 1e-9f, r01 = 0.5f * (KA[5] + KA[7]), r11 = KA[8] + 1e-9f;
      const float rd = r00 * r11 - r01 * r01;
      rows[o + 19u] = mk4(mat.y, mat.z, KA[0] > 1e-12f ? 1.0f / ks : 0.0f, 0.0f);
      rows[o + 20u] = mk4(r11 / rd, -r01 / rd, r00 / rd, 0.0f);
      rows[o + 21u] = mk4(0.0f, 0.0f, 0.0f, 0.0f);
      if (C.ANG_ART == 1u) {
        // The raw 5x5 response of (t1, t2, spin, roll1, roll2), upper triangle row by row, for the
        // articulated angular block (wgsl.js:2244-2267).
        v3 JA[5][2], JB[5][2], RA[5][2], RB[5][2];
        for (uint32_t q = 0; q < 2u; q++) {
          const v3 d = dirs[q + 1u];
          JA[q][0] = -d; JA[q][1] = -cross(fa, d);
          JB[q][0] = d; JB[q][1] = cross(fb, d);
          RA[q][0] = Ma[q + 1u][0]; RA[q][1] = Ma[q + 1u][1];
          RB[q][0] = Mb[q + 1u][0]; RB[q][1] = Mb[q + 1u][1];
        }
        for (uint32_t q = 0; q < 3u; q++) {
          JA[q + 2u][0] = splat3(0.0f); JA[q + 2u][1] = -dirs[q];
          JB[q + 2u][0] = splat3(0.0f); JB[q + 2u][1] = dirs[q];
          RA[q + 2u][0] = MA[q][0]; RA[q + 2u][1] = MA[q][1];
          RB[q + 2u][0] = MB[q][0]; RB[q + 2u][1] = MB[q][1];
        }
        float Hu[16];
        uint32_t idx = 0;
        for (uint32_t x = 0; x < 5u; x++)
          for (uint32_t y = x; y < 5u; y++)
            Hu[idx++] = ((dot(JA[x][0], RA[y][0]) + dot(JA[x][1], RA[y][1])) + dot(JB[x][0], RB[y][0])) +
                        dot(JB[x][1], RB[y][1]);
        Hu[15] = 0.0f;
        for (uint32_t q = 0; q < 4u; q++) rows[o + C.EO + q] = v4{Hu[q * 4u], Hu[q * 4u + 1u], Hu[q * 4u + 2u], Hu[q * 4u + 3u]};
      }
    }
  }
  // Phase 6b: contact torsion headers, then friction patches.
  if (C.TORS == 1u) for (uint32_t sp = 0; sp < nu; sp++) build_torsion(sp);
  if (C.PATCH == 1u) for (uint32_t sp = 0; sp < nu; sp++) build_patch(sp);
  // Phase 6c: coloring in walk order.
  uint32_t totp = std::min(sc[C.S_USTART + nu], MAXC);
  for (uint32_t c = 0; c < nc; c++) sc[C.S_ROWOF + c] = 0xffffffffu;
  std::fill(wmask.begin(), wmask.end(), 0u);
  std::fill(wcount.begin(), wcount.end(), 0u);
  for (uint32_t sp = 0; sp < nu; sp++) {
    sc[C.S_UTC + sp] = 0u;
    sc[C.S_UTP + sp] = C.LONGEST_FIRST == 0u ? 0u : 0xffffffffu;
  }
  for (uint32_t row = 0; row < totp; row++) {
    uint32_t sp = unit_of(row, nu);
    uint32_t c = sc[C.S_KEPT + sc[C.S_OSTART + sp] + row - sc[C.S_USTART + sp]];
    sc[C.S_RUNIT + row] = sp;
    sc[C.S_RCON + row] = c;
    if (c < nc) sc[C.S_ROWOF + c] = row;
  }
  uint32_t ncu = C.LONGEST_FIRST == 0u ? std::min(wnwalk, MAXC) : 0u;
  for (uint32_t i = 0; i < ncu; i++) {
    uint32_t wc = sc[C.S_WALK + i];
    uint32_t row = wc < MAXC ? sc[C.S_ROWOF + std::min(wc, MAXC - 1u)] : 0xffffffffu;
    uint32_t key = row < totp ? sc[C.S_UKEY + sc[C.S_RUNIT + std::min(row, MAXC - 1u)]] : 0xffffffffu;
    if (key == 0xffffffffu) continue;
    uint32_t col = first_free_color((int)(key & 0xffffu) - 1, (int)(key >> 16u) - 1);
    sc[C.S_PCOL + row] = col;
    wcount[col]++;
    uint32_t& utp = sc[C.S_UTP + sc[C.S_RUNIT + row]];
    utp = std::max(utp, ((col + 1u) << 16u) | wc);
  }
  if (C.LONGEST_FIRST == 0u) {
    for (uint32_t sp = 0; sp < nu; sp++) {
      uint32_t packed = sc[C.S_UTP + sp];
      sc[C.S_UTC + sp] = packed >> 16u;
      sc[C.S_UTP + sp] = packed != 0u ? sc[C.S_ROWOF + (packed & 0xffffu)] : 0xffffffffu;
    }
  } else {
    // propagation_color_order "longest_first" (wgsl.js:2331-2346): first-fit by row count first
    // (7 rows down to 1), then contact index; a unit's last row of its highest color carries its
    // torsion row.
    for (uint32_t lp = 0; lp < 8u; lp++)
      for (uint32_t c = 0; c < nc; c++) {
        uint32_t row = sc[C.S_ROWOF + c];
        if (row >= totp) continue;
        if (row_count(row) != 7u - lp) continue;
        uint32_t sp = sc[C.S_RUNIT + row];
        uint32_t key = sc[C.S_UKEY + sp];
        uint32_t col = first_free_color((int)(key & 0xffffu) - 1, (int)(key >> 16u) - 1);
        sc[C.S_PCOL + row] = col;
        wcount[col]++;
        if (col + 1u >= sc[C.S_UTC + sp]) {
          sc[C.S_UTC + sp] = col + 1u;
          sc[C.S_UTP + sp] = row;
        }
      }
  }
  {
    uint32_t acc = 0u, ncol = 0u;
    for (uint32_t c = 0; c <= NCOL; c++) {
      uint32_t n = wcount[c];
      sc[C.S_CSTART + c] = acc;
      wcount[c] = acc;
      acc += n;
      if (n > 0u) ncol = c + 1u;
    }
    sc[C.S_CSTART + NCOL + 1u] = acc;
    sc[C.S_META + 1u] = ncol;
  }
  for (uint32_t row = 0; row < totp; row++) {
    uint32_t slot = wcount[sc[C.S_PCOL + row]]++;
    if (slot < MAXC) sc[C.S_PORD + slot] = row;
  }
  // sort_overflow_color (wgsl.js:1740-1780): the serial color in contact order.
  {
    uint32_t o0 = std::min(sc[C.S_CSTART + NCOL], MAXC);
    uint32_t m = std::min(sc[C.S_CSTART + NCOL + 1u], MAXC) - o0;
    if (m >= 2u) {
      uint32_t k = 0u;
      for (uint32_t c = 0; c < nc && k < m; c++) {
        uint32_t row = sc[C.S_ROWOF + c];
        if (row < totp && sc[C.S_PCOL + row] == NCOL) { sc[C.S_PORD + o0 + k] = row; k++; }
      }
    }
  }
  // Phase 7: dense rows for same-articulation contacts, then loops and mimics.
  uint32_t nloop_rows = 0u;
  for (uint32_t k = 0; k < C.NLOOP; k++) nloop_rows += statF[C.SF_LOOP + k * 5u].w > 0.5f ? 2u : 1u;
  sc[C.S_META + 3u] = ndc + nloop_rows + C.NMIMIC;
  const uint32_t NDA = C.NDA, JDIM = C.JDIM, DHDR = C.DHDR, DPS = C.DPS;
  std::vector<float> J(JDIM), tau(NDA), y(NDA);
  uint32_t dslot = 0u;
  for (uint32_t c = 0; c < nc; c++) {
    if (sc[C.S_CSLOT + c] != 0xffffffffu || sc[C.S_CLOCAL + c] == 0u) continue;
    uint32_t slot = dslot++;
    if (slot >= C.MAXDENSE) continue;
    v4 c0 = contacts[c * 5u], c1 = contacts[c * 5u + 1u], cmeta = contacts[c * 5u + 2u];
    int a = f2i(cmeta.x), b = f2i(cmeta.y);
    uint32_t key = std::max(f2u(cmeta.z) | (f2u(cmeta.w) << 16u), 1u);
    v3 p = xyz(c0), n = xyz(c1);
    float phi = c0.w;
    float mu = phi <= C.F_FGAP ? c1.w * C.F_FSCALE : 0.0f;
    v3 t1 = cross(n, mk3(1.0f, 0.0f, 0.0f));
    if (dot(t1, t1) < 0.1f) t1 = cross(n, mk3(0.0f, 1.0f, 0.0f));
    t1 = normalize(t1);
    v3 t2 = cross(n, t1);
    uint32_t art_id = (uint32_t)body_art(a);
    u4 ai = art_info(art_id);
    std::fill(J.begin(), J.end(), 0.0f);
    add_gen_jac((uint32_t)body_link(b), p, 1.0f, n, t1, t2, ai.z, J.data());
    add_gen_jac((uint32_t)body_link(a), p, -1.0f, n, t1, t2, ai.z, J.data());
    uint32_t o = C.A_DENSE + slot * DPS;
    float K[9];
    for (uint32_t r = 0; r < 3u; r++) {
      for (uint32_t k = 0; k < NDA; k++) { tau[k] = k < ai.w ? J[r * NDA + k] : 0.0f; y[k] = 0.0f; }
      art_solve_gen(art_id, tau.data(), y.data());
      for (uint32_t k = 0; k < ai.w; k++) {
        art[o + DHDR + r * NDA + k] = J[r * NDA + k];
        art[o + DHDR + 3u * NDA + r * NDA + k] = y[k];
      }
      for (uint32_t s2 = 0; s2 < 3u; s2++) {
        float acc = 0.0f;
        for (uint32_t k = 0; k < ai.w; k++) acc += J[s2 * NDA + k] * y[k];
        K[s2 * 3u + r] = acc;
      }
    }
    float kscale = fmaxf_((K[0] + K[4]) + K[8], 1e-30f);
    float effn = 0.0f;
    if (K[0] > 1e-6f * kscale && K[0] > 1e-12f) effn = 1.0f / (K[0] + C.F_CFM);
    float k00 = (K[4] + 1e-6f * kscale) + C.F_CFM, k01 = 0.5f * (K[5] + K[7]), k11 = (K[8] + 1e-6f * kscale) + C.F_CFM;
    float det = k00 * k11 - k01 * k01;
    float rhs = phi < 0.0f ? fmaxf_((P.beta * phi) / P.dt, -depen_cap(a, b)) : (C.F_SPEC * phi) / P.dt;
    float e = contacts[c * 5u + 3u].x;
    bool bounce = false;
    if (e > 0.0f) {
      float vn0 = 0.0f;
      for (uint32_t k = 0; k < ai.w; k++) vn0 += J[k] * art[C.A_QD + ai.z + k];
      bounce = restitution_fires(e, phi, vn0);
      if (bounce) rhs = e * vn0;
    }
    float ln = 0.0f;
    v3 lf = splat3(0.0f);
    uint32_t h = key % WH;
    for (uint32_t probe = 0; probe < 32u; probe++) {
      uint32_t k = warm[rbase + h];
      if (k == 0u) break;
      if (k == key) {
        uint32_t vo = 2u * WH + (rbase + h) * 4u;
        ln = bitsf(warm[vo]) * P.warm_scale;
        lf = mk3(bitsf(warm[vo + 1u]), bitsf(warm[vo + 2u]), bitsf(warm[vo + 3u])) * P.warm_scale;
        break;
      }
      h = (h + 1u) % WH;
    }
    v2 lt = mk2(dot(lf, t1), dot(lf, t2));
    if (length(lt) > mu * ln) lt = lt * ((mu * ln) / fmaxf_(length(lt), 1e-12f));
    art[o] = (float)art_id; art[o + 1u] = (float)(key & 0xffffu); art[o + 2u] = (float)(key >> 16u); art[o + 3u] = mu;
    art[o + 4u] = rhs; art[o + 5u] = effn;
    art[o + 6u] = k11 / det; art[o + 7u] = -k01 / det; art[o + 8u] = k00 / det;
    art[o + 9u] = ln; art[o + 10u] = lt.x; art[o + 11u] = lt.y;
    st3(o + 12u, t1); st3(o + 15u, t2); st3(o + 18u, n);
    art[o + 21u] = 0.0f;
    art[o + 24u] = bounce ? 1.0f : row_weight(phi);
    art[o + 22u] = bounce ? 1e30f : phi;
  }
  for (uint32_t i = 0; i < C.NLOOP; i++) {
    v4 L0 = statF[C.SF_LOOP + i * 5u];
    int pl = f2i(L0.x);
    uint32_t cl = f2u(L0.y), art_id = f2u(L0.z);
    bool revolute = L0.w > 0.5f;
    uint32_t slot = ndc;
    for (uint32_t k = 0; k < i; k++) slot += statF[C.SF_LOOP + k * 5u].w > 0.5f ? 2u : 1u;
    if (slot + (revolute ? 1u : 0u) >= C.MAXDENSE) continue;
    v3 pa = xyz(statF[C.SF_LOOP + i * 5u + 1u]);
    v4 rp = mk4(0, 0, 0, 1);
    if (pl >= 0) { rp = link_rot((uint32_t)pl); pa = ld3(lo((uint32_t)pl) + L_POS) + qrot(rp, pa); }
    v4 rc = link_rot(cl);
    v3 pc = ld3(lo(cl) + L_POS) + qrot(rc, xyz(statF[C.SF_LOOP + i * 5u + 2u]));
    v3 pm = 0.5f * (pa + pc);
    u4 ai = art_info(art_id);
    std::fill(J.begin(), J.end(), 0.0f);
    v3 ex = mk3(1, 0, 0), ey = mk3(0, 1, 0), ez = mk3(0, 0, 1);
    add_gen_jac(cl, pm, 1.0f, ex, ey, ez, ai.z, J.data());
    if (pl >= 0) add_gen_jac((uint32_t)pl, pm, -1.0f, ex, ey, ez, ai.z, J.data());
    put_bilateral(C.A_DENSE + slot * DPS, art_id, J.data(), 3u, (P.beta * (pc - pa)) / P.dt);
    if (revolute) {
      v3 ap = qrot(rp, xyz(statF[C.SF_LOOP + i * 5u + 3u]));
      v3 ac = qrot(rc, xyz(statF[C.SF_LOOP + i * 5u + 4u]));
      v3 e1 = cross(ap, mk3(1, 0, 0));
      if (dot(e1, e1) < 1e-6f) e1 = cross(ap, mk3(0, 1, 0));
      e1 = normalize(e1);
      v3 e2 = cross(ap, e1);
      std::vector<float> Ja(JDIM, 0.0f);
      add_gen_ang(cl, 1.0f, e1, e2, ai.z, Ja.data());
      if (pl >= 0) add_gen_ang((uint32_t)pl, -1.0f, e1, e2, ai.z, Ja.data());
      v3 err = cross(ap, ac);
      put_bilateral(C.A_DENSE + (slot + 1u) * DPS, art_id, Ja.data(), 2u,
                    (P.beta * mk3(dot(e1, err), dot(e2, err), 0.0f)) / P.dt);
    }
  }
  for (uint32_t i = 0; i < C.NMIMIC; i++) {
    v4 M0 = statF[C.SF_MIMIC + i * 2u], M1 = statF[C.SF_MIMIC + i * 2u + 1u];
    uint32_t slot = ndc + nloop_rows + i;
    if (slot >= C.MAXDENSE) continue;
    std::fill(J.begin(), J.end(), 0.0f);
    J[f2u(M0.y)] = 1.0f;
    J[f2u(M0.z)] -= M0.w;
    float phi = (art[C.A_Q + f2u(M1.x)] - M0.w * art[C.A_Q + f2u(M1.y)]) - M1.z;
    put_bilateral(C.A_DENSE + slot * DPS, f2u(M0.x), J.data(), 1u, mk3((P.beta * phi) / P.dt, 0.0f, 0.0f));
  }
}

}  // namespace orc
