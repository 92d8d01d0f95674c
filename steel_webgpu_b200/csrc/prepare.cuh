#pragma once
// Prepare of one scene by one block (the body of k_prepare).
//
// Follows the reference's prepare pass (packages/steel-webgpu/src/wgsl.js:1222-2494) on its
// default option set: drive targets (wgsl.js:1800-1825), joint-limit gating and the
// articulation factorisation (wgsl.js:1856-1877), grouping of the canonically sorted contacts
// into body-pair units (wgsl.js:1889-2028), body-pair contact reduction (wgsl.js:2029-2105),
// row build with warm-start lookup (wgsl.js:2106-2269), friction patches (wgsl.js:1562-1725),
// greedy first-fit coloring in contact order (wgsl.js:2282-2364) and dense same-articulation,
// loop-closure and mimic rows (wgsl.js:2365-2492).
//
// Units are runs of one body pair in the sorted contact list; the reference reaches the same
// runs through a unit hash and a walk list, here they come straight from one block scan. Rows
// are numbered unit by unit in contact order, so rows are also in contact order, which makes
// the serial overflow color's contact-order sort the identity.
#include "team.cuh"
#include "art.cuh"
#include "batch.cuh"
#include "bulk.cuh"
#include "block.cuh"

namespace steel {

static __constant__ float BP_BX[20] = {-0.57095543f, -0.64404845f, -0.86918069f, -0.93522697f, -0.75091368f, 0.36427171f,
                                -0.17291149f, 0.47113684f, 0.11826704f, 0.17291155f, 0.0f, -0.11826707f,
                                -0.36427169f, 0.0f, -0.47113677f, 0.93522695f, 0.75091367f, 0.57095545f,
                                0.64404840f, 0.86918063f};
static __constant__ float BP_BY[20] = {0.75026579f, 0.17218052f, -0.36525859f, -0.11932883f, 0.57010308f, 0.86959472f,
                                0.64385240f, 0.47167205f, 0.93536185f, -0.64385245f, 0.0f, -0.93536184f,
                                -0.86959473f, 0.0f, -0.47167196f, 0.11932898f, -0.57010306f, -0.75026579f,
                                -0.17218051f, 0.36525872f};
static __constant__ float BP_BZ[20] = {0.33333337f, 0.74535593f, 0.33333330f, -0.33333339f, -0.33333336f, -0.33333337f,
                                -0.74535609f, 0.74535599f, 0.33333335f, 0.74535603f, 1.0f, -0.33333335f,
                                0.33333337f, -1.0f, -0.74535609f, 0.33333339f, 0.33333340f, -0.33333334f,
                                -0.74535597f, -0.33333332f};
static constexpr uint32_t AVN = 14u;

struct Prep {
  const SceneDev& S;
  const Params& P;
  Art ar;
  __device__ Prep(const SceneDev& s, const Params& p, float* lb) : S(s), P(p), ar(s, lb) {}

  __device__ uint32_t bkind(int b) const { return f2u(S.sf[S.SF_BODY + (uint32_t)b * 8u].y); }
  __device__ int bart(int b) const { return f2i(S.sf[S.SF_BODY + (uint32_t)b * 8u].z); }
  __device__ int blink(int b) const { return f2i(S.sf[S.SF_BODY + (uint32_t)b * 8u].w); }
  __device__ float bradius(int b) const { return b < 0 ? 1e30f : S.sf[S.SF_BODY + (uint32_t)b * 8u + 2u].w; }
  __device__ float depen_cap(int a, int b) const {
    float m = 1e20f;
    if (a >= 0) { float l = S.sf[S.SF_BODY + (uint32_t)a * 8u + 6u].w; if (l > 0.0f) m = fmn(m, l); }
    if (b >= 0) { float l = S.sf[S.SF_BODY + (uint32_t)b * 8u + 6u].w; if (l > 0.0f) m = fmn(m, l); }
    return m;
  }
  __device__ uint32_t* sc(uint32_t off) const { return S.sched + off; }
  // Sleep-island node of body b (artwgsl.js:49 node_asleep's index): a free body is its own node,
  // a link its articulation's (NB + a); static bodies have none.
  __device__ int bnode(int b) const {
    if (b < 0) return -1;
    uint32_t k = bkind(b);
    if (k == 1u) return b;
    if (k == 2u || k == 3u) return (int)S.NB + bart(b);
    return -1;
  }
  __device__ bool node_asleep(int n) const {
    return S.SLEEP == 1u && n >= 0 && S.art[S.A_SLP + (uint32_t)n * 4u + 1u] > 0.5f;
  }
  // Both sides asleep or static (wgsl.js:1732-1736): the contact makes no rows.
  __device__ bool pair_asleep(int a, int b) const {
    if (S.SLEEP == 0u) return false;
    int na = bnode(a), nb = bnode(b);
    return (na < 0 || node_asleep(na)) && (nb < 0 || node_asleep(nb));
  }

  // Twist change of body b for a unit (force, torque) impulse (wgsl.js:1299-1328).
  __device__ void response(int b, f3 f, f3 t, f3 out[2], bool unsplit = false) const {
    if (b < 0) { out[0] = sp3(0.0f); out[1] = sp3(0.0f); return; }
    uint32_t k = bkind(b);
    if (k == 1u) {
      float4 q = S.rot[b];
      m3 R = qmat(q);
      RO<float4> o = S.sf + S.SF_BODY + (uint32_t)b * 8u;
      m3 Ii = tr(mcols(v3(o[5]), v3(o[6]), v3(o[7])));
      out[0] = f * o[0].x;
      out[1] = mul(R, mul(Ii, mul(tr(R), t)));
      return;
    }
    // Kind 2 links answer the unsplit query from L_W2; immovable links (kind 3) from L_W.
    uint32_t wo = ar.lo((uint32_t)blink(b)) + ((unsplit && k == 2u) ? L_W2 : L_W);
    const float* W = ar.LB + wo;
    float x[6] = {f.x, f.y, f.z, t.x, t.y, t.z}, o[6];
    for (uint32_t r = 0; r < 6u; r++) {
      float s = 0.0f;
      for (uint32_t c = 0; c < 6u; c++) s += W[r * 6u + c] * x[c];
      o[r] = s;
    }
    out[0] = mf3(o[0], o[1], o[2]);
    out[1] = mf3(o[3], o[4], o[5]);
  }
  __device__ bool rest_fires(float e, float phi, float vn) const {
    if (S.REST == 0u || e <= 0.0f || vn >= -S.F_REST_SPEED) return false;
    return phi <= 1e-6f || phi + P.dt * vn <= 1e-6f;
  }
  __device__ void pre_twist(int b, f3 out[2]) const {
    out[0] = sp3(0.0f); out[1] = sp3(0.0f);
    if (b < 0) return;
    uint32_t k = bkind(b);
    if (k == 1u) { out[0] = v3(S.lv[b]); out[1] = v3(S.av[b]); return; }
    if (k == 2u) { uint32_t o = ar.lo((uint32_t)blink(b)) + L_V; out[0] = ar.ld3(o + 3u); out[1] = ar.ld3(o); }
  }
  __device__ float row_weight(float phi) const { return (phi > 0.0f || P.reg <= 0.0f) ? 1.0f : 1.0f / (1.0f + P.reg); }
  __device__ void warm_lookup(uint32_t key, float* ln, f3* lf) const {
    *ln = 0.0f;
    *lf = sp3(0.0f);
    const uint32_t WH = S.WH, rbase = P.parity * WH;
    uint32_t h = key % WH;
    for (uint32_t probe = 0; probe < 32u; probe++) {
      uint32_t k = S.warm_tab[rbase + h];
      if (k == 0u) break;
      if (k == key) {
        const uint32_t* vo = S.warm_tab + 2u * WH + (rbase + h) * 4u;
        *ln = ubits(vo[0]) * P.warm_scale;
        *lf = mf3(ubits(vo[1]), ubits(vo[2]), ubits(vo[3])) * P.warm_scale;
        break;
      }
      h = (h + 1u) % WH;
    }
  }

  // Body-pair reduction key of contact c (wgsl.js:1471-1495): group key words, plane position,
  // gap and position identity.
  __device__ void bp_contact(uint32_t c, uint32_t k[3], float* px, float* py, float* gap, uint32_t* pk) const {
    float4 c0 = S.con[c * 5u], c1 = S.con[c * 5u + 1u], cm = S.con[c * 5u + 2u], c4 = S.con[c * 5u + 4u];
    int a = f2i(cm.x), b = f2i(cm.y);
    uint32_t ga = f2u(c4.z), gb = f2u(c4.w);
    f3 ng = gb < ga ? -v3(c1) : v3(c1);
    int rb = a >= 0 ? a : b;
    f3 org = sp3(0.0f);
    if (rb >= 0) org = v3(S.pos[rb]) - qrot(S.rot[rb], v3(S.sf[S.SF_BODY + (uint32_t)rb * 8u + 1u]));
    uint32_t bin = 0u;
    float bd = -2.0f;
    for (uint32_t i = 0; i < 20u; i++) {
      float d = dot(ng, mf3(BP_BX[i], BP_BY[i], BP_BZ[i]));
      if (d > bd) { bd = d; bin = i; }
    }
    f3 fn_ = mf3(BP_BX[bin], BP_BY[bin], BP_BZ[bin]);
    f3 rv = fabsf(fn_.y) < 0.9f ? mf3(0.0f, 1.0f, 0.0f) : mf3(1.0f, 0.0f, 0.0f);
    f3 u = nrm(rv - dot(rv, fn_) * fn_);
    f3 v = cross(fn_, u);
    f3 x = v3(c0) - org;
    float pxv = dot(x, u), pyv = dot(x, v);
    uint32_t cx = (uint32_t)(f2i(clmp(floorf(pxv / S.F_BP_CELL + 0.5f), -31.0f, 31.0f)) + 31);
    uint32_t cy = (uint32_t)(f2i(clmp(floorf(pyv / S.F_BP_CELL + 0.5f), -31.0f, 31.0f)) + 31);
    uint32_t qx = (uint32_t)(f2i(clmp(floorf(pxv * 2000.0f), -32768.0f, 32767.0f)) + 32768);
    uint32_t qy = (uint32_t)(f2i(clmp(floorf(pyv * 2000.0f), -8192.0f, 8191.0f)) + 8192);
    k[0] = min(ga, gb); k[1] = max(ga, gb); k[2] = bin | (cx << 5u) | (cy << 11u);
    *px = pxv; *py = pyv; *gap = c0.w; *pk = (qx << 15u) | (qy << 1u) | 1u;
  }
  static __device__ uint32_t fflip(float f) {
    uint32_t i = __float_as_uint(f);
    return i ^ (((i >> 31u) != 0u ? 0xffffffffu : 0u) | 0x80000000u);
  }
  // Slot q's packed (score, identity) (wgsl.js:1498-1503).
  static __device__ void bp_value(float px, float py, float gap, uint32_t pk, uint32_t q, uint32_t* sc_, uint32_t* id) {
    if (q == 6u) { *sc_ = fflip(-gap); *id = pk; return; }
    if (q > 6u && gap > 0.0f) { *sc_ = 0u; *id = 0u; return; }
    float ang = (float)(q > 6u ? q - 7u : q) * 1.0471975511965976f;
    *sc_ = fflip(dot(mf2(px, py), mf2(fcos(ang), fsin(ang))));
    *id = pk;
  }
  static __device__ uint32_t anchor_hash(uint32_t pair, uint32_t k) { return max(mix32(pair * 2u + k), 1u); }

  // Friction patch of unit sp (wgsl.js:1562-1725).
  __device__ void build_patch(uint32_t sp) const {
    const uint32_t ROWS = S.ROWS, PO = S.PO;
    float4* rows = S.rows;
    uint32_t st = sc(S.S_USTART)[sp];
    uint32_t n = sc(S.S_USIZE)[sp];
    if (n == 0u) return;
    uint32_t pair = sc(S.S_UKEY)[sp];
    int a = (int)(pair & 0xffffu) - 1, b = (int)(pair >> 16u) - 1;
    f3 ca = sp3(0.0f), cb = sp3(0.0f);
    float4 qa = make_float4(0, 0, 0, 1);
    if (a >= 0) { ca = v3(S.pos[a]); qa = S.rot[a]; }
    if (b >= 0) cb = v3(S.pos[b]);
    float r = fmx(fmn(bradius(a), bradius(b)), 1e-4f);
    uint32_t seed = st;
    for (uint32_t i = st; i < st + n; i++) if (rows[i * ROWS + 1u].w < rows[seed * ROWS + 1u].w) seed = i;
    f3 ns = v3(rows[seed * ROWS]);
    const uint32_t* rcon = sc(S.S_RCON);
    float4 mus = S.con[S.MAXC * 5u + rcon[seed]];
    uint32_t first = seed;
    for (uint32_t i = st; i < st + n; i++) {
      uint32_t o = i * ROWS;
      f3 dseed = v3(rows[o + PO + 2u]) - v3(rows[seed * ROWS + PO + 2u]);
      float4 mui = S.con[S.MAXC * 5u + rcon[i]];
      if (dot(v3(rows[o]), ns) < 0.995f || mui.x != mus.x || mui.y != mus.y || fabsf(dot(dseed, ns)) > 0.02f * r ||
          len(dseed) > 2.0f * r)
        continue;
      rows[o + PO].w = 0.0f;
      f3 p = v3(rows[o + PO + 2u]), pf = v3(rows[first * ROWS + PO + 2u]);
      if (p.x < pf.x || (p.x == pf.x && (p.y < pf.y || (p.y == pf.y && p.z < pf.z)))) first = i;
    }
    f3 pf = v3(rows[first * ROWS + PO + 2u]);
    uint32_t second = first;
    float far = (1e-8f * r) * r;
    for (uint32_t i = st; i < st + n; i++) {
      if (rows[i * ROWS + PO].w != 0.0f) continue;
      f3 d = v3(rows[i * ROWS + PO + 2u]) - pf;
      if (dot(d, d) > far) { far = dot(d, d); second = i; }
    }
    uint32_t na = second != first ? 2u : 1u;
    f3 loc0 = v3(rows[first * ROWS + PO + 2u]), loc1 = v3(rows[second * ROWS + PO + 2u]);
    if (na == 2u) {
      f3 t0 = cross(ns, mf3(1.0f, 0.0f, 0.0f));
      if (dot(t0, t0) < 1e-6f) t0 = cross(ns, mf3(0.0f, 1.0f, 0.0f));
      t0 = nrm(t0);
      f3 t1 = nrm(cross(ns, t0));
      float sx = 0, sy = 0, sxx = 0, sxy = 0, syy = 0, cnt = 0;
      f3 cen = sp3(0.0f);
      for (uint32_t i = st; i < st + n; i++) {
        if (rows[i * ROWS + PO].w != 0.0f) continue;
        f3 pc = v3(rows[i * ROWS + PO + 2u]), d = pc - pf;
        float x = dot(d, t0), y = dot(d, t1);
        sx += x; sy += y; sxx += x * x; sxy += x * y; syy += y * y; cen += pc; cnt += 1.0f;
      }
      float xx = sxx - (sx * sx) / cnt, xy = sxy - (sx * sy) / cnt, yy = syy - (sy * sy) / cnt;
      float spread = sqrtf((xx - yy) * (xx - yy) + (4.0f * xy) * xy);
      if (spread > 1e-6f * (xx + yy)) {
        float big = 0.5f * ((xx + yy) + spread);
        f2 a2 = mf2(xy, big - xx);
        if (xx >= yy) a2 = mf2(big - yy, xy);
        a2 = nrm(a2);
        f3 ax = a2.x * t0 + a2.y * t1;
        float lo_ = 1e30f, hi = -1e30f;
        for (uint32_t i = st; i < st + n; i++) {
          if (rows[i * ROWS + PO].w != 0.0f) continue;
          float pr = dot(v3(rows[i * ROWS + PO + 2u]) - pf, ax);
          if (pr < lo_) { lo_ = pr; first = i; }
          if (pr > hi) { hi = pr; second = i; }
        }
        f3 centroid = cen / cnt;
        loc0 = centroid + dot(v3(rows[first * ROWS + PO + 2u]) - centroid, ax) * ax;
        loc1 = centroid + dot(v3(rows[second * ROWS + PO + 2u]) - centroid, ax) * ax;
        f3 across = nrm(cross(ns, ax));
        float tol = fmx(1e-5f * r, 0.05f * (hi - lo_));
        f3 e0 = sp3(0.0f), e1 = sp3(0.0f);
        float c0 = 0.0f, c1 = 0.0f;
        for (uint32_t i = st; i < st + n; i++) {
          if (rows[i * ROWS + PO].w != 0.0f) continue;
          f3 pc = v3(rows[i * ROWS + PO + 2u]);
          float pr = dot(pc - pf, ax);
          if (pr <= lo_ + tol) { e0 += pc; c0 += 1.0f; }
          if (pr >= hi - tol) { e1 += pc; c1 += 1.0f; }
        }
        e0 = e0 / fmx(c0, 1.0f);
        e1 = e1 / fmx(c1, 1.0f);
        loc0 += dot(e0 - centroid, across) * across + dot(e0 - centroid, ns) * ns;
        loc1 += dot(e1 - centroid, across) * across + dot(e1 - centroid, ns) * ns;
      }
    }
    float load = 0.0f;
    for (uint32_t i = st; i < st + n; i++) {
      if (rows[i * ROWS + PO].w != 0.0f) continue;
      load += rows[i * ROWS + 6u].x;
      if (i != first && !(na == 2u && i == second)) {
        float4 r6 = rows[i * ROWS + 6u];
        rows[i * ROWS + 6u] = make_float4(r6.x, 0.0f, 0.0f, r6.w);
      }
    }
    const uint32_t AK = 10u * S.WH, AVb = 10u * S.WH + 2u * S.AH;
    uint32_t rbase = AK + P.parity * S.AH;
    for (uint32_t k = 0; k < na; k++) {
      uint32_t i = k == 1u ? second : first;
      uint32_t o = i * ROWS;
      f3 loc = k == 1u ? loc1 : loc0;
      f3 nn = v3(rows[o]), t1 = v3(rows[o + 1u]), t2 = v3(rows[o + 2u]);
      f3 fra = loc - ca, frb = loc - cb;
      f3 Ma[2][2], Mb[2][2];
      f3 dirs[2] = {t1, t2};
      for (uint32_t q = 0; q < 2u; q++) {
        response(a, -dirs[q], -cross(fra, dirs[q]), Ma[q]);
        response(b, dirs[q], cross(frb, dirs[q]), Mb[q]);
        rows[o + 11u + q * 4u] = mf4(Ma[q][0], 0.0f);
        rows[o + 12u + q * 4u] = mf4(Ma[q][1], 0.0f);
        rows[o + 13u + q * 4u] = mf4(Mb[q][0], 0.0f);
        rows[o + 14u + q * 4u] = mf4(Mb[q][1], 0.0f);
      }
      float K[4];
      for (uint32_t x = 0; x < 2u; x++)
        for (uint32_t y = 0; y < 2u; y++) {
          f3 d = dirs[x];
          K[x * 2u + y] = ((dot(-d, Ma[y][0]) + dot(-cross(fra, d), Ma[y][1])) + dot(d, Mb[y][0])) +
                          dot(cross(frb, d), Mb[y][1]);
        }
      float ks = fmx(K[0] + K[3], 1e-30f);
      float k00 = K[0] + 1e-6f * ks, k01 = 0.5f * (K[1] + K[2]), k11 = K[3] + 1e-6f * ks;
      float det = k00 * k11 - k01 * k01;
      rows[o + 5u] = make_float4(k11 / det, -k01 / det, k00 / det, rows[o + 5u].w);
      rows[o + 2u] = mf4(t2, rows[o + 2u].w / (float)na);
      f3 e = sp3(0.0f), imp = sp3(0.0f);
      bool carried = false;
      float best = (4.0f * r) * r;
      const uint32_t* W = S.warm_tab;
      for (uint32_t kk = 0; kk < 2u; kk++) {
        uint32_t h = anchor_hash(pair, kk) % S.AH;
        for (uint32_t probe = 0; probe < 32u; probe++) {
          uint32_t key = W[rbase + h];
          if (key == 0u) break;
          uint32_t vo = AVb + (P.parity * S.AH + h) * AVN;
          if (key == anchor_hash(pair, kk) && W[vo] == pair && W[vo + 1u] == kk) {
            f3 ll = mf3(ubits(W[vo + 2u]), ubits(W[vo + 3u]), ubits(W[vo + 4u]));
            f3 el = mf3(ubits(W[vo + 5u]), ubits(W[vo + 6u]), ubits(W[vo + 7u]));
            f3 prev = ca + qrot(qa, ll);
            f3 dl = prev - loc;
            if (dot(dl, dl) <= best && fabsf(dot(dl, nn)) <= 0.05f * r) {
              f3 ew = qrot(qa, el);
              f3 on = qrot(qa, mf3(ubits(W[vo + 11u]), ubits(W[vo + 12u]), ubits(W[vo + 13u])));
              float cs = dot(on, nn);
              if (cs > 0.0f) { f3 ax = cross(on, nn), ce = cross(ax, ew); ew += ce + cross(ax, ce) / (1.0f + cs); }
              ew -= nn * dot(nn, ew);
              if (dot(ew, ew) <= (0.01f * r) * r) {
                e = ew; best = dot(dl, dl); carried = true;
                imp = qrot(qa, mf3(ubits(W[vo + 8u]), ubits(W[vo + 9u]), ubits(W[vo + 10u])));
              }
            }
            break;
          }
          h = (h + 1u) % S.AH;
        }
      }
      if (P.warm_scale > 0.0f) {
        float4 r6 = rows[o + 6u];
        f2 lw = mf2(r6.y, r6.z);
        if (carried) lw = mf2(dot(imp, t1), dot(imp, t2)) * P.warm_scale;
        float rad = fmx(rows[o + 2u].w * load, 0.0f);
        if (len(lw) > rad) lw = lw * (rad / len(lw));
        rows[o + 6u] = make_float4(r6.x, lw.x, lw.y, r6.w);
      }
      rows[o + PO] = mf4(fra, 2.0f);
      rows[o + PO + 1u] = mf4(frb, (float)k);
      rows[o + PO + 2u] = mf4(e, 0.0f);
      rows[o + PO + 3u] = mf4(qinv(qa, fra), __uint_as_float(pair));
    }
  }

  // Contact row idx for contact c (wgsl.js:2106-2269).
  // Contact torsion header of unit sp (wgsl.js:1526-1557; min_torsional_patch_radius): one spin
  // row per articulated unit about the normal of its touching coplanar cluster, the unit's rows
  // within 0.995 of the deepest row's normal and 2 mm of its plane; the radius is the members'
  // largest torsion radius. The header lives in the unit's first row: (Ma lin, mu),
  // (Ma ang, 1/K), (Mb lin, spin impulse), (Mb ang, r), (n, member).
  __device__ void build_torsion(uint32_t sp) const {
    const uint32_t ROWS = S.ROWS, TO = S.TO;
    float4* rows = S.rows;
    const uint32_t st = S.sched[S.S_USTART + sp];
    const uint32_t n = min(S.sched[S.S_USIZE + sp], S.MAXC - min(st, S.MAXC));
    if (n == 0u) return;
    const uint32_t pair = S.sched[S.S_UKEY + sp];
    const int a = (int)(pair & 0xffffu) - 1, b = (int)(pair >> 16u) - 1;
    const uint32_t L = st * ROWS;
    const bool art_u = (a >= 0 && bkind(a) >= 2u) || (b >= 0 && bkind(b) >= 2u);
    uint32_t seed = st;
    for (uint32_t i = st; i < st + n; i++)
      if (rows[i * ROWS + 1u].w < rows[seed * ROWS + 1u].w) seed = i;
    const f3 ns = v3(rows[seed * ROWS]), ps = v3(rows[seed * ROWS + TO + 4u]);
    float r = 0.0f;
    for (uint32_t i = st; i < st + n; i++) {
      const uint32_t o = i * ROWS;
      const bool member = art_u && rows[o + 6u].w <= 0.0f && dot(v3(rows[o]), ns) >= 0.995f &&
                          fabsf(dot(v3(rows[o + TO + 4u]) - ps, ns)) <= 0.002f;
      if (member) r = fmx(r, rows[o + TO + 3u].w);
      rows[o + TO + 4u].w = member ? 1.0f : 0.0f;
    }
    const float mu = rows[seed * ROWS + 2u].w;
    if (r <= 0.0f || mu <= 0.0f) { rows[L + TO] = make_float4(0, 0, 0, 0); return; }
    f3 Ma[2], Mb[2];
    response(a, sp3(0.0f), -ns, Ma);
    response(b, sp3(0.0f), ns, Mb);
    const float k = dot(-ns, Ma[1]) + dot(ns, Mb[1]);
    const float lead = rows[L + TO + 4u].w;
    rows[L + TO] = mf4(Ma[0], mu);
    rows[L + TO + 1u] = mf4(Ma[1], k > 1e-12f ? 1.0f / (k + S.F_CFM) : 0.0f);
    rows[L + TO + 2u] = mf4(Mb[0], 0.0f);
    rows[L + TO + 3u] = mf4(Mb[1], r);
    rows[L + TO + 4u] = mf4(ns, lead);
  }

  // row_count (wgsl.js:1507-1514): the rows a contact point solves (normal, a friction pair unless
  // it is a patch member, the angular three), for the longest-first color order.
  __device__ uint32_t row_count(uint32_t row) const {
    const float4* rows = S.rows;
    const uint32_t o = row * S.ROWS;
    uint32_t n = 1u;
    const bool member = S.EXTRA == 1u && rows[o + S.PO].w == 0.0f;
    if (rows[o + 2u].w > 0.0f && !member) n += 2u;
    if (S.ANG == 1u && (rows[o + 19u].x > 0.0f || rows[o + 19u].y > 0.0f)) n += 3u;
    return min(n, 7u);
  }
  __device__ void build_row(uint32_t idx, uint32_t c) const {
    const uint32_t ROWS = S.ROWS, PO = S.PO;
    float4* rows = S.rows;
    float4 c0 = S.con[c * 5u], c1 = S.con[c * 5u + 1u], cmeta = S.con[c * 5u + 2u];
    int a = f2i(cmeta.x), b = f2i(cmeta.y);
    uint32_t key = max(f2u(cmeta.z) | (f2u(cmeta.w) << 16u), 1u);
    f3 p = v3(c0), n = v3(c1);
    float phi = c0.w;
    float mu = phi <= S.F_FGAP ? c1.w * S.F_FSCALE : 0.0f;
    f3 t1 = cross(n, mf3(1.0f, 0.0f, 0.0f));
    if (dot(t1, t1) < 0.1f) t1 = cross(n, mf3(0.0f, 1.0f, 0.0f));
    t1 = nrm(t1);
    f3 t2 = cross(n, t1);
    f3 ca = sp3(0.0f), cb = sp3(0.0f);
    if (a >= 0) ca = v3(S.pos[a]);
    if (b >= 0) cb = v3(S.pos[b]);
    float half = S.SHARED == 1u ? 0.0f : 0.5f * phi;
    f3 ra = (p - n * half) - ca, rb = (p + n * half) - cb;
    f3 fa = ra, fb = rb;
    if (S.FSHARED == 1u) { fa = p - ca; fb = p - cb; }
    uint32_t o = idx * ROWS;
    f3 dirs[3] = {n, t1, t2};
    f3 Ma[3][2], Mb[3][2];
    for (uint32_t r = 0; r < 3u; r++) {
      f3 d = dirs[r];
      f3 aa = r == 0u ? ra : fa, ab = r == 0u ? rb : fb;
      response(a, -d, -cross(aa, d), Ma[r]);
      response(b, d, cross(ab, d), Mb[r]);
      rows[o + 7u + r * 4u] = mf4(Ma[r][0], 0.0f);
      rows[o + 8u + r * 4u] = mf4(Ma[r][1], 0.0f);
      rows[o + 9u + r * 4u] = mf4(Mb[r][0], 0.0f);
      rows[o + 10u + r * 4u] = mf4(Mb[r][1], 0.0f);
    }
    float K[9];
    for (uint32_t r = 0; r < 3u; r++)
      for (uint32_t s = 0; s < 3u; s++) {
        f3 d = dirs[r];
        f3 aa = r == 0u ? ra : fa, ab = r == 0u ? rb : fb;
        K[r * 3u + s] = ((dot(-d, Ma[s][0]) + dot(-cross(aa, d), Ma[s][1])) + dot(d, Mb[s][0])) + dot(cross(ab, d), Mb[s][1]);
      }
    if (S.EXTRA == 1u) {
      rows[o + PO] = mf4(fa, 1.0f);
      rows[o + PO + 1u] = mf4(fb, 0.0f);
      rows[o + PO + 2u] = mf4(p, 0.0f);
    }
    if (S.TORS == 1u) {
      rows[o + S.TO + 3u] = make_float4(0.0f, 0.0f, 0.0f, S.con[c * 5u + 3u].w);
      rows[o + S.TO + 4u] = mf4(p, 0.0f);
    }
    if (S.FMODE > 0u) {
      rows[o + S.FMO] = make_float4(K[0], 0.5f * (K[1] + K[3]), 0.5f * (K[2] + K[6]), 0.0f);
      rows[o + S.FMO + 1u] = make_float4(K[4], 0.5f * (K[5] + K[7]), K[8], 0.0f);
    }
    float kscale = fmx((K[0] + K[4]) + K[8], 1e-30f);
    float effn = 0.0f;
    if (K[0] > 1e-6f * kscale && K[0] > 1e-12f) effn = 1.0f / (K[0] + S.F_CFM);
    float k00 = (K[4] + 1e-6f * kscale) + S.F_CFM, k01 = 0.5f * (K[5] + K[7]), k11 = (K[8] + 1e-6f * kscale) + S.F_CFM;
    float det = k00 * k11 - k01 * k01;
    float rhs = phi < 0.0f ? fmx((P.beta * phi) / P.dt, -depen_cap(a, b)) : (S.F_SPEC * phi) / P.dt;
    float e = S.con[c * 5u + 3u].x;
    bool bounce = false;
    if (e > 0.0f) {
      f3 ta0[2], tb0[2];
      pre_twist(a, ta0);
      pre_twist(b, tb0);
      float vn0 = dot(n, (tb0[0] + cross(tb0[1], rb)) - (ta0[0] + cross(ta0[1], ra)));
      bounce = rest_fires(e, phi, vn0);
      if (bounce) rhs = e * vn0;
    }
    float ln;
    f3 lf;
    warm_lookup(key, &ln, &lf);
    f2 lt = mf2(dot(lf, t1), dot(lf, t2));
    float lim = mu * ln;
    float lm = len(lt);
    if (lm > lim) lt = lt * (lim / fmx(lm, 1e-12f));
    float effc = effn, rhsc = rhs;
    if (S.COMPL == 1u) {
      // contact_compliance (wgsl.js:2194-2206): a spring-damper normal row; the pair's series
      // stiffness and summed damping are split over the unit's kept points.
      const float4 kc4 = S.con[c * 5u + 4u];
      const float nk = (float)max(S.sched[S.S_USIZE + S.sched[S.S_RUNIT + idx]], 1u);
      const f2 kc = mf2(kc4.x / nk, kc4.y / nk);
      float gam = 0.0f;
      if (kc.x > 0.0f) {
        float ce = phi <= 0.0f ? kc.y : 0.0f;
        float den = P.dt * kc.x + ce;
        gam = 1.0f / (P.dt * den);
        rhsc = (kc.x * phi) / den;
        if (effn > 0.0f) effc = 1.0f / (1.0f / effn + gam);
      }
      rows[o + S.CO] = make_float4(gam, 0.0f, 0.0f, 0.0f);
    }
    rows[o + 0u] = mf4(n, effc);
    rows[o + 1u] = mf4(t1, rhsc);
    rows[o + 2u] = mf4(t2, mu);
    rows[o + 3u] = mf4(ra, (float)(key & 0xffffu));
    rows[o + 4u] = mf4(rb, (float)(key >> 16u));
    float wrow = row_weight(phi);
    if (wrow < 1.0f && ((a >= 0 && bkind(a) == 2u) || (b >= 0 && bkind(b) == 2u))) {
      f3 ua[2], ub[2];
      response(a, -n, -cross(ra, n), ua, true);
      response(b, n, cross(rb, n), ub, true);
      float du = ((dot(-n, ua[0]) + dot(-cross(ra, n), ua[1])) + dot(n, ub[0])) + dot(cross(rb, n), ub[1]);
      if (du > 0.0f && K[0] != du) wrow = (wrow * K[0]) / (wrow * K[0] + (1.0f - wrow) * du);
    }
    rows[o + 5u] = make_float4(k11 / det, -k01 / det, k00 / det, bounce ? 1.0f : wrow);
    rows[o + 6u] = make_float4(ln, lt.x, lt.y, bounce ? 1e30f : phi);
    if (S.ANG == 1u) {
      // Torsional (about n) and rolling (about t1, t2) rows of free bodies (wgsl.js:2223-2243):
      // angular-only Jacobians, the spin row's 1 / K and the rolling pair's inverse 2x2 block.
      const float4 mat = S.con[c * 5u + 3u];
      f3 MA[3][2], MB[3][2];
      for (uint32_t r = 0; r < 3u; r++) {
        const f3 d = dirs[r];
        response(a, sp3(0.0f), -d, MA[r]);
        response(b, sp3(0.0f), d, MB[r]);
        rows[o + 22u + r * 4u] = mf4(MA[r][0], 0.0f);
        rows[o + 23u + r * 4u] = mf4(MA[r][1], 0.0f);
        rows[o + 24u + r * 4u] = mf4(MB[r][0], 0.0f);
        rows[o + 25u + r * 4u] = mf4(MB[r][1], 0.0f);
      }
      float KA[9];
      for (uint32_t r = 0; r < 3u; r++)
        for (uint32_t s3 = 0; s3 < 3u; s3++) KA[r * 3u + s3] = dot(-dirs[r], MA[s3][1]) + dot(dirs[r], MB[s3][1]);
      const float ks = fmx(KA[0], 1e-12f);
      const float r00 = KA[4] + 1e-9f, r01 = 0.5f * (KA[5] + KA[7]), r11 = KA[8] + 1e-9f;
      const float rd = r00 * r11 - r01 * r01;
      rows[o + 19u] = make_float4(mat.y, mat.z, KA[0] > 1e-12f ? 1.0f / ks : 0.0f, 0.0f);
      rows[o + 20u] = make_float4(r11 / rd, -r01 / rd, r00 / rd, 0.0f);
      rows[o + 21u] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
      if (S.ANG_ART == 1u) {
        // The raw 5x5 response of (t1, t2, spin, roll1, roll2), upper triangle row by row, for the
        // articulated angular block (wgsl.js:2244-2267): row x's Jacobian against row y's response.
        f3 JA[5][2], JB[5][2], RA[5][2], RB[5][2];
        for (uint32_t q = 0; q < 2u; q++) {
          const f3 d = dirs[q + 1u];
          JA[q][0] = -d; JA[q][1] = -cross(fa, d);
          JB[q][0] = d; JB[q][1] = cross(fb, d);
          RA[q][0] = Ma[q + 1u][0]; RA[q][1] = Ma[q + 1u][1];
          RB[q][0] = Mb[q + 1u][0]; RB[q][1] = Mb[q + 1u][1];
        }
        for (uint32_t q = 0; q < 3u; q++) {
          JA[q + 2u][0] = sp3(0.0f); JA[q + 2u][1] = -dirs[q];
          JB[q + 2u][0] = sp3(0.0f); JB[q + 2u][1] = dirs[q];
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
        for (uint32_t q = 0; q < 4u; q++)
          rows[o + S.EO + q] = make_float4(Hu[q * 4u], Hu[q * 4u + 1u], Hu[q * 4u + 2u], Hu[q * 4u + 3u]);
      }
    }
  }

  // Dense row of a same-articulation contact (wgsl.js:2370-2444). scr: JDIM + 2 NDA + 18 MAXLP floats.
  __device__ void dense_row(uint32_t slot, uint32_t c, Lane scr) const {
    const uint32_t NDA = S.NDA, DHDR = S.DHDR, DPS = S.DPS;
    float* A = S.art;
    float4 c0 = S.con[c * 5u], c1 = S.con[c * 5u + 1u], cmeta = S.con[c * 5u + 2u];
    int a = f2i(cmeta.x), b = f2i(cmeta.y);
    uint32_t key = max(f2u(cmeta.z) | (f2u(cmeta.w) << 16u), 1u);
    f3 p = v3(c0), n = v3(c1);
    float phi = c0.w;
    float mu = phi <= S.F_FGAP ? c1.w * S.F_FSCALE : 0.0f;
    f3 t1 = cross(n, mf3(1.0f, 0.0f, 0.0f));
    if (dot(t1, t1) < 0.1f) t1 = cross(n, mf3(0.0f, 1.0f, 0.0f));
    t1 = nrm(t1);
    f3 t2 = cross(n, t1);
    uint32_t art_id = (uint32_t)bart(a);
    uint4 ai = ar.info(art_id);
    Lane J = scr;
    Lane Y = scr + 3u * NDA;
    Lane gs = Y + 3u * NDA;
    for (uint32_t k = 0; k < 3u * NDA; k++) { J[k] = 0.0f; Y[k] = 0.0f; }
    ar.gen_jac((uint32_t)blink(b), p, 1.0f, n, t1, t2, ai.z, J);
    ar.gen_jac((uint32_t)blink(a), p, -1.0f, n, t1, t2, ai.z, J);
    uint32_t o = S.A_DENSE + slot * DPS;
    float K[9];
    // Row r's right-hand side is J row r (zero beyond the articulation's dofs, as gen_jac leaves it).
    ar.solve_gen3(art_id, J, Y, gs);
    for (uint32_t r = 0; r < 3u; r++) {
      const Lane y = Y + r * NDA;
      for (uint32_t k = 0; k < ai.w; k++) {
        A[o + DHDR + r * NDA + k] = J[r * NDA + k];
        A[o + DHDR + 3u * NDA + r * NDA + k] = y[k];
      }
      for (uint32_t s2 = 0; s2 < 3u; s2++) {
        float acc = 0.0f;
        for (uint32_t k = 0; k < ai.w; k++) acc += J[s2 * NDA + k] * y[k];
        K[s2 * 3u + r] = acc;
      }
    }
    float kscale = fmx((K[0] + K[4]) + K[8], 1e-30f);
    float effn = 0.0f;
    if (K[0] > 1e-6f * kscale && K[0] > 1e-12f) effn = 1.0f / (K[0] + S.F_CFM);
    float k00 = (K[4] + 1e-6f * kscale) + S.F_CFM, k01 = 0.5f * (K[5] + K[7]), k11 = (K[8] + 1e-6f * kscale) + S.F_CFM;
    float det = k00 * k11 - k01 * k01;
    float rhs = phi < 0.0f ? fmx((P.beta * phi) / P.dt, -depen_cap(a, b)) : (S.F_SPEC * phi) / P.dt;
    float e = S.con[c * 5u + 3u].x;
    bool bounce = false;
    if (e > 0.0f) {
      float vn0 = 0.0f;
      for (uint32_t k = 0; k < ai.w; k++) vn0 += J[k] * A[S.A_QD + ai.z + k];
      bounce = rest_fires(e, phi, vn0);
      if (bounce) rhs = e * vn0;
    }
    float ln;
    f3 lf;
    warm_lookup(key, &ln, &lf);
    f2 lt = mf2(dot(lf, t1), dot(lf, t2));
    if (len(lt) > mu * ln) lt = lt * ((mu * ln) / fmx(len(lt), 1e-12f));
    A[o] = (float)art_id; A[o + 1u] = (float)(key & 0xffffu); A[o + 2u] = (float)(key >> 16u); A[o + 3u] = mu;
    A[o + 4u] = rhs; A[o + 5u] = effn;
    A[o + 6u] = k11 / det; A[o + 7u] = -k01 / det; A[o + 8u] = k00 / det;
    A[o + 9u] = ln; A[o + 10u] = lt.x; A[o + 11u] = lt.y;
    ar.ast3(o + 12u, t1); ar.ast3(o + 15u, t2); ar.ast3(o + 18u, n);
    A[o + 21u] = 0.0f;
    A[o + 24u] = bounce ? 1.0f : row_weight(phi);
    A[o + 22u] = bounce ? 1e30f : phi;
  }
  // Bilateral dense block (wgsl.js:1351-1369).
  __device__ void put_bilateral(uint32_t o, uint32_t art_id, const float* J, uint32_t nb, f3 rhs, float* scr) const {
    const uint32_t NDA = S.NDA;
    float* A = S.art;
    uint4 ai = ar.info(art_id);
    float* tau = scr;
    float* y = scr + NDA;
    float* gs = y + NDA;
    for (uint32_t r = 0; r < nb; r++) {
      for (uint32_t k = 0; k < NDA; k++) { tau[k] = k < ai.w ? J[r * NDA + k] : 0.0f; y[k] = 0.0f; }
      ar.solve_gen(art_id, tau, y, gs);
      float kk = 0.0f;
      for (uint32_t k = 0; k < ai.w; k++) {
        A[o + S.DHDR + r * NDA + k] = J[r * NDA + k];
        A[o + S.DHDR + 3u * NDA + r * NDA + k] = y[k];
        kk += J[r * NDA + k] * y[k];
      }
      A[o + 5u + r] = kk > 1e-12f ? 1.0f / kk : 0.0f;
    }
    A[o] = (float)art_id; A[o + 1u] = 0.0f; A[o + 2u] = 0.0f;
    A[o + 4u] = rhs.x; A[o + 22u] = rhs.y; A[o + 23u] = rhs.z;
    A[o + 9u] = 0.0f; A[o + 10u] = 0.0f; A[o + 11u] = 0.0f;
    A[o + 21u] = (float)nb;
  }
};

// Sleep islands (wgsl.js:1371-1457), by the whole block. Islands are nodes (free bodies,
// articulations) joined by contacts: roots hook under the smaller root (atomicMin) and paths are
// compressed until a round joins nothing, so each node ends pointing at its island's lowest node
// whatever the order of the atomics. A round that changes something joins two islands, so NN + 1
// rounds always suffice; the loop is bounded by that. Island flags OR onto the root: 1 supported
// (touches static geometry, or a fixed-base articulation), 2 vetoed (moving, driven, loop or
// mimic owner; picking is not carried), 4 some member younger than the quiet time. Ages and the
// asleep flags are in A_SLP (age, asleep) per node; S_META + 5 counts the sleeping nodes.
__device__ __forceinline__ void sleep_islands(const Prep& pr, uint32_t tid, uint32_t nt) {
  const SceneDev& S = pr.S;
  const Art& ar = pr.ar;
  const uint32_t NN = S.NB + S.NA;
  uint32_t* uf = S.sched + S.S_UF;
  uint32_t* uff = S.sched + S.S_UFF;
  float* A = S.art;
  __shared__ uint32_t changed;
  for (uint32_t n = tid; n < NN; n += nt) { uf[n] = n; uff[n] = 0u; }
  if (tid == 0u) S.sched[S.S_META + 5u] = 0u;
  __syncthreads();
  const uint32_t nc = min(S.counters[1], S.MAXC);
  for (uint32_t c = tid; c < nc; c += nt) {
    float4 m = S.con[c * 5u + 2u];
    int na = pr.bnode(f2i(m.x)), nb = pr.bnode(f2i(m.y));
    if ((na < 0 || nb < 0) && max(na, nb) >= 0 && S.con[c * 5u].w <= 1e-5f) atomicOr(&uff[max(na, nb)], 1u);
  }
  // Parent links change under other threads' atomics: read them volatile.
  auto find = [&](uint32_t n) {
    const volatile uint32_t* v = uf;
    uint32_t r = n;
    for (uint32_t k = 0; k < NN; k++) {
      uint32_t p = v[r];
      if (p == r) break;
      r = p;
    }
    return r;
  };
  for (uint32_t round = 0; round <= NN; round++) {
    if (tid == 0u) changed = 0u;
    __syncthreads();
    for (uint32_t c = tid; c < nc; c += nt) {
      float4 m = S.con[c * 5u + 2u];
      int na = pr.bnode(f2i(m.x)), nb = pr.bnode(f2i(m.y));
      if (na < 0 || nb < 0) continue;
      uint32_t ra = find((uint32_t)na), rb = find((uint32_t)nb);
      if (ra != rb) { atomicMin(&uf[max(ra, rb)], min(ra, rb)); changed = 1u; }
    }
    __syncthreads();
    for (uint32_t n = tid; n < NN; n += nt) {
      uint32_t r = find(n);
      reinterpret_cast<volatile uint32_t*>(uf)[n] = r;
    }
    __syncthreads();
    const bool more = changed != 0u;
    __syncthreads();  // every thread has read the flag before thread 0 clears it
    if (!more) break;
  }
  for (uint32_t n = tid; n < NN; n += nt) {
    bool moving = false, fixed = false, veto = false;
    if (n < S.NB) {
      if (pr.bkind((int)n) != 1u) continue;
      if (A[S.A_SLP + n * 4u + 1u] < 0.5f)
        moving = len(v3(S.lv[n])) > S.F_SLEEP_LIN || len(v3(S.av[n])) > S.F_SLEEP_ANG;
    } else {
      const uint32_t a = n - S.NB;
      uint4 ai = ar.info(a);
      fixed = ar.ltype(ai.x) != 4u;
      for (uint32_t k = 0; k < ai.y; k++) {
        SVec v = ar.ldsv(ar.lo(ai.x + k) + L_V);
        if (A[S.A_SLP + n * 4u + 1u] < 0.5f && (len(v.l) > S.F_SLEEP_LIN || len(v.a) > S.F_SLEEP_ANG)) moving = true;
      }
      for (uint32_t d = ai.z; d < ai.z + ai.w; d++) {
        float4 dr = ar.dof_drive(d);
        if (dr.y > 0.0f || dr.z > 0.0f) veto = true;
      }
      if (S.su[S.SU_ACON + a] != 0u) veto = true;
    }
    uint32_t f = (fixed ? 1u : 0u) | ((moving || veto) ? 2u : 0u) | (uff[n] & 1u);
    atomicOr(&uff[uf[n]], f);
  }
  __syncthreads();
  // Ages: reset in vetoed or unsupported islands, else grown to the quiet time.
  for (uint32_t n = tid; n < NN; n += nt) {
    if (n < S.NB && pr.bkind((int)n) != 1u) continue;
    uint32_t r = uf[n];
    uint32_t f = reinterpret_cast<volatile uint32_t*>(uff)[r];
    float age = A[S.A_SLP + n * 4u];
    if ((f & 2u) != 0u || (f & 1u) == 0u) age = 0.0f;
    else age = fmn(age + pr.P.dt, S.F_SLEEP_TIME);
    A[S.A_SLP + n * 4u] = age;
    if (age < S.F_SLEEP_TIME) atomicOr(&uff[r], 4u);
  }
  __syncthreads();
  for (uint32_t n = tid; n < NN; n += nt) {
    if (n < S.NB && pr.bkind((int)n) != 1u) continue;
    bool s = (uff[uf[n]] & 4u) == 0u;
    A[S.A_SLP + n * 4u + 1u] = s ? 1.0f : 0.0f;
    if (s) atomicAdd(&S.sched[S.S_META + 5u], 1u);
  }
}

// Prepare of scene sc by a team (all its threads): the calling block (TEAM false, the batched
// path), or every block of a cooperative launch on a batch of one large scene (TEAM true). In a
// team launch the passes over articulations, contacts, units and rows are spread over all blocks
// and meet at grid barriers; the passes built on block-wide scans and shared counters (contact
// classification, the unit scan, sleep islands, coloring and the color buckets) run on block 0
// exactly as in the one-block kernel, and their counts reach the other blocks through the team's
// words (B.team_bar[4..7]). Nothing is staged in shared memory; the per-thread scratch serves the
// first TSCR_T threads of the team (all threads of a block).
template <bool F64, bool TEAM>
__device__ __forceinline__ void prepare_scene(const BatchDev& B, uint32_t sc, Team<TEAM> tm) {
  extern __shared__ float4 psm4[];  // prep_smem_layout: link blocks, coloring
  __shared__ uint32_t stmp[40];
  __shared__ Params Ps;
  __shared__ SceneDev Ss;  // the scene's offsets and sizes, read everywhere in the serial passes
  const uint32_t tid = tm.rank(), nt = tm.size();
  const bool b0 = !TEAM || blockIdx.x == 0u;  // this block runs the block-wide passes
  if (B.active[sc] == 0u) return;  // not stepping in this frame (serving loop)
  copy_scene(Ss, B.scenes[sc]);
  const SceneDev& S = Ss;
  if (threadIdx.x == 0u) Ps = *B.scenes[sc].params;
  uint8_t* pb = reinterpret_cast<uint8_t*>(psm4);
  const uint32_t stage = TEAM ? 0u : S.stage;
  const PrepSmem lay = prep_smem_layout(stage, S.NL, S.NB, S.NCOLW, S.NCOL);
  const bool staged = (stage & STAGE_LINKS) != 0u;
  float* lb = staged ? reinterpret_cast<float*>(pb + lay.links) : S.art + S.A_LINK;
  // Link blocks into shared memory with one bulk copy (A_LINK is 16-byte aligned).
  __shared__ __align__(8) uint64_t stage_bar;
  if (staged && !stage_to_shared(lb, S.art + S.A_LINK, 4u * S.NL * LBLK, &stage_bar, B.wait_limit)) {
    if (threadIdx.x == 0u) atomicCAS(B.error, 0u, (uint32_t)ERR_STAGE_TIMEOUT);
    return;  // the whole block: the result above is the same in every thread
  }
  __syncthreads();
  const Params& P = Ps;
  Prep pr(S, P, lb);
  const Art& ar = pr.ar;
  float* A = S.art;
  uint32_t* sch = S.sched;
  // Threads that own a scratch slice: every thread of a block, the first TSCR_T of a team.
  const uint32_t sn = TEAM ? min(nt, S.TSCR_T) : nt;
  float* tscr = S.tscr + (size_t)tid * S.TSCR;  // dereferenced only by threads below sn

  // Phase 0: clear this substep's warm table halves and scratch; drive targets.
  const uint32_t wbase = (1u - P.parity) * S.WH;
  for (uint32_t i = tid; i < S.WH; i += nt) { S.warm_tab[wbase + i] = 0u; sch[S.S_WWIN + i] = 0u; }
  if (S.PATCH == 1u)
    for (uint32_t i = tid; i < S.AH; i += nt) S.warm_tab[10u * S.WH + (1u - P.parity) * S.AH + i] = 0u;
  for (uint32_t i = tid; i < S.NB * S.NCOLW; i += nt) sch[S.S_WMASK + i] = 0u;
  for (uint32_t i = tid; i < S.NCOL + 2u; i += nt) sch[S.S_WCOUNT + i] = 0u;
  for (uint32_t i = tid; i < S.NB; i += nt) sch[S.S_LINKHIT + i] = 0u;
  for (uint32_t i = tid; i < S.NL; i += nt) sch[S.S_JSPLIT + i] = 0u;
  for (uint32_t d = tid; d < P.driven; d += nt) {
    float ramp = ((P.phase + ((float)P.substep + 0.5f) * P.dt) * 60.0f) - 0.5f;
    float frame = clmp(S.TGT_HELD == 1u ? P.phase * 60.0f : ramp, 0.0f, (float)(P.path_frames - 1u));
    uint32_t a = f2u(frame);
    uint32_t b = min(a + 1u, P.path_frames - 1u);
    RO<float> path{reinterpret_cast<const float*>(S.sf.p + S.SF_PATH)};
    float pa = path[a * P.driven + d], pb = path[b * P.driven + d];
    float t = frame - (float)a;
    float value = pa * (1.0f - t) + pb * t;
    if (d < P.integral_count) {
      if (P.substep == 0u) {
        float err = clmp(value - A[S.A_Q + d], -0.08f, 0.08f);
        A[S.A_INT + d] = clmp(A[S.A_INT + d] + (3.0f * P.frame_dt) * err, -0.12f, 0.12f);
      }
      value += A[S.A_INT + d];
    }
    A[S.A_TGT + d] = value;
  }
  if (S.CTRL_KIND == 1u && tid == 0u) {
    float4 c = S.sf[S.SF_CTRL];
    A[S.A_TGTV + S.CTRL_B] = c.y * clmp(A[S.A_Q + S.CTRL_A] / c.x, 0.0f, 1.0f);
  }
  if (S.SLEEP == 1u) {
    if (TEAM) tm.sync();  // the clears and targets above, from every block
    if (b0) sleep_islands(pr, threadIdx.x, blockDim.x);
  }
  tm.sync();
  // Joint-limit gating, listed joint rows, FK and factorisation per articulation.
  auto gate = [&](uint32_t a) {
    uint4 ai = ar.info(a);
    // Joint velocity limits (wgsl.js:1829-1854): scale the articulation's scalar dof speeds so the
    // most exceeded limit is met, then mark the dofs near their limit (rows exist only there).
    // A driven dof under drive rows with the fused clamp is not scaled (artwgsl.js:54).
    auto fused = [&](uint32_t d) {
      const float4 dr = ar.dof_drive(d);
      return S.DRIVE_ROWS == 1u && S.FUSE_VLIM == 1u && (dr.y > 0.0f || dr.z > 0.0f);
    };
    if (S.VLIM_ON == 1u) {
      float ratio = 1.0f;
      for (uint32_t k = 0; k < ai.w; k++) {
        uint32_t d = ai.z + k;
        float vl = ar.dof_passive(d).z;
        if (vl < 0.0f || fused(d)) continue;
        float sp = fabsf(A[S.A_QD + d]);
        if (sp > vl) ratio = fmn(ratio, vl / sp);
      }
      if (ratio < 1.0f)
        for (uint32_t k = 0; k < ai.w; k++)
          if (ar.scalar_dof(ai.z + k) && !fused(ai.z + k)) A[S.A_QD + ai.z + k] *= ratio;
      bool any = false;
      for (uint32_t k = 0; k < ai.w; k++) {
        uint32_t d = ai.z + k;
        bool on = fabsf(A[S.A_QD + d]) >= S.F_VLIM_FRAC * ar.dof_passive(d).z;
        A[S.A_VLG + d] = on ? 1.0f : 0.0f;
        any = any || (on && ar.dof_passive(d).z >= 0.0f && ar.scalar_dof(d));
      }
      A[S.A_AVL + a] = any ? 1.0f : 0.0f;
    }
    uint32_t n = 0u;
    for (uint32_t k = 0; k < ai.w; k++) {
      uint32_t d = ai.z + k;
      float4 lim = ar.dof_limit(d);
      bool on = false;
      if (lim.z > 0.5f) {
        uint32_t l = f2u(lim.w);
        float q = A[S.A_Q + ar.lqs(l) + d - ar.ldof(l)];
        float g = S.F_JL_GAP + (S.F_JL_SPEED * P.dt) * fabsf(A[S.A_QD + d]);
        on = q <= lim.x + g || q >= lim.y - g;
      }
      A[S.A_LG + d] = on ? 1.0f : 0.0f;
      const float4 drv = ar.dof_drive(d);
      bool row = on || ar.dof_passive(d).y > 0.0f || S.JFL == 1u || (S.DRIVE_ROWS == 1u && (drv.y > 0.0f || drv.z > 0.0f));
      if (row && ar.scalar_dof(d)) { A[S.A_RL + ai.z + n] = (float)d; n++; }
    }
    A[S.A_RLN + a] = (float)n;
  };
  auto factor = [&](uint32_t a) {
    if (F64 && S.ART_F64 == 1u) ar.factor<true>(a, P);
    else ar.factor<false>(a, P);
  };
  if (S.NA <= (nt >> 5u)) {
    // Few articulations: a warp each, so the FK's per-link trigonometry and outputs run across
    // lanes and only the pose chain is serial.
    const uint32_t lane = tid & 31u;
    for (uint32_t a = tid >> 5u; a < S.NA; a += nt >> 5u) {
      if (lane == 0u) gate(a);
      __syncwarp();
      ar.fk_warp(a, lane);
      if (lane == 0u) factor(a);
      __syncwarp();
    }
  } else {
    for (uint32_t a = tid; a < S.NA; a += nt) {
      gate(a);
      ar.fk(a);
      factor(a);
    }
  }
  // Phase 1: classify the sorted contacts; units are runs of one body pair (block-wide scans: one
  // block).
  const uint32_t nc = min(S.counters[1], S.MAXC);
  uint32_t nu = 0u, nl = 0u, ndc = 0u;
  if (b0) {
    const uint32_t tid = threadIdx.x, nt = blockDim.x;
    const uint32_t ch = (nc + nt - 1u) / nt;
    const uint32_t c_lo = min(tid * ch, nc), c_hi = min(c_lo + ch, nc);
    uint32_t heads = 0u, listed = 0u, dn = 0u;
    auto pair_of = [&](uint32_t c) {
      float4 m = S.con[c * 5u + 2u];
      return (uint32_t)(f2i(m.x) + 1) | ((uint32_t)(f2i(m.y) + 1) << 16u);
    };
    auto is_dense = [&](uint32_t c) {
      float4 m = S.con[c * 5u + 2u];
      int a = f2i(m.x), b = f2i(m.y);
      return a >= 0 && b >= 0 && pr.bkind(a) == 2u && pr.bkind(b) == 2u && pr.bart(a) == pr.bart(b);
    };
    // Contacts between sleeping (or static) sides make no rows (wgsl.js:1905). A same-articulation
    // contact is asleep exactly when its articulation is, so every dense contact left has rows.
    auto asleep = [&](uint32_t c) {
      if (S.SLEEP == 0u) return false;
      float4 m = S.con[c * 5u + 2u];
      return pr.pair_asleep(f2i(m.x), f2i(m.y));
    };
    for (uint32_t c = c_lo; c < c_hi; c++) {
      if (asleep(c)) continue;
      if (is_dense(c)) { dn++; continue; }
      listed++;
      if (c == 0u || pair_of(c - 1u) != pair_of(c)) heads++;
    }
    uint32_t ubase = block_excl_scan(heads, stmp, &nu);
    uint32_t lbase = block_excl_scan(listed, stmp, &nl);
    uint32_t dbase = block_excl_scan(dn, stmp, &ndc);
    {
      uint32_t unit = ubase, pos = lbase, ds = dbase;
      for (uint32_t c = c_lo; c < c_hi; c++) {
        if (asleep(c)) {
          sch[S.S_UNITOF + c] = 0xffffffffu;
          sch[S.S_DSLOT + c] = 0xffffffffu;
          continue;
        }
        if (is_dense(c)) {
          sch[S.S_UNITOF + c] = 0xffffffffu;
          sch[S.S_DSLOT + c] = ds++;
          continue;
        }
        sch[S.S_DSLOT + c] = 0xffffffffu;
        uint32_t pk = pair_of(c);
        if (c == 0u || pair_of(c - 1u) != pk) {
          sch[S.S_UKEY + unit] = pk;
          sch[S.S_USTART0 + unit] = pos;
          unit++;
        }
        sch[S.S_UNITOF + c] = unit - 1u;
        sch[S.S_CORDER + pos] = c;
        pos++;
        float4 m = S.con[c * 5u + 2u];
        int a = f2i(m.x), b = f2i(m.y);
        if (a >= 0 && pr.bkind(a) == 2u) sch[S.S_LINKHIT + a] = 1u;
        if (b >= 0 && pr.bkind(b) == 2u) sch[S.S_LINKHIT + b] = 1u;
      }
    }
    if (tid == 0u) sch[S.S_USTART0 + nu] = nl;
    if (TEAM && tid == 0u) { B.team_bar[4] = nu; B.team_bar[5] = nl; B.team_bar[6] = ndc; }
  }
  tm.sync();
  if (TEAM) { nu = B.team_bar[4]; nl = B.team_bar[5]; ndc = B.team_bar[6]; }
  for (uint32_t u = tid; u < nu; u += nt) sch[S.S_USIZE + u] = sch[S.S_USTART0 + u + 1u] - sch[S.S_USTART0 + u];
  // Phase 2: joint split, link responses of contact-bearing links, H^-1 diagonals.
  for (uint32_t l = tid; l < S.NL; l += nt) {
    if (sch[S.S_LINKHIT + ar.lbody(l)] == 0u) continue;
    int j = (int)l;
    while (j >= 0) { atomicAdd(&sch[S.S_JSPLIT + j], 1u); j = ar.lparent((uint32_t)j); }
  }
  tm.sync();
  {
    uint32_t* pth = (uint32_t*)tscr;
    uint32_t* cnt = pth + S.MAXPATH;
    float* ub = (float*)(cnt + S.MAXPATH);
    for (uint32_t l = tid; tid < sn && l < S.NL; l += sn) {
      if (sch[S.S_LINKHIT + ar.lbody(l)] == 0u) continue;
      uint32_t np = ar.path(l, pth);
      for (uint32_t i = 0; i < np; i++) cnt[i] = sch[S.S_JSPLIT + pth[i]];
      ar.response(l, cnt, pth, ub);
    }
    for (uint32_t d = tid; tid < sn && d < S.ND; d += sn) {
      float4 lim = ar.dof_limit(d);
      const float4 drv = ar.dof_drive(d);
      if (lim.z > 0.5f || ar.dof_passive(d).y > 0.0f || ar.dof_passive(d).z >= 0.0f ||
          S.sf[S.SF_DOF + d * 5u + 3u].w > 0.0f || (S.DRIVE_ROWS == 1u && (drv.y > 0.0f || drv.z > 0.0f))) {
        uint32_t l = f2u(lim.w);
        A[S.A_HINV + d] = ar.dof_hinv(l, d - ar.ldof(l), pth, ub);
      }
    }
  }
  // Phase 5: body-pair contact reduction over each unit's listed contacts.
  for (uint32_t p = tid; p < nl; p += nt) {
    uint32_t k[3], pk;
    float px, py, gap;
    pr.bp_contact(sch[S.S_CORDER + p], k, &px, &py, &gap, &pk);
    sch[S.S_RK0 + p] = k[0]; sch[S.S_RK1 + p] = k[1]; sch[S.S_RK2 + p] = k[2];
    uint32_t* bpc = sch + S.S_BPC + p * 4u;
    bpc[0] = __float_as_uint(px); bpc[1] = __float_as_uint(py); bpc[2] = __float_as_uint(gap); bpc[3] = pk;
  }
  tm.sync();
  for (uint32_t p = tid; p < nl; p += nt) {
    uint32_t st = sch[S.S_USTART0 + sch[S.S_UNITOF + sch[S.S_CORDER + p]]];
    uint32_t k0 = sch[S.S_RK0 + p], k1 = sch[S.S_RK1 + p], k2 = sch[S.S_RK2 + p];
    uint32_t lead = p;
    for (uint32_t m = st; m < p; m++)
      if (sch[S.S_RK2 + m] == k2 && sch[S.S_RK0 + m] == k0 && sch[S.S_RK1 + m] == k1) { lead = m; break; }
    sch[S.S_LEAD + p] = lead;
    for (uint32_t q = 0; q < 26u; q++) sch[S.S_SLOT + p * 26u + q] = 0u;
  }
  tm.sync();
  for (uint32_t p = tid; p < nl; p += nt) {
    const uint32_t* bpc = sch + S.S_BPC + p * 4u;
    uint32_t* sl = sch + S.S_SLOT + sch[S.S_LEAD + p] * 26u;
    for (uint32_t q = 0; q < 13u; q++) {
      uint32_t s_, id;
      Prep::bp_value(__uint_as_float(bpc[0]), __uint_as_float(bpc[1]), __uint_as_float(bpc[2]), bpc[3], q, &s_, &id);
      if (id != 0u) atomicMax(&sl[q * 2u], s_);
    }
  }
  tm.sync();
  for (uint32_t p = tid; p < nl; p += nt) {
    const uint32_t* bpc = sch + S.S_BPC + p * 4u;
    uint32_t* sl = sch + S.S_SLOT + sch[S.S_LEAD + p] * 26u;
    for (uint32_t q = 0; q < 13u; q++) {
      uint32_t s_, id;
      Prep::bp_value(__uint_as_float(bpc[0]), __uint_as_float(bpc[1]), __uint_as_float(bpc[2]), bpc[3], q, &s_, &id);
      if (id != 0u && s_ == sl[q * 2u]) atomicMax(&sl[q * 2u + 1u], id);
    }
  }
  tm.sync();
  for (uint32_t p = tid; p < nl; p += nt) {
    const uint32_t* bpc = sch + S.S_BPC + p * 4u;
    const uint32_t* sl = sch + S.S_SLOT + sch[S.S_LEAD + p] * 26u;
    bool win = false;
    for (uint32_t q = 0; q < 13u; q++) {
      uint32_t s_, id;
      Prep::bp_value(__uint_as_float(bpc[0]), __uint_as_float(bpc[1]), __uint_as_float(bpc[2]), bpc[3], q, &s_, &id);
      if (id != 0u && s_ == sl[q * 2u] && id == sl[q * 2u + 1u]) win = true;
    }
    sch[S.S_KEEP + p] = (win || S.COMPL == 1u) ? 1u : 0u;  // compliant contacts stay whole
  }
  tm.sync();
  for (uint32_t u = tid; u < nu; u += nt) {
    uint32_t n = sch[S.S_USIZE + u], st = sch[S.S_USTART0 + u], kept = 0u;
    for (uint32_t j = 0; j < n; j++)
      if (sch[S.S_KEEP + st + j] != 0u) { sch[S.S_KEPT + st + kept] = sch[S.S_CORDER + st + j]; kept++; }
    sch[S.S_USIZE + u] = kept;
    sch[S.S_USTART + u] = kept;
  }
  for (uint32_t c = tid; c < nc; c += nt) sch[S.S_ROWOF + c] = 0xffffffffu;
  tm.sync();
  uint32_t total = 0u;
  if (b0) {
    total = block_scan_array(sch + S.S_USTART, nu, stmp);
    if (threadIdx.x == 0u) {
      sch[S.S_USTART + nu] = total;
      if (TEAM) B.team_bar[7] = total;
    }
  }
  if (TEAM) {
    tm.sync();
    total = B.team_bar[7];
  }
  for (uint32_t u = tid; u < nu; u += nt) {
    uint32_t st = sch[S.S_USTART + u], st0 = sch[S.S_USTART0 + u];
    for (uint32_t j = 0; j < sch[S.S_USIZE + u]; j++) {
      uint32_t c = sch[S.S_KEPT + st0 + j];
      sch[S.S_RUNIT + st + j] = u;
      sch[S.S_RCON + st + j] = c;
      sch[S.S_ROWOF + c] = st + j;
    }
  }
  tm.sync();
  // Phase 6: rows, then friction patches.
  for (uint32_t idx = tid; idx < total; idx += nt) pr.build_row(idx, sch[S.S_RCON + idx]);
  tm.sync();
  if (S.TORS == 1u) {
    for (uint32_t u = tid; u < nu; u += nt) pr.build_torsion(u);
    tm.sync();
  }
  if (S.PATCH == 1u)
    for (uint32_t u = tid; u < nu; u += nt) pr.build_patch(u);
  tm.sync();
  // Phase 6c on one block (shared counters and block-wide scans); in a team launch the other
  // blocks go on to the dense rows, which do not read the colors.
  if (b0) {
    const uint32_t tid = threadIdx.x, nt = blockDim.x;
    // Phase 6c: greedy first-fit coloring of the rows in contact order (the reference's serial pass,
    // W:1254-1267, reproduced in parallel rounds below; the longest-first order keeps a serial pass),
    // with the per-body color masks (in shared memory when staged) and the color counts in shared
    // memory; then the rows bucketed by color in row order (warp 0, match/ballot ranks).
    {
      uint32_t* wcount = reinterpret_cast<uint32_t*>(pb + lay.wcount);
      uint32_t* wmask = (stage & STAGE_WMASK) ? reinterpret_cast<uint32_t*>(pb + lay.wmask) : sch + S.S_WMASK;
      const uint32_t NCOLW = S.NCOLW;
      for (uint32_t i = tid; i < S.NCOL + 2u; i += nt) wcount[i] = 0u;
      if (stage & STAGE_WMASK)
        for (uint32_t i = tid; i < S.NB * NCOLW; i += nt) wmask[i] = 0u;
      if (S.LONGEST_FIRST == 0u) {
        // First-fit in row order, in parallel rounds with the same colors (Jones-Plassmann with the
        // row index as priority). Every body keeps its rows in row order and a frontier, the first
        // of them not yet colored; rows on one body are colored in that order, so when a row is the
        // frontier of both its bodies every earlier row touching them has its color, and the body
        // masks hold exactly the colors the serial pass would see. Such rows share no body, so one
        // round colors all of them without conflicts. A round only looks at the bodies whose
        // frontier moved in the previous one (all bodies in the first): phase A finds the ready rows
        // among their frontier rows (a row whose two bodies both look at it is listed once), phase B
        // colors them, advances the frontiers and lists the moved bodies for the next round. A row
        // is found in the round its last frontier reaches it, since that body is on the list. Each
        // round colors at least the lowest uncolored row, so the rounds end.
        uint32_t* bstart = sch + S.S_BSTART;  // [NB + 1] each body's first list entry
        uint32_t* bpos = sch + S.S_BPOS;      // [NB] fill cursor, then frontier
        uint32_t* rdy = sch + S.S_BREADY;     // [NB] rows found ready in a round
        uint32_t* blist = sch + S.S_BLIST;    // [2 * MAXC] rows of each body
        uint32_t* rkey = sch + S.S_RKEY;      // [MAXC] body-pair key of each row
        uint32_t* rflag = sch + S.S_RFLAG;    // [MAXC] the row is on the ready list
        uint32_t* wl[2] = {sch + S.S_WL, sch + S.S_WL + S.NB};  // [2][NB] bodies to look at
        __shared__ uint32_t wl_n[2], rdy_n;
        const uint32_t NB = S.NB;
        for (uint32_t b = tid; b <= NB; b += nt) bstart[b] = 0u;
        if (tid == 0u) { wl_n[0] = 0u; wl_n[1] = 0u; rdy_n = 0u; }
        __syncthreads();
        for (uint32_t r = tid; r < total; r += nt) {
          const uint32_t key = sch[S.S_UKEY + sch[S.S_RUNIT + r]];
          rkey[r] = key;
          rflag[r] = 0u;
          const int a = (int)(key & 0xffffu) - 1, b = (int)(key >> 16u) - 1;
          if (a >= 0) atomicAdd(&bstart[a], 1u);
          if (b >= 0 && b != a) atomicAdd(&bstart[b], 1u);
        }
        __syncthreads();
        block_scan_array(bstart, NB + 1u, stmp);
        for (uint32_t b = tid; b < NB; b += nt) bpos[b] = bstart[b];
        __syncthreads();
        for (uint32_t r = tid; r < total; r += nt) {
          const uint32_t key = rkey[r];
          const int a = (int)(key & 0xffffu) - 1, b = (int)(key >> 16u) - 1;
          if (a >= 0) blist[atomicAdd(&bpos[a], 1u)] = r;
          if (b >= 0 && b != a) blist[atomicAdd(&bpos[b], 1u)] = r;
        }
        __syncthreads();
        for (uint32_t b = tid; b < NB; b += nt) {  // each body's rows in row order
          const uint32_t s0 = bstart[b], s1 = bstart[b + 1u];
          for (uint32_t i = s0 + 1u; i < s1; i++) {
            const uint32_t v = blist[i];
            uint32_t j = i;
            while (j > s0 && blist[j - 1u] > v) { blist[j] = blist[j - 1u]; j--; }
            blist[j] = v;
          }
          bpos[b] = s0;
          if (s1 > s0) wl[0][atomicAdd(&wl_n[0], 1u)] = b;
        }
        __syncthreads();
        uint32_t cur = 0u;
        for (uint32_t round = 0; round <= total; round++) {
          const uint32_t n = wl_n[cur];
          if (n == 0u) break;  // the same value in every thread (read after the last barrier)
          for (uint32_t i = tid; i < n; i += nt) {
            const uint32_t b = wl[cur][i];
            const uint32_t p = bpos[b];
            if (p >= bstart[b + 1u]) continue;
            const uint32_t r = blist[p];
            const uint32_t key = rkey[r];
            const int x = (int)(key & 0xffffu) - 1, y = (int)(key >> 16u) - 1;
            const int other = x == (int)b ? y : x;
            if (other >= 0 && other != (int)b && blist[bpos[other]] != r) continue;
            if (atomicExch(&rflag[r], 1u) == 0u) rdy[atomicAdd(&rdy_n, 1u)] = r;
          }
          __syncthreads();
          const uint32_t nr = rdy_n;
          if (tid == 0u) wl_n[cur ^ 1u] = 0u;
          __syncthreads();
          for (uint32_t k = tid; k < nr; k += nt) {
            const uint32_t r = rdy[k];
            const uint32_t key = rkey[r];
            const int a = (int)(key & 0xffffu) - 1, c = (int)(key >> 16u) - 1;
            uint32_t col = S.NCOL;
            for (uint32_t w = 0; w < NCOLW; w++) {
              uint32_t used = 0u;
              if (a >= 0) used |= wmask[(uint32_t)a * NCOLW + w];
              if (c >= 0) used |= wmask[(uint32_t)c * NCOLW + w];
              if (used != 0xffffffffu) {
                uint32_t kk = (uint32_t)__ffs(~used) - 1u;
                if (a >= 0) wmask[(uint32_t)a * NCOLW + w] |= 1u << kk;
                if (c >= 0) wmask[(uint32_t)c * NCOLW + w] |= 1u << kk;
                col = w * 32u + kk;
                break;
              }
            }
            sch[S.S_PCOL + r] = col;
            atomicAdd(&wcount[col], 1u);
            // Advance the frontiers; a body with rows left is looked at in the next round.
            if (a >= 0 && ++bpos[a] < bstart[a + 1u]) wl[cur ^ 1u][atomicAdd(&wl_n[cur ^ 1u], 1u)] = (uint32_t)a;
            if (c >= 0 && c != a && ++bpos[c] < bstart[c + 1u]) wl[cur ^ 1u][atomicAdd(&wl_n[cur ^ 1u], 1u)] = (uint32_t)c;
          }
          __syncthreads();
          if (tid == 0u) rdy_n = 0u;
          cur ^= 1u;
          __syncthreads();
        }
      }
      __syncthreads();
      if (S.LONGEST_FIRST == 1u && tid == 0u) {
        // propagation_color_order "longest_first" (wgsl.js:2331-2346): first-fit by row count first
        // (7 rows down to 1), then contact index. A unit's torsion row is its last row of its highest
        // color; that color + 1 is kept as PCOL of the unit's current pick, so it needs no array.
        for (uint32_t u = 0; u < nu; u++) sch[S.S_UTP + u] = 0xffffffffu;
        for (uint32_t lp = 0; lp < 8u; lp++)
          for (uint32_t c = 0; c < nc; c++) {
            const uint32_t row = sch[S.S_ROWOF + c];
            if (row >= total || pr.row_count(row) != 7u - lp) continue;
            const uint32_t u = sch[S.S_RUNIT + row];
            const uint32_t key = sch[S.S_UKEY + u];
            const int a = (int)(key & 0xffffu) - 1, b = (int)(key >> 16u) - 1;
            uint32_t col = S.NCOL;
            for (uint32_t w = 0; w < NCOLW; w++) {
              uint32_t used = 0u;
              if (a >= 0) used |= wmask[(uint32_t)a * NCOLW + w];
              if (b >= 0) used |= wmask[(uint32_t)b * NCOLW + w];
              if (used != 0xffffffffu) {
                uint32_t k = (uint32_t)__ffs(~used) - 1u;
                if (a >= 0) wmask[(uint32_t)a * NCOLW + w] |= 1u << k;
                if (b >= 0) wmask[(uint32_t)b * NCOLW + w] |= 1u << k;
                col = w * 32u + k;
                break;
              }
            }
            sch[S.S_PCOL + row] = col;
            wcount[col]++;
            const uint32_t utp = sch[S.S_UTP + u];
            const uint32_t utc = utp == 0xffffffffu ? 0u : sch[S.S_PCOL + utp] + 1u;
            if (col + 1u >= utc) sch[S.S_UTP + u] = row;
          }
      }
      __syncthreads();
      if (tid == 0u) {
        uint32_t acc = 0u, ncol = 0u;
        for (uint32_t c = 0; c <= S.NCOL; c++) {
          uint32_t n = wcount[c];
          sch[S.S_CSTART + c] = acc;
          wcount[c] = acc;
          acc += n;
          if (n > 0u) ncol = c + 1u;
        }
        sch[S.S_CSTART + S.NCOL + 1u] = acc;
        sch[S.S_META + 0u] = nu;
        sch[S.S_META + 1u] = ncol;
        sch[S.S_META + 2u] = nc;
      }
      if (S.TORS == 1u && S.LONGEST_FIRST == 0u) {
        // Each unit's torsion row is its row of the highest color, the latest contact among equals:
        // (color + 1, contact) packed as the reference packs it, 16 bits of contact index
        // (wgsl.js:2288-2325).
        for (uint32_t u = tid; u < nu; u += nt) sch[S.S_UTP + u] = 0u;
        __syncthreads();
        for (uint32_t row = tid; row < total; row += nt)
          atomicMax(&sch[S.S_UTP + sch[S.S_RUNIT + row]], ((sch[S.S_PCOL + row] + 1u) << 16u) | sch[S.S_RCON + row]);
        __syncthreads();
        for (uint32_t u = tid; u < nu; u += nt) {
          uint32_t packed = sch[S.S_UTP + u];
          sch[S.S_UTP + u] = packed != 0u ? sch[S.S_ROWOF + (packed & 0xffffu)] : 0xffffffffu;
        }
      }
      __syncthreads();
      // Rows bucketed by color, row order kept within a color (a stable counting sort): the block
      // takes nt rows at a time; a row's place is its color's next free slot plus the rows of its
      // color in earlier warps of the chunk plus those before it in its warp (match ranks).
  #ifdef STEEL_BLOCK
      constexpr uint32_t BK_COLORS = 65u, BK_WARPS = STEEL_BLOCK / 32u;
  #else
      constexpr uint32_t BK_COLORS = 65u, BK_WARPS = BIG_THREADS / 32u;
  #endif
      __shared__ uint32_t bk_cnt[BK_WARPS][BK_COLORS], bk_off[BK_WARPS][BK_COLORS];
      const uint32_t nw = nt >> 5u, lane = tid & 31u, warp = tid >> 5u;
      if (S.NCOL + 1u <= BK_COLORS) {
        for (uint32_t i = tid; i < BK_WARPS * BK_COLORS; i += nt) (&bk_cnt[0][0])[i] = 0u;
        __syncthreads();
        for (uint32_t r0 = 0; r0 < total; r0 += nt) {
          const uint32_t row = r0 + tid;
          const bool in = row < total;
          const uint32_t col = in ? sch[S.S_PCOL + row] : 0xffffffffu;
          const uint32_t same = __match_any_sync(0xffffffffu, col);
          const uint32_t below = (uint32_t)__popc(same & ((1u << lane) - 1u));
          if (in && below == 0u) bk_cnt[warp][col] = (uint32_t)__popc(same);
          __syncthreads();
          for (uint32_t c = tid; c <= S.NCOL; c += nt) {
            uint32_t run = wcount[c];
            for (uint32_t w = 0; w < nw; w++) {
              bk_off[w][c] = run;
              run += bk_cnt[w][c];
              bk_cnt[w][c] = 0u;
            }
            wcount[c] = run;
          }
          __syncthreads();
          if (in) sch[S.S_PORD + bk_off[warp][col] + below] = row;
        }
      } else if (tid < 32u) {
        for (uint32_t r0 = 0; r0 < total; r0 += 32u) {
          const uint32_t row = r0 + tid;
          const bool in = row < total;
          const uint32_t col = in ? sch[S.S_PCOL + row] : 0xffffffffu;
          const uint32_t same = __match_any_sync(0xffffffffu, col);
          const uint32_t base = in ? wcount[col] : 0u;
          __syncwarp();
          if (in) {
            sch[S.S_PORD + base + (uint32_t)__popc(same & ((1u << tid) - 1u))] = row;
            if (tid == 31u - (uint32_t)__clz(same)) wcount[col] = base + (uint32_t)__popc(same);
          }
          __syncwarp();
        }
      }
    }
  }
  // Phase 7: dense rows for same-articulation contacts (slots in contact order), loops, mimics.
  uint32_t nloop_rows = 0u;
  for (uint32_t k = 0; k < S.NLOOP; k++) nloop_rows += S.sf[S.SF_LOOP + k * 5u].w > 0.5f ? 2u : 1u;
  if (tid == 0u) sch[S.S_META + 3u] = ndc + nloop_rows + S.NMIMIC;
  for (uint32_t c = tid; tid < sn && c < nc; c += sn) {
    uint32_t slot = sch[S.S_DSLOT + c];
    if (slot == 0xffffffffu || slot >= S.MAXDENSE) continue;
    pr.dense_row(slot, c, Lane{S.tscr + tid, sn});
  }
  tm.sync();  // the loop and mimic rows below use per-thread contiguous scratch slices
  const uint32_t JDIM = 3u * S.NDA;
  for (uint32_t i = tid; tid < sn && i < S.NLOOP; i += sn) {
    float4 L0 = S.sf[S.SF_LOOP + i * 5u];
    int pl = f2i(L0.x);
    uint32_t cl = f2u(L0.y), art_id = f2u(L0.z);
    bool revolute = L0.w > 0.5f;
    uint32_t slot = ndc;
    for (uint32_t k = 0; k < i; k++) slot += S.sf[S.SF_LOOP + k * 5u].w > 0.5f ? 2u : 1u;
    if (slot + (revolute ? 1u : 0u) >= S.MAXDENSE) continue;
    f3 pa = v3(S.sf[S.SF_LOOP + i * 5u + 1u]);
    float4 rp = make_float4(0, 0, 0, 1);
    if (pl >= 0) { rp = ar.link_rot((uint32_t)pl); pa = ar.ld3(ar.lo((uint32_t)pl) + L_POS) + qrot(rp, pa); }
    float4 rc = ar.link_rot(cl);
    f3 pc = ar.ld3(ar.lo(cl) + L_POS) + qrot(rc, v3(S.sf[S.SF_LOOP + i * 5u + 2u]));
    f3 pm = 0.5f * (pa + pc);
    uint4 ai = ar.info(art_id);
    float* J = tscr;
    float* rest = tscr + JDIM;
    for (uint32_t k = 0; k < JDIM; k++) J[k] = 0.0f;
    f3 ex = mf3(1, 0, 0), ey = mf3(0, 1, 0), ez = mf3(0, 0, 1);
    ar.gen_jac(cl, pm, 1.0f, ex, ey, ez, ai.z, J);
    if (pl >= 0) ar.gen_jac((uint32_t)pl, pm, -1.0f, ex, ey, ez, ai.z, J);
    pr.put_bilateral(S.A_DENSE + slot * S.DPS, art_id, J, 3u, (P.beta * (pc - pa)) / P.dt, rest);
    if (revolute) {
      f3 ap = qrot(rp, v3(S.sf[S.SF_LOOP + i * 5u + 3u]));
      f3 ac = qrot(rc, v3(S.sf[S.SF_LOOP + i * 5u + 4u]));
      f3 e1 = cross(ap, mf3(1, 0, 0));
      if (dot(e1, e1) < 1e-6f) e1 = cross(ap, mf3(0, 1, 0));
      e1 = nrm(e1);
      f3 e2 = cross(ap, e1);
      for (uint32_t k = 0; k < JDIM; k++) J[k] = 0.0f;
      ar.gen_ang(cl, 1.0f, e1, e2, ai.z, J);
      if (pl >= 0) ar.gen_ang((uint32_t)pl, -1.0f, e1, e2, ai.z, J);
      f3 err = cross(ap, ac);
      pr.put_bilateral(S.A_DENSE + (slot + 1u) * S.DPS, art_id, J, 2u,
                       (P.beta * mf3(dot(e1, err), dot(e2, err), 0.0f)) / P.dt, rest);
    }
  }
  for (uint32_t i = tid; tid < sn && i < S.NMIMIC; i += sn) {
    float4 M0 = S.sf[S.SF_MIMIC + i * 2u], M1 = S.sf[S.SF_MIMIC + i * 2u + 1u];
    uint32_t slot = ndc + nloop_rows + i;
    if (slot >= S.MAXDENSE) continue;
    float* J = tscr;
    for (uint32_t k = 0; k < JDIM; k++) J[k] = 0.0f;
    J[f2u(M0.y)] = 1.0f;
    J[f2u(M0.z)] -= M0.w;
    float phi = (A[S.A_Q + f2u(M1.x)] - M0.w * A[S.A_Q + f2u(M1.y)]) - M1.z;
    pr.put_bilateral(S.A_DENSE + slot * S.DPS, f2u(M0.x), J, 1u, mf3((P.beta * phi) / P.dt, 0.0f, 0.0f), tscr + JDIM);
  }
  if (staged) {
    __syncthreads();
    for (uint32_t i = tid; i < S.NL * LBLK; i += nt) S.art[S.A_LINK + i] = lb[i];
  }
}

}  // namespace steel
