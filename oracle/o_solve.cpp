// Test infrastructure (oracle): the solve kernel, wgsl.js:2501-3891 restated (default flag set).
#include <algorithm>
#include <cmath>

#include "oracle.h"
#include "smath_o.h"
#include "o_cone5.h"

namespace orc {

enum : uint32_t { L_V = 147, L_P = 201, L_ROT = 216, L_COM = 220, L_TAU = 223 };
static const uint32_t AVN = 14u;
static inline uint32_t anchor_hash(uint32_t pair, uint32_t k) { return std::max(hash_u32(pair * 2u + k), 1u); }
static inline m3 skew(v3 r) { return mcols(mk3(0.0f, r.z, -r.y), mk3(-r.z, 0.0f, r.x), mk3(r.y, -r.x, 0.0f)); }

m3 Oracle::gyro_inverse3(const m3& m) const {
  v3 a = m.c[0], b = m.c[1], c = m.c[2];
  v3 r0 = cross(b, c), r1 = cross(c, a), r2 = cross(a, b);
  float det = dot(a, r0);
  return mscale(transpose(mcols(r0, r1, r2)), 1.0f / det);
}
// gyroscopic_velocity (wgsl.js:2543-2562)
v3 Oracle::gyroscopic_velocity(const m3& inertia, v3 u0, float dt) const {
  m3 a = mscale(inertia, 1.0f / fmaxf_(inertia.c[0].x, fmaxf_(inertia.c[1].y, inertia.c[2].z)));
  m3 inv = gyro_inverse3(a);
  float speed = std::sqrt(fmaxf_(dot(u0, mul(a, u0)) * ((inv.c[0].x + inv.c[1].y) + inv.c[2].z), 0.0f));
  uint32_t n = f2u(clampf(std::ceil((2.0f * std::fabs(dt)) * speed), 1.0f, 32.0f));
  float h = dt / (float)n;
  v3 w = u0;
  for (uint32_t m = 0; m < n; m++) {
    v3 u = w;
    float energy = dot(u, mul(a, u));
    for (uint32_t it = 0; it < 8u; it++) {
      m3 S = mscale(0.5f * h, skew(mul(a, 0.5f * (u + w))));
      v3 c = mul(gyro_inverse3(msub(a, S)), mul(madd(a, S), u));
      v3 d = c - w;
      w = c;
      if (dot(d, mul(a, d)) <= 1e-12f * energy) break;
    }
  }
  return w;
}

// Friction modes (friction_mode, wgsl.js:2567-2652): the (normal, t1, t2) impulses of a contact
// point re-solved together on its 3x3 block, g0 = (G_nn, G_nt) and g1 = (G_tt: xx, xy, yy).
// Mode 1 and 2 bisect the normal impulse with the tangent pair re-solved and clipped at each
// trial (2 adds mu |u_t| to the normal target); mode 3 is the Coulomb-Newton root search.
static v2 tangent_step(v2 ut, v4 g1) {
  float det = g1.x * g1.z - g1.y * g1.y;
  if (std::fabs(det) <= 1e-20f) return mk2(0.0f, 0.0f);
  return mk2((-ut.x) * g1.z + ut.y * g1.y, ut.x * g1.y - ut.y * g1.x) / det;
}
static v2 clip_cone(v2 t, float lim) {
  float m = length(t);
  if (m > lim && m > 1e-20f) return t * (lim / m);
  return t;
}
// A singular block (fewer than two tangential mobilities) keeps the normal impulse and takes the
// fixed-normal pair on its disk.
v3 Oracle::fixed_normal_pair(v2 ut0, v4 g1, float mu, v3 lam) const {
  v2 t = friction_pair_solve(g1.x, g1.y, g1.z, ut0.x, ut0.y, lam.y, lam.z, fmaxf_(mu * lam.x, 0.0f), 1.0f);
  return mk3(lam.x, t.x, t.y);
}
v3 Oracle::contact_block(uint32_t mode, float un, v2 ut0, v4 g0, v4 g1, float vtarget0, float mu,
                          v3 lam) const {
  const float gnn = g0.x;
  const v2 gnt = mk2(g0.y, g0.z);
  const float trace = g1.x + g1.z;
  if (g1.x * g1.z - g1.y * g1.y <= (1e-6f * trace) * trace) return fixed_normal_pair(ut0, g1, mu, lam);
  if (gnn < 1e-20f) return lam;
  const v2 lt = mk2(lam.y, lam.z);
  float vt_n = vtarget0;
  if (mode == 2u) vt_n += mu * length(ut0);
  if (mode == 3u) {
    const float un_f = un - (gnn * lam.x + dot(gnt, lt));
    const v2 ut_f = ut0 - mk2((gnt.x * lam.x + g1.x * lt.x) + g1.y * lt.y, (gnt.y * lam.x + g1.y * lt.x) + g1.z * lt.y);
    if (un_f >= vt_n) return mk3(0.0f, 0.0f, 0.0f);
    const float bN = un_f - vt_n;
    const float A00 = g1.x - (gnt.x * gnt.x) / gnn, A01 = g1.y - (gnt.x * gnt.y) / gnn;
    const float A11 = g1.z - (gnt.y * gnt.y) / gnn;
    if (A00 * A11 - A01 * A01 <= (1e-6f * trace) * trace) return fixed_normal_pair(ut0, g1, mu, lam);
    const v2 c = ut_f - (bN / gnn) * gnt;
    const float id0 = 1.0f / (A00 * A11 - A01 * A01);
    v2 s = mk2(A11 * c.x - A01 * c.y, A00 * c.y - A01 * c.x) * id0;
    const float phi0 = length(s) - (mu * (dot(gnt, s) - bN)) / gnn;
    if (phi0 > 0.0f) {
      float hi = 1.0f;
      for (uint32_t e = 0; e < 30u; e++) {
        const float a = A00 + hi, d = A11 + hi, idt = 1.0f / (a * d - A01 * A01);
        const v2 sh = mk2(d * c.x - A01 * c.y, a * c.y - A01 * c.x) * idt;
        if (length(sh) - (mu * (dot(gnt, sh) - bN)) / gnn < 0.0f) break;
        hi *= 2.0f;
      }
      float lo = 0.0f, x = 0.5f * hi;
      const float tol = 1e-6f + 1e-6f * phi0;
      for (uint32_t k = 0; k < 50u; k++) {
        const float a = A00 + x, d = A11 + x, idt = 1.0f / (a * d - A01 * A01);
        const v2 sx = mk2(d * c.x - A01 * c.y, a * c.y - A01 * c.x) * idt;
        const v2 tx = mk2(d * sx.x - A01 * sx.y, a * sx.y - A01 * sx.x) * idt;
        const float ns = length(sx);
        const float fx = ns - (mu * (dot(gnt, sx) - bN)) / gnn;
        const float dfx = (-dot(sx, tx)) / ns + (mu * dot(gnt, tx)) / gnn;
        s = sx;
        if (std::fabs(fx) < tol || std::fabs(hi - lo) < 1e-6f * (1.0f + hi)) break;
        if (fx > 0.0f) lo = x; else hi = x;
        float xn = 0.5f * (lo + hi);
        if (dfx != 0.0f) {
          const float xt = x - fx / dfx;
          if (xt > lo && xt < hi) xn = xt;
        }
        x = xn;
      }
    }
    const v2 rt = mk2(-s.x, -s.y);
    // The finite search can end just below zero load; the exact root is non-negative.
    const float ln = fmaxf_((-(dot(gnt, rt) + bN)) / gnn, 0.0f);
    const float lim = fmaxf_(mu * ln, 0.0f);
    const float m = length(rt);
    const v2 t = m > lim ? rt * (lim / m) : rt;
    return mk3(ln, t.x, t.y);
  }
  const float u0 = (un - gnn * lam.x) - dot(gnt, lt);
  if (u0 >= vt_n) return mk3(0.0f, 0.0f, 0.0f);
  float lo = 0.0f;
  float hi = fmaxf_(fmaxf_(2.0f * lam.x, (vt_n - un) / gnn + lam.x), 1.0f);
  float flo = u0 - vt_n, fhi = -1.0f;
  for (uint32_t k = 0; k < 20u; k++) {
    const float mid = 0.5f * (lo + hi);
    const float dn = mid - lam.x;
    const v2 tr = clip_cone(lt + tangent_step(ut0 + gnt * dn, g1), mu * mid);
    const float u = (un + gnn * dn) + dot(gnt, tr - lt);
    if (u < vt_n) { lo = mid; flo = u - vt_n; } else { hi = mid; fhi = u - vt_n; }
  }
  float ln = 0.5f * (lo + hi);
  if (fhi >= 0.0f) ln = lo - (flo * (hi - lo)) / (fhi - flo);
  const v2 tf = clip_cone(lt + tangent_step(ut0 + gnt * (ln - lam.x), g1), mu * ln);
  return mk3(ln, tf.x, tf.y);
}

// friction_pair_solve (wgsl.js:2952-3011)
v2 Oracle::friction_pair_solve(float a0, float c0, float d0, float r0, float r1, float old0, float old1, float radius,
                               float omega) const {
  if (radius <= 0.0f) return mk2(0.0f, 0.0f);
  float scale = fmaxf_(fmaxf_(a0, d0), 1e-20f);
  float a = a0 / scale, c = c0 / scale, d = d0 / scale;
  float largest = 0.5f * ((a + d) + std::sqrt((a - d) * (a - d) + (4.0f * c) * c));
  float smallest = largest > 0.0f ? fmaxf_((a * d - c * c) / largest, 0.0f) : 0.0f;
  float vx = c, vy = largest - a;
  if (a >= d) { vx = largest - d; vy = c; }
  float vn = std::sqrt(vx * vx + vy * vy);
  if (vn > 0.0f) { vx /= vn; vy /= vn; } else { vx = 1.0f; vy = 0.0f; }
  float r0r = (vx * r0 + vy * r1) / scale;
  float r1r = ((-vy) * r0 + vx * r1) / scale;
  v2 res = mk2(old0, old1);
  bool sticking = false;
  if (largest > 0.0f && (smallest > 0.0f || r1r == 0.0f)) {
    float dx = r0r / largest;
    float dy = smallest > 0.0f ? r1r / smallest : 0.0f;
    res = mk2(old0 - (vx * dx - vy * dy), old1 - (vy * dx + vx * dy));
    sticking = length(res) <= radius;
  }
  if (!sticking) {
    float on = length(mk2(old0, old1)), rn = length(mk2(r0, r1));
    if (on > 0.0f && on <= radius && radius - on <= 2e-7f * radius && r0 * old0 + r1 * old1 <= 0.0f &&
        std::fabs(r0 * old1 - r1 * old0) <= (2e-7f * on) * rn)
      return mk2(old0, old1);
    float ox = vx * old0 + vy * old1, oy = (-vy) * old0 + vx * old1;
    float b0 = largest * ox - r0r, b1 = smallest * oy - r1r;
    float x = 0.0f, y = 0.0f;
    float hi = std::sqrt(b0 * b0 + b1 * b1) / radius;
    if (hi > 0.0f) {
      float lo = fmaxf_(fmaxf_(hi - largest, std::fabs(b1) / radius - smallest), 0.0f);
      float alpha = lo;
      bool done = false;
      for (uint32_t it = 0; it < 8u; it++) {
        float i0 = 1.0f / (largest + alpha);
        float i1 = smallest + alpha > 0.0f ? 1.0f / (smallest + alpha) : 0.0f;
        float tx = ox - (r0r + alpha * ox) * i0, ty = oy - (r1r + alpha * oy) * i1;
        float nrm = std::sqrt(tx * tx + ty * ty);
        if (std::fabs(nrm - radius) <= 2e-7f * radius || (alpha == 0.0f && nrm <= radius)) { x = tx; y = ty; done = true; break; }
        if (nrm > radius) lo = alpha; else hi = alpha;
        float slope = (tx * tx) * i0 + (ty * ty) * i1;
        float cand = alpha;
        if (slope > 0.0f) cand = alpha + (((nrm / radius - 1.0f) * nrm) * nrm) / slope;
        alpha = (cand > lo && cand < hi) ? cand : 0.5f * (lo + hi);
      }
      if (!done) {
        for (uint32_t it = 0; it < 24u; it++) {
          alpha = 0.5f * (lo + hi);
          if (length(mk2(b0 / (largest + alpha), b1 / (smallest + alpha))) > radius) lo = alpha; else hi = alpha;
        }
        x = b0 / (largest + hi);
        y = b1 / (smallest + hi);
      }
    }
    res = mk2((old0 + vx * (x - ox)) - vy * (y - oy), (old1 + vy * (x - ox)) + vx * (y - oy));
  }
  v2 old = mk2(old0, old1);
  v2 relaxed = old + omega * (res - old);
  float m = length(relaxed);
  return m > radius ? relaxed * (radius / m) : relaxed;
}

// snap_tw (wgsl.js:2930-2934): a body's twist at the end of the position iterations.
void Oracle::snap_tw(int b, v3 out[2]) const {
  if (b < 0) { out[0] = splat3(0.0f); out[1] = splat3(0.0f); return; }
  uint32_t o = C.A_SNAP + (uint32_t)b * 8u;
  out[0] = ld3(o);
  out[1] = ld3(o + 4u);
}
void Oracle::load_tw(int b, v3 out[2]) const {
  if (b < 0) { out[0] = splat3(0.0f); out[1] = splat3(0.0f); return; }
  out[0] = xyz(tw[(uint32_t)b * 2u]);
  out[1] = xyz(tw[(uint32_t)b * 2u + 1u]);
}
void Oracle::add_imp(int b, v3 f, v3 t) {
  if (b < 0) return;
  if (body_kind(b) != 2u) return;
  imp[(uint32_t)b * 2u] = imp[(uint32_t)b * 2u] + mk4(f, 0.0f);
  imp[(uint32_t)b * 2u + 1u] = imp[(uint32_t)b * 2u + 1u] + mk4(t, 0.0f);
}

void Oracle::solve_slot(uint32_t u, uint32_t mode, uint32_t it) {
  v4 sl = rows[C.MAXC * C.ROWS + 2u * u], sr = rows[C.MAXC * C.ROWS + 2u * u + 1u];
  solve_unit(f2u(sl.y), f2u(sl.x), f2i(sl.z), f2i(sl.w), f2u(sr.x), f2u(sr.y), mode, it);
}

// solve_unit (wgsl.js:3033-3231), fixed_normal friction with anchors.
void Oracle::solve_unit(uint32_t us, uint32_t row, int a, int b, uint32_t s0, uint32_t s1, uint32_t mode,
                        uint32_t it) {
  const uint32_t ROWS = C.ROWS, PO = C.PO;
  v3 ta[2], tb[2];
  load_tw(a, ta);
  load_tw(b, tb);
  uint32_t o = row * ROWS;
  v4 r0 = rows[o], r1 = rows[o + 1u], r2 = rows[o + 2u];
  v3 ra = xyz(rows[o + 3u]), rb = xyz(rows[o + 4u]);
  v3 n = xyz(r0), t1 = xyz(r1), t2 = xyz(r2);
  v4 lam = rows[o + 6u];
  float dn = 0.0f, dt1 = 0.0f, dt2 = 0.0f;
  if (mode == 0u) {
    dn = lam.x; dt1 = lam.y; dt2 = lam.z;
    for (uint32_t r = 0; r < 3u; r++) {
      float d = r == 0u ? dn : (r == 1u ? dt1 : dt2);
      ta[0] += xyz(rows[o + 7u + r * 4u]) * d; ta[1] += xyz(rows[o + 8u + r * 4u]) * d;
      tb[0] += xyz(rows[o + 9u + r * 4u]) * d; tb[1] += xyz(rows[o + 10u + r * 4u]) * d;
    }
    v3 fra = ra, frb = rb;
    if (C.EXTRA == 1u) { fra = xyz(rows[o + PO]); frb = xyz(rows[o + PO + 1u]); }
    v3 fn_ = n * dn, ft = t1 * dt1 + t2 * dt2;
    add_imp(a, -fn_ - ft, -cross(ra, fn_) - cross(fra, ft));
    add_imp(b, fn_ + ft, cross(rb, fn_) + cross(frb, ft));
  } else {
    v3 vrel = (tb[0] + cross(tb[1], rb)) - (ta[0] + cross(ta[1], ra));
    float jv = dot(n, vrel);
    float w = vpass ? 1.0f : rows[o + 5u].w;
    float res = jv + r1.w;
    if (C.COMPL == 1u) res += rows[o + C.CO].x * lam.x;
    float nl = fmaxf_(lam.x + C.F_OMEGA * ((((-res) * r0.w) * w) - (1.0f - w) * lam.x), 0.0f);
    dn = nl - lam.x;
    lam.x = nl;
    ta[0] += xyz(rows[o + 7u]) * dn; ta[1] += xyz(rows[o + 8u]) * dn;
    tb[0] += xyz(rows[o + 9u]) * dn; tb[1] += xyz(rows[o + 10u]) * dn;
    add_imp(a, -n * dn, -cross(ra, n * dn));
    add_imp(b, n * dn, cross(rb, n * dn));
    v3 fra = ra, frb = rb;
    float lim = r2.w * nl;
    float pooled = nl;
    v2 bias = mk2(0.0f, 0.0f);
    float role = 1.0f;
    if (C.EXTRA == 1u) {
      role = rows[o + PO].w;
      if (C.PATCH == 1u && role != 1.0f) art[C.A_ULOAD + us] += dn;
      fra = xyz(rows[o + PO]);
      frb = xyz(rows[o + PO + 1u]);
      if (C.PATCH == 1u && role == 2.0f) {
        float load = art[C.A_ULOAD + us];
        lim = r2.w * load;
        pooled = load;
        v3 e = xyz(rows[o + PO + 2u]);
        bias = vpass ? mk2(0.0f, 0.0f) : (C.F_ANCHOR_BETA * mk2(dot(t1, e), dot(t2, e))) / P.dt;
        rows[o + PO + 2u].w = lim;
      }
    }
    if (it < C.FSTART) { lam.y = 0.0f; lam.z = 0.0f; }
    if (C.FMODE > 0u && it >= C.FSTART) {
      // Coupled (normal, t1, t2) re-solve (wgsl.js:3081-3095); overwrites all three impulses.
      v3 vn = (tb[0] + cross(tb[1], rb)) - (ta[0] + cross(ta[1], ra));
      v3 vt = (tb[0] + cross(tb[1], frb)) - (ta[0] + cross(ta[1], fra));
      v3 nlam = contact_block(C.FMODE, dot(n, vn), mk2(dot(t1, vt), dot(t2, vt)), rows[o + C.FMO], rows[o + C.FMO + 1u],
                              -r1.w, r2.w, xyz(lam));
      v3 d = nlam - xyz(lam);
      if (C.PATCH == 1u && role != 1.0f) art[C.A_ULOAD + us] += d.x;
      ta[0] += (xyz(rows[o + 7u]) * d.x + xyz(rows[o + 11u]) * d.y) + xyz(rows[o + 15u]) * d.z;
      ta[1] += (xyz(rows[o + 8u]) * d.x + xyz(rows[o + 12u]) * d.y) + xyz(rows[o + 16u]) * d.z;
      tb[0] += (xyz(rows[o + 9u]) * d.x + xyz(rows[o + 13u]) * d.y) + xyz(rows[o + 17u]) * d.z;
      tb[1] += (xyz(rows[o + 10u]) * d.x + xyz(rows[o + 14u]) * d.y) + xyz(rows[o + 18u]) * d.z;
      v3 fn2 = n * d.x, ft = t1 * d.y + t2 * d.z;
      add_imp(a, (-fn2) - ft, (-cross(ra, fn2)) - cross(fra, ft));
      add_imp(b, fn2 + ft, cross(rb, fn2) + cross(frb, ft));
      lam = mk4(nlam, lam.w);
    } else if (role != 0.0f && it >= C.FSTART) {
      v3 vr2 = (tb[0] + cross(tb[1], frb)) - (ta[0] + cross(ta[1], fra));
      v4 ki = rows[o + 5u];
      float v1 = dot(t1, vr2) + bias.x, v2_ = dot(t2, vr2) + bias.y;
      float kd = ki.x * ki.z - ki.y * ki.y;
      v2 lt = friction_pair_solve(ki.z / kd, -ki.y / kd, ki.x / kd, v1, v2_, lam.y, lam.z, lim, C.F_OMEGA);
      dt1 = lt.x - lam.y;
      dt2 = lt.y - lam.z;
      lam.y = lt.x;
      lam.z = lt.y;
      ta[0] += xyz(rows[o + 11u]) * dt1 + xyz(rows[o + 15u]) * dt2;
      ta[1] += xyz(rows[o + 12u]) * dt1 + xyz(rows[o + 16u]) * dt2;
      tb[0] += xyz(rows[o + 13u]) * dt1 + xyz(rows[o + 17u]) * dt2;
      tb[1] += xyz(rows[o + 14u]) * dt1 + xyz(rows[o + 18u]) * dt2;
      v3 f = t1 * dt1 + t2 * dt2;
      add_imp(a, -f, -cross(fra, f));
      add_imp(b, f, cross(frb, f));
    }
    // Articulated torsional/rolling (wgsl.js:3080, 3112-3140): after the sliding pair, the block
    // over sliding, spin and rolling of a contact that touches an articulation.
    const bool art_u = (a >= 0 && body_kind(a) >= 2u) || (b >= 0 && body_kind(b) >= 2u);
    const bool ell = C.ANG_ART == 1u && C.ANG == 1u && art_u && (rows[o + 19u].x > 0.0f || rows[o + 19u].y > 0.0f);
    if (ell && it >= C.FSTART) {
      float H[25];
      uint32_t idx = 0;
      for (uint32_t x = 0; x < 5u; x++)
        for (uint32_t y = x; y < 5u; y++) {
          const v4 q = rows[o + C.EO + idx / 4u];
          const float hv = (&q.x)[idx % 4u];
          H[x * 5u + y] = hv;
          H[y * 5u + x] = hv;
          idx++;
        }
      const v3 vt = (tb[0] + cross(tb[1], frb)) - (ta[0] + cross(ta[1], fra));
      const v3 wr = tb[1] - ta[1];
      const v4 la0 = rows[o + 21u], g19 = rows[o + 19u];
      const float g[5] = {dot(t1, vt), dot(t2, vt), dot(n, wr), dot(t1, wr), dot(t2, wr)};
      const float mu5[5] = {r2.w, r2.w, g19.x, g19.y, g19.y};
      const float l5[5] = {lam.y, lam.z, la0.x, la0.y, la0.z};
      float nl5[5], d[5];
      ell_block5(H, g, mu5, l5, pooled, C.PYRAMID == 1u, C.F_CREEP, C.F_OMEGA, nl5);
      for (uint32_t k = 0; k < 5u; k++) d[k] = nl5[k] - l5[k];
      ta[0] += (((xyz(rows[o + 11u]) * d[0] + xyz(rows[o + 15u]) * d[1]) + xyz(rows[o + 22u]) * d[2]) + xyz(rows[o + 26u]) * d[3]) + xyz(rows[o + 30u]) * d[4];
      ta[1] += (((xyz(rows[o + 12u]) * d[0] + xyz(rows[o + 16u]) * d[1]) + xyz(rows[o + 23u]) * d[2]) + xyz(rows[o + 27u]) * d[3]) + xyz(rows[o + 31u]) * d[4];
      tb[0] += (((xyz(rows[o + 13u]) * d[0] + xyz(rows[o + 17u]) * d[1]) + xyz(rows[o + 24u]) * d[2]) + xyz(rows[o + 28u]) * d[3]) + xyz(rows[o + 32u]) * d[4];
      tb[1] += (((xyz(rows[o + 14u]) * d[0] + xyz(rows[o + 18u]) * d[1]) + xyz(rows[o + 25u]) * d[2]) + xyz(rows[o + 29u]) * d[3]) + xyz(rows[o + 33u]) * d[4];
      const v3 f = t1 * d[0] + t2 * d[1];
      const v3 tq = (n * d[2] + t1 * d[3]) + t2 * d[4];
      add_imp(a, -f, (-cross(fra, f)) - tq);
      add_imp(b, f, cross(frb, f) + tq);
      lam.y = nl5[0];
      lam.z = nl5[1];
      rows[o + 21u] = mk4(nl5[2], nl5[3], nl5[4], 0.0f);
    }
    rows[o + 6u] = lam;
    if (C.ANG == 1u) {
      // Spin within mu_t * N, rolling within a disk of mu_r * N (wgsl.js:3144-3170); under
      // friction patches only the region's first anchor carries them, with the pooled load.
      const v4 g = rows[o + 19u];
      const bool aon = !ell && (C.PATCH == 0u || role == 1.0f || (role == 2.0f && rows[o + PO + 1u].w == 0.0f));
      const float nl2 = pooled;
      if (aon && (g.x > 0.0f || g.y > 0.0f)) {
        const v4 la = rows[o + 21u];
        const v3 wrel = tb[1] - ta[1];
        const float ns = clampf(la.x - dot(n, wrel) * g.z, (-g.x) * nl2, g.x * nl2);
        const float ds = ns - la.x;
        ta[0] += xyz(rows[o + 22u]) * ds; ta[1] += xyz(rows[o + 23u]) * ds;
        tb[0] += xyz(rows[o + 24u]) * ds; tb[1] += xyz(rows[o + 25u]) * ds;
        const v3 w2 = tb[1] - ta[1];
        const v4 ri = rows[o + 20u];
        const float u1 = dot(t1, w2), u2 = dot(t2, w2);
        v2 lr = mk2(la.y, la.z) - mk2(ri.x * u1 + ri.y * u2, ri.y * u1 + ri.z * u2);
        const float rl = g.y * nl2;
        if (length(lr) > rl) lr = lr * (rl / fmaxf_(length(lr), 1e-12f));
        const float d1 = lr.x - la.y, d2 = lr.y - la.z;
        ta[0] += xyz(rows[o + 26u]) * d1 + xyz(rows[o + 30u]) * d2;
        ta[1] += xyz(rows[o + 27u]) * d1 + xyz(rows[o + 31u]) * d2;
        tb[0] += xyz(rows[o + 28u]) * d1 + xyz(rows[o + 32u]) * d2;
        tb[1] += xyz(rows[o + 29u]) * d1 + xyz(rows[o + 33u]) * d2;
        rows[o + 21u] = mk4(ns, lr.x, lr.y, 0.0f);
        const v3 tq = (n * ds + t1 * d1) + t2 * d2;
        add_imp(a, splat3(0.0f), -tq);
        add_imp(b, splat3(0.0f), tq);
      }
    }
  }
  // Contact torsion (wgsl.js:3185-3228) on the unit's last-colored row: sliding and spin share
  // the cluster's Coulomb budget mu * N.
  const uint32_t TO = C.TO;
  if (C.TORS == 1u && mode == 1u && row == sched[C.S_UTP + us] && rows[s0 * ROWS + TO].w > 0.0f) {
    uint32_t L = s0 * ROWS;
    float mu = rows[L + TO].w;
    float load = 0.0f, slide = 0.0f;
    for (uint32_t m = s0; m < s1; m++) {
      uint32_t om = m * ROWS;
      if (rows[om + TO + 4u].w < 0.5f) continue;
      v4 lm = rows[om + 6u];
      load += fmaxf_(lm.x, 0.0f);
      if (C.EXTRA == 0u || rows[om + PO].w != 0.0f) slide += length(mk2(lm.y, lm.z));
    }
    float budget = mu * load;
    if (slide > budget && slide > 0.0f) {
      // Later normals lowered the load: the members' tangent pairs are projected onto it.
      float scale = budget / slide;
      for (uint32_t m = s0; m < s1; m++) {
        uint32_t om = m * ROWS;
        if (rows[om + TO + 4u].w < 0.5f || (C.EXTRA == 1u && rows[om + PO].w == 0.0f)) continue;
        v4 lm = rows[om + 6u];
        float d1 = lm.y * (scale - 1.0f), d2 = lm.z * (scale - 1.0f);
        ta[0] += xyz(rows[om + 11u]) * d1 + xyz(rows[om + 15u]) * d2;
        ta[1] += xyz(rows[om + 12u]) * d1 + xyz(rows[om + 16u]) * d2;
        tb[0] += xyz(rows[om + 13u]) * d1 + xyz(rows[om + 17u]) * d2;
        tb[1] += xyz(rows[om + 14u]) * d1 + xyz(rows[om + 18u]) * d2;
        v3 fa = xyz(rows[om + 3u]), fb = xyz(rows[om + 4u]);
        if (C.EXTRA == 1u) { fa = xyz(rows[om + PO]); fb = xyz(rows[om + PO + 1u]); }
        v3 f = xyz(rows[om + 1u]) * d1 + xyz(rows[om + 2u]) * d2;
        add_imp(a, -f, -cross(fa, f));
        add_imp(b, f, cross(fb, f));
        rows[om + 6u] = mk4(lm.x, lm.y * scale, lm.z * scale, lm.w);
      }
      slide = budget;
    }
    float bound = rows[L + TO + 3u].w * fmaxf_(budget - slide, 0.0f);
    if (it < C.FSTART) bound = 0.0f;
    v3 ng = xyz(rows[L + TO + 4u]);
    float ls = rows[L + TO + 2u].w;
    float nls = clampf(ls - (C.F_OMEGA * dot(ng, tb[1] - ta[1])) * rows[L + TO + 1u].w, -bound, bound);
    float ds = nls - ls;
    if (ds != 0.0f) {
      ta[0] += xyz(rows[L + TO]) * ds;
      ta[1] += xyz(rows[L + TO + 1u]) * ds;
      tb[0] += xyz(rows[L + TO + 2u]) * ds;
      tb[1] += xyz(rows[L + TO + 3u]) * ds;
      rows[L + TO + 2u].w = nls;
      add_imp(a, splat3(0.0f), (-ng) * ds);
      add_imp(b, splat3(0.0f), ng * ds);
    }
  }
  if (a >= 0) { tw[(uint32_t)a * 2u] = mk4(ta[0], 0.0f); tw[(uint32_t)a * 2u + 1u] = mk4(ta[1], 0.0f); }
  if (b >= 0) { tw[(uint32_t)b * 2u] = mk4(tb[0], 0.0f); tw[(uint32_t)b * 2u + 1u] = mk4(tb[1], 0.0f); }
}

// subgroupAdd of a 32-lane subgroup (wgsl.js:3305 with SG = 1), pinned to a fixed order: an xor
// butterfly over lane offsets 16, 8, 4, 2, 1, each step adding lane l and lane l ^ offset. IEEE
// addition commutes, so every lane ends with the same bits; lane 0's value is returned.
static float lane_sum32(const float* part) {
  float v[32], t[32];
  for (uint32_t l = 0; l < 32u; l++) v[l] = part[l];
  for (uint32_t off = 16u; off > 0u; off >>= 1u) {
    for (uint32_t l = 0; l < 32u; l++) t[l] = v[l] + v[l ^ off];
    for (uint32_t l = 0; l < 32u; l++) v[l] = t[l];
  }
  return v[0];
}

// art_dense (wgsl.js:3306-3364) in its subgroup form: one 32-lane subgroup per articulation, lane
// l owns dofs l, l + 32, ... and accumulates its partial sums in dof order; lane_sum32 combines
// them. Per-dof updates are the same operations in either form.
bool Oracle::art_dense(uint32_t a, uint32_t mode, uint32_t it, uint32_t ph) {
  const uint32_t NDA = C.NDA, DHDR = C.DHDR, DPS = C.DPS;
  uint32_t nd = std::min(sched[C.S_META + 3u], C.MAXDENSE);
  u4 ai = art_info(a);
  bool touched = false;
  float part[32], p1[32], p2[32];
  for (uint32_t i = 0; i < nd; i++) {
    uint32_t o = C.A_DENSE + i * DPS;
    if (f2u(art[o]) != a) continue;
    touched = true;
    uint32_t jo = o + DHDR, yo = o + DHDR + 3u * NDA;
    v3 lam = mk3(art[o + 9u], art[o + 10u], art[o + 11u]);
    if ((art[o + 21u] > 0.5f) == (ph == 1u) && ph != 0u) continue;
    if (art[o + 21u] > 0.5f) {
      if (mode == 0u) continue;
      v3 nlam = lam;
      for (uint32_t r = 0; r < f2u(art[o + 21u]); r++) {
        for (uint32_t l = 0; l < 32u; l++) part[l] = 0.0f;
        for (uint32_t k = 0; k < ai.w; k++) part[k % 32u] += art[jo + r * NDA + k] * aqd[ai.z + k];
        float jv = lane_sum32(part);
        float rhs = vpass ? 0.0f : (r == 0u ? art[o + 4u] : (r == 1u ? art[o + 22u] : art[o + 23u]));
        float dl = ((-C.F_OMEGA) * (jv + rhs)) * art[o + 5u + r];
        setat(nlam, (int)r, at(nlam, (int)r) + dl);
        for (uint32_t k = 0; k < ai.w; k++) aqd[ai.z + k] += art[yo + r * NDA + k] * dl;
      }
      art[o + 9u] = nlam.x; art[o + 10u] = nlam.y; art[o + 11u] = nlam.z;
      continue;
    }
    if (mode == 0u) {
      for (uint32_t k = 0; k < ai.w; k++)
        aqd[ai.z + k] += (art[yo + k] * lam.x + art[yo + NDA + k] * lam.y) + art[yo + 2u * NDA + k] * lam.z;
      continue;
    }
    for (uint32_t l = 0; l < 32u; l++) part[l] = 0.0f;
    for (uint32_t k = 0; k < ai.w; k++) part[k % 32u] += art[jo + k] * aqd[ai.z + k];
    float jv = lane_sum32(part);
    float w = vpass ? 1.0f : art[o + 24u];
    float nl = fmaxf_(lam.x + C.F_OMEGA * ((((-(jv + art[o + 4u])) * art[o + 5u]) * w) - (1.0f - w) * lam.x), 0.0f);
    float dn = nl - lam.x;
    for (uint32_t l = 0; l < 32u; l++) { p1[l] = 0.0f; p2[l] = 0.0f; }
    for (uint32_t k = 0; k < ai.w; k++) {
      aqd[ai.z + k] += art[yo + k] * dn;
      p1[k % 32u] += art[jo + NDA + k] * aqd[ai.z + k];
      p2[k % 32u] += art[jo + 2u * NDA + k] * aqd[ai.z + k];
    }
    float s1 = lane_sum32(p1), s2 = lane_sum32(p2);
    float lim = it < C.FSTART ? 0.0f : art[o + 3u] * nl;
    float kd = art[o + 6u] * art[o + 8u] - art[o + 7u] * art[o + 7u];
    v2 lt = friction_pair_solve(art[o + 8u] / kd, -art[o + 7u] / kd, art[o + 6u] / kd, s1, s2, lam.y, lam.z, lim,
                                C.F_OMEGA);
    float d1 = lt.x - lam.y, d2 = lt.y - lam.z;
    for (uint32_t k = 0; k < ai.w; k++) aqd[ai.z + k] += art[yo + NDA + k] * d1 + art[yo + 2u * NDA + k] * d2;
    art[o + 9u] = nl; art[o + 10u] = lt.x; art[o + 11u] = lt.y;
  }
  return touched;
}
void Oracle::dense_phase(uint32_t mode, uint32_t it, uint32_t ph) {
  for (uint32_t a = 0; a < C.NA; a++)
    if (art_dense(a, mode, it, ph)) art_twists(a);
}
void Oracle::art_contact_impulses(uint32_t a) {
  u4 ai = art_info(a);
  bool hit = false;
  for (uint32_t k = 0; k < ai.y; k++) {
    uint32_t l = ai.x + k;
    uint32_t b = (uint32_t)link_body(l);
    v3 f = xyz(imp[b * 2u]), t = xyz(imp[b * 2u + 1u]);
    if (any_ne0(f) || any_ne0(t)) {
      hit = true;
      stsv(lo(l) + L_P, SV{-t, -f});
      imp[b * 2u] = mk4(0, 0, 0, 0);
      imp[b * 2u + 1u] = mk4(0, 0, 0, 0);
    }
  }
  if (hit) art_apply(a);
}
void Oracle::art_dof_impulse(uint32_t a, uint32_t l, uint32_t r, float dl) {
  art[lo(l) + L_TAU + r] = dl;
  art_apply(a);
}
void Oracle::art_propagate(uint32_t a, bool vlim, bool rowsOn) {
  u4 ai = art_info(a);
  if (rowsOn) {
    uint32_t n = f2u(art[C.A_RLN + a]);
    for (uint32_t i = 0; i < n; i++) {
      uint32_t d = f2u(art[C.A_RL + ai.z + i]);
      uint32_t l = f2u(dof_limit(d).w);
      art_dof_rows(a, l, d - link_dof(l), d, false, true);
    }
  }
  if (!(vlim && C.VLIM_ON == 1u && art[C.A_AVL + a] > 0.5f)) return;
  for (uint32_t k = 0; k < ai.y; k++) {
    uint32_t l = ai.x + k;
    uint32_t t = link_type(l);
    if (t != 1u && t != 0u && t != 6u) continue;  // revolute, prismatic, D6
    for (uint32_t r = 0; r < link_ndof(l); r++) art_dof_rows(a, l, r, link_dof(l) + r, true, false);
  }
}
// art_dof_rows (wgsl.js:3421-3468), joint friction and limit rows.
void Oracle::art_dof_rows(uint32_t a, uint32_t l, uint32_t r, uint32_t d, bool vlim, bool rowsOn) {
  float hinv = fmaxf_(art[C.A_HINV + d], 1e-12f);
  v4 pv = dof_passive(d);
  v4 dr = dof_drive(d);
  // drive_mode="rows" (wgsl.js:3425-3438): a PhysX-style drive row, cold-started each substep, no
  // relaxation; in the velocity pass only when velocity drives are active, against the snapshot.
  bool driven = rowsOn && C.DRIVE_ROWS == 1u && (dr.y > 0.0f || dr.z > 0.0f);
  if (driven && !(vpass && C.VEL_DRIVE_ACTIVE == 0u)) {
    float q = art[C.A_Q + link_qs(l) + r];
    float pd = 0.0f;
    if (vpass) pd = P.dt * art[C.A_SNAP + C.NB * 8u + d];
    float ca = P.dt * (P.dt * dr.y + dr.z);
    float x = 1.0f / (1.0f + ca * hinv);
    float bias = ((x * P.dt) * dr.z) * art[C.A_TGTV + d] + ((dr.y * x) * P.dt) * (((art[C.A_TGT + d] - q) - pd));
    float mx = dr.w > 0.0f ? dr.w * P.dt : 1e20f;
    float lam = art[C.A_DRV + d];
    float nl = clampf((lam * (1.0f - x) - (x * ca) * aqd[d]) + bias, -mx, mx);
    if (nl != lam) { art[C.A_DRV + d] = nl; art_dof_impulse(a, l, r, nl - lam); }
  }
  float fr = pv.y;
  if (C.JFL == 1u) fr += art[C.A_JFL + d];
  if (rowsOn && fr > 0.0f) {
    float lam = art[C.A_FRIC + d];
    float nl = clampf(lam - (C.F_OMEGA * aqd[d]) / hinv, -fr * P.dt, fr * P.dt);
    if (nl != lam) { art[C.A_FRIC + d] = nl; art_dof_impulse(a, l, r, nl - lam); }
  }
  v4 lim = dof_limit(d);
  if (rowsOn && art[C.A_LG + d] > 0.5f) {
    float q = art[C.A_Q + link_qs(l) + r];
    for (uint32_t side = 0; side < 2u; side++) {
      float sg = side == 0u ? 1.0f : -1.0f;
      float gap = side == 0u ? q - lim.x : lim.y - q;
      float lam = art[C.A_LIM + 2u * d + side];
      float rhs = gap / P.dt;
      if (gap < 0.0f) rhs = vpass ? 0.0f : fmaxf_((P.beta * gap) / P.dt, -P.max_depen);
      float nl = fmaxf_(lam - (C.F_OMEGA * (sg * aqd[d] + rhs)) / hinv, 0.0f);
      if (nl == lam) continue;
      art[C.A_LIM + 2u * d + side] = nl;
      art_dof_impulse(a, l, r, sg * (nl - lam));
    }
  }
  // Velocity limit (wgsl.js:3462-3467): a stateless push back onto |qd| <= limit, no bias.
  if (vlim && pv.z >= 0.0f && art[C.A_VLG + d] > 0.5f) {
    float over = aqd[d] - clampf(aqd[d], -pv.z, pv.z);
    if (over != 0.0f) art_dof_impulse(a, l, r, (-over) / hinv);
  }
}
// body_motion (wgsl.js:3472-3489)
v3 Oracle::body_motion(int b, v3 x) const {
  if (b < 0) return splat3(0.0f);
  v3 p0 = xyz(poses[C.P_PREV + (uint32_t)b * 2u]);
  v4 q0 = poses[C.P_PREV + (uint32_t)b * 2u + 1u];
  v3 p1 = xyz(poses[C.P_BODY + (uint32_t)b * 2u]);
  v4 q1 = poses[C.P_BODY + (uint32_t)b * 2u + 1u];
  v4 r = qmul(q1, qconj(q0));
  if (r.w < 0.0f) r = -r;
  float sn = length(xyz(r));
  v3 ang = 2.0f * xyz(r);
  v3 tr = p1 - p0;
  v3 lin = tr;
  if (sn > 1e-6f) {
    float half = atan2_o(sn, r.w);
    v3 axis = xyz(r) / sn;
    ang = (2.0f * half) * axis;
    float sc = (half * r.w) / sn;
    lin = sc * tr + ((1.0f - sc) * dot(axis, tr)) * axis;
  }
  return lin + cross(ang, x - 0.5f * (p0 + p1));
}

// nesterov_momentum (wgsl.js:3491-3557): MuJoCo's PGS acceleration on the contact rows. Each row's
// impulse is extrapolated by beta along its change since the last extrapolation, and the change
// e = y - lam reaches the twists and link impulses through the row's own response, as a sweep
// update would. rows[o + MO] keeps lam at the last extrapolation, rows[o + MO + 1] keeps e.
void Oracle::momentum_unit(uint32_t us, uint32_t row, float beta, bool init) {
  const uint32_t o = row * C.ROWS, MO = C.MO;
  v4 lam = rows[o + 6u];
  if (init) {
    rows[o + MO] = mk4(xyz(lam), 0.0f);
    rows[o + MO + 1u] = mk4(0.0f, 0.0f, 0.0f, 0.0f);
    return;
  }
  v3 y = xyz(lam) + beta * (xyz(lam) - xyz(rows[o + MO]));
  v3 e = y - xyz(lam);
  rows[o + MO] = mk4(xyz(lam), 0.0f);
  rows[o + MO + 1u] = mk4(e, 0.0f);
  if (e.x == 0.0f && e.y == 0.0f && e.z == 0.0f) return;
  rows[o + 6u] = mk4(y, lam.w);
  uint32_t key = sched[C.S_UKEY + us];
  int a = (int)(key & 0xffffu) - 1, b = (int)(key >> 16u) - 1;
  v3 ta[2], tb[2];
  load_tw(a, ta);
  load_tw(b, tb);
  ta[0] = ta[0] + ((xyz(rows[o + 7u]) * e.x + xyz(rows[o + 11u]) * e.y) + xyz(rows[o + 15u]) * e.z);
  ta[1] = ta[1] + ((xyz(rows[o + 8u]) * e.x + xyz(rows[o + 12u]) * e.y) + xyz(rows[o + 16u]) * e.z);
  tb[0] = tb[0] + ((xyz(rows[o + 9u]) * e.x + xyz(rows[o + 13u]) * e.y) + xyz(rows[o + 17u]) * e.z);
  tb[1] = tb[1] + ((xyz(rows[o + 10u]) * e.x + xyz(rows[o + 14u]) * e.y) + xyz(rows[o + 18u]) * e.z);
  v3 ra = xyz(rows[o + 3u]), rb = xyz(rows[o + 4u]);
  v3 fa = ra, fb = rb;
  if (C.EXTRA == 1u) { fa = xyz(rows[o + C.PO]); fb = xyz(rows[o + C.PO + 1u]); }
  v3 fn = xyz(rows[o]) * e.x;
  v3 ft = xyz(rows[o + 1u]) * e.y + xyz(rows[o + 2u]) * e.z;
  add_imp(a, (-fn) - ft, (-cross(ra, fn)) - cross(fa, ft));
  add_imp(b, fn + ft, cross(rb, fn) + cross(fb, ft));
  if (a >= 0) { tw[(uint32_t)a * 2u] = mk4(ta[0], 0.0f); tw[(uint32_t)a * 2u + 1u] = mk4(ta[1], 0.0f); }
  if (b >= 0) { tw[(uint32_t)b * 2u] = mk4(tb[0], 0.0f); tw[(uint32_t)b * 2u + 1u] = mk4(tb[1], 0.0f); }
}

// One momentum step before a position sweep (wgsl.js:3528-3557), with the O'Donoghue-Candes
// restart when the last sweep's correction opposed its extrapolation or friction switches on.
// The restart test sums per-invocation partials of the 256-invocation solve workgroup
// (wgsl.js:2503), each over rows tid, tid + 256, ..., then the partials in invocation order.
void Oracle::momentum_step(uint32_t ncol, uint32_t it) {
  const uint32_t NCOL = C.NCOL, WGS = 256u;
  const uint32_t nrows = wcs[NCOL + 1u];
  if (it > 0u) {
    float total = 0.0f;
    for (uint32_t t = 0; t < WGS; t++) {
      float part = 0.0f;
      for (uint32_t u = t; u < nrows; u += WGS) {
        uint32_t o = sched[C.S_PORD + u] * C.ROWS;
        v3 e = xyz(rows[o + C.MO + 1u]);
        part += dot((xyz(rows[o + 6u]) - xyz(rows[o + C.MO])) - e, e);
      }
      total += part;
    }
    float k = (total < 0.0f || it == C.FSTART) ? 0.0f : wmom_k + 1.0f;
    wmom_k = k;
    wmom_beta = k > 1.0f ? (k - 1.0f) / (k + 2.0f) : 0.0f;
  } else {
    wmom_k = 0.0f;
    wmom_beta = 0.0f;
  }
  const float beta = wmom_beta;
  for (uint32_t c = 0; c < NCOL; c++) {
    if (c >= ncol) break;
    for (uint32_t u = wcs[c]; u < wcs[c + 1u]; u++) {
      uint32_t row = sched[C.S_PORD + u];
      momentum_unit(sched[C.S_RUNIT + row], row, beta, it == 0u);
    }
  }
  for (uint32_t u = wcs[NCOL]; u < wcs[NCOL + 1u]; u++) {
    uint32_t row = sched[C.S_PORD + u];
    momentum_unit(sched[C.S_RUNIT + row], row, beta, it == 0u);
  }
  for (uint32_t a = 0; a < C.NA; a++) { art_contact_impulses(a); art_propagate(a, true, false); }
}

void Oracle::sweep(uint32_t mode, uint32_t ncol0, uint32_t it, uint32_t ph) {
  const uint32_t NCOL = C.NCOL;
  uint32_t ncol = ph == 2u ? 0u : ncol0;
  if (ph != 1u) for (uint32_t a = 0; a < C.NA; a++) art_propagate(a, false, true);
  if (C.PATCH == 1u && mode == 1u) {
    for (uint32_t us = 0; us < wn_x; us++) {
      uint32_t s0 = sched[C.S_USTART + us];
      float load = 0.0f;
      for (uint32_t m = s0; m < s0 + sched[C.S_USIZE + us]; m++)
        if (rows[m * C.ROWS + C.PO].w != 1.0f) load += rows[m * C.ROWS + 6u].x;
      art[C.A_ULOAD + us] = load;
    }
  }
  dense_phase(1u, it, ph);
  for (uint32_t c = 0; c < NCOL; c++) {
    if (c >= ncol) break;
    for (uint32_t u = wcs[c]; u < wcs[c + 1u]; u++) solve_slot(u, mode, it);
  }
  if (ph != 2u)
    for (uint32_t u = wcs[NCOL]; u < wcs[NCOL + 1u]; u++) solve_slot(std::min(u, C.MAXC - 1u), mode, it);
  for (uint32_t a = 0; a < C.NA; a++) { art_contact_impulses(a); if (ph != 1u) art_propagate(a, true, false); }
  if (C.VLIM_FREE == 1u) {
    for (uint32_t b = 0; b < C.NB; b++) {
      if (body_kind((int)b) != 1u || (body_flags((int)b) & 1u) != 0u) continue;
      v4 lim = body_limits((int)b);
      uint32_t g = C.A_VLG + C.ND + b * 6u;
      if (lim.y > 0.0f) {
        v3 v = xyz(tw[b * 2u]);
        for (int k = 0; k < 3; k++) if (art[g + k] > 0.5f) setat(v, k, clampf(at(v, k), -lim.y, lim.y));
        tw[b * 2u] = mk4(v, 0.0f);
      }
      if (lim.z > 0.0f) {
        v3 w = xyz(tw[b * 2u + 1u]);
        for (int k = 0; k < 3; k++) {
          float over = at(w, k) - clampf(at(w, k), -lim.z, lim.z);
          if (over == 0.0f || art[g + 3u + k] < 0.5f) continue;
          v3 e = splat3(0.0f);
          setat(e, k, 1.0f);
          m3 R = qmat(poses[C.P_BODY + b * 2u + 1u]);
          v3 iw = mul(R, mul(body_inv_inertia((int)b), mul(transpose(R), e)));
          w -= iw * (over / at(iw, k));
        }
        tw[b * 2u + 1u] = mk4(w, 0.0f);
      }
    }
  }
}

v4 Oracle::warm_row_value(uint32_t i, uint32_t nc) const {
  if (i < nc) {
    uint32_t o = i * C.ROWS;
    v4 lam = rows[o + 6u];
    return mk4(lam.x, xyz(rows[o + 1u]) * lam.y + xyz(rows[o + 2u]) * lam.z);
  }
  uint32_t o = C.A_DENSE + (i - nc) * C.DPS;
  return mk4(art[o + 9u], ld3(o + 12u) * art[o + 10u] + ld3(o + 15u) * art[o + 11u]);
}
uint32_t Oracle::warm_row_rank(uint32_t i, uint32_t nc) const {
  return std::min(fbits(fmaxf_(warm_row_value(i, nc).x, 0.0f)), 0xfffffffeu) + 1u;
}
uint32_t Oracle::warm_row_key(uint32_t i, uint32_t nc) const {
  if (i < nc) {
    uint32_t o = i * C.ROWS;
    return f2u(rows[o + 3u].w) | (f2u(rows[o + 4u].w) << 16u);
  }
  uint32_t o = C.A_DENSE + (i - nc) * C.DPS;
  if (art[o + 21u] > 0.5f) return 0xffffffffu;
  return f2u(art[o + 1u]) | (f2u(art[o + 2u]) << 16u);
}

// The solve kernel (wgsl.js:3634-3891).
void Oracle::k_solve() {
  const uint32_t NCOL = C.NCOL, WH = C.WH, ROWS = C.ROWS, PO = C.PO;
  uint32_t* sc = sched.data();
  wn_x = sc[C.S_META];
  wn_y = std::min(sc[C.S_META + 1u], NCOL);
  for (uint32_t i = 0; i < NCOL + 2u; i++) wcs[i] = sc[C.S_CSTART + i];
  for (uint32_t i = 0; i < C.ND; i++) aqd[i] = art[C.A_QDH + i];
  // Sleeping articulations start the solve at rest (wgsl.js:3640-3646; the reference's loop has no
  // barrier after the copy above, so its intent, these zeros, is what is restated).
  if (C.SLEEP == 1u)
    for (uint32_t a = 0; a < C.NA; a++) {
      if (!node_asleep((int)(C.NB + a))) continue;
      u4 ai = art_info(a);
      for (uint32_t d = ai.z; d < ai.z + ai.w; d++) aqd[d] = 0.0f;
    }
  for (uint32_t b = 0; b < C.NB; b++) {
    uint32_t kind = body_kind((int)b);
    imp[b * 2u] = mk4(0, 0, 0, 0);
    imp[b * 2u + 1u] = mk4(0, 0, 0, 0);
    // tw is workgroup memory in the reference (wgsl.js:2504), zero at the start of every dispatch.
    tw[b * 2u] = mk4(0, 0, 0, 0);
    tw[b * 2u + 1u] = mk4(0, 0, 0, 0);
    if (kind == 1u) {
      uint32_t fl = body_flags((int)b);
      v3 v = xyz(vel[b * 2u]) + ((node_asleep((int)b) || fl != 0u) ? splat3(0.0f) : xyz(P.gravity) * P.dt);
      v3 w = xyz(vel[b * 2u + 1u]);
      uint32_t bfo = C.A_BF + b * 8u;
      if ((fl & 1u) == 0u && (any_ne0(ld3(bfo)) || any_ne0(ld3(bfo + 4u)))) {
        m3 R = qmat(poses[C.P_BODY + b * 2u + 1u]);
        v += (ld3(bfo) * body_inv_mass((int)b)) * P.dt;
        w += mul(R, mul(body_inv_inertia((int)b), mul(transpose(R), ld3(bfo + 4u)))) * P.dt;
      }
      m3 I = body_inertia((int)b);
      bool iso = I.c[0].x == I.c[1].y && I.c[1].y == I.c[2].z && I.c[0].y == 0.0f && I.c[0].z == 0.0f && I.c[1].z == 0.0f;
      if ((fl & 1u) == 0u && !iso && any_ne0(w)) {
        m3 R = qmat(poses[C.P_BODY + b * 2u + 1u]);
        w = mul(R, gyroscopic_velocity(I, mul(transpose(R), w), P.dt));
      }
      tw[b * 2u] = mk4(v, 0.0f);
      tw[b * 2u + 1u] = mk4(w, 0.0f);
    }
  }
  for (uint32_t i = 0; i < 2u * C.ND; i++) art[C.A_LIM + i] = 0.0f;
  for (uint32_t i = 0; i < C.ND; i++) { art[C.A_FRIC + i] = 0.0f; art[C.A_DRV + i] = 0.0f; }
  uint32_t nslot = std::min(sc[C.S_CSTART + NCOL + 1u], C.MAXC);
  for (uint32_t u = 0; u < nslot; u++) {
    uint32_t row = sc[C.S_PORD + u], us = sc[C.S_RUNIT + row], key = sc[C.S_UKEY + us], s0 = sc[C.S_USTART + us];
    rows[C.MAXC * ROWS + 2u * u] = mk4((float)row, (float)us, (float)((int)(key & 0xffffu) - 1), (float)((int)(key >> 16u) - 1));
    rows[C.MAXC * ROWS + 2u * u + 1u] = mk4((float)s0, (float)(s0 + sc[C.S_USIZE + us]), 0.0f, 0.0f);
  }
  for (uint32_t a = 0; a < C.NA; a++) art_twists(a);
  dense_phase(0u, 0u, 0u);
  sweep(0u, wn_y, 0u, 0u);
  if (C.CTI == 1u) {
    // row_schedule "contact_then_internal" (wgsl.js:3693-3696): all contact iterations, then the
    // joint-internal rows.
    for (uint32_t it = 0; it < P.iterations; it++) {
      if (C.NEST == 1u) momentum_step(wn_y, it);
      sweep(1u, wn_y, it, 1u);
    }
    for (uint32_t it = 0; it < P.iterations; it++) sweep(1u, wn_y, it, 2u);
  } else {
    for (uint32_t it = 0; it < P.iterations; it++) {
      if (C.NEST == 1u) momentum_step(wn_y, it);
      sweep(1u, wn_y, it, 0u);
    }
  }
  // Velocity pass (velocity_iterations, wgsl.js:3700-3736): positions integrate with the velocities
  // reached here; further bias-free sweeps from the accumulated impulses set the output velocities.
  if (C.VELITERS > 0u) {
    for (uint32_t b = 0; b < C.NB; b++) {
      st3(C.A_SNAP + b * 8u, xyz(tw[b * 2u]));
      st3(C.A_SNAP + b * 8u + 4u, xyz(tw[b * 2u + 1u]));
    }
    for (uint32_t i = 0; i < C.ND; i++) art[C.A_SNAP + C.NB * 8u + i] = aqd[i];
    // Contact rhs without bias: 0, or a speculative gap still open at the snapshot velocity.
    for (uint32_t us = 0; us < wn_x; us++) {
      uint32_t key = sc[C.S_UKEY + us];
      int a = (int)(key & 0xffffu) - 1, b = (int)(key >> 16u) - 1;
      v3 ta[2], tb[2];
      load_tw(a, ta);
      load_tw(b, tb);
      uint32_t s0 = sc[C.S_USTART + us];
      for (uint32_t i = s0; i < s0 + sc[C.S_USIZE + us]; i++) {
        uint32_t o = i * ROWS;
        float phi = rows[o + 6u].w;
        if (phi >= 1e29f) continue;
        v3 n = xyz(rows[o]);
        float jv = dot(n, (tb[0] + cross(tb[1], xyz(rows[o + 4u]))) - (ta[0] + cross(ta[1], xyz(rows[o + 3u]))));
        rows[o + 1u].w = (phi > 0.0f && phi + P.dt * jv > 1e-6f) ? phi / P.dt : 0.0f;
      }
    }
    uint32_t nd = std::min(sc[C.S_META + 3u], C.MAXDENSE);
    for (uint32_t i = 0; i < nd; i++) {
      uint32_t o = C.A_DENSE + i * C.DPS;
      if (art[o + 21u] > 0.5f || art[o + 22u] >= 1e29f) continue;
      u4 ai = art_info(f2u(art[o]));
      float jv = 0.0f;
      for (uint32_t k = 0; k < ai.w; k++) jv += art[o + C.DHDR + k] * aqd[ai.z + k];
      float phi = art[o + 22u];
      art[o + 4u] = (phi > 0.0f && phi + P.dt * jv > 1e-6f) ? phi / P.dt : 0.0f;
    }
    vpass = true;
    for (uint32_t it = 0; it < C.VELITERS; it++) sweep(1u, wn_y, P.iterations + it, 0u);
    vpass = false;
  }
  // Warm-start table store (wgsl.js:3737-3767).
  uint32_t nc = sc[C.S_USTART + wn_x];
  uint32_t ndense = std::min(sc[C.S_META + 3u], C.MAXDENSE);
  uint32_t wbase = (1u - P.parity) * WH;
  for (uint32_t i = 0; i < nc + ndense; i++) {
    uint32_t key = warm_row_key(i, nc);
    sc[C.S_WSLOT + i] = 0xffffffffu;
    if (key == 0xffffffffu) continue;
    uint32_t h = key % WH;
    for (uint32_t probe = 0; probe < 32u; probe++) {
      uint32_t old = warm[wbase + h];
      if (old == 0u) warm[wbase + h] = key;
      if (old == 0u || old == key) {
        sc[C.S_WWIN + h] = std::max(sc[C.S_WWIN + h], warm_row_rank(i, nc));
        sc[C.S_WSLOT + i] = h;
        break;
      }
      h = (h + 1u) % WH;
    }
  }
  for (uint32_t i = 0; i < nc + ndense; i++) {
    uint32_t key = warm_row_key(i, nc);
    if (key == 0xffffffffu) continue;
    uint32_t h = sc[C.S_WSLOT + i];
    if (h >= WH || warm[wbase + h] != key || sc[C.S_WWIN + h] != warm_row_rank(i, nc)) continue;
    v4 v = warm_row_value(i, nc);
    uint32_t vo = 2u * WH + (wbase + h) * 4u;
    warm[vo] = fbits(v.x); warm[vo + 1u] = fbits(v.y); warm[vo + 2u] = fbits(v.z); warm[vo + 3u] = fbits(v.w);
  }
  // Integrate.
  if (C.PATCH == 1u) for (uint32_t b = 0; b < C.NB * 2u; b++) poses[C.P_PREV + b] = poses[C.P_BODY + b];
  for (uint32_t b = 0; b < C.NB; b++) {
    if (body_kind((int)b) != 1u) continue;
    v3 v = xyz(tw[b * 2u]), w = xyz(tw[b * 2u + 1u]);
    float damp = (body_flags((int)b) & 1u) != 0u ? 1.0f : 1.0f - body_limits((int)b).x * P.dt;
    vel[b * 2u] = mk4(v, 0.0f);
    vel[b * 2u + 1u] = mk4(w * damp, 0.0f);
    if (C.VELITERS > 0u) {
      v3 s2[2];
      snap_tw((int)b, s2);
      v = s2[0];
      w = s2[1];
    }
    if (node_asleep((int)b)) {
      vel[b * 2u] = mk4(0, 0, 0, 0);
      vel[b * 2u + 1u] = mk4(0, 0, 0, 0);
      continue;
    }
    v3 c = xyz(poses[C.P_BODY + b * 2u]) + v * P.dt;
    v4 q = poses[C.P_BODY + b * 2u + 1u];
    q = normalize(q + (0.5f * P.dt) * qmul(mk4(w, 0.0f), q));
    poses[C.P_BODY + b * 2u] = mk4(c, 0.0f);
    poses[C.P_BODY + b * 2u + 1u] = q;
  }
  for (uint32_t i = 0; i < C.ND; i++) {
    art[C.A_QD + i] = aqd[i];
    if (C.VELITERS > 0u) aqd[i] = art[C.A_SNAP + C.NB * 8u + i];
  }
  for (uint32_t l = 0; l < C.NL; l++) {
    if (link_type(l) != 4u || link_parent(l) >= 0) continue;
    float k = 1.0f - body_limits(link_body(l)).x * P.dt;
    uint32_t d = link_dof(l);
    art[C.A_QD + d + 3u] *= k; art[C.A_QD + d + 4u] *= k; art[C.A_QD + d + 5u] *= k;
  }
  for (uint32_t a = 0; a < C.NA; a++) {
    u4 ai = art_info(a);
    for (uint32_t k = 0; k < ai.y; k++) {
      uint32_t l = ai.x + k, qs = link_qs(l), d = link_dof(l), t = link_type(l);
      float* Q = &art[C.A_Q];
      if (t == 1u || t == 0u || t == 6u)
        for (uint32_t r = 0; r < link_ndof(l); r++) Q[qs + r] += aqd[d + r] * P.dt;
      if (t == 2u) {
        v3 w = mk3(aqd[d], aqd[d + 1u], aqd[d + 2u]);
        v4 q = mk4(Q[qs], Q[qs + 1], Q[qs + 2], Q[qs + 3]);
        q = normalize(q + (0.5f * P.dt) * qmul(mk4(w, 0.0f), q));
        Q[qs] = q.x; Q[qs + 1] = q.y; Q[qs + 2] = q.z; Q[qs + 3] = q.w;
      }
      if (t == 4u) {
        for (uint32_t c = 0; c < 3u; c++) Q[qs + c] += aqd[d + c] * P.dt;
        v3 w = mk3(aqd[d + 3u], aqd[d + 4u], aqd[d + 5u]);
        v4 q = mk4(Q[qs + 3], Q[qs + 4], Q[qs + 5], Q[qs + 6]);
        q = normalize(q + (0.5f * P.dt) * qmul(mk4(w, 0.0f), q));
        Q[qs + 3] = q.x; Q[qs + 4] = q.y; Q[qs + 5] = q.z; Q[qs + 6] = q.w;
      }
    }
    art_fk(a);
    for (uint32_t k = 0; k < ai.y; k++) {
      uint32_t l = ai.x + k;
      uint32_t b = (uint32_t)link_body(l);
      poses[C.P_BODY + b * 2u] = mk4(ld3(lo(l) + L_COM), 0.0f);
      poses[C.P_BODY + b * 2u + 1u] = link_rot(l);
    }
  }
  // Friction anchors: advance and store (wgsl.js:3832-3878).
  if (C.PATCH == 1u) {
    uint32_t ab = AK() + (1u - P.parity) * C.AH;
    const float keep_frac = (float)(1.0 - 1e-5);
    for (uint32_t i = 0; i < nc; i++) {
      uint32_t o = i * ROWS;
      if (rows[o + PO].w != 2.0f) continue;
      uint32_t pair = fbits(rows[o + PO + 3u].w);
      int a = (int)(pair & 0xffffu) - 1, b = (int)(pair >> 16u) - 1;
      v3 fra = xyz(rows[o + PO]), frb = xyz(rows[o + PO + 1u]);
      uint32_t k = f2u(rows[o + PO + 1u].w);
      v4 ex = rows[o + PO + 2u];
      float lim = ex.w;
      if (lim <= 0.0f) continue;
      v3 n = xyz(rows[o]), t1 = xyz(rows[o + 1u]), t2 = xyz(rows[o + 2u]);
      v3 ta[2], tb[2];
      load_tw(a, ta);
      load_tw(b, tb);
      if (C.VELITERS > 0u) { snap_tw(a, ta); snap_tw(b, tb); }
      v3 vrel = (tb[0] + cross(tb[1], frb)) - (ta[0] + cross(ta[1], fra));
      v4 lam = rows[o + 6u];
      v3 lt = t1 * lam.y + t2 * lam.z;
      float r = fmaxf_(fminf_(body_radius(a), body_radius(b)), 1e-4f);
      if (length(lt) >= keep_frac * lim && dot(vrel, lt) < (((-lim) * 1e-5f) * r) / P.dt) continue;
      v4 qa = mk4(0, 0, 0, 1);
      v3 ca = splat3(0.0f);
      if (a >= 0) { qa = poses[C.P_BODY + (uint32_t)a * 2u + 1u]; ca = xyz(poses[C.P_BODY + (uint32_t)a * 2u]); }
      v3 ll = xyz(rows[o + PO + 3u]);
      v3 x = ca + qrot(qa, ll);
      v3 e = (xyz(ex) + body_motion(b, x)) - body_motion(a, x);
      e -= n * dot(n, e);
      v3 el = qinvrot(qa, e);
      uint32_t hk = anchor_hash(pair, k);
      uint32_t h = hk % C.AH;
      for (uint32_t probe = 0; probe < 32u; probe++) {
        if (warm[ab + h] == 0u) {
          warm[ab + h] = hk;
          uint32_t vo = AV() + ((1u - P.parity) * C.AH + h) * AVN;
          v3 il = qinvrot(qa, lt), nl_ = qinvrot(qa, n);
          warm[vo + 11u] = fbits(nl_.x); warm[vo + 12u] = fbits(nl_.y); warm[vo + 13u] = fbits(nl_.z);
          warm[vo + 8u] = fbits(il.x); warm[vo + 9u] = fbits(il.y); warm[vo + 10u] = fbits(il.z);
          warm[vo] = pair; warm[vo + 1u] = k;
          warm[vo + 2u] = fbits(ll.x); warm[vo + 3u] = fbits(ll.y); warm[vo + 4u] = fbits(ll.z);
          warm[vo + 5u] = fbits(el.x); warm[vo + 6u] = fbits(el.y); warm[vo + 7u] = fbits(el.z);
          break;
        }
        h = (h + 1u) % C.AH;
      }
    }
  }
  stats[1] = std::max(stats[1], counters[1]);
  stats[2] = std::max(stats[2], wn_y);
  stats[3] = std::max(stats[3], wn_x);
  stats[4] = std::max(stats[4], counters[0]);
  stats[5] = counters[1];
  stats[6] = wn_y;
  stats[8] = sc[C.S_META + 5u];
  stats[7] = std::max(stats[7], sc[C.S_META + 3u]);
  counters[0] = 0u;
  counters[1] = 0u;
}

}  // namespace orc
