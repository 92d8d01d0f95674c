// Test infrastructure (oracle): shapes, broad, narrow and csort kernels.
// Restates wgsl.js:117-177 (shapes, broad), 182-1217 (narrow), 3899-3993 (csort, args).
#include <algorithm>
#include <cmath>

#include "oracle.h"

namespace orc {

static const uint32_t NLANE = 32u;
static const uint32_t GT_PLANE = 1u, GT_SPHERE = 3u, GT_CAPSULE = 4u, GT_CYL = 6u, GT_BOX = 7u, GT_CONE = 9u,
                      GT_CONVEX = 10u;
static const float MEPS = 1e-5f;
static const float COS_TILT = 0.9993908270190958f;
static const float SIN_TILT = 0.03489949670250097f;
static const float COS_DEEP = 0.9999984769132877f;
static const float WITNESS_TOL = 1e-3f;
static const float SAT_TIE = 1e-5f;
static const v2 PENT[5] = {{1.0f, 0.0f},
                           {0.30901699437494745f, 0.9510565162951535f},
                           {-0.8090169943749473f, 0.5877852522924732f},
                           {-0.8090169943749476f, -0.587785252292473f},
                           {0.30901699437494723f, -0.9510565162951536f}};

static inline float sel(float f, float t, bool c) { return c ? t : f; }

// --- shapes (wgsl.js:117-150) ---
void Oracle::k_shapes() {
  for (uint32_t s = 0; s < C.NS; s++) {
    uint32_t o = C.SF_SHAPE + s * 7u;
    int body = f2i(statF[o].x);
    uint32_t hull = f2u(statF[o].y);
    v3 bp = splat3(0.0f);
    v4 bq = mk4(0, 0, 0, 1);
    if (body >= 0) {
      v3 c = xyz(poses[C.P_BODY + (uint32_t)body * 2u]);
      bq = poses[C.P_BODY + (uint32_t)body * 2u + 1u];
      bp = c - qrot(bq, body_com_local(body));
    }
    v3 sp = bp + qrot(bq, xyz(statF[o + 1u]));
    v4 sq = normalize(qmul(bq, statF[o + 2u]));
    poses[C.P_SHAPE + s * 2u] = mk4(sp, 0.0f);
    poses[C.P_SHAPE + s * 2u + 1u] = sq;
    if (statF[o + 3u].x == 4.0f) {
      poses[C.P_AABB + s * 2u] = mk4(splat3(-1e6f), 0.0f);
      poses[C.P_AABB + s * 2u + 1u] = mk4(splat3(1e6f), 0.0f);
      continue;
    }
    v3 hc = xyz(statF[C.SF_HAABB + hull * 2u]);
    v3 hh = xyz(statF[C.SF_HAABB + hull * 2u + 1u]);
    m3 m = qmat(sq);
    v3 c = sp + mul(m, hc);
    v3 e = ((vabs(m.c[0]) * hh.x + vabs(m.c[1]) * hh.y) + vabs(m.c[2]) * hh.z) + splat3(statF[o].w);
    poses[C.P_AABB + s * 2u] = mk4(c - e, 0.0f);
    poses[C.P_AABB + s * 2u + 1u] = mk4(c + e, 0.0f);
  }
}

// --- broad (wgsl.js:154-177), all pairs in (i, j) order ---
void Oracle::k_broad() {
  for (uint32_t i = 0; i < C.NS; i++) {
    for (uint32_t j = i + 1; j < C.NS; j++) {
      int bi = f2i(statF[C.SF_SHAPE + i * 7u].x);
      int bj = f2i(statF[C.SF_SHAPE + j * 7u].x);
      if (bi == bj) continue;
      if (bi < 0 && bj < 0) continue;
      bool fi = bi < 0 || body_kind(bi) == 3u || (body_flags(bi) & 1u) != 0u;
      bool fj = bj < 0 || body_kind(bj) == 3u || (body_flags(bj) & 1u) != 0u;
      if (fi && fj) continue;
      uint32_t k = i * C.NS + j;
      if ((statU[C.SU_FILTER + (k >> 5u)] & (1u << (k & 31u))) != 0u) continue;
      v3 lo_i = xyz(poses[C.P_AABB + i * 2u]), hi_i = xyz(poses[C.P_AABB + i * 2u + 1u]);
      v3 lo_j = xyz(poses[C.P_AABB + j * 2u]), hi_j = xyz(poses[C.P_AABB + j * 2u + 1u]);
      if (lo_i.x > hi_j.x || lo_i.y > hi_j.y || lo_i.z > hi_j.z || lo_j.x > hi_i.x || lo_j.y > hi_i.y ||
          lo_j.z > hi_i.z)
        continue;
      uint32_t slot = counters[0]++;
      if (slot < C.MAXP) { pairs[slot * 2u] = i; pairs[slot * 2u + 1u] = j; }
    }
  }
}

// --- narrow helpers (wgsl.js:197-259) ---
FaceQ Oracle::face_query(uint32_t ha, uint32_t hb, v4 rq, v3 t, uint32_t lane) const {
  FaceQ best{-1e30f, 0u};
  uint32_t fo = hfo(ha), nf = hnf(ha), nv = hnv(hb);
  for (uint32_t f = lane; f < nf; f += NLANE) {
    v4 pl = fplane(fo + f);
    v3 nb = qinvrot(rq, xyz(pl));
    float m = 1e30f;
    for (uint32_t v = 0; v < nv; v++) m = fminf_(m, dot(nb, hv(hb, v)));
    float s = (m + dot(xyz(pl), t)) - pl.w;
    if (s > best.sep) best = FaceQ{s, f};
  }
  return best;
}
float Oracle::support_min(uint32_t h, v3 n) const {
  float m = 1e30f;
  for (uint32_t v = 0; v < hnv(h); v++) m = fminf_(m, dot(n, hv(h, v)));
  return m;
}
float Oracle::support_max(uint32_t h, v3 n) const {
  float m = -1e30f;
  for (uint32_t v = 0; v < hnv(h); v++) m = fmaxf_(m, dot(n, hv(h, v)));
  return m;
}
EdgeQ Oracle::edge_query(uint32_t ha, uint32_t hb, v4 rq, v3 t, uint32_t lane) const {
  EdgeQ best{-1e30f, splat3(0), splat3(0), splat3(0), splat3(0), splat3(0), 0u};
  uint32_t foa = hfo(ha), fob = hfo(hb);
  v3 cena = xyz(statF[C.SF_HAABB + ha * 2u]);
  v3 cenb = qrot(rq, xyz(statF[C.SF_HAABB + hb * 2u])) + t;
  uint32_t nea = hne(ha), neb = hne(hb);
  for (uint32_t k = lane; k < nea * neb; k += NLANE) {
    u4 ea_ = hedge(ha, k / neb), eb_ = hedge(hb, k % neb);
    v3 a = xyz(fplane(foa + ea_.z)), b = xyz(fplane(foa + ea_.w));
    v3 c = -qrot(rq, xyz(fplane(fob + eb_.z))), d = -qrot(rq, xyz(fplane(fob + eb_.w)));
    v3 bxa = cross(b, a), dxc = cross(d, c);
    float cba = dot(c, bxa), dba = dot(d, bxa), adc = dot(a, dxc), bdc = dot(b, dxc);
    if (cba * dba > 1e-3f || adc * bdc > 1e-3f || cba * bdc < -1e-3f) continue;
    uint32_t va0 = ea_.x, va1 = ea_.y, vb0 = eb_.x, vb1 = eb_.y;
    v3 a0 = hv(ha, va0), a1 = hv(ha, va1);
    v3 ea = a1 - a0;
    v3 b0 = qrot(rq, hv(hb, vb0)) + t, b1 = qrot(rq, hv(hb, vb1)) + t;
    v3 ax = cross(ea, b1 - b0);
    float l = length(ax);
    if (l < (1e-6f * length(ea)) * length(b1 - b0)) continue;
    ax = ax / l;
    if (dot(ax, cenb - cena) < 0.0f) ax = -ax;
    float amax = support_max(ha, ax);
    float bmin = dot(ax, t) + support_min(hb, qinvrot(rq, ax));
    float s = bmin - amax;
    float tol = 1e-4f + 1e-3f * (length(ea) + length(b1 - b0));
    if (dot(ax, a0) < amax - tol || dot(ax, a1) < amax - tol || dot(ax, b0) > bmin + tol || dot(ax, b1) > bmin + tol)
      continue;
    if (s > best.sep) best = EdgeQ{s, ax, a0, a1, b0, b1, (va0 << 24u) ^ (va1 << 16u) ^ (vb0 << 8u) ^ vb1};
  }
  return best;
}

static inline float combine(float a, float b, uint32_t mode) {
  if (mode == 1u) return fminf_(a, b);
  if (mode == 2u) return a * b;
  if (mode == 3u) return fmaxf_(a, b);
  return 0.5f * (a + b);
}

// emit (wgsl.js:269-307); the narrowphase writes craw.
void Oracle::emit(uint32_t sa, uint32_t sb, v3 p, v3 n, float phi, uint32_t key) {
  const uint32_t SA = C.SF_SHAPE + sa * 7u, SB = C.SF_SHAPE + sb * 7u;
  int ba = f2i(statF[SA].x), bb = f2i(statF[SB].x);
  v4 ma = statF[SA + 4u], mb = statF[SB + 4u];
  float mu = combine(statF[SA].z, statF[SB].z, C.FRICTION_COMBINE);
  bool art_c = (ba >= 0 && body_kind(ba) >= 2u) || (bb >= 0 && body_kind(bb) >= 2u);
  float mt = 0.0f, mr = 0.0f;
  if (art_c) {
    if (C.ANG_ART == 1u) { mt = combine(ma.y, mb.y, C.FRICTION_COMBINE); mr = combine(ma.z, mb.z, C.FRICTION_COMBINE); }
  } else {
    mt = fmaxf_(sel(0.0f, ma.y, ma.w >= 4.0f), sel(0.0f, mb.y, mb.w >= 4.0f));
    mr = fmaxf_(sel(0.0f, ma.z, ma.w >= 6.0f), sel(0.0f, mb.z, mb.w >= 6.0f));
    if (C.F_FR_MUT >= 0.0f) mt = C.F_FR_MUT;
    if (C.F_FR_MUR >= 0.0f) mr = C.F_FR_MUR;
  }
  float tr = sel(0.0f, fmaxf_(statF[SA + 3u].w, statF[SB + 3u].w), art_c);
  v3 mat = mk3(combine(clampf(ma.x, 0.0f, 1.0f), clampf(mb.x, 0.0f, 1.0f), C.RESTITUTION_COMBINE), mt, mr);
  int a = ba, b = bb;
  v3 nn = n;
  v2 smu = mk2(statF[SA].z, statF[SB].z);
  if (a > b) { a = bb; b = ba; nn = -n; smu = mk2(smu.y, smu.x); }
  uint32_t k = counters[1]++;
  if (k >= C.MAXC) return;
  craw[C.MAXC * 5u + k] = mk4(smu.x, smu.y, 0.0f, 0.0f);
  craw[k * 5u] = mk4(p, phi);
  craw[k * 5u + 1u] = mk4(nn, mu);
  craw[k * 5u + 2u] = mk4((float)a, (float)b, (float)(key & 0xffffu), (float)(key >> 16u));
  craw[k * 5u + 3u] = mk4(mat, tr);
  float ka = statF[SA + 5u].x, kb = statF[SB + 5u].x;
  float kc = sel(0.0f, (ka * kb) / (ka + kb), ka > 0.0f && kb > 0.0f);
  float ga = statF[SA + 5u].z, gb = statF[SB + 5u].z;
  if (ba > bb) { float t = ga; ga = gb; gb = t; }
  craw[k * 5u + 4u] = mk4(kc, statF[SA + 5u].y + statF[SB + 5u].y, ga, gb);
}

// Lane-major support scan: the subgroup max/min-lane reduction of wgsl.js:312-331.
v3 Oracle::sup_lane(uint32_t h, v3 d) const {
  float best = -1e30f;
  v3 bp = splat3(0.0f);
  uint32_t nv = hnv(h);
  for (uint32_t l = 0; l < NLANE; l++)
    for (uint32_t v = l; v < nv; v += NLANE) {
      v3 x = hv(h, v);
      float s = dot(d, x);
      if (s > best) { best = s; bp = x; }
    }
  return bp;
}
v3 Oracle::sup_md(uint32_t ha, uint32_t hb, v4 rq, v3 t, float r, v3 d) const {
  v3 sb = qrot(rq, sup_lane(hb, qinvrot(rq, d))) + t;
  v3 sa = sup_lane(ha, -d);
  return (sb - sa) + (2.0f * r) * normalize(d);
}

// MPR (wgsl.js:342-389).
v4 Oracle::mpr(uint32_t ha, uint32_t hb, v4 rq, v3 t, float r) const {
  const v4 none = mk4(0.0f, 0.0f, 1.0f, -1.0f);
  v3 v0 = (qrot(rq, xyz(statF[C.SF_HAABB + hb * 2u])) + t) - xyz(statF[C.SF_HAABB + ha * 2u]);
  if (dot(v0, v0) < 1e-14f) v0 = mk3(1e-5f, 0.0f, 0.0f);
  v3 n = -v0;
  v3 v1 = sup_md(ha, hb, rq, t, r, n);
  if (dot(v1, n) <= 0.0f) return none;
  n = cross(v1, v0);
  if (dot(n, n) < 1e-14f) {
    v3 nn = normalize(v1 - v0);
    return mk4(nn, dot(v1, nn));
  }
  v3 v2 = sup_md(ha, hb, rq, t, r, n);
  if (dot(v2, n) <= 0.0f) return none;
  n = cross(v1 - v0, v2 - v0);
  if (dot(n, v0) > 0.0f) { v3 tmp = v1; v1 = v2; v2 = tmp; n = -n; }
  v3 v3_ = splat3(0.0f);
  bool found = false;
  for (uint32_t i = 0; i < 32u; i++) {
    v3_ = sup_md(ha, hb, rq, t, r, n);
    if (dot(v3_, n) <= 0.0f) return none;
    if (dot(cross(v1, v3_), v0) < 0.0f) { v2 = v3_; n = cross(v1 - v0, v3_ - v0); continue; }
    if (dot(cross(v3_, v2), v0) < 0.0f) { v1 = v3_; n = cross(v3_ - v0, v2 - v0); continue; }
    found = true;
    break;
  }
  if (!found) return none;
  for (uint32_t i = 0; i < 32u; i++) {
    n = cross(v2 - v1, v3_ - v1);
    float ln = length(n);
    if (ln < 1e-12f) break;
    n = n / ln;
    if (dot(n, v1 - v0) < 0.0f) n = -n;
    v3 v4_ = sup_md(ha, hb, rq, t, r, n);
    float d1 = dot(n, v1);
    if (dot(v4_, n) - d1 < 1e-6f || i == 31u) {
      if (d1 < 0.0f) return none;
      return mk4(n, d1);
    }
    if (dot(v4_, n) < 0.0f) return none;
    v3 c = cross(v4_, v0);
    if (dot(v1, c) > 0.0f) {
      if (dot(v2, c) > 0.0f) v1 = v4_; else v3_ = v4_;
    } else {
      if (dot(v3_, c) > 0.0f) v2 = v4_; else v1 = v4_;
    }
  }
  float d1 = dot(n, v1);
  if (d1 < 0.0f) return none;
  return mk4(n, d1);
}

static void closest_seg(v3 a0, v3 a1, v3 b0, v3 b1, v3 out[2]) {
  v3 d1 = a1 - a0, d2 = b1 - b0, r = a0 - b0;
  float a = dot(d1, d1), e = dot(d2, d2), f = dot(d2, r);
  float s = 0.0f, t = 0.0f;
  if (a <= 1e-12f && e <= 1e-12f) { out[0] = a0; out[1] = b0; return; }
  if (a <= 1e-12f) {
    t = clampf(f / e, 0.0f, 1.0f);
  } else {
    float c = dot(d1, r);
    if (e <= 1e-12f) {
      s = clampf(-c / a, 0.0f, 1.0f);
    } else {
      float b = dot(d1, d2), den = a * e - b * b;
      if (den > 1e-12f) s = clampf((b * f - c * e) / den, 0.0f, 1.0f);
      t = (b * s + f) / e;
      if (t < 0.0f) { t = 0.0f; s = clampf(-c / a, 0.0f, 1.0f); }
      else if (t > 1.0f) { t = 1.0f; s = clampf((b - c) / a, 0.0f, 1.0f); }
    }
  }
  out[0] = a0 + d1 * s;
  out[1] = b0 + d2 * t;
}

static void sphere_sphere(v3 p1, float r1, v3 p2, float r2, v4 out[2]) {
  v3 dv = p2 - p1;
  float l = length(dv);
  v3 n = (l == 0.0f) ? mk3(1.0f, 0.0f, 0.0f) : dv / l;
  float d = l - (r1 + r2);
  out[0] = mk4(p1 + n * (r1 + 0.5f * d), d);
  out[1] = mk4(n, 0.0f);
}

// prim_prim (wgsl.js:424-454).
void Oracle::prim_prim(uint32_t sa, uint32_t sb, v3 pa, v4 qa, v3 pb, v4 qb, float thresh) {
  v4 A = statF[C.SF_SHAPE + sa * 7u + 6u], B = statF[C.SF_SHAPE + sb * 7u + 6u];
  v3 ua = qrot(qa, mk3(0.0f, 0.0f, A.z)), ub = qrot(qb, mk3(0.0f, 0.0f, B.z));
  uint32_t base = hash_u32(sa * 7919u + sb * 104729u);
  v4 c[2][2] = {};
  uint32_t nc = 1u;
  if (f2u(A.x) == GT_SPHERE) {
    v3 a = pb - ub, ab = (pb + ub) - a;
    sphere_sphere(pa, A.y, a + clampf(dot(pa - a, ab) / (dot(ab, ab) + 1e-6f), 0.0f, 1.0f) * ab, B.y, c[0]);
  } else {
    v3 dif = pa - pb;
    float ma = dot(ua, ua), mb = -dot(ua, ub), mc = dot(ub, ub);
    float u = -dot(ua, dif), v = dot(ub, dif);
    float det = ma * mc - mb * mb;
    if (std::fabs(det) >= 1e-15f) {
      float inv_det = 1.0f / det;
      float x1 = (mc * u - mb * v) * inv_det, x2 = (ma * v - mb * u) * inv_det;
      if (x1 > 1.0f) { x1 = 1.0f; x2 = (v - mb) / mc; } else if (x1 < -1.0f) { x1 = -1.0f; x2 = (v + mb) / mc; }
      if (x2 > 1.0f) { x2 = 1.0f; x1 = clampf((u - mb) / ma, -1.0f, 1.0f); }
      else if (x2 < -1.0f) { x2 = -1.0f; x1 = clampf((u + mb) / ma, -1.0f, 1.0f); }
      sphere_sphere(pa + ua * x1, A.y, pb + ub * x2, B.y, c[0]);
    } else {
      sphere_sphere(pa + ua, A.y, pb + ub * clampf((v - mb) / mc, -1.0f, 1.0f), B.y, c[0]);
      sphere_sphere(pa - ua, A.y, pb + ub * clampf((v + mb) / mc, -1.0f, 1.0f), B.y, c[1]);
      c[1][1] = c[0][1];
      nc = 2u;
    }
  }
  for (uint32_t i = 0; i < nc; i++)
    if (c[i][0].w <= thresh) emit(sa, sb, xyz(c[i][0]), xyz(c[0][1]), c[i][0].w, hash_u32(base ^ (i * 977u + 13u)));
}

// plane_contacts (wgsl.js:458-540).
void Oracle::plane_contacts(uint32_t pl, uint32_t os, v3 pp, v4 pq, v3 op, v4 oq, float thresh, bool flip) {
  v3 n = qrot(pq, mk3(0.0f, 0.0f, 1.0f));
  uint32_t sa = flip ? os : pl, sb = flip ? pl : os;
  v3 nab = flip ? -n : n;
  uint32_t base = hash_u32(sa * 7919u + sb * 104729u);
  v4 g = statF[C.SF_SHAPE + os * 7u + 6u];
  uint32_t gt = f2u(g.x);
  float d[4] = {1e30f, 1e30f, 1e30f, 1e30f};
  v3 x[4] = {};
  uint32_t nc = 0u;
  if (gt == GT_SPHERE || gt == GT_CAPSULE) {
    v3 u = qrot(oq, mk3(0.0f, 0.0f, g.z));
    uint32_t cnt = gt == GT_SPHERE ? 1u : 2u;
    for (uint32_t i = 0; i < cnt; i++) {
      v3 e = op + (i == 1u ? -u : u);
      d[i] = dot(n, e - pp) - g.y;
      x[i] = e - n * (g.y + 0.5f * d[i]);
    }
    nc = cnt;
  } else if (gt == GT_BOX) {
    float cd0 = dot(op - pp, n);
    uint32_t worst = 0u;
    m3 rot = qmat(oq);
    for (uint32_t i = 0; i < 8u; i++) {
      v3 c = mul(rot, mk3((i & 1u) ? g.y : -g.y, (i & 2u) ? g.z : -g.z, (i & 4u) ? g.w : -g.w));
      float cd = cd0 + dot(n, c);
      if (cd > thresh) continue;
      v3 cp = (c + op) - (0.5f * n) * cd;
      if (nc < 4u) {
        d[nc] = cd; x[nc] = cp;
        if (nc == 0u || cd > d[worst]) worst = nc;
        nc++;
      } else if (cd < d[worst]) {
        d[worst] = cd; x[worst] = cp;
        worst = 0u;
        for (uint32_t k = 1; k < 4u; k++) if (d[k] > d[worst]) worst = k;
      }
    }
  } else if (gt == GT_CYL) {
    v3 ax = qrot(oq, mk3(0.0f, 0.0f, 1.0f));
    float dna = dot(n, ax);
    if (dna > 0.0f) { ax = -ax; dna = -dna; }
    v3 cap = op + ax * g.z;
    v3 pa = -n + ax * dna;
    float l2 = dot(pa, pa);
    bool has = l2 > 1e-10f;
    if (has) pa = pa * (1.0f / std::sqrt(l2));
    bool flat = -dna >= 0.9238795325112867f;
    v3 pf = splat3(0.0f);
    if (flat || !has) {
      v3 rf = mk3(1.0f, 0.0f, 0.0f);
      if (std::fabs(dot(ax, rf)) > 0.9f) rf = mk3(0.0f, 1.0f, 0.0f);
      pf = normalize(rf - ax * dot(ax, rf));
    }
    v3 dp = has ? pa : pf;
    v3 dpt = cap + dp * g.y;
    d[0] = dot(dpt - pp, n);
    x[0] = dpt - n * (d[0] * 0.5f);
    nc = 1u;
    float mt = 0.01f * fmaxf_(g.y, g.z);
    v3 cand[3] = {};
    uint32_t ncand = 0u;
    if (flat) {
      v3 u = pf * g.y, v = cross(ax, pf) * g.y;
      cand[0] = cap + u;
      cand[1] = (cap - 0.5f * u) + 0.8660254f * v;
      cand[2] = (cap - 0.5f * u) - 0.8660254f * v;
      ncand = 3u;
    } else {
      v3 u = dp * g.y, v = cross(ax, dp) * g.y;
      cand[0] = (op - ax * g.z) + u;
      float dpv = dot((cap + v) - pp, n), dnv = dot((cap - v) - pp, n);
      cand[1] = dpv <= dnv ? cap + v : cap - v;
      ncand = 2u;
    }
    for (uint32_t k = 0; k < ncand; k++) {
      float dk = dot(cand[k] - pp, n);
      v3 pk = cand[k] - n * (dk * 0.5f);
      if (nc < 4u && dot(pk - x[0], pk - x[0]) > mt * mt) { d[nc] = dk; x[nc] = pk; nc++; }
    }
  }
  for (uint32_t i = 0; i < nc; i++)
    if (d[i] <= thresh) emit(sa, sb, x[i], nab, d[i], hash_u32(base ^ (i + 7u)));
}

// Segment paths (wgsl.js:543-624).
FaceQ Oracle::face_query_seg(uint32_t h, v3 e0, v3 e1, float r, uint32_t lane) const {
  FaceQ best{-1e30f, 0u};
  uint32_t fo = hfo(h);
  for (uint32_t f = lane; f < hnf(h); f += NLANE) {
    v4 pl = fplane(fo + f);
    float s = (fminf_(dot(xyz(pl), e0), dot(xyz(pl), e1)) - pl.w) - r;
    if (s > best.sep) best = FaceQ{s, f};
  }
  return best;
}
bool Oracle::seg_hits_hull(uint32_t h, v3 e0, v3 e1) const {
  float t0 = 0.0f, t1 = 1.0f;
  for (uint32_t f = 0; f < hnf(h); f++) {
    v4 pl = fplane(hfo(h) + f);
    float d0 = dot(xyz(pl), e0) - pl.w, d1 = dot(xyz(pl), e1) - pl.w;
    if (d0 > 0.0f && d1 > 0.0f) return false;
    if (d0 > 0.0f) t0 = fmaxf_(t0, d0 / (d0 - d1));
    else if (d1 > 0.0f) t1 = fminf_(t1, d0 / (d0 - d1));
  }
  return t0 <= t1;
}
SegQ Oracle::seg_hull_query(uint32_t h, v3 e0, v3 e1, uint32_t lane) const {
  SegQ best{1e30f, splat3(0), splat3(0), 0u, 1u};
  uint32_t fo = hfo(h);
  for (uint32_t f = lane; f < hnf(h); f += NLANE) {
    v4 pl = fplane(fo + f);
    uint32_t sr = fstart(fo + f), cr = fcount(fo + f);
    bool in0 = dot(xyz(pl), e0) > pl.w, in1 = dot(xyz(pl), e1) > pl.w;
    for (uint32_t k = 0; k < cr; k++) {
      v3 r0 = hv(h, fvert(sr + k)), r1 = hv(h, fvert(sr + (k + 1u) % cr));
      v3 out = cross(r1 - r0, xyz(pl));
      if (dot(e0 - r0, out) > 0.0f) in0 = false;
      if (dot(e1 - r0, out) > 0.0f) in1 = false;
      v3 c[2];
      closest_seg(e0, e1, r0, r1, c);
      float d2 = dot(c[0] - c[1], c[0] - c[1]);
      if (d2 < best.d2) best = SegQ{d2, c[0], c[1], f, 1u};
    }
    if (in0) {
      float sd = dot(xyz(pl), e0) - pl.w;
      if (sd * sd <= best.d2 * 1.0001f) best = SegQ{sd * sd, e0, e0 - xyz(pl) * sd, f, 0u};
    }
    if (in1) {
      float sd = dot(xyz(pl), e1) - pl.w;
      if (sd * sd <= best.d2 * 1.0001f) best = SegQ{sd * sd, e1, e1 - xyz(pl) * sd, f, 0u};
    }
  }
  return best;
}
void Oracle::seg_on_face(uint32_t hs, uint32_t ps, uint32_t h, uint32_t f, v3 e0, v3 e1, float r, v3 wp, v4 wq,
                         float thresh, bool flip) {
  v4 pl = fplane(hfo(h) + f);
  float t0 = 0.0f, t1 = 1.0f;
  uint32_t sr = fstart(hfo(h) + f), cr = fcount(hfo(h) + f);
  for (uint32_t k = 0; k < cr; k++) {
    v3 r0 = hv(h, fvert(sr + k)), r1 = hv(h, fvert(sr + (k + 1u) % cr));
    v3 out = cross(r1 - r0, xyz(pl));
    float d0 = dot(e0 - r0, out), d1 = dot(e1 - r0, out);
    if (d0 > 0.0f && d1 > 0.0f) { t0 = 2.0f; break; }
    if (d0 > 0.0f) t0 = fmaxf_(t0, d0 / (d0 - d1));
    if (d1 > 0.0f) t1 = fminf_(t1, d0 / (d0 - d1));
  }
  float ts[2] = {t0, t1};
  uint32_t n = 2u;
  if (t0 > t1) {
    ts[0] = dot(xyz(pl), e0) <= dot(xyz(pl), e1) ? 0.0f : 1.0f;
    n = 1u;
  } else if (t1 - t0 < 1e-4f || length(e1 - e0) < 1e-7f) {
    n = 1u;
  }
  v3 nw = qrot(wq, xyz(pl));
  uint32_t sa = flip ? ps : hs, sb = flip ? hs : ps;
  uint32_t base = hash_u32(sa * 7919u + sb * 104729u);
  for (uint32_t i = 0; i < n; i++) {
    v3 x = e0 + (e1 - e0) * ts[i];
    float sd = dot(xyz(pl), x) - pl.w;
    float phi = sd - r;
    if (phi > thresh) continue;
    v3 mid = x - xyz(pl) * (0.5f * (sd + r));
    emit(sa, sb, wp + qrot(wq, mid), flip ? -nw : nw, phi, hash_u32(base ^ (f * 131u + i * 7u + 3u)));
  }
}

// --- Newton's generic convex manifold (wgsl.js:644-977) ---
Geo Oracle::geo(uint32_t s) const {
  v4 g = statF[C.SF_SHAPE + s * 7u + 6u];
  Geo r{f2u(g.x), mk3(g.y, g.z, g.w), f2u(statF[C.SF_SHAPE + s * 7u].y)};
  if (r.t == GT_SPHERE || r.t == GT_CAPSULE) r.s.x = 1e-4f;
  return r;
}
v3 Oracle::gsup(const Geo& g, v3 d) const {
  if (g.t == GT_BOX) {
    float th = 1e-10f * fmaxf_(std::fabs(d.x), fmaxf_(std::fabs(d.y), std::fabs(d.z)));
    return mk3(d.x >= -th ? g.s.x : -g.s.x, d.y >= -th ? g.s.y : -g.s.y, d.z >= -th ? g.s.z : -g.s.z);
  }
  if (g.t == GT_SPHERE || g.t == GT_CAPSULE) {
    float l2 = dot(d, d);
    v3 p = (l2 > 1e-12f ? d * inverse_sqrt(l2) : mk3(1.0f, 0.0f, 0.0f)) * g.s.x;
    if (g.t == GT_CAPSULE) p.z = p.z + (d.z >= 0.0f ? g.s.y : -g.s.y);
    return p;
  }
  if (g.t == GT_CYL) {
    v3 xy = mk3(d.x, d.y, 0.0f);
    float l2 = dot(xy, xy);
    v3 p = l2 > 1e-12f ? (xy * inverse_sqrt(l2)) * g.s.x : mk3(g.s.x, 0.0f, 0.0f);
    if (d.z > 0.0f) p.z = g.s.y; else if (d.z < 0.0f) p.z = -g.s.y;
    return p;
  }
  float best = -1e10f;
  v3 bp = splat3(0.0f);
  for (uint32_t v = 0; v < hnv(g.h); v++) {
    v3 x = hv(g.h, v);
    float s = dot(x, d);
    if (s > best) { best = s; bp = x; }
  }
  return bp;
}
v3 Oracle::fsup(const Geo& g, v3 d, v3 n) const {
  v3 p = gsup(g, d);
  if ((g.t == GT_CAPSULE || (g.t == GT_CYL && g.s.z == 0.0f)) && std::fabs(n.z) <= 1e-4f) {
    v3 rad = normalize(mk3(n.x, n.y, 0.0f)) * g.s.x;
    p = mk3(rad.x, rad.y, d.z >= 0.0f ? g.s.y : -g.s.y);
  }
  return p;
}
static inline bool planar_geo(const Geo& g) { return g.t == GT_BOX || g.t == GT_CONVEX; }

struct Trk { v3 r, p, n; float a2; bool np; };
static Trk trk_add(Trk t, v3 x, uint32_t id, bool chk) {
  Trk o = t;
  if (id == 0u) { o.r = x; o.a2 = 0.0f; o.n = splat3(0.0f); o.np = false; }
  else if (id == 1u) { o.p = x; }
  else {
    if (chk && o.a2 > 0.0f) {
      float off = dot(o.n, x - o.r);
      if (off * off > (MEPS * MEPS) * o.a2) o.np = true;
    }
    v3 c = cross(o.p - o.r, x - o.r);
    float a2 = dot(c, c);
    if (a2 > o.a2) { o.a2 = a2; o.n = c; }
    o.p = x;
  }
  return o;
}
static bool trk_anchor(const Trk& t, v3 x) {
  float off = dot(t.n, x - t.r);
  return !t.np && off * off <= (MEPS * MEPS) * t.a2;
}
struct Proj { float d; v3 n; };
static v3 line_proj_n(v3 dir, v3 rn) {
  v3 nn = cross(cross(dir, rn), dir);
  float l = length(nn);
  return l > 1e-12f ? nn * (1.0f / l) : rn;
}
static void make_proj(const Trk& ta, v3 pa, const Trk& tb, v3 pb, v3 n, Proj out[2]) {
  Proj A{0.0f, splat3(0.0f)}, B{0.0f, splat3(0.0f)};
  if (ta.a2 == 0.0f && tb.a2 == 0.0f) {
    A.n = line_proj_n(ta.p - ta.r, n); A.d = -dot(0.5f * (ta.r + ta.p), A.n);
    B.n = line_proj_n(tb.p - tb.r, n); B.d = -dot(0.5f * (tb.r + tb.p), B.n);
    out[0] = A; out[1] = B;
    return;
  }
  if (ta.a2 > 0.0f) { A.n = ta.n * (1.0f / std::sqrt(fmaxf_(1e-12f, ta.a2))); A.d = -dot(pa, A.n); }
  if (tb.a2 > 0.0f) { B.n = tb.n * (1.0f / std::sqrt(fmaxf_(1e-12f, tb.a2))); B.d = -dot(pb, B.n); }
  if (ta.a2 == 0.0f) { A.n = line_proj_n(ta.p - ta.r, B.n); A.d = -dot(0.5f * (ta.r + ta.p), A.n); }
  if (tb.a2 == 0.0f) { B.n = line_proj_n(tb.p - tb.r, A.n); B.d = -dot(0.5f * (tb.r + tb.p), B.n); }
  out[0] = A; out[1] = B;
}
static v3 proj_on(const Proj& pr, v3 x, v3 n) {
  float den = dot(n, pr.n);
  if (std::fabs(den) < 1e-12f) return x;
  return x + n * (-(dot(x, pr.n) + pr.d) / den);
}
static inline float sarea(v2 a, v2 b, v2 q) { return (b.x - a.x) * (q.y - a.y) - (b.y - a.y) * (q.x - a.x); }
static bool add_nodup(v2* arr, int cnt, v2 v) {
  if (cnt > 0) { v2 d = arr[0] - v; if (dot(d, d) < MEPS * MEPS) return false; }
  if (cnt > 1) { v2 d = arr[cnt - 1] - v; if (dot(d, d) < MEPS * MEPS) return false; }
  arr[cnt] = v;
  return true;
}
static int trim_in_place(v2 s0, v2 s1, v2* lp, int cnt0) {
  int cnt = cnt0;
  if (cnt < 3) return cnt;
  v2 ia = mk2(0, 0), ib = mk2(0, 0);
  int ca = -1, cb = -1;
  bool keep = false;
  bool prev_out = sarea(s0, s1, lp[0]) <= 0.0f;
  for (int i = 0; i < cnt; i++) {
    int nx = (i + 1) % cnt;
    bool out = sarea(s0, s1, lp[nx]) <= 0.0f;
    if (out != prev_out) {
      v2 a = lp[i], b = lp[nx];
      float sa = sarea(s0, s1, a), sb = sarea(s0, s1, b);
      float t = std::fabs(sa) / std::fabs(sa - sb);
      v2 x = (1.0f - t) * a + t * b;
      if (ca < 0) { ca = i; keep = !prev_out; ia = x; } else { cb = i; ib = x; }
    }
    prev_out = out;
  }
  if (ca >= 0 && cb >= 0) {
    int li = -1, ncnt = cnt, i = 0;
    for (int guard = 0; guard < 24 && i < cnt; guard++) {
      if (keep) { li++; lp[li] = lp[i]; }
      if (i == ca || i == cb) {
        v2 pt = i == ca ? ia : ib;
        if (li == i && !keep) {
          li++;
          for (int k = std::min(ncnt, 9); k > li; k--) lp[k] = lp[k - 1];
          lp[li] = pt;
          ncnt++; i++; cb++; cnt++;
        } else {
          li++; lp[li] = pt;
        }
        keep = !keep;
      }
      i++;
    }
    return li + 1;
  }
  return prev_out ? 0 : cnt;
}
static int trim_all(v2* tp, int tn, v2* lp, int ln) {
  if (tn <= 1) return std::min(1, ln);
  if (tn == 2 || ln == 2) {
    v2 st = lp[0], en = lp[1];
    if (tn == 2) { st = tp[0]; en = tp[1]; }
    v2 dir = en - st;
    float l2 = dot(dir, dir);
    if (l2 <= MEPS * MEPS) return 0;
    float lo = 0.0f, hi = 1.0f;
    if (tn == 2 && ln == 2) {
      v2 os = lp[0], od = lp[1] - os;
      float cr = dir.x * od.y - dir.y * od.x;
      if (std::fabs(cr) > 1e-6f * std::sqrt(l2 * dot(od, od))) return 0;
      float t0 = dot(os - st, dir) / l2, t1 = dot(lp[1] - st, dir) / l2;
      lo = fmaxf_(lo, fminf_(t0, t1));
      hi = fminf_(hi, fmaxf_(t0, t1));
    } else {
      bool useLoop = tn == 2;
      int pc = useLoop ? ln : tn;
      for (int i = 0; i < pc; i++) {
        v2 e0 = useLoop ? lp[i] : tp[i];
        v2 e1 = useLoop ? lp[(i + 1) % pc] : tp[(i + 1) % pc];
        float a = sarea(e0, e1, st), b = sarea(e0, e1, en);
        if (a < 0.0f && b < 0.0f) return 0;
        if (a < 0.0f) lo = fmaxf_(lo, a / (a - b));
        else if (b < 0.0f) hi = fminf_(hi, a / (a - b));
      }
    }
    if (hi <= lo) return 0;
    lp[0] = st + lo * dir;
    lp[1] = st + hi * dir;
    return 2;
  }
  int c = ln;
  v2 t0 = tp[0];
  for (int i = 0; i < tn; i++) {
    v2 s1 = (i == tn - 1) ? t0 : tp[i + 1];
    c = trim_in_place(tp[i], s1, lp, c);
  }
  return c;
}
static int remove_zero_edges(v2* lp, int cnt) {
  if (cnt < 2) return 0;
  int w = 0;
  for (int r = 1; r < cnt; r++) {
    v2 d = lp[r] - lp[w];
    if (dot(d, d) > MEPS * MEPS) { w++; lp[w] = lp[r]; }
  }
  int n = w + 1;
  if (w > 0) { v2 d = lp[w] - lp[0]; if (dot(d, d) < MEPS * MEPS) n = w; }
  return n < 2 ? 0 : n;
}
static void calipers(const v2* h, int n, int out[4]) {
  int p1 = 0, p3 = 1;
  v2 d0 = h[0] - h[1];
  float md = dot(d0, d0);
  const float te = 1e-3f;
  int j = 1;
  for (int i = 0; i < n; i++) {
    v2 hi = h[i], hi1 = h[(i + 1) % n];
    for (int g = 0; g < 16; g++) {
      if (sarea(hi, hi1, h[(j + 1) % n]) > sarea(hi, hi1, h[j])) j = (j + 1) % n; else break;
    }
    v2 hj = h[j];
    v2 a = hi - hj;
    if (dot(a, a) > md * (1.0f + te)) { md = dot(a, a); p1 = i; p3 = j; }
    v2 b = hi1 - hj;
    if (dot(b, b) > md * (1.0f + te)) { md = dot(b, b); p1 = (i + 1) % n; p3 = j; }
  }
  int p2 = 0, p4 = 0;
  float m1 = 0.0f, m2 = 0.0f;
  v2 q1 = h[p1], q3 = h[p3];
  for (int i = 0; i < n; i++) {
    float ar = sarea(q1, q3, h[i]);
    if (ar > m1 * (1.0f + te)) { m1 = ar; p2 = i; }
    else if (-ar > m2 * (1.0f + te)) { m2 = -ar; p4 = i; }
  }
  out[0] = p1; out[1] = p2; out[2] = p3; out[3] = p4;
}
static void onb(v3 n, v3 out[2]) {
  if (n.z < 0.0f) {
    float a = 1.0f / (1.0f - n.z), b = (n.x * n.y) * a;
    out[0] = mk3(1.0f - (n.x * n.x) * a, -b, n.x);
    out[1] = mk3(b, (n.y * n.y) * a - 1.0f, -n.y);
    return;
  }
  float a = 1.0f / (1.0f + n.z), b = (-n.x * n.y) * a;
  out[0] = mk3(1.0f - (n.x * n.x) * a, b, -n.x);
  out[1] = mk3(b, 1.0f - (n.y * n.y) * a, -n.y);
}
bool Oracle::plane_supporting(const Geo& g, v3 dir, float d) const {
  float off = dot(dir, gsup(g, dir)) + d;
  return off * off <= (MEPS * MEPS) * dot(dir, dir);
}

struct Man { v3 p[5]; float d[5]; uint32_t n; };

// build_manifold (wgsl.js:875-937). Takes the oracle for the support maps.
static Man build_manifold(const Oracle& O, const Geo& ga, const Geo& gb, v4 rq, v3 rt, v3 wa, v3 wb, v3 n) {
  Man out{};
  out.n = 0u;
  v3 fna = n;
  if (ga.t == GT_CYL && gb.t == GT_CYL && ga.s.z == 0.0f && gb.s.z == 0.0f) {
    v3 axb = qrot(rq, mk3(0.0f, 0.0f, 1.0f));
    v3 ro = mk3(rt.x, rt.y, 0.0f);
    if (axb.x * axb.x + axb.y * axb.y <= 1e-12f && std::fabs(rt.z) < ga.s.y + gb.s.y && dot(ro, ro) > 1e-20f) {
      v3 rn = normalize(ro);
      if (dot(n, rn) >= COS_TILT) fna = rn;
    }
  }
  v3 tb[2];
  onb(n, tb);
  bool pa = planar_geo(ga), pb = planar_geo(gb);
  v3 center = 0.5f * (wa + wb);
  v2 A[10] = {}, B[10] = {};
  int ac = 0, bc = 0;
  Trk ta{splat3(0), splat3(0), splat3(0), 0.0f, false};
  Trk tbk = ta;
  v3 lnb = qinvrot(rq, -n), lfb = qinvrot(rq, -fna);
  v3 lta = qinvrot(rq, -tb[0]), ltb = qinvrot(rq, -tb[1]);
  for (uint32_t e = 0; e < 5u; e++) {
    v2 cs = PENT[e] * SIN_TILT;
    v3 x = O.fsup(ga, (n * COS_TILT + cs.x * tb[0]) + cs.y * tb[1], fna);
    v3 xa = x - center;
    if (add_nodup(A, ac, mk2(dot(tb[0], xa), dot(tb[1], xa)))) { ac++; ta = trk_add(ta, x, (uint32_t)(ac - 1), pa); }
    v3 y = qrot(rq, O.fsup(gb, (lnb * COS_TILT + cs.x * lta) + cs.y * ltb, lfb)) + rt;
    v3 yb = y - center;
    if (add_nodup(B, bc, mk2(dot(tb[0], yb), dot(tb[1], yb)))) { bc++; tbk = trk_add(tbk, y, (uint32_t)(bc - 1), pb); }
  }
  uint32_t cnt = 0u;
  float ndot = 0.0f;
  if (ac >= 2 && bc >= 2 && !(pa && !trk_anchor(ta, wa)) && !(pb && !trk_anchor(tbk, wb))) {
    Proj pr[2];
    make_proj(ta, wa, tbk, wb, n, pr);
    bool ok = std::fabs(dot(n, pr[0].n)) >= COS_TILT && std::fabs(dot(n, pr[1].n)) >= COS_TILT;
    if (ok && pa && (ta.a2 == 0.0f || dot(cross(n, pr[0].n), cross(n, pr[0].n)) > 0.0f)) {
      bool flip = dot(pr[0].n, n) < 0.0f;
      ok = O.plane_supporting(ga, flip ? -pr[0].n : pr[0].n, flip ? -pr[0].d : pr[0].d);
    }
    if (ok && pb && (tbk.a2 == 0.0f || dot(cross(n, pr[1].n), cross(n, pr[1].n)) > 0.0f)) {
      bool flip = dot(pr[1].n, n) > 0.0f;
      v3 db = flip ? -pr[1].n : pr[1].n;
      float dd = flip ? -pr[1].d : pr[1].d;
      ok = O.plane_supporting(gb, qinvrot(rq, db), dd + dot(db, rt));
    }
    if (ok) {
      ndot = std::fabs(dot(pr[0].n, pr[1].n));
      int lc = remove_zero_edges(B, trim_all(A, ac, B, bc));
      if (lc > 1) {
        int idx[4] = {0, 1, 2, 3};
        if (lc > 4) { calipers(B, lc, idx); lc = 4; }
        for (int i = 0; i < lc; i++) {
          v2 q = B[idx[i]];
          v3 pl = (q.x * tb[0] + q.y * tb[1]) + center;
          v3 a = proj_on(pr[0], pl, n), b = proj_on(pr[1], pl, n);
          out.p[cnt] = 0.5f * (a + b);
          out.d[cnt] = dot(b - a, n);
          cnt++;
        }
      } else {
        ndot = 0.0f;
      }
    }
  }
  if (ndot < COS_DEEP || cnt == 0u) {
    out.p[cnt] = 0.5f * (wa + wb);
    out.d[cnt] = dot(wb - wa, n);
    cnt++;
  }
  out.n = cnt;
  return out;
}

static inline bool is_discrete(uint32_t t) { return t == GT_BOX || t == GT_CONVEX || t == GT_PLANE; }

void Oracle::gen_run(uint32_t sa, uint32_t sb, const Geo& ga, const Geo& gb, v3 pa, v4 qa, v4 rq, v3 rt, v3 wa,
                     v3 wb, v3 n, float thresh) {
  Man m = build_manifold(*this, ga, gb, rq, rt, wa, wb, n);
  v3 nw = qrot(qa, n);
  float ra = (ga.t == GT_SPHERE || ga.t == GT_CAPSULE) ? statF[C.SF_SHAPE + sa * 7u + 6u].y : 0.0f;
  float rb = (gb.t == GT_SPHERE || gb.t == GT_CAPSULE) ? statF[C.SF_SHAPE + sb * 7u + 6u].y : 0.0f;
  bool axA = ga.t == GT_CYL || ga.t == GT_CONE, axB = gb.t == GT_CYL || gb.t == GT_CONE;
  bool roll = false;
  v3 rpos = splat3(0.0f), rn = splat3(0.0f);
  if ((is_discrete(ga.t) && axB) || (is_discrete(gb.t) && axA)) {
    bool onB = is_discrete(ga.t) && axB;
    v3 ax = onB ? qrot(qmul(qa, rq), mk3(0.0f, 0.0f, 1.0f)) : qrot(qa, mk3(0.0f, 0.0f, 1.0f));
    v3 an = onB ? nw : -nw;
    if (std::fabs(dot(ax, an)) <= SIN_TILT) {
      roll = true;
      rpos = onB ? pa + qrot(qa, rt) : pa;
      rn = normalize(cross(ax, an));
    }
  }
  uint32_t base = hash_u32(sa * 7919u + sb * 104729u);
  for (uint32_t i = 0; i < m.n; i++) {
    v3 p = ((pa + qrot(qa, m.p[i])) + nw * (0.5f * ra)) - nw * (0.5f * rb);
    float d = (m.d[i] - ra) - rb;
    if (roll) p = p - rn * dot(p - rpos, rn);
    if (d > thresh) continue;
    emit(sa, sb, p, nw, d, hash_u32(base ^ (i * 0x9e3779b1u + 0x51u)));
  }
}

float Oracle::hull_out(uint32_t h, v3 x) const {
  float m = -1e30f;
  for (uint32_t f = 0; f < hnf(h); f++) {
    v4 pl = fplane(hfo(h) + f);
    m = fmaxf_(m, dot(xyz(pl), x) - pl.w);
  }
  return m;
}
v3 Oracle::ray_face(uint32_t h, v3 o, v3 n, v3 s) const {
  float best = -2.0f;
  v4 pl = mk4(0, 0, 0, 0);
  for (uint32_t f = 0; f < hnf(h); f++) {
    v4 q = fplane(hfo(h) + f);
    if (dot(xyz(q), n) > best) { best = dot(xyz(q), n); pl = q; }
  }
  v3 x = o + n * ((pl.w - dot(xyz(pl), o)) / dot(xyz(pl), n));
  if (std::fabs(dot(x - s, n)) > WITNESS_TOL) return o + n * dot(s - o, n);
  return x;
}
void Oracle::sup_witness(const Geo& ga, const Geo& gb, v4 rq, v3 rt, v3 n, bool refA, v3 out[2]) const {
  v3 sA = gsup(ga, n);
  v3 lb = gsup(gb, qinvrot(rq, -n));
  v3 sB = qrot(rq, lb) + rt;
  v3 wb[2] = {ray_face(ga.h, sB, n, sA), sB};
  v3 wa[2] = {sA, qrot(rq, ray_face(gb.h, qinvrot(rq, sA - rt), qinvrot(rq, -n), lb)) + rt};
  float ob = fmaxf_(hull_out(ga.h, wb[0]), hull_out(gb.h, qinvrot(rq, wb[1] - rt)));
  float oa = fmaxf_(hull_out(ga.h, wa[0]), hull_out(gb.h, qinvrot(rq, wa[1] - rt)));
  if ((refA && !(oa < ob - 1e-6f)) || (!refA && ob < oa - 1e-6f)) { out[0] = wb[0]; out[1] = wb[1]; return; }
  out[0] = wa[0]; out[1] = wa[1];
}
void Oracle::sat_generic(uint32_t sa, uint32_t sb, uint32_t ha, uint32_t hb, v3 pa, v4 qa, v4 rBA, v3 tBA,
                         float thresh, FaceQ fa, FaceQ fb, const EdgeQ& eq) {
  Geo ga = geo(sa), gb = geo(sb);
  if (eq.sep > fmaxf_(fa.sep, fb.sep) + SAT_TIE) {
    v3 c[2];
    closest_seg(eq.a0, eq.a1, eq.b0, eq.b1, c);
    gen_emit(sa, sb, ga, gb, pa, qa, rBA, tBA, c[0], c[1], eq.axis, thresh);
    return;
  }
  bool refA = !(fb.sep > fa.sep + SAT_TIE);
  v3 n = refA ? xyz(fplane(hfo(ha) + fa.face)) : -qrot(rBA, xyz(fplane(hfo(hb) + fb.face)));
  v3 w[2];
  sup_witness(ga, gb, rBA, tBA, n, refA, w);
  gen_emit(sa, sb, ga, gb, pa, qa, rBA, tBA, w[0], w[1], n, thresh);
}
void Oracle::plane_convex(uint32_t sa, uint32_t sb, v3 pa, v4 qa, v3 pb, v4 qb, float thresh) {
  Geo gb = geo(sb);
  v3 nw = qrot(qa, mk3(0.0f, 0.0f, 1.0f));
  float L = 10.0f * (length(xyz(statF[C.SF_HAABB + gb.h * 2u])) + length(xyz(statF[C.SF_HAABB + gb.h * 2u + 1u])));
  v3 c = pb - nw * (dot(pb - pa, nw) + L);
  v4 rq = qmul(qconj(qa), qb);
  v3 rt = qinvrot(qa, pb - c);
  v3 n = mk3(0.0f, 0.0f, 1.0f);
  v3 wb = qrot(rq, gsup(gb, qinvrot(rq, -n))) + rt;
  float sep = wb.z - L;
  if (sep > thresh) return;
  gen_emit(sa, sb, Geo{GT_BOX, mk3(L, L, L), 0u}, gb, c, qa, rq, rt, wb - n * sep, wb, n, thresh);
}
void Oracle::capsule_generic(uint32_t c, uint32_t h, v3 pc, v4 qc, v3 wp, v4 wq, v3 wc, v3 wh, v3 nh,
                             float thresh) {
  if (dot(wh - wc, nh) - statF[C.SF_SHAPE + c * 7u + 6u].y > thresh) return;
  v4 rq = qmul(qconj(qc), wq);
  v3 rt = qinvrot(qc, wp - pc);
  gen_emit(c, h, geo(c), geo(h), pc, qc, rq, rt, qrot(rq, wc) + rt, qrot(rq, wh) + rt, qrot(rq, nh), thresh);
}
void Oracle::mpr_generic(uint32_t sa, uint32_t sb, uint32_t ha, uint32_t hb, v3 pa, v4 qa, v4 rBA, v3 tBA,
                         float thresh, v3 n) {
  float alA = -2.0f;
  for (uint32_t f = 0; f < hnf(ha); f++) alA = fmaxf_(alA, dot(xyz(fplane(hfo(ha) + f)), n));
  float alB = -2.0f;
  for (uint32_t f = 0; f < hnf(hb); f++) alB = fmaxf_(alB, -dot(qrot(rBA, xyz(fplane(hfo(hb) + f))), n));
  Geo ga = geo(sa), gb = geo(sb);
  v3 w[2];
  sup_witness(ga, gb, rBA, tBA, n, alA >= alB, w);
  gen_emit(sa, sb, ga, gb, pa, qa, rBA, tBA, w[0], w[1], n, thresh);
}

// Workgroup reductions over the 32 lanes (wgsl.js:1051-1061, 1114-1122, 1181-1191): the first lane
// with the strictly best value wins.
template <class Q, class F> static Q lane_reduce(F per_lane, bool want_max, float (*val)(const Q&)) {
  Q best = per_lane(0u);
  for (uint32_t k = 1; k < NLANE; k++) {
    Q q = per_lane(k);
    if (want_max ? (val(q) > val(best)) : (val(q) < val(best))) best = q;
  }
  return best;
}
static float fq_val(const FaceQ& q) { return q.sep; }
static float eq_val(const EdgeQ& q) { return q.sep; }
static float sq_val(const SegQ& q) { return q.d2; }

// narrow_pair (wgsl.js:1072-1195)
void Oracle::narrow_pair(uint32_t pi) {
  uint32_t p0 = pairs[pi * 2u], p1 = pairs[pi * 2u + 1u];
  bool swp = geo_type(p0) > geo_type(p1);
  uint32_t sa = swp ? p1 : p0, sb = swp ? p0 : p1;
  uint32_t ha = f2u(statF[C.SF_SHAPE + sa * 7u].y), hb = f2u(statF[C.SF_SHAPE + sb * 7u].y);
  v3 pa = xyz(poses[C.P_SHAPE + sa * 2u]);
  v4 qa = poses[C.P_SHAPE + sa * 2u + 1u];
  v3 pb = xyz(poses[C.P_SHAPE + sb * 2u]);
  v4 qb = poses[C.P_SHAPE + sb * 2u + 1u];
  float thresh = fminf_(statF[C.SF_SHAPE + sa * 7u].w + statF[C.SF_SHAPE + sb * 7u].w, C.F_GAP_GATE);
  v4 rBA = qmul(qconj(qa), qb);
  v3 tBA = qinvrot(qa, pb - pa);
  v4 rAB = qconj(rBA);
  v3 tAB = qinvrot(qb, pa - pb);
  v4 ka = shape_prim(sa), kb = shape_prim(sb);
  if (ka.x == 4.0f || kb.x == 4.0f) {
    if (geo_type(sb) == GT_CONVEX) plane_convex(sa, sb, pa, qa, pb, qb, thresh);
    else plane_contacts(sa, sb, pa, qa, pb, qb, thresh, false);
    return;
  }
  if (ka.x != 0.0f && kb.x != 0.0f) { prim_prim(sa, sb, pa, qa, pb, qb, thresh); return; }
  if (ka.x != 0.0f || kb.x != 0.0f) {
    bool flip = ka.x != 0.0f;
    uint32_t hs = flip ? sb : sa, ps = flip ? sa : sb;
    uint32_t h = flip ? hb : ha;
    v4 pr = flip ? ka : kb;
    v4 rq = flip ? rAB : rBA;
    v3 rt = flip ? tAB : tBA;
    v3 u = qrot(rq, mk3(0.0f, 0.0f, pr.z));
    v3 e0 = rt - u, e1 = rt + u;
    FaceQ fq = lane_reduce<FaceQ>([&](uint32_t l) { return face_query_seg(h, e0, e1, pr.y, l); }, true, fq_val);
    if (fq.sep > thresh) return;
    v3 wp = flip ? pb : pa;
    v4 wq = flip ? qb : qa;
    if (fq.sep + pr.y > 1e-6f || (pr.x == 2.0f && !seg_hits_hull(h, e0, e1))) {
      SegQ q = lane_reduce<SegQ>([&](uint32_t l) { return seg_hull_query(h, e0, e1, l); }, false, sq_val);
      if (pr.x == 2.0f) {
        float d = std::sqrt(q.d2);
        if (d >= 1e-9f) {
          v3 nh = (q.ph - q.ps) / d;
          capsule_generic(ps, hs, flip ? pa : pb, flip ? qa : qb, wp, wq, q.ps + nh * 1e-4f, q.ph, nh, thresh);
        }
      } else {
        float d = std::sqrt(q.d2);
        float phi = d - pr.y;
        v3 n = (q.ps - q.ph) / fmaxf_(d, 1e-9f);
        if (phi > thresh || d < 1e-9f) {
        } else if (dot(n, xyz(fplane(hfo(h) + fq.face))) > 0.999f) {
          seg_on_face(hs, ps, h, fq.face, e0, e1, pr.y, wp, wq, thresh, flip);
        } else {
          uint32_t sa2 = flip ? ps : hs, sb2 = flip ? hs : ps;
          v3 nw = qrot(wq, n);
          uint32_t key = hash_u32(hash_u32(sa2 * 7919u + sb2 * 104729u) ^ (q.face * 131u + q.kind * 17u + 0x9e37u));
          emit(sa2, sb2, wp + qrot(wq, q.ph + n * (0.5f * phi)), flip ? -nw : nw, phi, key);
        }
      }
      return;
    }
    if (pr.x == 2.0f) {
      v4 pl = fplane(hfo(h) + fq.face);
      v3 x = dot(xyz(pl), e0) <= dot(xyz(pl), e1) ? e0 : e1;
      capsule_generic(ps, hs, flip ? pa : pb, flip ? qa : qb, wp, wq, x - xyz(pl) * 1e-4f,
                      x - xyz(pl) * (dot(xyz(pl), x) - pl.w), -xyz(pl), thresh);
    } else {
      seg_on_face(hs, ps, h, fq.face, e0, e1, pr.y, wp, wq, thresh, flip);
    }
    return;
  }
  FaceQ fa = lane_reduce<FaceQ>([&](uint32_t l) { return face_query(ha, hb, rBA, tBA, l); }, true, fq_val);
  if (fa.sep > thresh) return;
  FaceQ fb = lane_reduce<FaceQ>([&](uint32_t l) { return face_query(hb, ha, rAB, tAB, l); }, true, fq_val);
  if (fb.sep > thresh) return;
  EdgeQ none{-1e30f, splat3(0), splat3(0), splat3(0), splat3(0), splat3(0), 0u};
  bool small = hnv(ha) <= 16u && hnv(hb) <= 16u;
  if (!small) {
    v4 m = mpr(ha, hb, rBA, tBA, 0.5f * thresh);
    if (m.w >= 0.0f) {
      v3 n = -xyz(m);
      float sep = (dot(n, tBA) + support_min(hb, qinvrot(rBA, n))) - support_max(ha, n);
      if (fmaxf_(fa.sep, fb.sep) > sep + 1e-4f) sat_generic(sa, sb, ha, hb, pa, qa, rBA, tBA, thresh, fa, fb, none);
      else mpr_generic(sa, sb, ha, hb, pa, qa, rBA, tBA, thresh, n);
    }
    return;
  }
  EdgeQ eq = lane_reduce<EdgeQ>([&](uint32_t l) { return edge_query(ha, hb, rBA, tBA, l); }, true, eq_val);
  if (eq.sep > thresh) return;
  sat_generic(sa, sb, ha, hb, pa, qa, rBA, tBA, thresh, fa, fb, eq);
}

void Oracle::k_narrow() {
  uint32_t np = std::min(counters[0], C.MAXP);  // args (wgsl.js:3985-3993)
  for (uint32_t pi = 0; pi < np; pi++) {
    job.on = false;
    narrow_pair(pi);
    if (job.on) {
      GenJob j = job;
      gen_run(j.sa, j.sb, j.ga, j.gb, j.pa, j.qa, j.rq, j.rt, j.wa, j.wb, j.n, j.thresh);
    }
  }
}

// csort (wgsl.js:3899-3982): canonical order by (pair, feature key, point-bit hash, raw index).
void Oracle::k_csort() {
  uint32_t nc = std::min(counters[1], C.MAXC);
  std::vector<u4> keys(nc);
  for (uint32_t c = 0; c < nc; c++) {
    v4 p = craw[c * 5u], m = craw[c * 5u + 2u];
    uint32_t pair = (uint32_t)(f2i(m.x) + 1) | ((uint32_t)(f2i(m.y) + 1) << 16u);
    uint32_t feat = f2u(m.z) | (f2u(m.w) << 16u);
    uint32_t bits = hash_u32(hash_u32(hash_u32(fbits(p.x)) ^ fbits(p.y)) ^ fbits(p.z)) ^ fbits(p.w);
    keys[c] = {pair, feat, bits, c};
  }
  std::sort(keys.begin(), keys.end(), [](const u4& a, const u4& b) {
    if (a.x != b.x) return a.x < b.x;
    if (a.y != b.y) return a.y < b.y;
    if (a.z != b.z) return a.z < b.z;
    return a.w < b.w;
  });
  for (uint32_t i = 0; i < nc; i++) {
    uint32_t c = keys[i].w;
    for (uint32_t q = 0; q < 5u; q++) contacts[i * 5u + q] = craw[c * 5u + q];
    contacts[C.MAXC * 5u + i] = craw[C.MAXC * 5u + c];
  }
}

}  // namespace orc
