// Test infrastructure (oracle): the articulation library, artwgsl.js:57-596 restated.
#include <algorithm>

#include "oracle.h"
#include "smath_o.h"

namespace orc {

// Link block offsets (artwgsl.js:8-26).
enum : uint32_t {
  L_S = 0, L_U = 36, L_DI = 72, L_IA = 108, L_C = 135, L_PA = 141, L_V = 147, L_W = 153, L_A = 189, L_UU = 195,
  L_P = 201, L_DV = 207, L_POS = 213, L_ROT = 216, L_COM = 220, L_TAU = 223, L_JR = 229, L_W2 = 232
};

static inline SV sv0() { return SV{splat3(0.0f), splat3(0.0f)}; }
static inline SV sadd(SV x, SV y) { return SV{x.a + y.a, x.l + y.l}; }
static inline SV sscale(SV x, float s) { return SV{x.a * s, x.l * s}; }
static inline float sdot(SV m, SV f) { return dot(m.a, f.a) + dot(m.l, f.l); }
static inline SV crm(SV v, SV m) { return SV{cross(v.a, m.a), cross(v.a, m.l) + cross(v.l, m.a)}; }
static inline SV crf(SV v, SV f) { return SV{cross(v.a, f.a) + cross(v.l, f.l), cross(v.a, f.l)}; }
static inline m3 skew3(v3 r) { return mcols(mk3(0.0f, r.z, -r.y), mk3(-r.z, 0.0f, r.x), mk3(r.y, -r.x, 0.0f)); }
static inline m3 outer3(v3 x, v3 y) { return mcols(x * y.x, x * y.y, x * y.z); }
static inline SV mshift(SV m, v3 r) { return SV{m.a, m.l + cross(m.a, r)}; }
static inline SV fshift(SV f, v3 r) { return SV{f.a + cross(r, f.l), f.l}; }
static inline v4 qaxis(v3 axis, float angle) {
  return mk4(axis * sin_o(0.5f * angle), cos_o(0.5f * angle));
}
static inline v3 unit3(uint32_t c) { return c == 0 ? mk3(1, 0, 0) : (c == 1 ? mk3(0, 1, 0) : mk3(0, 0, 1)); }

// Double 3-vectors and column-major 3x3 blocks for the FP64 articulated-inertia option (ART_F64),
// with the float path's evaluation orders.
struct d3 { double x, y, z; };
struct dm3 { d3 c[3]; };
static inline d3 dv(v3 v) { return {(double)v.x, (double)v.y, (double)v.z}; }
static inline v3 fv(d3 v) { return mk3((float)v.x, (float)v.y, (float)v.z); }
static inline d3 operator+(d3 a, d3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
static inline d3 operator-(d3 a, d3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
static inline d3 operator*(d3 a, double s) { return {a.x * s, a.y * s, a.z * s}; }
static inline d3 operator*(double s, d3 a) { return {s * a.x, s * a.y, s * a.z}; }
static inline double ddot(d3 a, d3 b) { return (a.x * b.x + a.y * b.y) + a.z * b.z; }
static inline dm3 dcols(d3 a, d3 b, d3 c) { return {{a, b, c}}; }
static inline dm3 dm(const m3& m) { return dcols(dv(m.c[0]), dv(m.c[1]), dv(m.c[2])); }
static inline m3 fm(const dm3& m) { return mcols(fv(m.c[0]), fv(m.c[1]), fv(m.c[2])); }
static inline d3 dmul(const dm3& m, d3 v) { return (m.c[0] * v.x + m.c[1] * v.y) + m.c[2] * v.z; }
static inline dm3 dmul(const dm3& a, const dm3& b) { return dcols(dmul(a, b.c[0]), dmul(a, b.c[1]), dmul(a, b.c[2])); }
static inline dm3 dtr(const dm3& m) {
  return dcols(d3{m.c[0].x, m.c[1].x, m.c[2].x}, d3{m.c[0].y, m.c[1].y, m.c[2].y}, d3{m.c[0].z, m.c[1].z, m.c[2].z});
}
static inline dm3 dadd(const dm3& a, const dm3& b) { return dcols(a.c[0] + b.c[0], a.c[1] + b.c[1], a.c[2] + b.c[2]); }
static inline dm3 dsub(const dm3& a, const dm3& b) { return dcols(a.c[0] - b.c[0], a.c[1] - b.c[1], a.c[2] - b.c[2]); }
static inline dm3 dscale(double s, const dm3& a) { return dcols(s * a.c[0], s * a.c[1], s * a.c[2]); }
static inline dm3 douter(d3 x, d3 y) { return dcols(x * y.x, x * y.y, x * y.z); }
static inline dm3 dskew(d3 r) { return dcols(d3{0.0, r.z, -r.y}, d3{-r.z, 0.0, r.x}, d3{r.y, -r.x, 0.0}); }
static inline double dmax(double a, double b) { return b > a ? b : a; }

SV Oracle::imul(uint32_t o, SV m) const {
  m3 A = ldm(o), B = ldm(o + 9u), Cm = ldm(o + 18u);
  return SV{mul(A, m.a) + mul(B, m.l), mul(transpose(B), m.a) + mul(Cm, m.l)};
}
v3 Oracle::link_r(uint32_t l) const {
  int par = link_parent(l);
  if (par < 0) return splat3(0.0f);
  return ld3(lo(l) + L_COM) - ld3(lo((uint32_t)par) + L_COM);
}
void Oracle::add_shifted_inertia(uint32_t o, const m3& A, const m3& B, const m3& Cm, v3 r) {
  m3 R = skew3(r);
  stm(o, msub(madd(msub(madd(ldm(o), A), mul(B, R)), mul(R, transpose(B))), mul(mul(R, Cm), R)));
  stm(o + 9u, madd(madd(ldm(o + 9u), B), mul(R, Cm)));
  stm(o + 18u, madd(ldm(o + 18u), Cm));
}
int Oracle::body_node(int b) const {
  if (b < 0) return -1;
  uint32_t k = body_kind(b);
  if (k == 1u) return b;
  if (k == 2u || k == 3u) return (int)C.NB + body_art(b);
  return -1;
}

// art_fk (artwgsl.js:98-187)
void Oracle::art_fk(uint32_t a) {
  u4 ai = art_info(a);
  for (uint32_t k = 0; k < ai.y; k++) {
    uint32_t l = ai.x + k;
    uint32_t o = C.SF_LINK + l * 6u;
    v3 pp = splat3(0.0f);
    v4 pq = mk4(0, 0, 0, 1);
    int par = link_parent(l);
    if (par >= 0) { pp = ld3(lo((uint32_t)par) + L_POS); pq = mk4(ld3(lo((uint32_t)par) + L_ROT), art[lo((uint32_t)par) + L_ROT + 3u]); }
    v3 jp = pp + qrot(pq, xyz(statF[o + 1u]));
    v4 jq = qmul(pq, statF[o + 2u]);
    v3 axis = xyz(statF[o + 5u]);
    v4 mq = mk4(0, 0, 0, 1);
    v3 mp = splat3(0.0f);
    uint32_t t = link_type(l);
    uint32_t qs = link_qs(l);
    const float* Q = &art[C.A_Q];
    if (t == 1u) mq = qaxis(axis, Q[qs]);
    if (t == 0u) mp = axis * Q[qs];
    if (t == 2u) mq = normalize(mk4(Q[qs], Q[qs + 1], Q[qs + 2], Q[qs + 3]));
    uint32_t d0 = link_dof(l);
    uint32_t nlin = f2u(statF[o + 5u].w);
    uint32_t nang = link_ndof(l) - nlin;
    v3 ang[3] = {};
    if (t == 6u) {
      for (uint32_t c = 0; c < nlin; c++) mp += dof_axis(d0 + c) * Q[qs + c];
      uint32_t iq = qs + nlin;
      if (nang == 1u) { ang[0] = dof_axis(d0 + nlin); mq = qaxis(ang[0], Q[iq]); }
      if (nang == 2u) {
        v3 x0 = normalize(dof_axis(d0 + nlin));
        v3 x2 = normalize(cross(x0, dof_axis(d0 + nlin + 1u)));
        ang[0] = x0;
        v4 q0 = qaxis(x0, Q[iq]);
        ang[1] = qrot(q0, cross(x2, x0));
        mq = qmul(qaxis(ang[1], Q[iq + 1u]), q0);
      }
      if (nang == 3u) {
        ang[0] = dof_axis(d0 + nlin);
        v4 q0 = qaxis(ang[0], Q[iq]);
        ang[1] = qrot(q0, dof_axis(d0 + nlin + 1u));
        v4 q1 = qaxis(ang[1], Q[iq + 1u]);
        ang[2] = qrot(qmul(q1, q0), dof_axis(d0 + nlin + 2u));
        mq = qmul(qaxis(ang[2], Q[iq + 2u]), qmul(q1, q0));
      }
    }
    if (t == 4u) {
      mp = mk3(Q[qs], Q[qs + 1], Q[qs + 2]);
      mq = normalize(mk4(Q[qs + 3], Q[qs + 4], Q[qs + 5], Q[qs + 6]));
    }
    v4 cq = qmul(jq, mq);
    v3 cp = jp + qrot(jq, mp);
    v4 iq = qconj(statF[o + 4u]);
    v4 lq = normalize(qmul(cq, iq));
    v3 lp = cp + qrot(cq, -qrot(iq, xyz(statF[o + 3u])));
    uint32_t L = lo(l);
    st3(L + L_POS, lp);
    st3(L + L_ROT, xyz(lq));
    art[L + L_ROT + 3u] = lq.w;
    v3 com = lp + qrot(lq, body_com_local(link_body(l)));
    st3(L + L_COM, com);
    v3 aw = qrot(jq, axis);
    v3 rj = com - jp;
    for (uint32_t c = 0; c < C.JM; c++) stsv(L + L_S + c * 6u, sv0());
    if (t == 1u) stsv(L + L_S, SV{aw, cross(aw, rj)});
    if (t == 0u) stsv(L + L_S, SV{splat3(0.0f), aw});
    if (t == 2u)
      for (uint32_t c = 0; c < 3u; c++) { v3 ew = qrot(jq, unit3(c)); stsv(L + L_S + c * 6u, SV{ew, cross(ew, rj)}); }
    v3 rf = com - cp;
    st3(L + L_JR, rf);
    if (t == 6u) {
      for (uint32_t c = 0; c < nlin; c++) stsv(L + L_S + c * 6u, SV{splat3(0.0f), qrot(jq, dof_axis(d0 + c))});
      for (uint32_t c = 0; c < nang; c++) {
        v3 ew = qrot(jq, ang[c]);
        stsv(L + L_S + (nlin + c) * 6u, SV{ew, cross(ew, rf)});
      }
    }
    if (t == 4u) {
      for (uint32_t c = 0; c < 3u; c++) {
        v3 ew = qrot(jq, unit3(c));
        stsv(L + L_S + c * 6u, SV{splat3(0.0f), ew});
        stsv(L + L_S + (c + 3u) * 6u, SV{ew, cross(ew, rf)});
      }
    }
  }
}

// inv_spd (artwgsl.js:192-207): Gauss-Jordan on the leading n x n block.
static void inv_spd(float* D, uint32_t n, uint32_t JM, float* Di) {
  for (uint32_t i = 0; i < JM * JM; i++) Di[i] = 0.0f;
  for (uint32_t i = 0; i < n; i++) Di[i * JM + i] = 1.0f;
  for (uint32_t c = 0; c < n; c++) {
    float pv = 1.0f / fmaxf_(D[c * JM + c], 1e-12f);
    for (uint32_t k = 0; k < n; k++) { D[c * JM + k] *= pv; Di[c * JM + k] *= pv; }
    for (uint32_t r = 0; r < n; r++) {
      if (r == c) continue;
      float f = D[r * JM + c];
      if (f == 0.0f) continue;
      for (uint32_t k = 0; k < n; k++) {
        D[r * JM + k] -= f * D[c * JM + k];
        Di[r * JM + k] -= f * Di[c * JM + k];
      }
    }
  }
}

// inv_spd in double, same steps (ART_F64).
static void inv_spd64(double* D, uint32_t n, uint32_t JM, double* Di) {
  for (uint32_t i = 0; i < JM * JM; i++) Di[i] = 0.0;
  for (uint32_t i = 0; i < n; i++) Di[i * JM + i] = 1.0;
  for (uint32_t c = 0; c < n; c++) {
    double pv = 1.0 / dmax(D[c * JM + c], 1e-12);
    for (uint32_t k = 0; k < n; k++) { D[c * JM + k] *= pv; Di[c * JM + k] *= pv; }
    for (uint32_t r = 0; r < n; r++) {
      if (r == c) continue;
      double f = D[r * JM + c];
      if (f == 0.0) continue;
      for (uint32_t k = 0; k < n; k++) {
        D[r * JM + k] -= f * D[c * JM + k];
        Di[r * JM + k] -= f * Di[c * JM + k];
      }
    }
  }
}

// Diagonal terms and generalized force of dof d, the r-th of link l (artwgsl.js:290-318): the
// armature, implicit damping and the implicit PD drive are added to Drr (D[r][r], float or double);
// the drive's saturation test reads Drr rounded to float.
template <class T>
float Oracle::dof_tau(uint32_t l, uint32_t r, T& Drr) const {
  uint32_t d = link_dof(l) + r;
  v4 dr = dof_drive(d);
  Drr += (T)dr.x;
  float damp = dof_passive(d).x;
  Drr += (T)P.dt * (T)damp;
  float tau = (-damp) * art[C.A_QD + d] + art[C.A_JF + d];
  v2 sp = dof_spring(d);
  if (sp.x != 0.0f) tau += sp.x * (sp.y - art[C.A_Q + link_qs(l) + r]);
  if (C.DRIVE_ROWS == 0u && (dr.y > 0.0f || dr.z > 0.0f)) {
    float q = art[C.A_Q + link_qs(l) + r], qd = art[C.A_QD + d];
    float err = art[C.A_TGT + d] - q;
    float tv = art[C.A_TGTV + d];
    float mm = fmaxf_((float)Drr, 1e-9f);
    float qdn = (mm * qd + P.dt * (dr.y * err + dr.z * tv)) / ((mm + P.dt * dr.z) + (P.dt * P.dt) * dr.y);
    float ti = dr.y * (err - P.dt * qdn) + dr.z * (tv - qdn);
    if (std::fabs(ti) <= dr.w || dr.w <= 0.0f) {
      Drr += ((T)P.dt * (T)P.dt) * (T)dr.y + (T)P.dt * (T)dr.z;
      tau += (dr.y * err - (P.dt * dr.y) * qd) + dr.z * (tv - qd);
    } else {
      tau += clampf(ti, -dr.w, dr.w);
    }
  }
  return tau;
}

// Backward step of link l with the articulated-inertia branch in double (ART_F64): U = I^A S,
// D = S^T U and its inverse, the projected inertia I^A - U D^-1 U^T and its shifted sum into the
// parent are computed in double from the stored float blocks and rounded once on store; the bias
// forces stay float as in the FP32 path.
void Oracle::art_back_f64(uint32_t l) {
  const uint32_t JM = C.JM, L = lo(l), n = link_ndof(l);
  SV pA = ldsv(L + L_PA);
  dm3 A = dm(ldm(L + L_IA)), B = dm(ldm(L + L_IA + 9u)), Cm = dm(ldm(L + L_IA + 18u));
  d3 Ua[6], Ul[6];
  for (uint32_t c = 0; c < n; c++) {
    SV s = ldS(l, c);
    d3 sa = dv(s.a), sl = dv(s.l);
    Ua[c] = dmul(A, sa) + dmul(B, sl);
    Ul[c] = dmul(dtr(B), sa) + dmul(Cm, sl);
    stsv(L + L_U + c * 6u, SV{fv(Ua[c]), fv(Ul[c])});
  }
  double D[36] = {0};
  float u[6] = {0};
  for (uint32_t r = 0; r < n; r++) {
    SV s = ldS(l, r);
    for (uint32_t c = 0; c < n; c++) D[r * JM + c] = ddot(dv(s.a), Ua[c]) + ddot(dv(s.l), Ul[c]);
    float tau = dof_tau(l, r, D[r * JM + r]);
    u[r] = tau - sdot(s, pA);
  }
  double Di[36];
  inv_spd64(D, n, JM, Di);
  for (uint32_t i = 0; i < JM * JM; i++) art[L + L_DI + i] = (float)Di[i];
  for (uint32_t r = 0; r < JM; r++) art[L + L_UU + r] = u[r];
  int par = link_parent(l);
  if (par < 0) return;
  SV Duu = sv0();
  for (uint32_t r = 0; r < n; r++) {
    float du = 0.0f;
    for (uint32_t c = 0; c < n; c++) {
      double w = Di[r * JM + c];
      A = dsub(A, dscale(w, douter(Ua[r], Ua[c])));
      B = dsub(B, dscale(w, douter(Ua[r], Ul[c])));
      Cm = dsub(Cm, dscale(w, douter(Ul[r], Ul[c])));
      du += ldDI(l, r, c) * u[c];
    }
    Duu = sadd(Duu, sscale(ldU(l, r), du));
  }
  stm(L + L_IA, fm(A));
  stm(L + L_IA + 9u, fm(B));
  stm(L + L_IA + 18u, fm(Cm));
  SV pa = sadd(sadd(pA, imul(L + L_IA, ldsv(L + L_C))), Duu);
  uint32_t P0 = lo((uint32_t)par);
  v3 r = link_r(l);
  dm3 R = dskew(dv(r));
  dm3 PA = dm(ldm(P0 + L_IA)), PB = dm(ldm(P0 + L_IA + 9u)), PC = dm(ldm(P0 + L_IA + 18u));
  stm(P0 + L_IA, fm(dsub(dadd(dsub(dadd(PA, A), dmul(B, R)), dmul(R, dtr(B))), dmul(dmul(R, Cm), R))));
  stm(P0 + L_IA + 9u, fm(dadd(dadd(PB, B), dmul(R, Cm))));
  stm(P0 + L_IA + 18u, fm(dadd(PC, Cm)));
  stsv(P0 + L_PA, sadd(ldsv(P0 + L_PA), fshift(pa, r)));
}

// art_factor (artwgsl.js:210-369)
void Oracle::art_factor(uint32_t a) {
  u4 ai = art_info(a);
  v3 g = xyz(P.gravity);
  const uint32_t JM = C.JM;
  for (uint32_t k = 0; k < ai.y; k++) {
    uint32_t l = ai.x + k, L = lo(l);
    int par = link_parent(l);
    SV vp = sv0();
    if (par >= 0) vp = mshift(ldsv(lo((uint32_t)par) + L_V), link_r(l));
    SV sq = sv0();
    for (uint32_t c = 0; c < link_ndof(l); c++) sq = sadd(sq, sscale(ldS(l, c), art[C.A_QD + link_dof(l) + c]));
    SV v = sadd(vp, sq);
    stsv(L + L_V, v);
    SV cb = crm(vp, sq);
    if (link_type(l) == 6u) {
      uint32_t nlin = f2u(statF[C.SF_LINK + l * 6u + 5u].w);
      v3 ca = splat3(0.0f);
      for (uint32_t j = nlin; j < link_ndof(l); j++)
        for (uint32_t kk = j + 1u; kk < link_ndof(l); kk++)
          ca += (cross(ldS(l, j).a, ldS(l, kk).a) * art[C.A_QD + link_dof(l) + j]) * art[C.A_QD + link_dof(l) + kk];
      cb = sadd(cb, SV{ca, cross(ca, ld3(L + L_JR))});
    }
    uint32_t jt = link_type(l);
    if (jt == 4u || jt == 6u) {
      uint32_t nlin = jt == 4u ? 3u : f2u(statF[C.SF_LINK + l * 6u + 5u].w);
      v3 vo = splat3(0.0f), wj = splat3(0.0f);
      for (uint32_t c = 0; c < link_ndof(l); c++) {
        SV sc = ldS(l, c);
        float q = art[C.A_QD + link_dof(l) + c];
        if (c < nlin) vo += sc.l * q; else wj += sc.a * q;
      }
      cb = sadd(cb, SV{splat3(0.0f), -cross(wj, vo)});
    }
    stsv(L + L_C, cb);
    int b = link_body(l);
    float m = body_mass(b);
    m3 R = qmat(link_rot(l));
    m3 Ic = mul(mul(R, body_inertia(b)), transpose(R));
    stm(L + L_IA, Ic);
    stm(L + L_IA + 9u, mcols(splat3(0), splat3(0), splat3(0)));
    stm(L + L_IA + 18u, mcols(mk3(m, 0, 0), mk3(0, m, 0), mk3(0, 0, m)));
    SV pa0 = crf(v, imul(L + L_IA, v));
    if ((f2u(statF[C.SF_BODY + (uint32_t)b * 8u + 7u].w) & 2u) != 0u) pa0 = sadd(pa0, SV{splat3(0.0f), m * g});
    pa0 = sadd(pa0, SV{-ld3(C.A_BF + (uint32_t)b * 8u + 4u), -ld3(C.A_BF + (uint32_t)b * 8u)});
    stsv(L + L_PA, pa0);
  }
  for (uint32_t kk = 0; kk < ai.y; kk++) {
    uint32_t l = ai.x + ai.y - 1u - kk, L = lo(l);
    if (C.ART_F64 == 1u) {
      art_back_f64(l);
      continue;
    }
    uint32_t n = link_ndof(l);
    SV pA = ldsv(L + L_PA);
    float D[36] = {0};
    float u[6] = {0};
    for (uint32_t c = 0; c < n; c++) stsv(L + L_U + c * 6u, imul(L + L_IA, ldS(l, c)));
    for (uint32_t r = 0; r < n; r++) {
      for (uint32_t c = 0; c < n; c++) D[r * JM + c] = sdot(ldS(l, r), ldU(l, c));
      float tau = dof_tau(l, r, D[r * JM + r]);
      u[r] = tau - sdot(ldS(l, r), pA);
    }
    float Di[36];
    inv_spd(D, n, JM, Di);
    for (uint32_t i = 0; i < JM * JM; i++) art[L + L_DI + i] = Di[i];
    for (uint32_t r = 0; r < JM; r++) art[L + L_UU + r] = u[r];
    int par = link_parent(l);
    if (par < 0) continue;
    m3 A = ldm(L + L_IA), B = ldm(L + L_IA + 9u), Cm = ldm(L + L_IA + 18u);
    SV Duu = sv0();
    for (uint32_t r = 0; r < n; r++) {
      SV Ur = ldU(l, r);
      float du = 0.0f;
      for (uint32_t c = 0; c < n; c++) {
        SV Uc = ldU(l, c);
        float w = ldDI(l, r, c);
        A = msub(A, mscale(w, outer3(Ur.a, Uc.a)));
        B = msub(B, mscale(w, outer3(Ur.a, Uc.l)));
        Cm = msub(Cm, mscale(w, outer3(Ur.l, Uc.l)));
        du += w * u[c];
      }
      Duu = sadd(Duu, sscale(Ur, du));
    }
    stm(L + L_IA, A);
    stm(L + L_IA + 9u, B);
    stm(L + L_IA + 18u, Cm);
    SV cbias = ldsv(L + L_C);
    SV pa = sadd(sadd(pA, imul(L + L_IA, cbias)), Duu);
    uint32_t P0 = lo((uint32_t)par);
    v3 r = link_r(l);
    add_shifted_inertia(P0 + L_IA, A, B, Cm, r);
    stsv(P0 + L_PA, sadd(ldsv(P0 + L_PA), fshift(pa, r)));
  }
  for (uint32_t k = 0; k < ai.y; k++) {
    uint32_t l = ai.x + k, L = lo(l);
    int par = link_parent(l);
    SV ap = SV{splat3(0.0f), -g};
    if (par >= 0) ap = mshift(ldsv(lo((uint32_t)par) + L_A), link_r(l));
    SV a1 = sadd(ap, ldsv(L + L_C));
    uint32_t n = link_ndof(l);
    SV acc = a1;
    for (uint32_t r = 0; r < n; r++) {
      float qdd = 0.0f;
      for (uint32_t c = 0; c < n; c++) qdd += ldDI(l, r, c) * (art[L + L_UU + c] - sdot(ldU(l, c), a1));
      uint32_t d = link_dof(l) + r;
      art[C.A_QDH + d] = art[C.A_QD + d] + P.dt * qdd;
      acc = sadd(acc, sscale(ldS(l, r), qdd));
    }
    stsv(L + L_A, acc);
    if (C.JFL == 1u) {
      // joint_friction_load_coefficient (artwgsl.js:361-367): the joint's transmitted force and
      // torque under the free dynamics (I^A a + p^A at the child COM) raise its friction bound.
      SV f = sadd(imul(L + L_IA, acc), ldsv(L + L_PA));
      float fm = length(f.l) + length(f.a);
      for (uint32_t r = 0; r < n; r++) {
        uint32_t d = link_dof(l) + r;
        art[C.A_JFL + d] = statF[C.SF_DOF + d * 5u + 3u].w * fm;
      }
    }
  }
}

uint32_t Oracle::link_path(uint32_t l0, uint32_t* path) const {
  uint32_t n = 0;
  int l = (int)l0;
  for (;;) {
    if (l < 0 || n >= C.MAXPATH) break;
    path[n] = (uint32_t)l;
    n++;
    l = link_parent((uint32_t)l);
  }
  return n;
}

// dof_hinv via path_test (artwgsl.js:375-414, 513-518): F = 0, unit generalized impulse at (l, r).
float Oracle::dof_hinv(uint32_t l, uint32_t rr) const {
  const uint32_t JM = C.JM;
  std::vector<uint32_t> path(C.MAXPATH);
  uint32_t np = link_path(l, path.data());
  std::vector<float> ub(C.MAXPATH * JM, 0.0f);
  SV p = sscale(sv0(), -1.0f);
  for (uint32_t i = 0; i < np; i++) {
    uint32_t pl = path[i], n = link_ndof(pl);
    float u[6] = {0};
    for (uint32_t r = 0; r < n; r++) {
      float t = (pl == l && r == rr) ? 1.0f : 0.0f;
      u[r] = t - sdot(ldS(pl, r), p);
      ub[i * JM + r] = u[r];
    }
    for (uint32_t r = 0; r < n; r++) {
      float du = 0.0f;
      for (uint32_t c = 0; c < n; c++) du += ldDI(pl, r, c) * u[c];
      p = sadd(p, sscale(ldU(pl, r), du));
    }
    p = fshift(p, link_r(pl));
  }
  SV dv = sv0();
  float out = 0.0f;
  for (uint32_t ii = 0; ii < np; ii++) {
    uint32_t i = np - 1u - ii, pl = path[i], n = link_ndof(pl);
    dv = mshift(dv, link_r(pl));
    float dq[6] = {0};
    for (uint32_t r = 0; r < n; r++) {
      dq[r] = 0.0f;
      for (uint32_t c = 0; c < n; c++) dq[r] += ldDI(pl, r, c) * (ub[i * JM + c] - sdot(ldU(pl, c), dv));
    }
    for (uint32_t r = 0; r < n; r++) {
      dv = sadd(dv, sscale(ldS(pl, r), dq[r]));
      if (pl == l && r == rr) out = dq[r];
    }
  }
  return out;
}

// link_response (artwgsl.js:431-510)
void Oracle::link_response(uint32_t l, const uint32_t* split_count) {
  const uint32_t JM = C.JM, PD = C.MAXPATH * JM;
  std::vector<uint32_t> path(C.MAXPATH);
  uint32_t np = link_path(l, path.data());
  std::vector<float> ub(6 * PD, 0.0f);
  SV p[6];
  for (uint32_t e = 0; e < 6u; e++) {
    v3 f = splat3(0.0f), t = splat3(0.0f);
    if (e < 3u) setat(f, (int)e, 1.0f); else setat(t, (int)e - 3, 1.0f);
    p[e] = SV{-t, -f};
  }
  SV S[6], U[6];
  float DI[36] = {0};
  for (uint32_t i = 0; i < np; i++) {
    uint32_t pl = path[i], n = link_ndof(pl);
    for (uint32_t c = 0; c < n; c++) { S[c] = ldS(pl, c); U[c] = ldU(pl, c); }
    for (uint32_t x = 0; x < n * JM; x++) DI[x] = art[lo(pl) + L_DI + x];
    v3 r = link_r(pl);
    for (uint32_t e = 0; e < 6u; e++) {
      float u[6] = {0};
      for (uint32_t c = 0; c < n; c++) { u[c] = 0.0f - sdot(S[c], p[e]); ub[e * PD + i * JM + c] = u[c]; }
      SV pe = p[e];
      for (uint32_t rr = 0; rr < n; rr++) {
        float du = 0.0f;
        for (uint32_t c = 0; c < n; c++) du += DI[rr * JM + c] * u[c];
        pe = sadd(pe, sscale(U[rr], du));
      }
      p[e] = fshift(pe, r);
    }
  }
  SV dv[6];
  for (uint32_t e = 0; e < 6u; e++) dv[e] = sv0();
  for (uint32_t ii = 0; ii < np; ii++) {
    uint32_t i = np - 1u - ii, pl = path[i], n = link_ndof(pl);
    for (uint32_t c = 0; c < n; c++) { S[c] = ldS(pl, c); U[c] = ldU(pl, c); }
    for (uint32_t x = 0; x < n * JM; x++) DI[x] = art[lo(pl) + L_DI + x];
    v3 r = link_r(pl);
    for (uint32_t e = 0; e < 6u; e++) {
      SV d = mshift(dv[e], r);
      float dq[6] = {0};
      for (uint32_t rr = 0; rr < n; rr++) {
        dq[rr] = 0.0f;
        for (uint32_t c = 0; c < n; c++) dq[rr] += DI[rr * JM + c] * (ub[e * PD + i * JM + c] - sdot(U[c], d));
      }
      for (uint32_t rr = 0; rr < n; rr++) d = sadd(d, sscale(S[rr], dq[rr]));
      dv[e] = d;
    }
  }
  float W[36];
  for (uint32_t e = 0; e < 6u; e++) {
    W[0 * 6 + e] = dv[e].l.x; W[1 * 6 + e] = dv[e].l.y; W[2 * 6 + e] = dv[e].l.z;
    W[3 * 6 + e] = dv[e].a.x; W[4 * 6 + e] = dv[e].a.y; W[5 * 6 + e] = dv[e].a.z;
  }
  for (uint32_t k = 0; k < 36u; k++) art[lo(l) + L_W2 + k] = W[k];
  for (uint32_t i = 0; i < np; i++) {
    float extra = (float)split_count[i] - 1.0f;
    if (extra <= 0.0f) continue;
    uint32_t pl = path[i], n = link_ndof(pl);
    for (uint32_t x = 0; x < n * JM; x++) DI[x] = art[lo(pl) + L_DI + x];
    float t[36] = {0};
    for (uint32_t cc = 0; cc < 6u; cc++)
      for (uint32_t x = 0; x < n; x++) {
        float v = 0.0f;
        for (uint32_t y = 0; y < n; y++) v += DI[x * JM + y] * ub[cc * PD + i * JM + y];
        t[cc * 6u + x] = v;
      }
    for (uint32_t rr = 0; rr < 6u; rr++)
      for (uint32_t cc = 0; cc < 6u; cc++) {
        float sv = 0.0f;
        for (uint32_t x = 0; x < n; x++) sv += ub[rr * PD + i * JM + x] * t[cc * 6u + x];
        W[rr * 6u + cc] += extra * sv;
      }
  }
  for (uint32_t k = 0; k < 36u; k++) art[lo(l) + L_W + k] = W[k];
}

// add_gen_jac / add_gen_ang (artwgsl.js:525-554)
void Oracle::add_gen_jac(uint32_t x, v3 p, float sgn, v3 d0, v3 d1, v3 d2, uint32_t ds, float* J) const {
  int l = (int)x;
  while (l >= 0) {
    uint32_t k = (uint32_t)l;
    v3 c = ld3(lo(k) + L_COM);
    for (uint32_t r = 0; r < link_ndof(k); r++) {
      SV S = ldS(k, r);
      v3 v = S.l + cross(S.a, p - c);
      uint32_t i = link_dof(k) + r - ds;
      J[i] += sgn * dot(d0, v);
      J[C.NDA + i] += sgn * dot(d1, v);
      J[2u * C.NDA + i] += sgn * dot(d2, v);
    }
    l = link_parent(k);
  }
}
void Oracle::add_gen_ang(uint32_t x, float sgn, v3 d0, v3 d1, uint32_t ds, float* J) const {
  int l = (int)x;
  while (l >= 0) {
    uint32_t k = (uint32_t)l;
    for (uint32_t r = 0; r < link_ndof(k); r++) {
      v3 w = ldS(k, r).a;
      uint32_t i = link_dof(k) + r - ds;
      J[i] += sgn * dot(d0, w);
      J[C.NDA + i] += sgn * dot(d1, w);
    }
    l = link_parent(k);
  }
}

// art_solve_gen (artwgsl.js:557-596)
void Oracle::art_solve_gen(uint32_t a, const float* tau, float* out) const {
  u4 ai = art_info(a);
  std::vector<SV> p(ai.y), dvs(ai.y);
  std::vector<float> uu(ai.y * 6u, 0.0f);
  for (uint32_t k = 0; k < ai.y; k++) p[k] = sv0();
  for (uint32_t kk = 0; kk < ai.y; kk++) {
    uint32_t k = ai.y - 1u - kk, l = ai.x + k, n = link_ndof(l);
    float u[6] = {0};
    for (uint32_t r = 0; r < n; r++) u[r] = tau[link_dof(l) + r - ai.z] - sdot(ldS(l, r), p[k]);
    for (uint32_t r = 0; r < 6u; r++) uu[k * 6u + r] = u[r];
    int par = link_parent(l);
    if (par >= 0) {
      SV pp = p[k];
      for (uint32_t r = 0; r < n; r++) {
        float du = 0.0f;
        for (uint32_t c = 0; c < n; c++) du += ldDI(l, r, c) * u[c];
        pp = sadd(pp, sscale(ldU(l, r), du));
      }
      uint32_t pk = (uint32_t)par - ai.x;
      p[pk] = sadd(p[pk], fshift(pp, link_r(l)));
    }
  }
  for (uint32_t k = 0; k < ai.y; k++) {
    uint32_t l = ai.x + k;
    int par = link_parent(l);
    SV dv = sv0();
    if (par >= 0) dv = mshift(dvs[(uint32_t)par - ai.x], link_r(l));
    uint32_t n = link_ndof(l);
    float dq[6] = {0};
    for (uint32_t r = 0; r < n; r++) {
      dq[r] = 0.0f;
      for (uint32_t c = 0; c < n; c++) dq[r] += ldDI(l, r, c) * (uu[k * 6u + c] - sdot(ldU(l, c), dv));
    }
    for (uint32_t r = 0; r < n; r++) {
      dv = sadd(dv, sscale(ldS(l, r), dq[r]));
      out[link_dof(l) + r - ai.z] = dq[r];
    }
    dvs[k] = dv;
  }
}

// art_twists (wgsl.js:3240-3251), art_apply (wgsl.js:3254-3299)
void Oracle::set_link_twist(uint32_t l, SV v) {
  uint32_t b = (uint32_t)link_body(l);
  tw[b * 2u] = mk4(v.l, 0.0f);
  tw[b * 2u + 1u] = mk4(v.a, 0.0f);
}
void Oracle::art_twists(uint32_t a) {
  u4 ai = art_info(a);
  for (uint32_t k = 0; k < ai.y; k++) {
    uint32_t l = ai.x + k;
    int par = link_parent(l);
    SV v = sv0();
    if (par >= 0) v = mshift(ldsv(lo((uint32_t)par) + L_V), link_r(l));
    for (uint32_t r = 0; r < link_ndof(l); r++) v = sadd(v, sscale(ldS(l, r), aqd[link_dof(l) + r]));
    stsv(lo(l) + L_V, v);
    set_link_twist(l, v);
  }
}
void Oracle::art_apply(uint32_t a) {
  u4 ai = art_info(a);
  for (uint32_t kk = 0; kk < ai.y; kk++) {
    uint32_t l = ai.x + ai.y - 1u - kk, L = lo(l);
    uint32_t n = link_ndof(l);
    SV p = ldsv(L + L_P);
    float u[6] = {0};
    for (uint32_t r = 0; r < n; r++) {
      u[r] = art[L + L_TAU + r] - sdot(ldS(l, r), p);
      art[L + L_UU + r] = u[r];
    }
    int par = link_parent(l);
    if (par >= 0) {
      SV pp = p;
      for (uint32_t r = 0; r < n; r++) {
        float du = 0.0f;
        for (uint32_t c = 0; c < n; c++) du += ldDI(l, r, c) * u[c];
        pp = sadd(pp, sscale(ldU(l, r), du));
      }
      uint32_t P0 = lo((uint32_t)par) + L_P;
      stsv(P0, sadd(ldsv(P0), fshift(pp, link_r(l))));
    }
  }
  for (uint32_t k = 0; k < ai.y; k++) {
    uint32_t l = ai.x + k, L = lo(l);
    int par = link_parent(l);
    SV dv = sv0();
    if (par >= 0) dv = mshift(ldsv(lo((uint32_t)par) + L_DV), link_r(l));
    uint32_t n = link_ndof(l);
    float dq[6] = {0};
    for (uint32_t r = 0; r < n; r++) {
      dq[r] = 0.0f;
      for (uint32_t c = 0; c < n; c++) dq[r] += ldDI(l, r, c) * (art[L + L_UU + c] - sdot(ldU(l, c), dv));
    }
    for (uint32_t r = 0; r < n; r++) {
      dv = sadd(dv, sscale(ldS(l, r), dq[r]));
      aqd[link_dof(l) + r] += dq[r];
    }
    stsv(L + L_DV, dv);
    SV v = sadd(ldsv(L + L_V), dv);
    stsv(L + L_V, v);
    set_link_twist(l, v);
    stsv(L + L_P, sv0());
    for (uint32_t r = 0; r < C.JM; r++) art[L + L_TAU + r] = 0.0f;
  }
}

}  // namespace orc
