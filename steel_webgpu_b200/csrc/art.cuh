// Articulated-body (Featherstone) device library for one articulation per thread.
//
// Follows packages/steel-webgpu/src/artwgsl.js: link FK (artwgsl.js:98-187), the articulated
// inertia factorisation with implicit PD drives in D (artwgsl.js:210-369), the split COM
// response of a contact-bearing link (artwgsl.js:431-510), the H^-1 diagonal of a dof
// (artwgsl.js:513-518), generalized Jacobians and solves (artwgsl.js:525-596) and the impulse
// propagation of the solve (wgsl.js:3240-3299). Spatial quantities are expressed at each link's
// COM with world orientation. Per-link records keep the reference's 268-float block layout in
// the scene's articulation buffer; path-length temporaries live in a per-thread slice of global
// scratch (deep chains do not fit in registers).
#pragma once
#include "common.cuh"

namespace steel {

enum : uint32_t {
  L_S = 0, L_U = 36, L_DI = 72, L_IA = 108, L_C = 135, L_PA = 141, L_V = 147, L_W = 153, L_A = 189, L_UU = 195,
  L_P = 201, L_DV = 207, L_POS = 213, L_ROT = 216, L_COM = 220, L_TAU = 223, L_JR = 229, L_W2 = 232, LBLK = 268
};

struct SVec { f3 a, l; };
// A thread's scratch interleaved with the other threads of its block: element i at p[i * s]
// (p = scratch + thread index, s = block size). Threads that walk the same articulation in step
// then touch consecutive words instead of one cache line each.
struct Lane {
  float* p;
  uint32_t s;
  __device__ float& operator[](uint32_t i) const { return p[(size_t)i * s]; }
  __device__ Lane operator+(uint32_t i) const { return Lane{p + (size_t)i * s, s}; }
};
SD SVec sv0() { return SVec{sp3(0.0f), sp3(0.0f)}; }
SD SVec sadd(SVec x, SVec y) { return SVec{x.a + y.a, x.l + y.l}; }
SD SVec sscl(SVec x, float s) { return SVec{x.a * s, x.l * s}; }
SD float sdot(SVec m, SVec f) { return dot(m.a, f.a) + dot(m.l, f.l); }
SD SVec crm(SVec v, SVec m) { return SVec{cross(v.a, m.a), cross(v.a, m.l) + cross(v.l, m.a)}; }
SD SVec crf(SVec v, SVec f) { return SVec{cross(v.a, f.a) + cross(v.l, f.l), cross(v.a, f.l)}; }
SD m3 skew(f3 r) { return mcols(mf3(0.0f, r.z, -r.y), mf3(-r.z, 0.0f, r.x), mf3(r.y, -r.x, 0.0f)); }
SD m3 outer(f3 x, f3 y) { return mcols(x * y.x, x * y.y, x * y.z); }
SD SVec mshift(SVec m, f3 r) { return SVec{m.a, m.l + cross(m.a, r)}; }
SD SVec fshift(SVec f, f3 r) { return SVec{f.a + cross(r, f.l), f.l}; }
SD float4 qaxis(f3 axis, float angle) { return mf4(axis * fsin(0.5f * angle), fcos(0.5f * angle)); }
SD f3 unit_axis(uint32_t c) { return c == 0 ? mf3(1, 0, 0) : (c == 1 ? mf3(0, 1, 0) : mf3(0, 0, 1)); }

// Double 3-vectors and column-major 3x3 blocks for the FP64 articulated-inertia option (ART_F64),
// evaluated in the float path's orders (no contraction: the library builds with --fmad=false).
struct d3 { double x, y, z; };
struct dm3 { d3 c[3]; };
SD d3 dv(f3 v) { return d3{(double)v.x, (double)v.y, (double)v.z}; }
SD f3 fv(d3 v) { return mf3((float)v.x, (float)v.y, (float)v.z); }
SD d3 operator+(d3 a, d3 b) { return d3{a.x + b.x, a.y + b.y, a.z + b.z}; }
SD d3 operator-(d3 a, d3 b) { return d3{a.x - b.x, a.y - b.y, a.z - b.z}; }
SD d3 operator*(d3 a, double s) { return d3{a.x * s, a.y * s, a.z * s}; }
SD d3 operator*(double s, d3 a) { return d3{s * a.x, s * a.y, s * a.z}; }
SD double ddot(d3 a, d3 b) { return (a.x * b.x + a.y * b.y) + a.z * b.z; }
SD dm3 dcols(d3 a, d3 b, d3 c) { return dm3{{a, b, c}}; }
SD dm3 dm(const m3& m) { return dcols(dv(m.c[0]), dv(m.c[1]), dv(m.c[2])); }
SD m3 fm(const dm3& m) { return mcols(fv(m.c[0]), fv(m.c[1]), fv(m.c[2])); }
SD d3 dmul(const dm3& m, d3 v) { return (m.c[0] * v.x + m.c[1] * v.y) + m.c[2] * v.z; }
SD dm3 dmul(const dm3& a, const dm3& b) { return dcols(dmul(a, b.c[0]), dmul(a, b.c[1]), dmul(a, b.c[2])); }
SD dm3 dtr(const dm3& m) {
  return dcols(d3{m.c[0].x, m.c[1].x, m.c[2].x}, d3{m.c[0].y, m.c[1].y, m.c[2].y}, d3{m.c[0].z, m.c[1].z, m.c[2].z});
}
SD dm3 dadd(const dm3& a, const dm3& b) { return dcols(a.c[0] + b.c[0], a.c[1] + b.c[1], a.c[2] + b.c[2]); }
SD dm3 dsub(const dm3& a, const dm3& b) { return dcols(a.c[0] - b.c[0], a.c[1] - b.c[1], a.c[2] - b.c[2]); }
SD dm3 dscl(double s, const dm3& a) { return dcols(s * a.c[0], s * a.c[1], s * a.c[2]); }
SD dm3 douter(d3 x, d3 y) { return dcols(x * y.x, x * y.y, x * y.z); }
SD dm3 dskew(d3 r) { return dcols(d3{0.0, r.z, -r.y}, d3{-r.z, 0.0, r.x}, d3{r.y, -r.x, 0.0}); }
SD double dmx(double a, double b) { return b > a ? b : a; }

struct Art {
  const SceneDev& S;
  float* A;   // the scene's articulation buffer
  float* LB;  // link blocks: LB + lo(l) is link l's LBLK floats
  // Static records and the dof stride, read once: the serial passes address them on every link.
  RO<float4> LR, DR, BR;  // link (6 vec4), dof (5 vec4) and body (8 vec4) records
  uint32_t JMc;
  __device__ Art(const SceneDev& s)
      : S(s), A(s.art), LB(s.art + s.A_LINK), LR(s.sf + s.SF_LINK), DR(s.sf + s.SF_DOF), BR(s.sf + s.SF_BODY),
        JMc(s.JM) {}
  __device__ Art(const SceneDev& s, float* lb)
      : S(s), A(s.art), LB(lb), LR(s.sf + s.SF_LINK), DR(s.sf + s.SF_DOF), BR(s.sf + s.SF_BODY), JMc(s.JM) {}

  __device__ float4 lrec(uint32_t l, uint32_t k) const { return LR[l * 6u + k]; }
  __device__ uint32_t ltype(uint32_t l) const { return f2u(lrec(l, 0).x); }
  __device__ int lparent(uint32_t l) const { return f2i(lrec(l, 0).y); }
  __device__ uint32_t ldof(uint32_t l) const { return f2u(lrec(l, 0).z); }
  __device__ int lbody(uint32_t l) const { return f2i(lrec(l, 0).w); }
  __device__ uint32_t lndof(uint32_t l) const { return f2u(lrec(l, 1).w); }
  __device__ uint32_t lqs(uint32_t l) const { return f2u(lrec(l, 3).w); }
  __device__ float4 dof_drive(uint32_t d) const { return DR[d * 5u]; }
  __device__ float4 dof_limit(uint32_t d) const { return DR[d * 5u + 1u]; }
  __device__ float4 dof_passive(uint32_t d) const { return DR[d * 5u + 2u]; }
  __device__ f3 dof_axis(uint32_t d) const { return v3(DR[d * 5u + 3u]); }
  __device__ bool scalar_dof(uint32_t d) const { return DR[d * 5u + 2u].w > 0.5f; }
  __device__ uint4 info(uint32_t a) const {
    RO<uint32_t> p = S.su + S.SU_ART + a * 4u;
    return make_uint4(p[0], p[1], p[2], p[3]);
  }
  __device__ float bmass(int b) const { return BR[(uint32_t)b * 8u + 1u].w; }
  __device__ m3 binertia(int b) const {
    RO<float4> o = BR + (uint32_t)b * 8u;
    return tr(mcols(v3(o[2]), v3(o[3]), v3(o[4])));
  }
  __device__ uint32_t lo(uint32_t l) const { return l * LBLK; }
  // Link-block fields (offsets from lo(l)) live at LB, which is either the scene's art buffer or a
  // shared-memory copy of its link blocks; every other art field is addressed through A.
  __device__ f3 ld3(uint32_t o) const { return mf3(LB[o], LB[o + 1], LB[o + 2]); }
  __device__ void st3(uint32_t o, f3 v) const { LB[o] = v.x; LB[o + 1] = v.y; LB[o + 2] = v.z; }
  __device__ f3 ald3(uint32_t o) const { return mf3(A[o], A[o + 1], A[o + 2]); }
  __device__ void ast3(uint32_t o, f3 v) const { A[o] = v.x; A[o + 1] = v.y; A[o + 2] = v.z; }
  __device__ SVec ldsv(uint32_t o) const { return SVec{ld3(o), ld3(o + 3u)}; }
  __device__ void stsv(uint32_t o, SVec s) const { st3(o, s.a); st3(o + 3u, s.l); }
  __device__ m3 ldm(uint32_t o) const { return mcols(ld3(o), ld3(o + 3u), ld3(o + 6u)); }
  __device__ void stm(uint32_t o, const m3& m) const { st3(o, m.c[0]); st3(o + 3u, m.c[1]); st3(o + 6u, m.c[2]); }
  __device__ SVec imul(uint32_t o, SVec m) const {
    m3 Am = ldm(o), Bm = ldm(o + 9u), Cm = ldm(o + 18u);
    return SVec{mul(Am, m.a) + mul(Bm, m.l), mul(tr(Bm), m.a) + mul(Cm, m.l)};
  }
  __device__ SVec ldS(uint32_t l, uint32_t k) const { return ldsv(lo(l) + L_S + k * 6u); }
  __device__ SVec ldU(uint32_t l, uint32_t k) const { return ldsv(lo(l) + L_U + k * 6u); }
  __device__ float ldDI(uint32_t l, uint32_t r, uint32_t c) const { return LB[lo(l) + L_DI + r * JMc + c]; }
  __device__ f3 link_r(uint32_t l) const {
    int par = lparent(l);
    if (par < 0) return sp3(0.0f);
    return ld3(lo(l) + L_COM) - ld3(lo((uint32_t)par) + L_COM);
  }
  __device__ float4 link_rot(uint32_t l) const { return mf4(ld3(lo(l) + L_ROT), LB[lo(l) + L_ROT + 3u]); }

  // Link poses, COMs and world motion subspaces (artwgsl.js:98-187), in three parts per link:
  // the joint's own motion from its coordinates (fk_joint), the pose chain from the parent's pose
  // (fk_pose), and the COM, motion subspace and joint offset from the link's pose (fk_out).
  struct FkJoint {
    float4 mq;
    f3 mp;
    f3 ang[3];
    uint32_t nlin, nang;
  };
  __device__ FkJoint fk_joint(uint32_t l) const {
    const float* Q = A + S.A_Q;
    const float4 r0 = lrec(l, 0), r1 = lrec(l, 1), r3 = lrec(l, 3), r5 = lrec(l, 5);
    FkJoint j;
    j.mq = make_float4(0, 0, 0, 1);
    j.mp = sp3(0.0f);
    j.ang[0] = sp3(0.0f); j.ang[1] = sp3(0.0f); j.ang[2] = sp3(0.0f);
    const f3 axis = v3(r5);
    const uint32_t t = f2u(r0.x), qs = f2u(r3.w), d0 = f2u(r0.z);
    if (t == 1u) j.mq = qaxis(axis, Q[qs]);
    if (t == 0u) j.mp = axis * Q[qs];
    if (t == 2u) j.mq = nrm4(make_float4(Q[qs], Q[qs + 1], Q[qs + 2], Q[qs + 3]));
    j.nlin = f2u(r5.w);
    j.nang = f2u(r1.w) - j.nlin;
    if (t == 6u) {
      for (uint32_t c = 0; c < j.nlin; c++) j.mp += dof_axis(d0 + c) * Q[qs + c];
      uint32_t iq = qs + j.nlin;
      if (j.nang == 1u) { j.ang[0] = dof_axis(d0 + j.nlin); j.mq = qaxis(j.ang[0], Q[iq]); }
      if (j.nang == 2u) {
        f3 x0 = nrm(dof_axis(d0 + j.nlin));
        f3 x2 = nrm(cross(x0, dof_axis(d0 + j.nlin + 1u)));
        j.ang[0] = x0;
        float4 q0 = qaxis(x0, Q[iq]);
        j.ang[1] = qrot(q0, cross(x2, x0));
        j.mq = qmul(qaxis(j.ang[1], Q[iq + 1u]), q0);
      }
      if (j.nang == 3u) {
        j.ang[0] = dof_axis(d0 + j.nlin);
        float4 q0 = qaxis(j.ang[0], Q[iq]);
        j.ang[1] = qrot(q0, dof_axis(d0 + j.nlin + 1u));
        float4 q1 = qaxis(j.ang[1], Q[iq + 1u]);
        j.ang[2] = qrot(qmul(q1, q0), dof_axis(d0 + j.nlin + 2u));
        j.mq = qmul(qaxis(j.ang[2], Q[iq + 2u]), qmul(q1, q0));
      }
    }
    if (t == 4u) {
      j.mp = mf3(Q[qs], Q[qs + 1], Q[qs + 2]);
      j.mq = nrm4(make_float4(Q[qs + 3], Q[qs + 4], Q[qs + 5], Q[qs + 6]));
    }
    return j;
  }
  // Joint frame (jp, jq), child frame (cp, cq) and link pose (lp, lq) from the parent's pose.
  __device__ void fk_pose(uint32_t l, f3 pp, float4 pq, float4 mq, f3 mp, f3& jp, float4& jq, f3& cp, f3& lp,
                          float4& lq) const {
    const float4 r1 = lrec(l, 1), r2 = lrec(l, 2), r3 = lrec(l, 3), r4 = lrec(l, 4);
    jp = pp + qrot(pq, v3(r1));
    jq = qmul(pq, r2);
    const float4 cq = qmul(jq, mq);
    cp = jp + qrot(jq, mp);
    const float4 iq = qconj(r4);
    lq = nrm4(qmul(cq, iq));
    lp = cp + qrot(cq, -qrot(iq, v3(r3)));
  }
  __device__ void fk_store_pose(uint32_t l, f3 lp, float4 lq) const {
    const uint32_t L = lo(l);
    st3(L + L_POS, lp);
    st3(L + L_ROT, v3(lq));
    LB[L + L_ROT + 3u] = lq.w;
  }
  __device__ void fk_out(uint32_t l, const FkJoint& j, f3 jp, float4 jq, f3 cp, f3 lp, float4 lq) const {
    const float4 r0 = lrec(l, 0), r5 = lrec(l, 5);
    const uint32_t t = f2u(r0.x), d0 = f2u(r0.z), L = lo(l);
    const f3 axis = v3(r5);
    f3 com = lp + qrot(lq, v3(BR[(uint32_t)f2i(r0.w) * 8u + 1u]));
    st3(L + L_COM, com);
    f3 aw = qrot(jq, axis);
    f3 rj = com - jp;
    for (uint32_t c = 0; c < S.JM; c++) stsv(L + L_S + c * 6u, sv0());
    if (t == 1u) stsv(L + L_S, SVec{aw, cross(aw, rj)});
    if (t == 0u) stsv(L + L_S, SVec{sp3(0.0f), aw});
    if (t == 2u)
      for (uint32_t c = 0; c < 3u; c++) { f3 ew = qrot(jq, unit_axis(c)); stsv(L + L_S + c * 6u, SVec{ew, cross(ew, rj)}); }
    f3 rf = com - cp;
    st3(L + L_JR, rf);
    if (t == 6u) {
      for (uint32_t c = 0; c < j.nlin; c++) stsv(L + L_S + c * 6u, SVec{sp3(0.0f), qrot(jq, dof_axis(d0 + c))});
      for (uint32_t c = 0; c < j.nang; c++) {
        f3 ew = qrot(jq, j.ang[c]);
        stsv(L + L_S + (j.nlin + c) * 6u, SVec{ew, cross(ew, rf)});
      }
    }
    if (t == 4u) {
      for (uint32_t c = 0; c < 3u; c++) {
        f3 ew = qrot(jq, unit_axis(c));
        stsv(L + L_S + c * 6u, SVec{sp3(0.0f), ew});
        stsv(L + L_S + (c + 3u) * 6u, SVec{ew, cross(ew, rf)});
      }
    }
  }
  __device__ void fk(uint32_t a) const {
    const uint4 ai = info(a);
    for (uint32_t k = 0; k < ai.y; k++) {
      const uint32_t l = ai.x + k;
      f3 pp = sp3(0.0f);
      float4 pq = make_float4(0, 0, 0, 1);
      const int par = lparent(l);
      if (par >= 0) { pp = ld3(lo((uint32_t)par) + L_POS); pq = link_rot((uint32_t)par); }
      const FkJoint j = fk_joint(l);
      f3 jp, cp, lp;
      float4 jq, lq;
      fk_pose(l, pp, pq, j.mq, j.mp, jp, jq, cp, lp, lq);
      fk_store_pose(l, lp, lq);
      fk_out(l, j, jp, jq, cp, lp, lq);
    }
  }
  // fk() by one warp (all 32 lanes call it): lane k evaluates the joint motion of link k of each
  // 32-link chunk (the trigonometry) and afterwards its COM and motion subspace; between the two,
  // every lane runs the pose chain with the broadcast joint motions (same operations as fk()),
  // lane 0 stores the poses and each link's owner keeps its frames. A chain link's parent pose is
  // the previous link's, kept in registers.
  __device__ void fk_warp(uint32_t a, uint32_t lane) const {
    const uint4 ai = info(a);
    const uint32_t full = 0xffffffffu;
    f3 pprev = sp3(0.0f);
    float4 qprev = make_float4(0, 0, 0, 1);
    for (uint32_t c0 = 0; c0 < ai.y; c0 += 32u) {
      const uint32_t nl = min(32u, ai.y - c0);
      FkJoint j{};
      if (lane < nl) j = fk_joint(ai.x + c0 + lane);
      f3 ojp = sp3(0.0f), ocp = sp3(0.0f), olp = sp3(0.0f);
      float4 ojq = make_float4(0, 0, 0, 1), olq = make_float4(0, 0, 0, 1);
      for (uint32_t k = 0; k < nl; k++) {
        const uint32_t l = ai.x + c0 + k;
        const float4 mq = make_float4(__shfl_sync(full, j.mq.x, (int)k), __shfl_sync(full, j.mq.y, (int)k),
                                      __shfl_sync(full, j.mq.z, (int)k), __shfl_sync(full, j.mq.w, (int)k));
        const f3 mp = mf3(__shfl_sync(full, j.mp.x, (int)k), __shfl_sync(full, j.mp.y, (int)k),
                          __shfl_sync(full, j.mp.z, (int)k));
        f3 pp = sp3(0.0f);
        float4 pq = make_float4(0, 0, 0, 1);
        const int par = lparent(l);
        if (par >= 0) {
          if ((uint32_t)par + 1u == l) { pp = pprev; pq = qprev; }
          else { pp = ld3(lo((uint32_t)par) + L_POS); pq = link_rot((uint32_t)par); }
        }
        f3 jp, cp, lp;
        float4 jq, lq;
        fk_pose(l, pp, pq, mq, mp, jp, jq, cp, lp, lq);
        if (lane == 0u) fk_store_pose(l, lp, lq);
        __syncwarp();
        if (lane == k) { ojp = jp; ojq = jq; ocp = cp; olp = lp; olq = lq; }
        pprev = lp;
        qprev = lq;
      }
      if (lane < nl) fk_out(ai.x + c0 + lane, j, ojp, ojq, ocp, olp, olq);
      __syncwarp();
    }
  }

  // Gauss-Jordan inverse of the leading n x n block (artwgsl.js:192-207).
  static __device__ void inv_spd(float* D, uint32_t n, uint32_t JM, float* Di) {
    for (uint32_t i = 0; i < JM * JM; i++) Di[i] = 0.0f;
    for (uint32_t i = 0; i < n; i++) Di[i * JM + i] = 1.0f;
    for (uint32_t c = 0; c < n; c++) {
      float pv = 1.0f / fmx(D[c * JM + c], 1e-12f);
      for (uint32_t k = 0; k < n; k++) { D[c * JM + k] *= pv; Di[c * JM + k] *= pv; }
      for (uint32_t r = 0; r < n; r++) {
        if (r == c) continue;
        float f = D[r * JM + c];
        if (f == 0.0f) continue;
        for (uint32_t k = 0; k < n; k++) { D[r * JM + k] -= f * D[c * JM + k]; Di[r * JM + k] -= f * Di[c * JM + k]; }
      }
    }
  }

  // Diagonal terms and generalized force of dof d (the r-th of its link, joint coordinates from
  // qs): joint damping, spring, and the implicit PD drive folded into D (artwgsl.js:290-318).
  // Drr (float, or double under ART_F64) holds D[r][r] = S_r . U_r on entry and gains the drive
  // and damping terms; the drive's saturation test reads it rounded to float.
  template <class T>
  __device__ float dof_tau(uint32_t d, uint32_t qs, uint32_t r, T& Drr, const Params& P) const {
    // Every input is loaded first, so the loads overlap.
    const float4 dr = dof_drive(d), pas = dof_passive(d), spr = DR[d * 5u + 4u];
    const float qd = A[S.A_QD + d], jf = A[S.A_JF + d], q = A[S.A_Q + qs + r];
    const float tgt = A[S.A_TGT + d], tv = A[S.A_TGTV + d];
    Drr += (T)dr.x;
    float damp = pas.x;
    Drr += (T)P.dt * (T)damp;
    float tau = (-damp) * qd + jf;
    if (spr.x != 0.0f) tau += spr.x * (spr.y - q);
    if (S.DRIVE_ROWS == 0u && (dr.y > 0.0f || dr.z > 0.0f)) {
      float err = tgt - q;
      float mm = fmx((float)Drr, 1e-9f);
      float qdn = (mm * qd + P.dt * (dr.y * err + dr.z * tv)) / ((mm + P.dt * dr.z) + (P.dt * P.dt) * dr.y);
      float ti = dr.y * (err - P.dt * qdn) + dr.z * (tv - qdn);
      if (fabsf(ti) <= dr.w || dr.w <= 0.0f) {
        Drr += ((T)P.dt * (T)P.dt) * (T)dr.y + (T)P.dt * (T)dr.z;
        tau += (dr.y * err - (P.dt * dr.y) * qd) + dr.z * (tv - qd);
      } else {
        tau += clmp(ti, -dr.w, dr.w);
      }
    }
    return tau;
  }

  // Backward step of link l with the articulated-inertia branch in double (ART_F64, not a
  // reference option): U = I^A S, D = S^T U and its Gauss-Jordan inverse (artwgsl.js:192-207), the
  // projected inertia I^A - U D^-1 U^T and its shifted sum into the parent (artwgsl.js:90-95, 342)
  // are computed in double from the stored float blocks and rounded once on store, so the
  // accumulation toward the root cancels in double; bias forces stay float as in the FP32 step.
  __device__ void back_f64(uint32_t l, const Params& P) const {
    const uint32_t JM = JMc, L = lo(l), n = lndof(l), d0 = ldof(l), qs = lqs(l);
    const SVec pA = ldsv(L + L_PA);
    dm3 Am = dm(ldm(L + L_IA)), Bm = dm(ldm(L + L_IA + 9u)), Cm = dm(ldm(L + L_IA + 18u));
    d3 Ua[6], Ul[6];
    for (uint32_t c = 0; c < n; c++) {
      SVec s = ldS(l, c);
      d3 sa = dv(s.a), sl = dv(s.l);
      Ua[c] = dmul(Am, sa) + dmul(Bm, sl);
      Ul[c] = dmul(dtr(Bm), sa) + dmul(Cm, sl);
      stsv(L + L_U + c * 6u, SVec{fv(Ua[c]), fv(Ul[c])});
    }
    double D[36], Di[36];
    float u[6];
    for (uint32_t i = 0; i < 36u; i++) D[i] = 0.0;
    for (uint32_t r = 0; r < n; r++) {
      SVec s = ldS(l, r);
      for (uint32_t c = 0; c < n; c++) D[r * JM + c] = ddot(dv(s.a), Ua[c]) + ddot(dv(s.l), Ul[c]);
      float tau = dof_tau(d0 + r, qs, r, D[r * JM + r], P);
      u[r] = tau - sdot(s, pA);
    }
    for (uint32_t i = 0; i < JM * JM; i++) Di[i] = 0.0;
    for (uint32_t i = 0; i < n; i++) Di[i * JM + i] = 1.0;
    for (uint32_t c = 0; c < n; c++) {
      double pv = 1.0 / dmx(D[c * JM + c], 1e-12);
      for (uint32_t k = 0; k < n; k++) { D[c * JM + k] *= pv; Di[c * JM + k] *= pv; }
      for (uint32_t r = 0; r < n; r++) {
        if (r == c) continue;
        double f = D[r * JM + c];
        if (f == 0.0) continue;
        for (uint32_t k = 0; k < n; k++) { D[r * JM + k] -= f * D[c * JM + k]; Di[r * JM + k] -= f * Di[c * JM + k]; }
      }
    }
    for (uint32_t i = 0; i < JM * JM; i++) LB[L + L_DI + i] = (float)Di[i];
    for (uint32_t r = 0; r < JM; r++) LB[L + L_UU + r] = r < n ? u[r] : 0.0f;
    int par = lparent(l);
    if (par < 0) return;
    SVec Duu = sv0();
    for (uint32_t r = 0; r < n; r++) {
      float du = 0.0f;
      for (uint32_t c = 0; c < n; c++) {
        double w = Di[r * JM + c];
        Am = dsub(Am, dscl(w, douter(Ua[r], Ua[c])));
        Bm = dsub(Bm, dscl(w, douter(Ua[r], Ul[c])));
        Cm = dsub(Cm, dscl(w, douter(Ul[r], Ul[c])));
        du += ldDI(l, r, c) * u[c];
      }
      Duu = sadd(Duu, sscl(ldU(l, r), du));
    }
    stm(L + L_IA, fm(Am));
    stm(L + L_IA + 9u, fm(Bm));
    stm(L + L_IA + 18u, fm(Cm));
    SVec pa = sadd(sadd(pA, imul(L + L_IA, ldsv(L + L_C))), Duu);
    uint32_t P0 = lo((uint32_t)par);
    f3 r = link_r(l);
    dm3 Rs = dskew(dv(r));
    dm3 PA = dm(ldm(P0 + L_IA)), PB = dm(ldm(P0 + L_IA + 9u)), PC = dm(ldm(P0 + L_IA + 18u));
    stm(P0 + L_IA, fm(dsub(dadd(dsub(dadd(PA, Am), dmul(Bm, Rs)), dmul(Rs, dtr(Bm))), dmul(dmul(Rs, Cm), Rs))));
    stm(P0 + L_IA + 9u, fm(dadd(dadd(PB, Bm), dmul(Rs, Cm))));
    stm(P0 + L_IA + 18u, fm(dadd(PC, Cm)));
    stsv(P0 + L_PA, sadd(ldsv(P0 + L_PA), fshift(pa, r)));
  }

  // Articulated inertias, U = I^A S, D^-1 with implicit drives, free velocity (artwgsl.js:210-369).
  // F64: the backward pass's articulated-inertia branch in double (back_f64), for scenes with
  // ART_F64; it is a separate instance so the FP32 kernels keep their registers.
  template <bool F64>
  __device__ void factor(uint32_t a, const Params& P) const {
    uint4 ai = info(a);
    f3 g = v3(P.gravity);
    const uint32_t JM = S.JM;
    for (uint32_t k = 0; k < ai.y; k++) {
      uint32_t l = ai.x + k, L = lo(l);
      int par = lparent(l);
      uint32_t nd = lndof(l), d0 = ldof(l);
      // Global inputs first (qd of the link's dofs, the body's applied wrench), so they overlap.
      const uint32_t bo = S.A_BF + (uint32_t)lbody(l) * 8u;
      const f3 bforce = ald3(bo), btorque = ald3(bo + 4u);
      float qdv[6];
#pragma unroll
      for (uint32_t c = 0; c < 6u; c++) qdv[c] = c < nd ? A[S.A_QD + d0 + c] : 0.0f;
      SVec vp = sv0();
      if (par >= 0) vp = mshift(ldsv(lo((uint32_t)par) + L_V), link_r(l));
      SVec sq = sv0();
#pragma unroll
      for (uint32_t c = 0; c < 6u; c++) {
        if (c >= nd) break;
        sq = sadd(sq, sscl(ldS(l, c), qdv[c]));
      }
      SVec v = sadd(vp, sq);
      stsv(L + L_V, v);
      SVec cb = crm(vp, sq);
      uint32_t jt = ltype(l);
      if (jt == 6u) {
        uint32_t nlin = f2u(lrec(l, 5).w);
        f3 ca = sp3(0.0f);
        for (uint32_t j = nlin; j < nd; j++)
          for (uint32_t kk = j + 1u; kk < nd; kk++)
            ca += (cross(ldS(l, j).a, ldS(l, kk).a) * A[S.A_QD + d0 + j]) * A[S.A_QD + d0 + kk];
        cb = sadd(cb, SVec{ca, cross(ca, ld3(L + L_JR))});
      }
      if (jt == 4u || jt == 6u) {
        uint32_t nlin = jt == 4u ? 3u : f2u(lrec(l, 5).w);
        f3 vo = sp3(0.0f), wj = sp3(0.0f);
        for (uint32_t c = 0; c < nd; c++) {
          SVec sc = ldS(l, c);
          float q = A[S.A_QD + d0 + c];
          if (c < nlin) vo += sc.l * q; else wj += sc.a * q;
        }
        cb = sadd(cb, SVec{sp3(0.0f), -cross(wj, vo)});
      }
      stsv(L + L_C, cb);
      int b = lbody(l);
      float m = bmass(b);
      m3 R = qmat(link_rot(l));
      m3 Ic = mul(mul(R, binertia(b)), tr(R));
      stm(L + L_IA, Ic);
      stm(L + L_IA + 9u, mcols(sp3(0), sp3(0), sp3(0)));
      stm(L + L_IA + 18u, mcols(mf3(m, 0, 0), mf3(0, m, 0), mf3(0, 0, m)));
      SVec pa0 = crf(v, imul(L + L_IA, v));
      if ((f2u(BR[(uint32_t)b * 8u + 7u].w) & 2u) != 0u) pa0 = sadd(pa0, SVec{sp3(0.0f), m * g});
      pa0 = sadd(pa0, SVec{-btorque, -bforce});
      stsv(L + L_PA, pa0);
    }
    for (uint32_t kk = 0; kk < ai.y; kk++) {
      uint32_t l = ai.x + ai.y - 1u - kk, L = lo(l);
      if (F64) {
        back_f64(l, P);
        continue;
      }
      uint32_t n = lndof(l), d0 = ldof(l), qs = lqs(l);
      SVec pA = ldsv(L + L_PA);
      float u[6] = {0, 0, 0, 0, 0, 0};
#pragma unroll
      for (uint32_t c = 0; c < 6u; c++)
        if (c < n) stsv(L + L_U + c * 6u, imul(L + L_IA, ldS(l, c)));
      if (n == 1u) {
        // One dof: D is 1 x 1 and its Gauss-Jordan inverse is 1 * (1 / max(D, 1e-12)).
        float d00 = sdot(ldS(l, 0u), ldU(l, 0u));
        float tau = dof_tau(d0, qs, 0u, d00, P);
        u[0] = tau - sdot(ldS(l, 0u), pA);
        float di = 1.0f * (1.0f / fmx(d00, 1e-12f));
        for (uint32_t i = 0; i < JM * JM; i++) LB[L + L_DI + i] = i == 0u ? di : 0.0f;
      } else {
        float D[36];
        for (uint32_t i = 0; i < 36u; i++) D[i] = 0.0f;
        for (uint32_t r = 0; r < n; r++) {
          for (uint32_t c = 0; c < n; c++) D[r * JM + c] = sdot(ldS(l, r), ldU(l, c));
          float tau = dof_tau(d0 + r, qs, r, D[r * JM + r], P);
          float ur = tau - sdot(ldS(l, r), pA);
#pragma unroll
          for (uint32_t c = 0; c < 6u; c++) if (c == r) u[c] = ur;
        }
        float Di[36];
        inv_spd(D, n, JM, Di);
        for (uint32_t i = 0; i < JM * JM; i++) LB[L + L_DI + i] = Di[i];
      }
#pragma unroll
      for (uint32_t r = 0; r < 6u; r++) if (r < JM) LB[L + L_UU + r] = u[r];
      int par = lparent(l);
      if (par < 0) continue;
      m3 Am = ldm(L + L_IA), Bm = ldm(L + L_IA + 9u), Cm = ldm(L + L_IA + 18u);
      SVec Duu = sv0();
      for (uint32_t r = 0; r < n; r++) {
        SVec Ur = ldU(l, r);
        float du = 0.0f;
#pragma unroll
        for (uint32_t c = 0; c < 6u; c++) {
          if (c >= n) break;
          SVec Uc = ldU(l, c);
          float w = ldDI(l, r, c);
          Am = msub(Am, mscl(w, outer(Ur.a, Uc.a)));
          Bm = msub(Bm, mscl(w, outer(Ur.a, Uc.l)));
          Cm = msub(Cm, mscl(w, outer(Ur.l, Uc.l)));
          du += w * u[c];
        }
        Duu = sadd(Duu, sscl(Ur, du));
      }
      stm(L + L_IA, Am);
      stm(L + L_IA + 9u, Bm);
      stm(L + L_IA + 18u, Cm);
      SVec pa = sadd(sadd(pA, imul(L + L_IA, ldsv(L + L_C))), Duu);
      uint32_t P0 = lo((uint32_t)par);
      f3 r = link_r(l);
      m3 Rs = skew(r);
      stm(P0 + L_IA, msub(madd(msub(madd(ldm(P0 + L_IA), Am), mul(Bm, Rs)), mul(Rs, tr(Bm))), mul(mul(Rs, Cm), Rs)));
      stm(P0 + L_IA + 9u, madd(madd(ldm(P0 + L_IA + 9u), Bm), mul(Rs, Cm)));
      stm(P0 + L_IA + 18u, madd(ldm(P0 + L_IA + 18u), Cm));
      stsv(P0 + L_PA, sadd(ldsv(P0 + L_PA), fshift(pa, r)));
    }
    for (uint32_t k = 0; k < ai.y; k++) {
      uint32_t l = ai.x + k, L = lo(l);
      int par = lparent(l);
      SVec ap = SVec{sp3(0.0f), -g};
      if (par >= 0) ap = mshift(ldsv(lo((uint32_t)par) + L_A), link_r(l));
      SVec a1 = sadd(ap, ldsv(L + L_C));
      uint32_t n = lndof(l), d0 = ldof(l);
      SVec acc = a1;
      for (uint32_t r = 0; r < n; r++) {
        float qdd = 0.0f;
        for (uint32_t c = 0; c < n; c++) qdd += ldDI(l, r, c) * (LB[L + L_UU + c] - sdot(ldU(l, c), a1));
        A[S.A_QDH + d0 + r] = A[S.A_QD + d0 + r] + P.dt * qdd;
        acc = sadd(acc, sscl(ldS(l, r), qdd));
      }
      stsv(L + L_A, acc);
      if (S.JFL == 1u) {
        // joint_friction_load_coefficient (artwgsl.js:361-367): the joint's transmitted force and
        // torque under the free dynamics (I^A a + p^A at the child COM) raise its friction bound.
        const SVec f = sadd(imul(L + L_IA, acc), ldsv(L + L_PA));
        const float fm = len(f.l) + len(f.a);
        for (uint32_t r = 0; r < n; r++) A[S.A_JFL + d0 + r] = DR[(d0 + r) * 5u + 3u].w * fm;
      }
    }
  }

  __device__ uint32_t path(uint32_t l0, uint32_t* pth) const {
    uint32_t n = 0;
    int l = (int)l0;
    while (l >= 0 && n < S.MAXPATH) { pth[n] = (uint32_t)l; n++; l = lparent((uint32_t)l); }
    return n;
  }

  // Diagonal of H^-1 for dof r of link l (path_test with F = 0, artwgsl.js:375-414, 513-518).
  // ub: scratch of MAXPATH * JM floats.
  __device__ float dof_hinv(uint32_t l, uint32_t rr, uint32_t* pth, float* ub) const {
    const uint32_t JM = S.JM;
    uint32_t np = path(l, pth);
    SVec p = sscl(sv0(), -1.0f);
    for (uint32_t i = 0; i < np; i++) {
      uint32_t pl = pth[i], n = lndof(pl);
      float u[6] = {0, 0, 0, 0, 0, 0};
      for (uint32_t r = 0; r < n; r++) {
        float t = (pl == l && r == rr) ? 1.0f : 0.0f;
        u[r] = t - sdot(ldS(pl, r), p);
        ub[i * JM + r] = u[r];
      }
      for (uint32_t r = 0; r < n; r++) {
        float du = 0.0f;
        for (uint32_t c = 0; c < n; c++) du += ldDI(pl, r, c) * u[c];
        p = sadd(p, sscl(ldU(pl, r), du));
      }
      p = fshift(p, link_r(pl));
    }
    SVec dv = sv0();
    float out = 0.0f;
    for (uint32_t ii = 0; ii < np; ii++) {
      uint32_t i = np - 1u - ii, pl = pth[i], n = lndof(pl);
      dv = mshift(dv, link_r(pl));
      float dq[6] = {0, 0, 0, 0, 0, 0};
      for (uint32_t r = 0; r < n; r++) {
        dq[r] = 0.0f;
        for (uint32_t c = 0; c < n; c++) dq[r] += ldDI(pl, r, c) * (ub[i * JM + c] - sdot(ldU(pl, c), dv));
      }
      for (uint32_t r = 0; r < n; r++) {
        dv = sadd(dv, sscl(ldS(pl, r), dq[r]));
        if (pl == l && r == rr) out = dq[r];
      }
    }
    return out;
  }

  // Split COM response of link l (artwgsl.js:431-510). split: per path link, the number of
  // contact-bearing links whose root path crosses it. ub: scratch of 6 * MAXPATH * JM floats.
  __device__ void response(uint32_t l, const uint32_t* split, uint32_t* pth, float* ub) const {
    const uint32_t JM = S.JM, PD = S.MAXPATH * JM;
    uint32_t np = path(l, pth);
    SVec p[6];
    for (uint32_t e = 0; e < 6u; e++) {
      f3 f = sp3(0.0f), t = sp3(0.0f);
      if (e < 3u) setc(f, (int)e, 1.0f); else setc(t, (int)e - 3, 1.0f);
      p[e] = SVec{-t, -f};
    }
    for (uint32_t i = 0; i < np; i++) {
      uint32_t pl = pth[i], n = lndof(pl);
      f3 r = link_r(pl);
      for (uint32_t e = 0; e < 6u; e++) {
        float u[6] = {0, 0, 0, 0, 0, 0};
        for (uint32_t c = 0; c < n; c++) { u[c] = 0.0f - sdot(ldS(pl, c), p[e]); ub[e * PD + i * JM + c] = u[c]; }
        SVec pe = p[e];
        for (uint32_t rr = 0; rr < n; rr++) {
          float du = 0.0f;
          for (uint32_t c = 0; c < n; c++) du += ldDI(pl, rr, c) * u[c];
          pe = sadd(pe, sscl(ldU(pl, rr), du));
        }
        p[e] = fshift(pe, r);
      }
    }
    SVec dv[6];
    for (uint32_t e = 0; e < 6u; e++) dv[e] = sv0();
    for (uint32_t ii = 0; ii < np; ii++) {
      uint32_t i = np - 1u - ii, pl = pth[i], n = lndof(pl);
      f3 r = link_r(pl);
      for (uint32_t e = 0; e < 6u; e++) {
        SVec d = mshift(dv[e], r);
        float dq[6] = {0, 0, 0, 0, 0, 0};
        for (uint32_t rr = 0; rr < n; rr++) {
          dq[rr] = 0.0f;
          for (uint32_t c = 0; c < n; c++) dq[rr] += ldDI(pl, rr, c) * (ub[e * PD + i * JM + c] - sdot(ldU(pl, c), d));
        }
        for (uint32_t rr = 0; rr < n; rr++) d = sadd(d, sscl(ldS(pl, rr), dq[rr]));
        dv[e] = d;
      }
    }
    float W[36];
    for (uint32_t e = 0; e < 6u; e++) {
      W[0 * 6 + e] = dv[e].l.x; W[1 * 6 + e] = dv[e].l.y; W[2 * 6 + e] = dv[e].l.z;
      W[3 * 6 + e] = dv[e].a.x; W[4 * 6 + e] = dv[e].a.y; W[5 * 6 + e] = dv[e].a.z;
    }
    for (uint32_t k = 0; k < 36u; k++) LB[lo(l) + L_W2 + k] = W[k];
    for (uint32_t i = 0; i < np; i++) {
      float extra = (float)split[i] - 1.0f;
      if (extra <= 0.0f) continue;
      uint32_t pl = pth[i], n = lndof(pl);
      float t[36];
      for (uint32_t cc = 0; cc < 6u; cc++)
        for (uint32_t x = 0; x < n; x++) {
          float v = 0.0f;
          for (uint32_t y = 0; y < n; y++) v += ldDI(pl, x, y) * ub[cc * PD + i * JM + y];
          t[cc * 6u + x] = v;
        }
      for (uint32_t rr = 0; rr < 6u; rr++)
        for (uint32_t cc = 0; cc < 6u; cc++) {
          float sv = 0.0f;
          for (uint32_t x = 0; x < n; x++) sv += ub[rr * PD + i * JM + x] * t[cc * 6u + x];
          W[rr * 6u + cc] += extra * sv;
        }
    }
    for (uint32_t k = 0; k < 36u; k++) LB[lo(l) + L_W + k] = W[k];
  }

  // Generalized Jacobians (artwgsl.js:525-554).
  template <class PJ>
  __device__ void gen_jac(uint32_t x, f3 p, float sgn, f3 d0, f3 d1, f3 d2, uint32_t ds, PJ J) const {
    int l = (int)x;
    while (l >= 0) {
      uint32_t k = (uint32_t)l;
      f3 c = ld3(lo(k) + L_COM);
      for (uint32_t r = 0; r < lndof(k); r++) {
        SVec Sv = ldS(k, r);
        f3 v = Sv.l + cross(Sv.a, p - c);
        uint32_t i = ldof(k) + r - ds;
        J[i] += sgn * dot(d0, v);
        J[S.NDA + i] += sgn * dot(d1, v);
        J[2u * S.NDA + i] += sgn * dot(d2, v);
      }
      l = lparent(k);
    }
  }
  __device__ void gen_ang(uint32_t x, float sgn, f3 d0, f3 d1, uint32_t ds, float* J) const {
    int l = (int)x;
    while (l >= 0) {
      uint32_t k = (uint32_t)l;
      for (uint32_t r = 0; r < lndof(k); r++) {
        f3 w = ldS(k, r).a;
        uint32_t i = ldof(k) + r - ds;
        J[i] += sgn * dot(d0, w);
        J[S.NDA + i] += sgn * dot(d1, w);
      }
      l = lparent(k);
    }
  }
  // qd change of articulation a for generalized impulse tau (artwgsl.js:557-596).
  // scratch: 18 * MAXLP floats.
  __device__ void solve_gen(uint32_t a, const float* tau, float* out, float* scr) const {
    uint4 ai = info(a);
    float* p = scr;                  // 6 per link
    float* uu = scr + 6u * S.MAXLP;  // 6 per link
    float* dvs = scr + 12u * S.MAXLP;
    for (uint32_t k = 0; k < 6u * ai.y; k++) p[k] = 0.0f;
    auto ldp = [&](float* base, uint32_t k) { return SVec{mf3(base[k * 6], base[k * 6 + 1], base[k * 6 + 2]), mf3(base[k * 6 + 3], base[k * 6 + 4], base[k * 6 + 5])}; };
    auto stp = [&](float* base, uint32_t k, SVec v) {
      base[k * 6] = v.a.x; base[k * 6 + 1] = v.a.y; base[k * 6 + 2] = v.a.z;
      base[k * 6 + 3] = v.l.x; base[k * 6 + 4] = v.l.y; base[k * 6 + 5] = v.l.z;
    };
    for (uint32_t kk = 0; kk < ai.y; kk++) {
      uint32_t k = ai.y - 1u - kk, l = ai.x + k, n = lndof(l);
      float u[6] = {0, 0, 0, 0, 0, 0};
      SVec pk = ldp(p, k);
#pragma unroll
      for (uint32_t r = 0; r < 6u; r++) {
        if (r >= n) break;
        u[r] = tau[ldof(l) + r - ai.z] - sdot(ldS(l, r), pk);
      }
#pragma unroll
      for (uint32_t r = 0; r < 6u; r++) uu[k * 6u + r] = u[r];
      int par = lparent(l);
      if (par >= 0) {
        SVec pp = pk;
#pragma unroll
        for (uint32_t r = 0; r < 6u; r++) {
          if (r >= n) break;
          float du = 0.0f;
#pragma unroll
          for (uint32_t c = 0; c < 6u; c++) {
            if (c >= n) break;
            du += ldDI(l, r, c) * u[c];
          }
          pp = sadd(pp, sscl(ldU(l, r), du));
        }
        uint32_t pi = (uint32_t)par - ai.x;
        stp(p, pi, sadd(ldp(p, pi), fshift(pp, link_r(l))));
      }
    }
    for (uint32_t k = 0; k < ai.y; k++) {
      uint32_t l = ai.x + k;
      int par = lparent(l);
      SVec dv = sv0();
      if (par >= 0) dv = mshift(ldp(dvs, (uint32_t)par - ai.x), link_r(l));
      uint32_t n = lndof(l);
      float dq[6] = {0, 0, 0, 0, 0, 0};
#pragma unroll
      for (uint32_t r = 0; r < 6u; r++) {
        if (r >= n) break;
        dq[r] = 0.0f;
#pragma unroll
        for (uint32_t c = 0; c < 6u; c++) {
          if (c >= n) break;
          dq[r] += ldDI(l, r, c) * (uu[k * 6u + c] - sdot(ldU(l, c), dv));
        }
      }
#pragma unroll
      for (uint32_t r = 0; r < 6u; r++) {
        if (r >= n) break;
        dv = sadd(dv, sscl(ldS(l, r), dq[r]));
        out[ldof(l) + r - ai.z] = dq[r];
      }
      stp(dvs, k, dv);
    }
  }

  // solve_gen3 on a serial chain: p and dv carried in registers, u staged in uu (18 per link).
  template <class PF>
  __device__ void solve_gen3_chain(uint4 ai, PF J, PF Y, PF uu) const {
    const uint32_t NDA = S.NDA;
    SVec pc[3] = {sv0(), sv0(), sv0()};  // p of the link being visited (its child's contribution)
    for (uint32_t kk = 0; kk < ai.y; kk++) {
      uint32_t k = ai.y - 1u - kk, l = ai.x + k, n = lndof(l);
      bool has_parent = k > 0u || lparent(l) >= 0;
      f3 rl = link_r(l);
      uint32_t dl = ldof(l) - ai.z;
#pragma unroll
      for (uint32_t rs = 0; rs < 3u; rs++) {
        const PF tau = J + rs * NDA;
        float u[6] = {0, 0, 0, 0, 0, 0};
        SVec pk = pc[rs];
#pragma unroll
        for (uint32_t r = 0; r < 6u; r++) {
          if (r >= n) break;
          u[r] = tau[dl + r] - sdot(ldS(l, r), pk);
        }
#pragma unroll
        for (uint32_t r = 0; r < 6u; r++) {
          if (r >= n) break;
          uu[(k * 3u + rs) * 6u + r] = u[r];
        }
        if (has_parent) {
          SVec pp = pk;
#pragma unroll
          for (uint32_t r = 0; r < 6u; r++) {
            if (r >= n) break;
            float du = 0.0f;
#pragma unroll
            for (uint32_t c = 0; c < 6u; c++) {
              if (c >= n) break;
              du += ldDI(l, r, c) * u[c];
            }
            pp = sadd(pp, sscl(ldU(l, r), du));
          }
          pc[rs] = sadd(sv0(), fshift(pp, rl));
        }
      }
    }
    SVec dc[3] = {sv0(), sv0(), sv0()};  // dv of the parent of the link being visited
    for (uint32_t k = 0; k < ai.y; k++) {
      uint32_t l = ai.x + k;
      bool has_parent = lparent(l) >= 0;
      f3 rl = link_r(l);
      uint32_t n = lndof(l), dl = ldof(l) - ai.z;
#pragma unroll
      for (uint32_t rs = 0; rs < 3u; rs++) {
        SVec dv = sv0();
        if (has_parent) dv = mshift(dc[rs], rl);
        float dq[6] = {0, 0, 0, 0, 0, 0};
#pragma unroll
        for (uint32_t r = 0; r < 6u; r++) {
          if (r >= n) break;
          dq[r] = 0.0f;
#pragma unroll
          for (uint32_t c = 0; c < 6u; c++) {
            if (c >= n) break;
            dq[r] += ldDI(l, r, c) * (uu[(k * 3u + rs) * 6u + c] - sdot(ldU(l, c), dv));
          }
        }
#pragma unroll
        for (uint32_t r = 0; r < 6u; r++) {
          if (r >= n) break;
          dv = sadd(dv, sscl(ldS(l, r), dq[r]));
          Y[rs * NDA + dl + r] = dq[r];
        }
        dc[rs] = dv;
      }
    }
  }

  // solve_gen for three right-hand sides in one walk of the articulation: row r of J (NDA
  // floats, zero beyond the articulation's dofs) is the generalized impulse of right-hand side r,
  // row r of Y receives its qd change. Each right-hand side goes through exactly the operations of
  // solve_gen. scratch: 54 * MAXLP floats.
  template <class PF>
  __device__ void solve_gen3(uint32_t a, PF J, PF Y, PF scr) const {
    uint4 ai = info(a);
    const uint32_t NDA = S.NDA, M = S.MAXLP;
    // A serial chain (every link's parent is the previous link) has one child per link, so the
    // impulse accumulated into a parent and the velocity change handed to a child can stay in
    // registers; the sums are the same (the parent's accumulator starts at zero).
    bool chain = true;
    for (uint32_t k = 1; k < ai.y; k++) chain = chain && lparent(ai.x + k) == (int)(ai.x + k - 1u);
    if (chain) { solve_gen3_chain(ai, J, Y, scr + 18u * M); return; }
    PF p = scr;                     // per link, 3 x 6
    PF uu = scr + 18u * M;          // per link, 3 x 6
    PF dvs = scr + 36u * M;         // per link, 3 x 6
    for (uint32_t k = 0; k < 18u * ai.y; k++) p[k] = 0.0f;
    auto ldp = [&](PF base, uint32_t k) {
      return SVec{mf3(base[k * 6], base[k * 6 + 1], base[k * 6 + 2]), mf3(base[k * 6 + 3], base[k * 6 + 4], base[k * 6 + 5])};
    };
    auto stp = [&](PF base, uint32_t k, SVec v) {
      base[k * 6] = v.a.x; base[k * 6 + 1] = v.a.y; base[k * 6 + 2] = v.a.z;
      base[k * 6 + 3] = v.l.x; base[k * 6 + 4] = v.l.y; base[k * 6 + 5] = v.l.z;
    };
    for (uint32_t kk = 0; kk < ai.y; kk++) {
      uint32_t k = ai.y - 1u - kk, l = ai.x + k, n = lndof(l);
      int par = lparent(l);
      f3 rl = link_r(l);
      uint32_t dl = ldof(l) - ai.z;
#pragma unroll
      for (uint32_t rs = 0; rs < 3u; rs++) {
        const PF tau = J + rs * NDA;
        float u[6] = {0, 0, 0, 0, 0, 0};
        SVec pk = ldp(p, k * 3u + rs);
#pragma unroll
        for (uint32_t r = 0; r < 6u; r++) {
          if (r >= n) break;
          u[r] = tau[dl + r] - sdot(ldS(l, r), pk);
        }
#pragma unroll
        for (uint32_t r = 0; r < 6u; r++) {
          if (r >= n) break;
          uu[(k * 3u + rs) * 6u + r] = u[r];
        }
        if (par >= 0) {
          SVec pp = pk;
#pragma unroll
          for (uint32_t r = 0; r < 6u; r++) {
            if (r >= n) break;
            float du = 0.0f;
#pragma unroll
            for (uint32_t c = 0; c < 6u; c++) {
              if (c >= n) break;
              du += ldDI(l, r, c) * u[c];
            }
            pp = sadd(pp, sscl(ldU(l, r), du));
          }
          uint32_t pi = ((uint32_t)par - ai.x) * 3u + rs;
          stp(p, pi, sadd(ldp(p, pi), fshift(pp, rl)));
        }
      }
    }
    for (uint32_t k = 0; k < ai.y; k++) {
      uint32_t l = ai.x + k;
      int par = lparent(l);
      f3 rl = link_r(l);
      uint32_t n = lndof(l), dl = ldof(l) - ai.z;
#pragma unroll
      for (uint32_t rs = 0; rs < 3u; rs++) {
        SVec dv = sv0();
        if (par >= 0) dv = mshift(ldp(dvs, ((uint32_t)par - ai.x) * 3u + rs), rl);
        float dq[6] = {0, 0, 0, 0, 0, 0};
#pragma unroll
        for (uint32_t r = 0; r < 6u; r++) {
          if (r >= n) break;
          dq[r] = 0.0f;
#pragma unroll
          for (uint32_t c = 0; c < 6u; c++) {
            if (c >= n) break;
            dq[r] += ldDI(l, r, c) * (uu[(k * 3u + rs) * 6u + c] - sdot(ldU(l, c), dv));
          }
        }
#pragma unroll
        for (uint32_t r = 0; r < 6u; r++) {
          if (r >= n) break;
          dv = sadd(dv, sscl(ldS(l, r), dq[r]));
          Y[rs * NDA + dl + r] = dq[r];
        }
        stp(dvs, k * 3u + rs, dv);
      }
    }
  }

  // Solve-side propagation (wgsl.js:3233-3299). tw: body twists (v, w), aqd: generalized velocities.
  __device__ void set_twist(uint32_t l, SVec v, float4* tw) const {
    uint32_t b = (uint32_t)lbody(l);
    tw[b * 2u] = mf4(v.l, 0.0f);
    tw[b * 2u + 1u] = mf4(v.a, 0.0f);
  }
  __device__ void twists(uint32_t a, const float* aqd, float4* tw) const {
    uint4 ai = info(a);
    for (uint32_t k = 0; k < ai.y; k++) {
      uint32_t l = ai.x + k;
      int par = lparent(l);
      SVec v = sv0();
      if (par >= 0) v = mshift(ldsv(lo((uint32_t)par) + L_V), link_r(l));
      for (uint32_t r = 0; r < lndof(l); r++) v = sadd(v, sscl(ldS(l, r), aqd[ldof(l) + r]));
      stsv(lo(l) + L_V, v);
      set_twist(l, v, tw);
    }
  }
  // twists() by one warp (all 32 lanes call it). The per-link inputs that do not depend on the
  // recursion -- the parent, the COM offset to it and, for a one-dof link, S qd -- are computed
  // by lane k for link k of each 32-link chunk and broadcast with shuffles; every lane then runs
  // the recursion with the same operations in the same order as twists(), and lane 0 stores.
  // A chain link's parent twist is the previous link's, kept in registers.
  __device__ void twists_warp(uint32_t a, const float* aqd, float4* tw, uint32_t lane) const {
    const uint4 ai = info(a);
    const uint32_t full = 0xffffffffu;
    SVec vprev = sv0();
    for (uint32_t c0 = 0; c0 < ai.y; c0 += 32u) {
      const uint32_t nl = min(32u, ai.y - c0);
      int par = -1;
      uint32_t nd = 0u;
      f3 r = sp3(0.0f);
      SVec prod = sv0();
      if (lane < nl) {
        const uint32_t l = ai.x + c0 + lane;
        par = lparent(l);
        nd = lndof(l);
        if (par >= 0) r = link_r(l);
        if (nd == 1u) prod = sscl(ldS(l, 0u), aqd[ldof(l)]);
      }
      for (uint32_t k = 0; k < nl; k++) {
        const uint32_t l = ai.x + c0 + k;
        const int p = __shfl_sync(full, par, (int)k);
        const uint32_t n = __shfl_sync(full, nd, (int)k);
        const f3 rr = mf3(__shfl_sync(full, r.x, (int)k), __shfl_sync(full, r.y, (int)k), __shfl_sync(full, r.z, (int)k));
        const SVec pr = SVec{mf3(__shfl_sync(full, prod.a.x, (int)k), __shfl_sync(full, prod.a.y, (int)k),
                                 __shfl_sync(full, prod.a.z, (int)k)),
                             mf3(__shfl_sync(full, prod.l.x, (int)k), __shfl_sync(full, prod.l.y, (int)k),
                                 __shfl_sync(full, prod.l.z, (int)k))};
        SVec v = sv0();
        if (p >= 0) v = mshift((uint32_t)p + 1u == l ? vprev : ldsv(lo((uint32_t)p) + L_V), rr);
        if (n == 1u) {
          v = sadd(v, pr);
        } else {
          for (uint32_t q = 0; q < n; q++) v = sadd(v, sscl(ldS(l, q), aqd[ldof(l) + q]));
        }
        if (lane == 0u) {
          stsv(lo(l) + L_V, v);
          set_twist(l, v, tw);
        }
        __syncwarp();
        vprev = v;
      }
    }
  }
  __device__ void apply(uint32_t a, float* aqd, float4* tw) const {
    uint4 ai = info(a);
    for (uint32_t kk = 0; kk < ai.y; kk++) {
      uint32_t l = ai.x + ai.y - 1u - kk, L = lo(l);
      uint32_t n = lndof(l);
      SVec p = ldsv(L + L_P);
      float u[6] = {0, 0, 0, 0, 0, 0};
#pragma unroll
      for (uint32_t r = 0; r < 6u; r++) {
        if (r >= n) break;
        u[r] = LB[L + L_TAU + r] - sdot(ldS(l, r), p);
        LB[L + L_UU + r] = u[r];
      }
      int par = lparent(l);
      if (par >= 0) {
        SVec pp = p;
#pragma unroll
        for (uint32_t r = 0; r < 6u; r++) {
          if (r >= n) break;
          float du = 0.0f;
#pragma unroll
          for (uint32_t c = 0; c < 6u; c++) {
            if (c >= n) break;
            du += ldDI(l, r, c) * u[c];
          }
          pp = sadd(pp, sscl(ldU(l, r), du));
        }
        uint32_t P0 = lo((uint32_t)par) + L_P;
        stsv(P0, sadd(ldsv(P0), fshift(pp, link_r(l))));
      }
    }
    for (uint32_t k = 0; k < ai.y; k++) {
      uint32_t l = ai.x + k, L = lo(l);
      int par = lparent(l);
      SVec dv = sv0();
      if (par >= 0) dv = mshift(ldsv(lo((uint32_t)par) + L_DV), link_r(l));
      uint32_t n = lndof(l);
      float dq[6] = {0, 0, 0, 0, 0, 0};
#pragma unroll
      for (uint32_t r = 0; r < 6u; r++) {
        if (r >= n) break;
        dq[r] = 0.0f;
#pragma unroll
        for (uint32_t c = 0; c < 6u; c++) {
          if (c >= n) break;
          dq[r] += ldDI(l, r, c) * (LB[L + L_UU + c] - sdot(ldU(l, c), dv));
        }
      }
#pragma unroll
      for (uint32_t r = 0; r < 6u; r++) {
        if (r >= n) break;
        dv = sadd(dv, sscl(ldS(l, r), dq[r]));
        aqd[ldof(l) + r] += dq[r];
      }
      stsv(L + L_DV, dv);
      SVec v = sadd(ldsv(L + L_V), dv);
      stsv(L + L_V, v);
      set_twist(l, v, tw);
      stsv(L + L_P, sv0());
      for (uint32_t r = 0; r < S.JM; r++) LB[L + L_TAU + r] = 0.0f;
    }
  }
};

}  // namespace steel
