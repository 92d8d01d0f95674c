#pragma once
// Solve of one scene by one block (the body of k_solve).
//
// Follows the reference's solve pass (packages/steel-webgpu/src/wgsl.js:2501-3891) on its
// default option set: free-body gravity, wrench and gyroscopic prologue (wgsl.js:3647-3675),
// the slot table (wgsl.js:3679-3686), the warm-apply sweep and `iterations` colored
// Gauss-Seidel sweeps (wgsl.js:3559-3611) of fixed-normal contact rows with friction anchors
// (wgsl.js:3033-3231, 2952-3011), dense same-articulation rows (wgsl.js:3306-3377), exact
// Featherstone impulse propagation and joint limit / friction rows after each sweep
// (wgsl.js:3380-3468), the warm-start table (wgsl.js:3737-3767), integration of bodies and
// joints with FK (wgsl.js:3768-3828) and the friction-anchor advance (wgsl.js:3832-3878).
// Rows of one color touch disjoint bodies, so a color's rows run in parallel across the block
// with one barrier per color; the overflow color runs serially in contact order.
#include "art.cuh"
#include "batch.cuh"
#include "block.cuh"
#include "bulk.cuh"
#include "cone5.cuh"
#include "team.cuh"

namespace steel {

static constexpr uint32_t AVN_S = 14u;

template <bool TEAM>
struct SolverT {
  const SceneDev& S;
  const Params& P;
  Art ar;
  float4* tw;
  float4* imp;
  float* aqd;
  bool vpass = false;  // velocity pass (wgsl.js:2928): rows without position bias or regularization
  Team<TEAM> tm;       // the threads that solve the scene: the block, or every block of a team launch
  __device__ SolverT(Team<TEAM> tm_, const SceneDev& s, const Params& p, float* lb, float4* tw_, float4* imp_,
                     float* aqd_)
      : S(s), P(p), ar(s, lb), tw(tw_), imp(imp_), aqd(aqd_), tm(tm_) {}

  __device__ uint32_t bkind(int b) const { return f2u(S.sf[S.SF_BODY + (uint32_t)b * 8u].y); }
  __device__ uint32_t bflags(int b) const { return b < 0 ? 0u : f2u(S.sf[S.SF_BODY + (uint32_t)b * 8u + 7u].w); }
  __device__ float bradius(int b) const { return b < 0 ? 1e30f : S.sf[S.SF_BODY + (uint32_t)b * 8u + 2u].w; }
  __device__ m3 binv_inertia(int b) const {
    RO<float4> o = S.sf + S.SF_BODY + (uint32_t)b * 8u;
    return tr(mcols(v3(o[5]), v3(o[6]), v3(o[7])));
  }
  // A body's twist at the end of the position iterations (wgsl.js:2930-2934).
  __device__ void snap_tw(int b, f3 out[2]) const {
    if (b < 0) { out[0] = sp3(0.0f); out[1] = sp3(0.0f); return; }
    const uint32_t o = S.A_SNAP + (uint32_t)b * 8u;
    out[0] = ar.ald3(o);
    out[1] = ar.ald3(o + 4u);
  }
  __device__ void load_tw(int b, f3 out[2]) const {
    if (b < 0) { out[0] = sp3(0.0f); out[1] = sp3(0.0f); return; }
    out[0] = v3(tw[(uint32_t)b * 2u]);
    out[1] = v3(tw[(uint32_t)b * 2u + 1u]);
  }
  __device__ void add_imp(int b, f3 f, f3 t) const {
    if (b < 0 || bkind(b) != 2u) return;
    imp[(uint32_t)b * 2u] = add4(imp[(uint32_t)b * 2u], mf4(f, 0.0f));
    imp[(uint32_t)b * 2u + 1u] = add4(imp[(uint32_t)b * 2u + 1u], mf4(t, 0.0f));
  }
  static __device__ m3 inverse3(const m3& m) {
    f3 a = m.c[0], b = m.c[1], c = m.c[2];
    f3 r0 = cross(b, c), r1 = cross(c, a), r2 = cross(a, b);
    float det = dot(a, r0);
    return mscl(1.0f / det, tr(mcols(r0, r1, r2)));
  }
  // Energy-preserving Cayley microsteps of the free-body gyroscopic term (wgsl.js:2543-2562).
  static __device__ f3 gyro(const m3& inertia, f3 u0, float dt) {
    m3 a = mscl(1.0f / fmx(inertia.c[0].x, fmx(inertia.c[1].y, inertia.c[2].z)), inertia);
    m3 inv = inverse3(a);
    float speed = sqrtf(fmx(dot(u0, mul(a, u0)) * ((inv.c[0].x + inv.c[1].y) + inv.c[2].z), 0.0f));
    uint32_t n = f2u(clmp(ceilf((2.0f * fabsf(dt)) * speed), 1.0f, 32.0f));
    float h = dt / (float)n;
    f3 w = u0;
    for (uint32_t m = 0; m < n; m++) {
      f3 u = w;
      float energy = dot(u, mul(a, u));
      for (uint32_t it = 0; it < 8u; it++) {
        m3 Sk = mscl(0.5f * h, skew(mul(a, 0.5f * (u + w))));
        f3 c = mul(inverse3(msub(a, Sk)), mul(madd(a, Sk), u));
        f3 d = c - w;
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
  static __device__ f2 tangent_step(f2 ut, float4 g1) {
    float det = g1.x * g1.z - g1.y * g1.y;
    if (fabsf(det) <= 1e-20f) return mf2(0.0f, 0.0f);
    return mf2((-ut.x) * g1.z + ut.y * g1.y, ut.x * g1.y - ut.y * g1.x) / det;
  }
  static __device__ f2 clip_cone(f2 t, float lim) {
    float m = len(t);
    if (m > lim && m > 1e-20f) return t * (lim / m);
    return t;
  }
  // A singular block (fewer than two tangential mobilities) keeps the normal impulse and takes the
  // fixed-normal pair on its disk.
  static __device__ f3 fixed_normal_pair(f2 ut0, float4 g1, float mu, f3 lam) {
    f2 t = friction_pair(g1.x, g1.y, g1.z, ut0.x, ut0.y, lam.y, lam.z, fmx(mu * lam.x, 0.0f), 1.0f);
    return mf3(lam.x, t.x, t.y);
  }
  static __device__ f3 contact_block(uint32_t mode, float un, f2 ut0, float4 g0, float4 g1, float vtarget0, float mu,
                          f3 lam) {
    const float gnn = g0.x;
    const f2 gnt = mf2(g0.y, g0.z);
    const float trace = g1.x + g1.z;
    if (g1.x * g1.z - g1.y * g1.y <= (1e-6f * trace) * trace) return fixed_normal_pair(ut0, g1, mu, lam);
    if (gnn < 1e-20f) return lam;
    const f2 lt = mf2(lam.y, lam.z);
    float vt_n = vtarget0;
    if (mode == 2u) vt_n += mu * len(ut0);
    if (mode == 3u) {
      const float un_f = un - (gnn * lam.x + dot(gnt, lt));
      const f2 ut_f = ut0 - mf2((gnt.x * lam.x + g1.x * lt.x) + g1.y * lt.y, (gnt.y * lam.x + g1.y * lt.x) + g1.z * lt.y);
      if (un_f >= vt_n) return mf3(0.0f, 0.0f, 0.0f);
      const float bN = un_f - vt_n;
      const float A00 = g1.x - (gnt.x * gnt.x) / gnn, A01 = g1.y - (gnt.x * gnt.y) / gnn;
      const float A11 = g1.z - (gnt.y * gnt.y) / gnn;
      if (A00 * A11 - A01 * A01 <= (1e-6f * trace) * trace) return fixed_normal_pair(ut0, g1, mu, lam);
      const f2 c = ut_f - (bN / gnn) * gnt;
      const float id0 = 1.0f / (A00 * A11 - A01 * A01);
      f2 s = mf2(A11 * c.x - A01 * c.y, A00 * c.y - A01 * c.x) * id0;
      const float phi0 = len(s) - (mu * (dot(gnt, s) - bN)) / gnn;
      if (phi0 > 0.0f) {
        float hi = 1.0f;
        for (uint32_t e = 0; e < 30u; e++) {
          const float a = A00 + hi, d = A11 + hi, idt = 1.0f / (a * d - A01 * A01);
          const f2 sh = mf2(d * c.x - A01 * c.y, a * c.y - A01 * c.x) * idt;
          if (len(sh) - (mu * (dot(gnt, sh) - bN)) / gnn < 0.0f) break;
          hi *= 2.0f;
        }
        float lo = 0.0f, x = 0.5f * hi;
        const float tol = 1e-6f + 1e-6f * phi0;
        for (uint32_t k = 0; k < 50u; k++) {
          const float a = A00 + x, d = A11 + x, idt = 1.0f / (a * d - A01 * A01);
          const f2 sx = mf2(d * c.x - A01 * c.y, a * c.y - A01 * c.x) * idt;
          const f2 tx = mf2(d * sx.x - A01 * sx.y, a * sx.y - A01 * sx.x) * idt;
          const float ns = len(sx);
          const float fx = ns - (mu * (dot(gnt, sx) - bN)) / gnn;
          const float dfx = (-dot(sx, tx)) / ns + (mu * dot(gnt, tx)) / gnn;
          s = sx;
          if (fabsf(fx) < tol || fabsf(hi - lo) < 1e-6f * (1.0f + hi)) break;
          if (fx > 0.0f) lo = x; else hi = x;
          float xn = 0.5f * (lo + hi);
          if (dfx != 0.0f) {
            const float xt = x - fx / dfx;
            if (xt > lo && xt < hi) xn = xt;
          }
          x = xn;
        }
      }
      const f2 rt = mf2(-s.x, -s.y);
      // The finite search can end just below zero load; the exact root is non-negative.
      const float ln = fmx((-(dot(gnt, rt) + bN)) / gnn, 0.0f);
      const float lim = fmx(mu * ln, 0.0f);
      const float m = len(rt);
      const f2 t = m > lim ? rt * (lim / m) : rt;
      return mf3(ln, t.x, t.y);
    }
    const float u0 = (un - gnn * lam.x) - dot(gnt, lt);
    if (u0 >= vt_n) return mf3(0.0f, 0.0f, 0.0f);
    float lo = 0.0f;
    float hi = fmx(fmx(2.0f * lam.x, (vt_n - un) / gnn + lam.x), 1.0f);
    float flo = u0 - vt_n, fhi = -1.0f;
    for (uint32_t k = 0; k < 20u; k++) {
      const float mid = 0.5f * (lo + hi);
      const float dn = mid - lam.x;
      const f2 tr = clip_cone(lt + tangent_step(ut0 + gnt * dn, g1), mu * mid);
      const float u = (un + gnn * dn) + dot(gnt, tr - lt);
      if (u < vt_n) { lo = mid; flo = u - vt_n; } else { hi = mid; fhi = u - vt_n; }
    }
    float ln = 0.5f * (lo + hi);
    if (fhi >= 0.0f) ln = lo - (flo * (hi - lo)) / (fhi - flo);
    const f2 tf = clip_cone(lt + tangent_step(ut0 + gnt * (ln - lam.x), g1), mu * ln);
    return mf3(ln, tf.x, tf.y);
  }
  // Friction pair update on its 2x2 block with a disk bound (wgsl.js:2952-3011).
  static __device__ f2 friction_pair(float a0, float c0, float d0, float r0, float r1, float old0, float old1,
                                     float radius, float omega) {
    if (radius <= 0.0f) return mf2(0.0f, 0.0f);
    float scale = fmx(fmx(a0, d0), 1e-20f);
    float a = a0 / scale, c = c0 / scale, d = d0 / scale;
    float largest = 0.5f * ((a + d) + sqrtf((a - d) * (a - d) + (4.0f * c) * c));
    float smallest = largest > 0.0f ? fmx((a * d - c * c) / largest, 0.0f) : 0.0f;
    float vx = c, vy = largest - a;
    if (a >= d) { vx = largest - d; vy = c; }
    float vn = sqrtf(vx * vx + vy * vy);
    if (vn > 0.0f) { vx /= vn; vy /= vn; } else { vx = 1.0f; vy = 0.0f; }
    float r0r = (vx * r0 + vy * r1) / scale;
    float r1r = ((-vy) * r0 + vx * r1) / scale;
    f2 res = mf2(old0, old1);
    bool sticking = false;
    if (largest > 0.0f && (smallest > 0.0f || r1r == 0.0f)) {
      float dx = r0r / largest;
      float dy = smallest > 0.0f ? r1r / smallest : 0.0f;
      res = mf2(old0 - (vx * dx - vy * dy), old1 - (vy * dx + vx * dy));
      sticking = len(res) <= radius;
    }
    if (!sticking) {
      float on = len(mf2(old0, old1)), rn = len(mf2(r0, r1));
      if (on > 0.0f && on <= radius && radius - on <= 2e-7f * radius && r0 * old0 + r1 * old1 <= 0.0f &&
          fabsf(r0 * old1 - r1 * old0) <= (2e-7f * on) * rn)
        return mf2(old0, old1);
      float ox = vx * old0 + vy * old1, oy = (-vy) * old0 + vx * old1;
      float b0 = largest * ox - r0r, b1 = smallest * oy - r1r;
      float x = 0.0f, y = 0.0f;
      float hi = sqrtf(b0 * b0 + b1 * b1) / radius;
      if (hi > 0.0f) {
        float lo = fmx(fmx(hi - largest, fabsf(b1) / radius - smallest), 0.0f);
        float alpha = lo;
        bool done = false;
        for (uint32_t it = 0; it < 8u; it++) {
          float i0 = 1.0f / (largest + alpha);
          float i1 = smallest + alpha > 0.0f ? 1.0f / (smallest + alpha) : 0.0f;
          float tx = ox - (r0r + alpha * ox) * i0, ty = oy - (r1r + alpha * oy) * i1;
          float nr = sqrtf(tx * tx + ty * ty);
          if (fabsf(nr - radius) <= 2e-7f * radius || (alpha == 0.0f && nr <= radius)) { x = tx; y = ty; done = true; break; }
          if (nr > radius) lo = alpha; else hi = alpha;
          float slope = (tx * tx) * i0 + (ty * ty) * i1;
          float cand = alpha;
          if (slope > 0.0f) cand = alpha + (((nr / radius - 1.0f) * nr) * nr) / slope;
          alpha = (cand > lo && cand < hi) ? cand : 0.5f * (lo + hi);
        }
        if (!done) {
          for (uint32_t it = 0; it < 24u; it++) {
            alpha = 0.5f * (lo + hi);
            if (len(mf2(b0 / (largest + alpha), b1 / (smallest + alpha))) > radius) lo = alpha; else hi = alpha;
          }
          x = b0 / (largest + hi);
          y = b1 / (smallest + hi);
        }
      }
      res = mf2((old0 + vx * (x - ox)) - vy * (y - oy), (old1 + vy * (x - ox)) + vx * (y - oy));
    }
    f2 old = mf2(old0, old1);
    f2 relaxed = old + omega * (res - old);
    float m = len(relaxed);
    return m > radius ? relaxed * (radius / m) : relaxed;
  }

  // One contact row of unit us (wgsl.js:3033-3231, default option set). mode 0 applies the warm
  // impulses, mode 1 solves.
  // Contact torsion (wgsl.js:3185-3228), run by a unit's last-colored row in position sweeps:
  // sliding and spin share the cluster's Coulomb budget mu * N.
  __device__ void torsion(uint32_t us, int a, int b, uint32_t it, f3 ta[2], f3 tb[2]) const {
    const uint32_t ROWS = S.ROWS, PO = S.PO, TO = S.TO;
    float4* rows = S.rows;
    const uint32_t s0 = S.sched[S.S_USTART + us], s1 = s0 + S.sched[S.S_USIZE + us];
    const uint32_t L = s0 * ROWS;
    if (!(rows[L + TO].w > 0.0f)) return;
    const float mu = rows[L + TO].w;
    float load = 0.0f, slide = 0.0f;
    for (uint32_t m = s0; m < s1; m++) {
      const uint32_t om = m * ROWS;
      if (rows[om + TO + 4u].w < 0.5f) continue;
      const float4 lm = rows[om + 6u];
      load += fmx(lm.x, 0.0f);
      if (S.EXTRA == 0u || rows[om + PO].w != 0.0f) slide += len(mf2(lm.y, lm.z));
    }
    const float budget = mu * load;
    if (slide > budget && slide > 0.0f) {
      // Later normals lowered the load: the members' tangent pairs are projected onto it.
      const float scale = budget / slide;
      for (uint32_t m = s0; m < s1; m++) {
        const uint32_t om = m * ROWS;
        if (rows[om + TO + 4u].w < 0.5f || (S.EXTRA == 1u && rows[om + PO].w == 0.0f)) continue;
        const float4 lm = rows[om + 6u];
        const float d1 = lm.y * (scale - 1.0f), d2 = lm.z * (scale - 1.0f);
        ta[0] += v3(rows[om + 11u]) * d1 + v3(rows[om + 15u]) * d2;
        ta[1] += v3(rows[om + 12u]) * d1 + v3(rows[om + 16u]) * d2;
        tb[0] += v3(rows[om + 13u]) * d1 + v3(rows[om + 17u]) * d2;
        tb[1] += v3(rows[om + 14u]) * d1 + v3(rows[om + 18u]) * d2;
        f3 fa = v3(rows[om + 3u]), fb = v3(rows[om + 4u]);
        if (S.EXTRA == 1u) { fa = v3(rows[om + PO]); fb = v3(rows[om + PO + 1u]); }
        const f3 f = v3(rows[om + 1u]) * d1 + v3(rows[om + 2u]) * d2;
        add_imp(a, -f, -cross(fa, f));
        add_imp(b, f, cross(fb, f));
        rows[om + 6u] = make_float4(lm.x, lm.y * scale, lm.z * scale, lm.w);
      }
      slide = budget;
    }
    float bound = rows[L + TO + 3u].w * fmx(budget - slide, 0.0f);
    if (it < S.FSTART) bound = 0.0f;
    const f3 ng = v3(rows[L + TO + 4u]);
    const float ls = rows[L + TO + 2u].w;
    const float nls = clmp(ls - (S.F_OMEGA * dot(ng, tb[1] - ta[1])) * rows[L + TO + 1u].w, -bound, bound);
    const float ds = nls - ls;
    if (ds != 0.0f) {
      ta[0] += v3(rows[L + TO]) * ds;
      ta[1] += v3(rows[L + TO + 1u]) * ds;
      tb[0] += v3(rows[L + TO + 2u]) * ds;
      tb[1] += v3(rows[L + TO + 3u]) * ds;
      rows[L + TO + 2u].w = nls;
      add_imp(a, sp3(0.0f), (-ng) * ds);
      add_imp(b, sp3(0.0f), ng * ds);
    }
  }
  // The articulated angular block of one contact row: H unpacked from the row's upper triangle, the
  // rows' velocity residual, the cone solve, then the impulse change applied to both bodies. Twists
  // and impulses go in and out by value, so the contact loop's own stay in registers.
  struct AngOut {
    f3 ta0, ta1, tb0, tb1;
    float l1, l2;
  };
  __device__ __noinline__ AngOut ang_block(uint32_t o, int a, int b, f3 n, f3 t1, f3 t2, f3 fra, f3 frb, float mu,
                                           float pooled, float ly, float lz, f3 ta0, f3 ta1, f3 tb0, f3 tb1) const {
    float4* rows = S.rows;
    f3 ta[2] = {ta0, ta1}, tb[2] = {tb0, tb1};
    float H[25];
    uint32_t idx = 0;
    for (uint32_t x = 0; x < 5u; x++)
      for (uint32_t y = x; y < 5u; y++) {
        const float4 q = rows[o + S.EO + idx / 4u];
        const uint32_t m = idx % 4u;
        const float hv = m == 0u ? q.x : (m == 1u ? q.y : (m == 2u ? q.z : q.w));
        H[x * 5u + y] = hv;
        H[y * 5u + x] = hv;
        idx++;
      }
    const f3 vt = (tb[0] + cross(tb[1], frb)) - (ta[0] + cross(ta[1], fra));
    const f3 wr = tb[1] - ta[1];
    const float4 la0 = rows[o + 21u], g19 = rows[o + 19u];
    const float g[5] = {dot(t1, vt), dot(t2, vt), dot(n, wr), dot(t1, wr), dot(t2, wr)};
    const float mu5[5] = {mu, mu, g19.x, g19.y, g19.y};
    const float l5[5] = {ly, lz, la0.x, la0.y, la0.z};
    float nl5[5], d[5];
    ell_block5(H, g, mu5, l5, pooled, S.PYRAMID == 1u, S.F_CREEP, S.F_OMEGA, nl5);
    for (uint32_t k = 0; k < 5u; k++) d[k] = nl5[k] - l5[k];
    ta[0] += (((v3(rows[o + 11u]) * d[0] + v3(rows[o + 15u]) * d[1]) + v3(rows[o + 22u]) * d[2]) + v3(rows[o + 26u]) * d[3]) + v3(rows[o + 30u]) * d[4];
    ta[1] += (((v3(rows[o + 12u]) * d[0] + v3(rows[o + 16u]) * d[1]) + v3(rows[o + 23u]) * d[2]) + v3(rows[o + 27u]) * d[3]) + v3(rows[o + 31u]) * d[4];
    tb[0] += (((v3(rows[o + 13u]) * d[0] + v3(rows[o + 17u]) * d[1]) + v3(rows[o + 24u]) * d[2]) + v3(rows[o + 28u]) * d[3]) + v3(rows[o + 32u]) * d[4];
    tb[1] += (((v3(rows[o + 14u]) * d[0] + v3(rows[o + 18u]) * d[1]) + v3(rows[o + 25u]) * d[2]) + v3(rows[o + 29u]) * d[3]) + v3(rows[o + 33u]) * d[4];
    const f3 f = t1 * d[0] + t2 * d[1];
    const f3 tq = (n * d[2] + t1 * d[3]) + t2 * d[4];
    add_imp(a, -f, (-cross(fra, f)) - tq);
    add_imp(b, f, cross(frb, f) + tq);
    rows[o + 21u] = make_float4(nl5[2], nl5[3], nl5[4], 0.0f);
    return AngOut{ta[0], ta[1], tb[0], tb[1], nl5[0], nl5[1]};
  }
  // EXT compiles the articulated angular block in (the solve kernel's EXT instance, launched for
  // batches with a scene that has it or the contact-then-internal schedule); the EXT = false kernel
  // is the plain contact loop.
  template <bool EXT>
  __device__ void solve_row(uint32_t us, uint32_t row, int a, int b, uint32_t mode, uint32_t it) const {
    const uint32_t ROWS = S.ROWS, PO = S.PO;
    float4* rows = S.rows;
    f3 ta[2], tb[2];
    load_tw(a, ta);
    load_tw(b, tb);
    uint32_t o = row * ROWS;
    float4 r0 = rows[o], r1 = rows[o + 1u], r2 = rows[o + 2u];
    f3 ra = v3(rows[o + 3u]), rb = v3(rows[o + 4u]);
    f3 n = v3(r0), t1 = v3(r1), t2 = v3(r2);
    float4 lam = rows[o + 6u];
    if (mode == 0u) {
      float dn = lam.x, dt1 = lam.y, dt2 = lam.z;
      for (uint32_t r = 0; r < 3u; r++) {
        float d = r == 0u ? dn : (r == 1u ? dt1 : dt2);
        ta[0] += v3(rows[o + 7u + r * 4u]) * d; ta[1] += v3(rows[o + 8u + r * 4u]) * d;
        tb[0] += v3(rows[o + 9u + r * 4u]) * d; tb[1] += v3(rows[o + 10u + r * 4u]) * d;
      }
      f3 fra = ra, frb = rb;
      if (S.EXTRA == 1u) { fra = v3(rows[o + PO]); frb = v3(rows[o + PO + 1u]); }
      f3 fn_ = n * dn, ft = t1 * dt1 + t2 * dt2;
      add_imp(a, -fn_ - ft, -cross(ra, fn_) - cross(fra, ft));
      add_imp(b, fn_ + ft, cross(rb, fn_) + cross(frb, ft));
    } else {
      f3 vrel = (tb[0] + cross(tb[1], rb)) - (ta[0] + cross(ta[1], ra));
      float jv = dot(n, vrel);
      float w = vpass ? 1.0f : rows[o + 5u].w;
      float res = jv + r1.w;
      if (S.COMPL == 1u) res += rows[o + S.CO].x * lam.x;
      float nl = fmx(lam.x + S.F_OMEGA * ((((-res) * r0.w) * w) - (1.0f - w) * lam.x), 0.0f);
      float dn = nl - lam.x;
      lam.x = nl;
      ta[0] += v3(rows[o + 7u]) * dn; ta[1] += v3(rows[o + 8u]) * dn;
      tb[0] += v3(rows[o + 9u]) * dn; tb[1] += v3(rows[o + 10u]) * dn;
      add_imp(a, -n * dn, -cross(ra, n * dn));
      add_imp(b, n * dn, cross(rb, n * dn));
      f3 fra = ra, frb = rb;
      float lim = r2.w * nl;
      float pooled = nl;
      f2 bias = mf2(0.0f, 0.0f);
      float role = 1.0f;
      if (S.EXTRA == 1u) {
        role = rows[o + PO].w;
        if (S.PATCH == 1u && role != 1.0f) S.art[S.A_ULOAD + us] += dn;
        fra = v3(rows[o + PO]);
        frb = v3(rows[o + PO + 1u]);
        if (S.PATCH == 1u && role == 2.0f) {
          float load = S.art[S.A_ULOAD + us];
          lim = r2.w * load;
          pooled = load;
          f3 e = v3(rows[o + PO + 2u]);
          bias = vpass ? mf2(0.0f, 0.0f) : (S.F_ANCHOR_BETA * mf2(dot(t1, e), dot(t2, e))) / P.dt;
          rows[o + PO + 2u].w = lim;
        }
      }
      if (it < S.FSTART) { lam.y = 0.0f; lam.z = 0.0f; }
      if (S.FMODE > 0u && it >= S.FSTART) {
        // Coupled (normal, t1, t2) re-solve (wgsl.js:3081-3095); overwrites all three impulses.
        const f3 vn = (tb[0] + cross(tb[1], rb)) - (ta[0] + cross(ta[1], ra));
        const f3 vt = (tb[0] + cross(tb[1], frb)) - (ta[0] + cross(ta[1], fra));
        const f3 nlam = contact_block(S.FMODE, dot(n, vn), mf2(dot(t1, vt), dot(t2, vt)), rows[o + S.FMO],
                                      rows[o + S.FMO + 1u], -r1.w, r2.w, v3(lam));
        const f3 d = nlam - v3(lam);
        if (S.PATCH == 1u && role != 1.0f) S.art[S.A_ULOAD + us] += d.x;
        ta[0] += (v3(rows[o + 7u]) * d.x + v3(rows[o + 11u]) * d.y) + v3(rows[o + 15u]) * d.z;
        ta[1] += (v3(rows[o + 8u]) * d.x + v3(rows[o + 12u]) * d.y) + v3(rows[o + 16u]) * d.z;
        tb[0] += (v3(rows[o + 9u]) * d.x + v3(rows[o + 13u]) * d.y) + v3(rows[o + 17u]) * d.z;
        tb[1] += (v3(rows[o + 10u]) * d.x + v3(rows[o + 14u]) * d.y) + v3(rows[o + 18u]) * d.z;
        const f3 fn2 = n * d.x, ft = t1 * d.y + t2 * d.z;
        add_imp(a, (-fn2) - ft, (-cross(ra, fn2)) - cross(fra, ft));
        add_imp(b, fn2 + ft, cross(rb, fn2) + cross(frb, ft));
        lam = mf4(nlam, lam.w);
      } else if (role != 0.0f && it >= S.FSTART) {
        f2 lt = mf2(0.0f, 0.0f);  // friction_pair's zero-radius exit: no tangential velocities needed
        if (!(lim <= 0.0f)) {
          f3 vr2 = (tb[0] + cross(tb[1], frb)) - (ta[0] + cross(ta[1], fra));
          float4 ki = rows[o + 5u];
          float v1 = dot(t1, vr2) + bias.x, v2_ = dot(t2, vr2) + bias.y;
          float kd = ki.x * ki.z - ki.y * ki.y;
          lt = friction_pair(ki.z / kd, -ki.y / kd, ki.x / kd, v1, v2_, lam.y, lam.z, lim, S.F_OMEGA);
        }
        float dt1 = lt.x - lam.y, dt2 = lt.y - lam.z;
        lam.y = lt.x;
        lam.z = lt.y;
        ta[0] += v3(rows[o + 11u]) * dt1 + v3(rows[o + 15u]) * dt2;
        ta[1] += v3(rows[o + 12u]) * dt1 + v3(rows[o + 16u]) * dt2;
        tb[0] += v3(rows[o + 13u]) * dt1 + v3(rows[o + 17u]) * dt2;
        tb[1] += v3(rows[o + 14u]) * dt1 + v3(rows[o + 18u]) * dt2;
        f3 f = t1 * dt1 + t2 * dt2;
        add_imp(a, -f, -cross(fra, f));
        add_imp(b, f, cross(frb, f));
      }
      // Articulated torsional/rolling (wgsl.js:3080, 3112-3140): after the sliding pair, the block
      // over sliding, spin and rolling of a contact that touches an articulation.
      const bool art_u = (a >= 0 && bkind(a) >= 2u) || (b >= 0 && bkind(b) >= 2u);
      const bool ell = EXT && S.ANG_ART == 1u && S.ANG == 1u && art_u && (rows[o + 19u].x > 0.0f || rows[o + 19u].y > 0.0f);
      if (ell && it >= S.FSTART) {
        const AngOut r = ang_block(o, a, b, n, t1, t2, fra, frb, r2.w, pooled, lam.y, lam.z, ta[0], ta[1], tb[0], tb[1]);
        ta[0] = r.ta0; ta[1] = r.ta1; tb[0] = r.tb0; tb[1] = r.tb1;
        lam.y = r.l1;
        lam.z = r.l2;
      }
      rows[o + 6u] = lam;
      if (S.ANG == 1u) {
        // Spin within mu_t * N, rolling within a disk of mu_r * N (wgsl.js:3144-3170); under
        // friction patches only the region's first anchor carries them, with the pooled load.
        const float4 g = rows[o + 19u];
        const bool aon = !ell && (S.PATCH == 0u || role == 1.0f || (role == 2.0f && rows[o + PO + 1u].w == 0.0f));
        const float nl2 = pooled;
        if (aon && (g.x > 0.0f || g.y > 0.0f)) {
          const float4 la = rows[o + 21u];
          const f3 wrel = tb[1] - ta[1];
          const float ns = clmp(la.x - dot(n, wrel) * g.z, (-g.x) * nl2, g.x * nl2);
          const float ds = ns - la.x;
          ta[0] += v3(rows[o + 22u]) * ds; ta[1] += v3(rows[o + 23u]) * ds;
          tb[0] += v3(rows[o + 24u]) * ds; tb[1] += v3(rows[o + 25u]) * ds;
          const f3 w2 = tb[1] - ta[1];
          const float4 ri = rows[o + 20u];
          const float u1 = dot(t1, w2), u2 = dot(t2, w2);
          f2 lr = mf2(la.y, la.z) - mf2(ri.x * u1 + ri.y * u2, ri.y * u1 + ri.z * u2);
          const float rl = g.y * nl2;
          if (len(lr) > rl) lr = lr * (rl / fmx(len(lr), 1e-12f));
          const float d1 = lr.x - la.y, d2 = lr.y - la.z;
          ta[0] += v3(rows[o + 26u]) * d1 + v3(rows[o + 30u]) * d2;
          ta[1] += v3(rows[o + 27u]) * d1 + v3(rows[o + 31u]) * d2;
          tb[0] += v3(rows[o + 28u]) * d1 + v3(rows[o + 32u]) * d2;
          tb[1] += v3(rows[o + 29u]) * d1 + v3(rows[o + 33u]) * d2;
          rows[o + 21u] = make_float4(ns, lr.x, lr.y, 0.0f);
          const f3 tq = (n * ds + t1 * d1) + t2 * d2;
          add_imp(a, sp3(0.0f), -tq);
          add_imp(b, sp3(0.0f), tq);
        }
      }
      if (S.TORS == 1u && row == S.sched[S.S_UTP + us]) torsion(us, a, b, it, ta, tb);
    }
    if (a >= 0) { tw[(uint32_t)a * 2u] = mf4(ta[0], 0.0f); tw[(uint32_t)a * 2u + 1u] = mf4(ta[1], 0.0f); }
    if (b >= 0) { tw[(uint32_t)b * 2u] = mf4(tb[0], 0.0f); tw[(uint32_t)b * 2u + 1u] = mf4(tb[1], 0.0f); }
  }
  template <bool EXT>
  __device__ void solve_slot(uint32_t u, uint32_t mode, uint32_t it) const {
    float4 sl = S.slots[2u * u];
    solve_row<EXT>(f2u(sl.y), f2u(sl.x), f2i(sl.z), f2i(sl.w), mode, it);
  }


  // subgroupAdd over the warp (wgsl.js:3305, subgroups on), pinned to an xor butterfly over lane
  // offsets 16, 8, 4, 2, 1. IEEE addition commutes, so every lane ends with the same bits.
  static __device__ float lane_sum(float x) {
    for (uint32_t off = 16u; off > 0u; off >>= 1u) x += __shfl_xor_sync(0xffffffffu, x, off);
    return x;
  }
  // Each articulation's dense rows in slot order (S_DSTART / S_DLIST), by a stable counting sort
  // once per solve, so the dense passes walk their own rows instead of filtering all of them (the
  // order within an articulation, the one the Gauss-Seidel pass needs, is kept). All threads of
  // one block call it (in a team launch, block 0's).
  __device__ void dense_lists(uint32_t* tmp) const {
    const uint32_t tid = threadIdx.x, nt = blockDim.x, lane = tid & 31u, warp = tid >> 5u, nw = nt >> 5u;
    const uint32_t nd = min(S.sched[S.S_META + 3u], S.MAXDENSE);
    uint32_t* start = S.sched + S.S_DSTART;
    uint32_t* off = S.sched + S.S_DOFF;
    uint32_t* list = S.sched + S.S_DLIST;
    const float* A = S.art;
    for (uint32_t a = tid; a <= S.NA; a += nt) start[a] = 0u;
    __syncthreads();
    for (uint32_t i = tid; i < nd; i += nt) atomicAdd(&start[f2u(A[S.A_DENSE + i * S.DPS])], 1u);
    __syncthreads();
    block_scan_array(start, S.NA + 1u, tmp);
    for (uint32_t a = tid; a < S.NA; a += nt) off[a] = start[a];
    __syncthreads();
    // Blocks of nt rows in order; inside one, warps in order and lanes ranked among equal ids.
    for (uint32_t c0 = 0; c0 < nd; c0 += nt) {
      const uint32_t i = c0 + tid;
      const bool v = i < nd;
      const uint32_t art = v ? f2u(A[S.A_DENSE + i * S.DPS]) : 0xffffffffu;
      const uint32_t peers = __match_any_sync(0xffffffffu, art);
      const uint32_t rank = (uint32_t)__popc(peers & ((1u << lane) - 1u));
      for (uint32_t w = 0; w < nw; w++) {
        if (warp == w && v) list[off[art] + rank] = i;
        __syncthreads();
        if (warp == w && v && lane == 31u - (uint32_t)__clz(peers)) off[art] += (uint32_t)__popc(peers);
        __syncthreads();
      }
    }
  }
  // Dense same-articulation rows of articulation a (wgsl.js:3306-3364), one warp: lane l owns
  // dofs l, l + 32, ... (so lanes never touch each other's qd entries) and its partial sums
  // are combined with lane_sum. The lanes keep their qd entries in registers for the whole pass
  // (no other warp touches a's dofs meanwhile) and store them back at the end. The rows are
  // Gauss-Seidel, one after another, but their data are not: a's rows come from its slot-ordered
  // list (dense_lists), and each lane holds its slice of a row (J and Y rows of its dofs, up to
  // DENSE_REG of them) and the row's header in registers, the next row's loaded while this one
  // is solved. Called by all 32 lanes; returns whether a row belongs to a.
  static constexpr uint32_t DENSE_REG = 2u;  // articulations of up to 64 dofs keep rows in registers
  struct DenseRow {
    float J[3][DENSE_REG], Y[3][DENSE_REG];
    float m3_, m4, m5, m6, m7, m8, nbil, m22, m23, m24;
    f3 lam;
  };
  __device__ void dense_load(uint32_t o, uint32_t lane, uint32_t nw, DenseRow& d) const {
    const float* A = S.art;
    const uint32_t NDA = S.NDA, jo = o + S.DHDR, yo = o + S.DHDR + 3u * NDA;
#pragma unroll
    for (uint32_t j = 0; j < DENSE_REG; j++) {
      uint32_t k = lane + 32u * j;
      bool v = k < nw;
#pragma unroll
      for (uint32_t r = 0; r < 3u; r++) {
        d.J[r][j] = v ? A[jo + r * NDA + k] : 0.0f;
        d.Y[r][j] = v ? A[yo + r * NDA + k] : 0.0f;
      }
    }
    d.m3_ = A[o + 3u]; d.m4 = A[o + 4u]; d.m5 = A[o + 5u]; d.m6 = A[o + 6u]; d.m7 = A[o + 7u]; d.m8 = A[o + 8u];
    d.nbil = A[o + 21u]; d.m22 = A[o + 22u]; d.m23 = A[o + 23u]; d.m24 = A[o + 24u];
    d.lam = mf3(A[o + 9u], A[o + 10u], A[o + 11u]);
  }
  __device__ bool dense(uint32_t a, uint32_t mode, uint32_t it, uint32_t ph, uint32_t lane) const {
    const uint32_t DPS = S.DPS, base0 = S.A_DENSE;
    const uint32_t nd = min(S.sched[S.S_META + 3u], S.MAXDENSE);
    const uint4 ai = ar.info(a);
    if (ai.w > 32u * DENSE_REG) return dense_wide(a, mode, it, ph, lane, nd, ai);
    const uint32_t* dl = S.sched + S.S_DLIST;
    const uint32_t k0 = S.sched[S.S_DSTART + a], k1 = S.sched[S.S_DSTART + a + 1u];
    if (k0 >= k1) return false;
    float* qg = aqd + ai.z;
    float q[DENSE_REG];
#pragma unroll
    for (uint32_t j = 0; j < DENSE_REG; j++) q[j] = lane + 32u * j < ai.w ? qg[lane + 32u * j] : 0.0f;
    uint32_t row = dl[k0];
    DenseRow cur;
    dense_load(base0 + row * DPS, lane, ai.w, cur);
    for (uint32_t k = k0; k < k1; k++) {
      const bool more = k + 1u < k1;
      const uint32_t nrow = more ? dl[k + 1u] : row;
      DenseRow nxt;
      if (more) dense_load(base0 + nrow * DPS, lane, ai.w, nxt);
      dense_row(cur, base0 + row * DPS, ai, mode, it, ph, lane, q);
      cur = nxt;
      row = nrow;
    }
    (void)nd;
#pragma unroll
    for (uint32_t j = 0; j < DENSE_REG; j++)
      if (lane + 32u * j < ai.w) qg[lane + 32u * j] = q[j];
    return true;
  }
  // One dense row (wgsl.js:3320-3362) from its registers; lane 0 stores the new impulses.
  __device__ void dense_row(const DenseRow& d, uint32_t o, uint4 ai, uint32_t mode, uint32_t it, uint32_t ph,
                            uint32_t lane, float (&q)[DENSE_REG]) const {
    float* A = S.art;
    const f3 lam = d.lam;
    if ((d.nbil > 0.5f) == (ph == 1u) && ph != 0u) return;
    if (d.nbil > 0.5f) {
      if (mode == 0u) return;
      f3 nlam = lam;
      const uint32_t nr = f2u(d.nbil);
#pragma unroll
      for (uint32_t r = 0; r < 3u; r++) {
        if (r >= nr) break;
        float part = 0.0f;
#pragma unroll
        for (uint32_t j = 0; j < DENSE_REG; j++) {
          uint32_t k = lane + 32u * j;
          if (k < ai.w) part += d.J[r][j] * q[j];
        }
        float jv = lane_sum(part);
        float rhs = vpass ? 0.0f : (r == 0u ? d.m4 : (r == 1u ? d.m22 : d.m23));
        float dl = ((-S.F_OMEGA) * (jv + rhs)) * A[o + 5u + r];
        setc(nlam, (int)r, comp(nlam, (int)r) + dl);
#pragma unroll
        for (uint32_t j = 0; j < DENSE_REG; j++) {
          uint32_t k = lane + 32u * j;
          if (k < ai.w) q[j] += d.Y[r][j] * dl;
        }
      }
      if (lane == 0u) { A[o + 9u] = nlam.x; A[o + 10u] = nlam.y; A[o + 11u] = nlam.z; }
      return;
    }
    if (mode == 0u) {
#pragma unroll
      for (uint32_t j = 0; j < DENSE_REG; j++) {
        uint32_t k = lane + 32u * j;
        if (k < ai.w) q[j] += (d.Y[0][j] * lam.x + d.Y[1][j] * lam.y) + d.Y[2][j] * lam.z;
      }
      return;
    }
    float part = 0.0f;
#pragma unroll
    for (uint32_t j = 0; j < DENSE_REG; j++) {
      uint32_t k = lane + 32u * j;
      if (k < ai.w) part += d.J[0][j] * q[j];
    }
    float jv = lane_sum(part);
    const float w = vpass ? 1.0f : d.m24;
    float nl = fmx(lam.x + S.F_OMEGA * ((((-(jv + d.m4)) * d.m5) * w) - (1.0f - w) * lam.x), 0.0f);
    float dn = nl - lam.x;
    float lim = it < S.FSTART ? 0.0f : d.m3_ * nl;
    float p1 = 0.0f, p2 = 0.0f;
#pragma unroll
    for (uint32_t j = 0; j < DENSE_REG; j++) {
      uint32_t k = lane + 32u * j;
      if (k < ai.w) {
        q[j] += d.Y[0][j] * dn;
        p1 += d.J[1][j] * q[j];
        p2 += d.J[2][j] * q[j];
      }
    }
    // friction_pair's zero-radius exit returns (0, 0) without the tangential sums (a separated or
    // unloaded contact, or before the friction iterations): skip their lane reductions.
    f2 lt = mf2(0.0f, 0.0f);
    if (!(lim <= 0.0f)) {
      float s1 = lane_sum(p1), s2 = lane_sum(p2);
      float kd = d.m6 * d.m8 - d.m7 * d.m7;
      lt = friction_pair(d.m8 / kd, -d.m7 / kd, d.m6 / kd, s1, s2, lam.y, lam.z, lim, S.F_OMEGA);
    }
    float d1 = lt.x - lam.y, d2 = lt.y - lam.z;
#pragma unroll
    for (uint32_t j = 0; j < DENSE_REG; j++) {
      uint32_t k = lane + 32u * j;
      if (k < ai.w) q[j] += d.Y[1][j] * d1 + d.Y[2][j] * d2;
    }
    if (lane == 0u) { A[o + 9u] = nl; A[o + 10u] = lt.x; A[o + 11u] = lt.y; }
  }
  // The same for articulations of more than 32 * DENSE_REG dofs, reading rows as it goes.
  __device__ bool dense_wide(uint32_t a, uint32_t mode, uint32_t it, uint32_t ph, uint32_t lane, uint32_t nd,
                             uint4 ai) const {
    const uint32_t NDA = S.NDA, DHDR = S.DHDR, DPS = S.DPS;
    float* A = S.art;
    bool touched = false;
    for (uint32_t i = 0; i < nd; i++) {
      uint32_t o = S.A_DENSE + i * DPS;
      if (f2u(A[o]) != a) continue;
      touched = true;
      uint32_t jo = o + DHDR, yo = o + DHDR + 3u * NDA;
      f3 lam = mf3(A[o + 9u], A[o + 10u], A[o + 11u]);
      if ((A[o + 21u] > 0.5f) == (ph == 1u) && ph != 0u) continue;
      if (A[o + 21u] > 0.5f) {
        if (mode == 0u) continue;
        f3 nlam = lam;
        for (uint32_t r = 0; r < f2u(A[o + 21u]); r++) {
          float part = 0.0f;
          for (uint32_t k = lane; k < ai.w; k += 32u) part += A[jo + r * NDA + k] * aqd[ai.z + k];
          float jv = lane_sum(part);
          float rhs = vpass ? 0.0f : (r == 0u ? A[o + 4u] : (r == 1u ? A[o + 22u] : A[o + 23u]));
          float dl = ((-S.F_OMEGA) * (jv + rhs)) * A[o + 5u + r];
          setc(nlam, (int)r, comp(nlam, (int)r) + dl);
          for (uint32_t k = lane; k < ai.w; k += 32u) aqd[ai.z + k] += A[yo + r * NDA + k] * dl;
        }
        if (lane == 0u) { A[o + 9u] = nlam.x; A[o + 10u] = nlam.y; A[o + 11u] = nlam.z; }
        continue;
      }
      if (mode == 0u) {
        for (uint32_t k = lane; k < ai.w; k += 32u)
          aqd[ai.z + k] += (A[yo + k] * lam.x + A[yo + NDA + k] * lam.y) + A[yo + 2u * NDA + k] * lam.z;
        continue;
      }
      float part = 0.0f;
      for (uint32_t k = lane; k < ai.w; k += 32u) part += A[jo + k] * aqd[ai.z + k];
      float jv = lane_sum(part);
      float w = vpass ? 1.0f : A[o + 24u];
      float nl = fmx(lam.x + S.F_OMEGA * ((((-(jv + A[o + 4u])) * A[o + 5u]) * w) - (1.0f - w) * lam.x), 0.0f);
      float dn = nl - lam.x;
      float lim = it < S.FSTART ? 0.0f : A[o + 3u] * nl;
      float p1 = 0.0f, p2 = 0.0f;
      for (uint32_t k = lane; k < ai.w; k += 32u) {
        aqd[ai.z + k] += A[yo + k] * dn;
        p1 += A[jo + NDA + k] * aqd[ai.z + k];
        p2 += A[jo + 2u * NDA + k] * aqd[ai.z + k];
      }
      f2 lt = mf2(0.0f, 0.0f);
      if (!(lim <= 0.0f)) {  // friction_pair's zero-radius exit, as in dense_row
        float s1 = lane_sum(p1), s2 = lane_sum(p2);
        float kd = A[o + 6u] * A[o + 8u] - A[o + 7u] * A[o + 7u];
        lt = friction_pair(A[o + 8u] / kd, -A[o + 7u] / kd, A[o + 6u] / kd, s1, s2, lam.y, lam.z, lim, S.F_OMEGA);
      }
      float d1 = lt.x - lam.y, d2 = lt.y - lam.z;
      for (uint32_t k = lane; k < ai.w; k += 32u) aqd[ai.z + k] += A[yo + NDA + k] * d1 + A[yo + 2u * NDA + k] * d2;
      if (lane == 0u) { A[o + 9u] = nl; A[o + 10u] = lt.x; A[o + 11u] = lt.y; }
    }
    return touched;
  }
  // Exact articulation update from the contact impulses on its links (wgsl.js:3380-3394).
  __device__ void contact_impulses(uint32_t a) const {
    uint4 ai = ar.info(a);
    bool hit = false;
    for (uint32_t k = 0; k < ai.y; k++) {
      uint32_t l = ai.x + k;
      uint32_t b = (uint32_t)ar.lbody(l);
      f3 f = v3(imp[b * 2u]), t = v3(imp[b * 2u + 1u]);
      if (nonzero(f) || nonzero(t)) {
        hit = true;
        ar.stsv(ar.lo(l) + L_P, SVec{-t, -f});
        imp[b * 2u] = make_float4(0, 0, 0, 0);
        imp[b * 2u + 1u] = make_float4(0, 0, 0, 0);
      }
    }
    if (hit) ar.apply(a, aqd, tw);
  }
  // Joint friction and limit rows over the dofs listed in prepare (wgsl.js:3404-3468).
  __device__ void joint_rows(uint32_t a) const {
    float* A = S.art;
    uint4 ai = ar.info(a);
    uint32_t n = f2u(A[S.A_RLN + a]);
    for (uint32_t i = 0; i < n; i++) {
      uint32_t d = f2u(A[S.A_RL + ai.z + i]);
      uint32_t l = f2u(ar.dof_limit(d).w);
      uint32_t r = d - ar.ldof(l);
      float hinv = fmx(A[S.A_HINV + d], 1e-12f);
      const float4 dr = ar.dof_drive(d);
      // drive_mode="rows" (wgsl.js:3425-3438): a PhysX-style drive row, cold-started each substep,
      // no relaxation; in the velocity pass only when velocity drives are active.
      if (S.DRIVE_ROWS == 1u && (dr.y > 0.0f || dr.z > 0.0f) && !(vpass && S.VEL_DRIVE_ACTIVE == 0u)) {
        float q = A[S.A_Q + ar.lqs(l) + r];
        float pd = 0.0f;
        if (vpass) pd = P.dt * A[S.A_SNAP + S.NB * 8u + d];
        float ca = P.dt * (P.dt * dr.y + dr.z);
        float x = 1.0f / (1.0f + ca * hinv);
        float bias = ((x * P.dt) * dr.z) * A[S.A_TGTV + d] + ((dr.y * x) * P.dt) * ((A[S.A_TGT + d] - q) - pd);
        float mx = dr.w > 0.0f ? dr.w * P.dt : 1e20f;
        float lam = A[S.A_DRV + d];
        float nl = clmp((lam * (1.0f - x) - (x * ca) * aqd[d]) + bias, -mx, mx);
        if (nl != lam) { A[S.A_DRV + d] = nl; ar.LB[ar.lo(l) + L_TAU + r] = nl - lam; ar.apply(a, aqd, tw); }
      }
      float fr = ar.dof_passive(d).y;
      if (S.JFL == 1u) fr += A[S.A_JFL + d];
      if (fr > 0.0f) {
        float lam = A[S.A_FRIC + d];
        float nl = clmp(lam - (S.F_OMEGA * aqd[d]) / hinv, -fr * P.dt, fr * P.dt);
        if (nl != lam) { A[S.A_FRIC + d] = nl; ar.LB[ar.lo(l) + L_TAU + r] = nl - lam; ar.apply(a, aqd, tw); }
      }
      float4 lim = ar.dof_limit(d);
      if (A[S.A_LG + d] > 0.5f) {
        float q = A[S.A_Q + ar.lqs(l) + r];
        for (uint32_t side = 0; side < 2u; side++) {
          float sg = side == 0u ? 1.0f : -1.0f;
          float gap = side == 0u ? q - lim.x : lim.y - q;
          float lam = A[S.A_LIM + 2u * d + side];
          float rhs = gap / P.dt;
          if (gap < 0.0f) rhs = vpass ? 0.0f : fmx((P.beta * gap) / P.dt, -P.max_depen);
          float nl = fmx(lam - (S.F_OMEGA * (sg * aqd[d] + rhs)) / hinv, 0.0f);
          if (nl == lam) continue;
          A[S.A_LIM + 2u * d + side] = nl;
          ar.LB[ar.lo(l) + L_TAU + r] = sg * (nl - lam);
          ar.apply(a, aqd, tw);
        }
      }
    }
  }
  // Joint velocity limits after the contact impulses (wgsl.js:3413-3419, 3462-3467): a stateless
  // push back onto |qd| <= limit for the marked dofs of revolute, prismatic and D6 links.
  __device__ void vlim_rows(uint32_t a) const {
    float* A = S.art;
    if (A[S.A_AVL + a] <= 0.5f) return;
    uint4 ai = ar.info(a);
    for (uint32_t k = 0; k < ai.y; k++) {
      uint32_t l = ai.x + k, t = ar.ltype(l);
      if (t != 1u && t != 0u && t != 6u) continue;
      for (uint32_t r = 0; r < ar.lndof(l); r++) {
        uint32_t d = ar.ldof(l) + r;
        float hinv = fmx(A[S.A_HINV + d], 1e-12f);
        float4 pv = ar.dof_passive(d);
        if (pv.z >= 0.0f && A[S.A_VLG + d] > 0.5f) {
          float over = aqd[d] - clmp(aqd[d], -pv.z, pv.z);
          if (over != 0.0f) { ar.LB[ar.lo(l) + L_TAU + r] = (-over) / hinv; ar.apply(a, aqd, tw); }
        }
      }
    }
  }
  // Displacement of world point x under body b's motion this substep (wgsl.js:3472-3489).
  __device__ f3 body_motion(int b, f3 x) const {
    if (b < 0) return sp3(0.0f);
    f3 p0 = v3(S.ppos[b]), p1 = v3(S.pos[b]);
    float4 q0 = S.prot[b], q1 = S.rot[b];
    float4 r = qmul(q1, qconj(q0));
    if (r.w < 0.0f) r = neg4(r);
    float sn = len(v3(r));
    f3 ang = 2.0f * v3(r);
    f3 trv = p1 - p0;
    f3 lin = trv;
    if (sn > 1e-6f) {
      float half = fatan2(sn, r.w);
      f3 axis = v3(r) / sn;
      ang = (2.0f * half) * axis;
      float scv = (half * r.w) / sn;
      lin = scv * trv + ((1.0f - scv) * dot(axis, trv)) * axis;
    }
    return lin + cross(ang, x - 0.5f * (p0 + p1));
  }

  // Dense rows of every articulation, one warp each, then the twists of the articulations they
  // moved (wgsl.js:3366-3377). Articulations share no qd, rows or links, so each warp goes on to
  // its next articulation without a block barrier.
  __device__ void dense_phase(uint32_t mode, uint32_t it, uint32_t ph) const {
    const uint32_t lane = threadIdx.x & 31u, warp = tm.rank() >> 5u, nw = tm.size() >> 5u;
    for (uint32_t a = warp; a < S.NA; a += nw) {
      bool touched = dense(a, mode, it, ph, lane);
      __syncwarp();
      if (touched) ar.twists_warp(a, aqd, tw, lane);
      __syncwarp();
    }
    tm.sync();
  }
  // nesterov_momentum (wgsl.js:3491-3557): MuJoCo's PGS acceleration on the contact rows. Each
  // row's impulse is extrapolated by beta along its change since the last extrapolation, and the
  // change e = y - lam reaches the twists and link impulses through the row's own response, as a
  // sweep update would. rows[o + MO] keeps lam at the last extrapolation, rows[o + MO + 1] keeps e.
  __device__ void momentum_unit(uint32_t us, uint32_t row, float beta, bool init) const {
    float4* R = S.rows + (size_t)row * S.ROWS;
    const uint32_t MO = S.MO;
    const float4 lam = R[6];
    if (init) {
      R[MO] = mf4(v3(lam), 0.0f);
      R[MO + 1u] = make_float4(0, 0, 0, 0);
      return;
    }
    f3 y = v3(lam) + beta * (v3(lam) - v3(R[MO]));
    f3 e = y - v3(lam);
    R[MO] = mf4(v3(lam), 0.0f);
    R[MO + 1u] = mf4(e, 0.0f);
    if (e.x == 0.0f && e.y == 0.0f && e.z == 0.0f) return;
    R[6] = mf4(y, lam.w);
    uint32_t key = S.sched[S.S_UKEY + us];
    int a = (int)(key & 0xffffu) - 1, b = (int)(key >> 16u) - 1;
    f3 ta[2], tb[2];
    load_tw(a, ta);
    load_tw(b, tb);
    ta[0] = ta[0] + ((v3(R[7]) * e.x + v3(R[11]) * e.y) + v3(R[15]) * e.z);
    ta[1] = ta[1] + ((v3(R[8]) * e.x + v3(R[12]) * e.y) + v3(R[16]) * e.z);
    tb[0] = tb[0] + ((v3(R[9]) * e.x + v3(R[13]) * e.y) + v3(R[17]) * e.z);
    tb[1] = tb[1] + ((v3(R[10]) * e.x + v3(R[14]) * e.y) + v3(R[18]) * e.z);
    f3 ra = v3(R[3]), rb = v3(R[4]);
    f3 fa = ra, fb = rb;
    if (S.EXTRA == 1u) { fa = v3(R[S.PO]); fb = v3(R[S.PO + 1u]); }
    f3 fn = v3(R[0]) * e.x;
    f3 ft = v3(R[1]) * e.y + v3(R[2]) * e.z;
    add_imp(a, (-fn) - ft, (-cross(ra, fn)) - cross(fa, ft));
    add_imp(b, fn + ft, cross(rb, fn) + cross(fb, ft));
    if (a >= 0) { tw[(uint32_t)a * 2u] = mf4(ta[0], 0.0f); tw[(uint32_t)a * 2u + 1u] = mf4(ta[1], 0.0f); }
    if (b >= 0) { tw[(uint32_t)b * 2u] = mf4(tb[0], 0.0f); tw[(uint32_t)b * 2u + 1u] = mf4(tb[1], 0.0f); }
  }
  // One momentum step before a position sweep (wgsl.js:3528-3557), with the O'Donoghue-Candes
  // restart when the last sweep's correction opposed its extrapolation or friction switches on.
  // The restart test keeps the reference's sum: partials of its 256-invocation solve workgroup
  // (wgsl.js:2503), each over rows t, t + 256, ..., added in invocation order by one thread; each
  // thread of this block computes the partials of invocations tid and tid + 128.
  __device__ void momentum_step(uint32_t ncol, uint32_t it, const uint32_t* wcs) const {
    const uint32_t tid = threadIdx.x, nt = blockDim.x;
    constexpr uint32_t WGS = 256u;
    __shared__ float wred[WGS];
    __shared__ float wmom[2];  // (k, beta), carried across the iterations of one solve
    if (it > 0u) {
      const uint32_t nrows = wcs[S.NCOL + 1u];
      for (uint32_t t = tid; t < WGS; t += nt) {
        float part = 0.0f;
        for (uint32_t u = t; u < nrows; u += WGS) {
          const float4* R = S.rows + (size_t)S.sched[S.S_PORD + u] * S.ROWS;
          f3 e = v3(R[S.MO + 1u]);
          part += dot((v3(R[6]) - v3(R[S.MO])) - e, e);
        }
        wred[t] = part;
      }
      __syncthreads();
      if (tid == 0u) {
        float total = 0.0f;
        for (uint32_t i = 0; i < WGS; i++) total += wred[i];
        float k = (total < 0.0f || it == S.FSTART) ? 0.0f : wmom[0] + 1.0f;
        wmom[0] = k;
        wmom[1] = k > 1.0f ? (k - 1.0f) / (k + 2.0f) : 0.0f;
      }
    } else if (tid == 0u) {
      wmom[0] = 0.0f;
      wmom[1] = 0.0f;
    }
    __syncthreads();
    const float beta = wmom[1];
    for (uint32_t c = 0; c < ncol; c++) {
      for (uint32_t u = wcs[c] + tid; u < wcs[c + 1u]; u += nt) {
        uint32_t row = S.sched[S.S_PORD + u];
        momentum_unit(S.sched[S.S_RUNIT + row], row, beta, it == 0u);
      }
      __syncthreads();
    }
    if (tid == 0u)
      for (uint32_t u = wcs[S.NCOL]; u < wcs[S.NCOL + 1u]; u++) {
        uint32_t row = S.sched[S.S_PORD + u];
        momentum_unit(S.sched[S.S_RUNIT + row], row, beta, it == 0u);
      }
    __syncthreads();
    for (uint32_t a = tid; a < S.NA; a += nt) {
      contact_impulses(a);
      if (S.VLIM_ON == 1u) vlim_rows(a);
    }
    __syncthreads();
  }
  // One sweep (wgsl.js:3559-3611).
  template <bool EXT>
  // ph: 0 every row; 1 contacts only (no joint-internal rows, no velocity-limit rows, no internal
  // dense rows); 2 joint-internal rows only (no contact slots, no contact dense rows). The two
  // partial sweeps serve row_schedule "contact_then_internal" (wgsl.js:3559-3590).
  __device__ void sweep(uint32_t mode, uint32_t ncol0, uint32_t it, const uint32_t* wcs, uint32_t nu, uint32_t ph) const {
    const uint32_t tid = tm.rank(), nt = tm.size();
    const uint32_t ncol = ph == 2u ? 0u : ncol0;
    if (ph != 1u)
      for (uint32_t a = tid; a < S.NA; a += nt) joint_rows(a);
    if (S.PATCH == 1u && mode == 1u) {
      // Four units per thread at a time, their loads issued together (each unit's sum keeps its
      // row order).
      constexpr uint32_t UL = 4u;
      for (uint32_t us0 = tid; us0 < nu; us0 += UL * nt) {
        uint32_t s0[UL], n[UL];
#pragma unroll
        for (uint32_t k = 0; k < UL; k++) {
          const uint32_t us = us0 + k * nt;
          s0[k] = us < nu ? S.sched[S.S_USTART + us] : 0u;
          n[k] = us < nu ? S.sched[S.S_USIZE + us] : 0u;
        }
        float load[UL];
#pragma unroll
        for (uint32_t k = 0; k < UL; k++) {
          load[k] = 0.0f;
          for (uint32_t m = s0[k]; m < s0[k] + n[k]; m++)
            if (S.rows[m * S.ROWS + S.PO].w != 1.0f) load[k] += S.rows[m * S.ROWS + 6u].x;
        }
#pragma unroll
        for (uint32_t k = 0; k < UL; k++)
          if (us0 + k * nt < nu) S.art[S.A_ULOAD + us0 + k * nt] = load[k];
      }
    }
    tm.sync();
    dense_phase(1u, it, ph);
    for (uint32_t c = 0; c < ncol; c++) {
      for (uint32_t u = wcs[c] + tid; u < wcs[c + 1u]; u += nt) solve_slot<EXT>(u, mode, it);
      tm.sync();
    }
    if (tid == 0u && ph != 2u)
      for (uint32_t u = wcs[S.NCOL]; u < wcs[S.NCOL + 1u]; u++) solve_slot<EXT>(u, mode, it);
    tm.sync();
    for (uint32_t a = tid; a < S.NA; a += nt) {
      contact_impulses(a);
      if (S.VLIM_ON == 1u && ph != 1u) vlim_rows(a);
    }
    tm.sync();
    if (S.VLIM_FREE == 1u) {
      for (uint32_t b = tid; b < S.NB; b += nt) {
        if (bkind((int)b) != 1u || (bflags((int)b) & 1u) != 0u) continue;
        RO<float4> o = S.sf + S.SF_BODY + b * 8u;
        float limv = o[4].w, lima = o[5].w;
        uint32_t g = S.A_VLG + S.ND + b * 6u;
        if (limv > 0.0f) {
          f3 v = v3(tw[b * 2u]);
          for (int k = 0; k < 3; k++) if (S.art[g + k] > 0.5f) setc(v, k, clmp(comp(v, k), -limv, limv));
          tw[b * 2u] = mf4(v, 0.0f);
        }
        if (lima > 0.0f) {
          f3 w = v3(tw[b * 2u + 1u]);
          for (int k = 0; k < 3; k++) {
            float over = comp(w, k) - clmp(comp(w, k), -lima, lima);
            if (over == 0.0f || S.art[g + 3u + k] < 0.5f) continue;
            f3 e = sp3(0.0f);
            setc(e, k, 1.0f);
            m3 R = qmat(S.rot[b]);
            f3 iw = mul(R, mul(binv_inertia((int)b), mul(tr(R), e)));
            w -= iw * (over / comp(iw, k));
          }
          tw[b * 2u + 1u] = mf4(w, 0.0f);
        }
      }
      tm.sync();
    }
  }
  __device__ float4 warm_value(uint32_t i, uint32_t nc) const {
    if (i < nc) {
      uint32_t o = i * S.ROWS;
      float4 lam = S.rows[o + 6u];
      return mf4(lam.x, v3(S.rows[o + 1u]) * lam.y + v3(S.rows[o + 2u]) * lam.z);
    }
    uint32_t o = S.A_DENSE + (i - nc) * S.DPS;
    return mf4(S.art[o + 9u], ar.ald3(o + 12u) * S.art[o + 10u] + ar.ald3(o + 15u) * S.art[o + 11u]);
  }
  __device__ uint32_t warm_rank(uint32_t i, uint32_t nc) const {
    return min(__float_as_uint(fmx(warm_value(i, nc).x, 0.0f)), 0xfffffffeu) + 1u;
  }
  __device__ uint32_t warm_key(uint32_t i, uint32_t nc) const {
    if (i < nc) { uint32_t o = i * S.ROWS; return f2u(S.rows[o + 3u].w) | (f2u(S.rows[o + 4u].w) << 16u); }
    uint32_t o = S.A_DENSE + (i - nc) * S.DPS;
    if (S.art[o + 21u] > 0.5f) return 0xffffffffu;
    return f2u(S.art[o + 1u]) | (f2u(S.art[o + 2u]) << 16u);
  }
};

// Solve of scene sc by a team (all its threads): the calling block (TEAM false, the batched path),
// or every block of a cooperative launch on a batch of one large scene (TEAM true). A team launch
// stages nothing in shared memory: twists, impulses, qd and link blocks stay in global memory,
// where every block sees them after a grid barrier. Each block keeps its own copy of the scene
// descriptor, the parameters and the color starts.
template <bool EXT, bool TEAM>
__device__ __forceinline__ void solve_scene(const BatchDev& B, uint32_t sc, Team<TEAM> tm) {
  extern __shared__ float4 ssm4[];  // solve_smem_layout: [tw | imp], qd, color starts, link blocks
  __shared__ Params Ps;
  __shared__ SceneDev Ss;  // the scene's offsets and sizes, read everywhere in the serial passes
  const uint32_t tid = tm.rank(), nt = tm.size();
  if (B.active[sc] == 0u) return;  // not stepping in this frame (serving loop)
  copy_scene(Ss, B.scenes[sc]);
  const SceneDev& S = Ss;
  if (threadIdx.x == 0u) Ps = *S.params;
  uint8_t* sb = reinterpret_cast<uint8_t*>(ssm4);
  const uint32_t stage = TEAM ? 0u : S.stage;
  const SolveSmem lay = solve_smem_layout(stage, S.NB, S.ND, S.NCOL, S.NL);
  const bool staged_links = (stage & STAGE_LINKS) != 0u, staged_bodies = (stage & STAGE_BODIES) != 0u;
  uint32_t* wcs = reinterpret_cast<uint32_t*>(sb + lay.wcs);
  float* lb = staged_links ? reinterpret_cast<float*>(sb + lay.links) : S.art + S.A_LINK;
  const uint32_t nu = S.sched[S.S_META];
  const uint32_t ncol = min(S.sched[S.S_META + 1u], S.NCOL);
  for (uint32_t i = threadIdx.x; i < S.NCOL + 2u; i += blockDim.x) wcs[i] = S.sched[S.S_CSTART + i];
  // Link blocks into shared memory with one bulk copy (A_LINK is 16-byte aligned).
  __shared__ __align__(8) uint64_t stage_bar;
  if (staged_links && !stage_to_shared(lb, S.art + S.A_LINK, 4u * S.NL * LBLK, &stage_bar, B.wait_limit)) {
    if (threadIdx.x == 0u) atomicCAS(B.error, 0u, (uint32_t)ERR_STAGE_TIMEOUT);
    return;  // the whole block: the result above is the same in every thread
  }
  __syncthreads();
  const Params& P = Ps;
  SolverT<TEAM> sv(tm, S, P, lb, staged_bodies ? reinterpret_cast<float4*>(sb + lay.tw) : S.tw,
                   staged_bodies ? reinterpret_cast<float4*>(sb + lay.imp) : S.imp,
                   (stage & STAGE_QD) ? reinterpret_cast<float*>(sb + lay.aqd) : S.aqd);
  float* A = S.art;
  // Prologue (wgsl.js:3635-3691).
  for (uint32_t i = tid; i < S.ND; i += nt) sv.aqd[i] = A[S.A_QDH + i];
  auto asleep = [&](uint32_t n) { return S.SLEEP == 1u && A[S.A_SLP + n * 4u + 1u] > 0.5f; };
  if (S.SLEEP == 1u) {
    // Sleeping articulations start the solve at rest (wgsl.js:3640-3646). The reference zeroes
    // them with no barrier after the copy above; the zeros are its intent and are what runs here.
    tm.sync();
    for (uint32_t a = tid; a < S.NA; a += nt) {
      if (!asleep(S.NB + a)) continue;
      uint4 ai = sv.ar.info(a);
      for (uint32_t d = ai.z; d < ai.z + ai.w; d++) sv.aqd[d] = 0.0f;
    }
  }
  for (uint32_t b = tid; b < S.NB; b += nt) {
    uint32_t kind = sv.bkind((int)b);
    sv.imp[b * 2u] = make_float4(0, 0, 0, 0);
    sv.imp[b * 2u + 1u] = make_float4(0, 0, 0, 0);
    // The reference keeps twists in workgroup memory, which starts at zero in every dispatch.
    sv.tw[b * 2u] = make_float4(0, 0, 0, 0);
    sv.tw[b * 2u + 1u] = make_float4(0, 0, 0, 0);
    if (kind != 1u) continue;
    uint32_t fl = sv.bflags((int)b);
    f3 v = v3(S.lv[b]) + ((asleep(b) || fl != 0u) ? sp3(0.0f) : v3(P.gravity) * P.dt);
    f3 w = v3(S.av[b]);
    uint32_t bfo = S.A_BF + b * 8u;
    f3 bf = mf3(A[bfo], A[bfo + 1], A[bfo + 2]), bt = mf3(A[bfo + 4], A[bfo + 5], A[bfo + 6]);
    RO<float4> o = S.sf + S.SF_BODY + b * 8u;
    if ((fl & 1u) == 0u && (nonzero(bf) || nonzero(bt))) {
      m3 R = qmat(S.rot[b]);
      v += (bf * o[0].x) * P.dt;
      w += mul(R, mul(sv.binv_inertia((int)b), mul(tr(R), bt))) * P.dt;
    }
    m3 I = tr(mcols(v3(o[2]), v3(o[3]), v3(o[4])));
    bool iso = I.c[0].x == I.c[1].y && I.c[1].y == I.c[2].z && I.c[0].y == 0.0f && I.c[0].z == 0.0f && I.c[1].z == 0.0f;
    if ((fl & 1u) == 0u && !iso && nonzero(w)) {
      m3 R = qmat(S.rot[b]);
      w = mul(R, SolverT<TEAM>::gyro(I, mul(tr(R), w), P.dt));
    }
    sv.tw[b * 2u] = mf4(v, 0.0f);
    sv.tw[b * 2u + 1u] = mf4(w, 0.0f);
  }
  for (uint32_t i = tid; i < 2u * S.ND; i += nt) A[S.A_LIM + i] = 0.0f;
  for (uint32_t i = tid; i < S.ND; i += nt) { A[S.A_FRIC + i] = 0.0f; A[S.A_DRV + i] = 0.0f; }
  const uint32_t nslot = wcs[S.NCOL + 1u];
  for (uint32_t u = tid; u < nslot; u += nt) {
    uint32_t row = S.sched[S.S_PORD + u], us = S.sched[S.S_RUNIT + row], key = S.sched[S.S_UKEY + us];
    S.slots[2u * u] = make_float4((float)row, (float)us, (float)((int)(key & 0xffffu) - 1), (float)((int)(key >> 16u) - 1));
  }
  tm.sync();
  // Few articulations: a warp each (the chain recursion shortened); many: a thread each.
  if (S.NA <= (nt >> 5u)) {
    for (uint32_t a = tid >> 5u; a < S.NA; a += nt >> 5u) sv.ar.twists_warp(a, sv.aqd, sv.tw, tid & 31u);
  } else {
    for (uint32_t a = tid; a < S.NA; a += nt) sv.ar.twists(a, sv.aqd, sv.tw);
  }
  tm.sync();
  {
    // The dense lists are built by one block (the whole team's block 0), then published.
    __shared__ uint32_t dtmp[33];
    if (!TEAM || blockIdx.x == 0u) sv.dense_lists(dtmp);
    if (TEAM) tm.sync();
  }
  sv.dense_phase(0u, 0u, 0u);
  sv.sweep<EXT>(0u, ncol, 0u, wcs, nu, 0u);
  // row_schedule "contact_then_internal" (wgsl.js:3693-3696): all contact iterations (phase 1),
  // then the joint-internal rows (phase 2); otherwise one pass of full sweeps (phase 0).
  // Only the EXT instance carries it.
  const bool cti = EXT && S.CTI == 1u;
  const uint32_t npass = cti ? 2u : 1u;
  for (uint32_t pass = 0; pass < npass; pass++)
    for (uint32_t it = 0; it < P.iterations; it++) {
      // Nesterov momentum keeps block-wide sums: a team launch is never made for a scene with it.
      if (!TEAM && S.NEST == 1u && pass == 0u) sv.momentum_step(ncol, it, wcs);
      sv.sweep<EXT>(1u, ncol, it, wcs, nu, cti ? pass + 1u : 0u);
    }
  // Velocity pass (velocity_iterations, wgsl.js:3700-3736): positions integrate with the velocities
  // reached here; further bias-free sweeps from the accumulated impulses set the output velocities.
  if (S.VELITERS > 0u) {
    for (uint32_t b = tid; b < S.NB; b += nt) {
      sv.ar.ast3(S.A_SNAP + b * 8u, v3(sv.tw[b * 2u]));
      sv.ar.ast3(S.A_SNAP + b * 8u + 4u, v3(sv.tw[b * 2u + 1u]));
    }
    for (uint32_t i = tid; i < S.ND; i += nt) A[S.A_SNAP + S.NB * 8u + i] = sv.aqd[i];
    // Contact rhs without bias: 0, or a speculative gap still open at the snapshot velocity.
    for (uint32_t us = tid; us < nu; us += nt) {
      const uint32_t key = S.sched[S.S_UKEY + us];
      const int a = (int)(key & 0xffffu) - 1, b = (int)(key >> 16u) - 1;
      f3 ta[2], tb[2];
      sv.load_tw(a, ta);
      sv.load_tw(b, tb);
      const uint32_t s0 = S.sched[S.S_USTART + us];
      for (uint32_t i = s0; i < s0 + S.sched[S.S_USIZE + us]; i++) {
        float4* R = S.rows + (size_t)i * S.ROWS;
        const float phi = R[6].w;
        if (phi >= 1e29f) continue;
        const f3 n = v3(R[0]);
        const float jv = dot(n, (tb[0] + cross(tb[1], v3(R[4]))) - (ta[0] + cross(ta[1], v3(R[3]))));
        R[1].w = (phi > 0.0f && phi + P.dt * jv > 1e-6f) ? phi / P.dt : 0.0f;
      }
    }
    const uint32_t ndv = min(S.sched[S.S_META + 3u], S.MAXDENSE);
    for (uint32_t i = tid; i < ndv; i += nt) {
      const uint32_t o = S.A_DENSE + i * S.DPS;
      if (A[o + 21u] > 0.5f || A[o + 22u] >= 1e29f) continue;
      const uint4 ai = sv.ar.info(f2u(A[o]));
      float jv = 0.0f;
      for (uint32_t k = 0; k < ai.w; k++) jv += A[o + S.DHDR + k] * sv.aqd[ai.z + k];
      const float phi = A[o + 22u];
      A[o + 4u] = (phi > 0.0f && phi + P.dt * jv > 1e-6f) ? phi / P.dt : 0.0f;
    }
    tm.sync();
    sv.vpass = true;
    for (uint32_t it = 0; it < S.VELITERS; it++) sv.sweep<EXT>(1u, ncol, P.iterations + it, wcs, nu, 0u);
    sv.vpass = false;
  }
  // Warm-start table (wgsl.js:3737-3767): rows sharing a key keep the largest normal impulse.
  const uint32_t nc = S.sched[S.S_USTART + nu];
  const uint32_t ndense = min(S.sched[S.S_META + 3u], S.MAXDENSE);
  const uint32_t WH = S.WH, wbase = (1u - P.parity) * WH;
  uint32_t* wslot = S.sched + S.S_WSLOT;
  uint32_t* wwin = S.sched + S.S_WWIN;
  for (uint32_t i = tid; i < nc + ndense; i += nt) {
    uint32_t key = sv.warm_key(i, nc);
    wslot[i] = 0xffffffffu;
    if (key == 0xffffffffu) continue;
    uint32_t h = key % WH;
    for (uint32_t probe = 0; probe < 32u; probe++) {
      uint32_t old = atomicCAS(&S.warm_tab[wbase + h], 0u, key);
      if (old == 0u || old == key) { atomicMax(&wwin[h], sv.warm_rank(i, nc)); wslot[i] = h; break; }
      h = (h + 1u) % WH;
    }
  }
  tm.sync();
  for (uint32_t i = tid; i < nc + ndense; i += nt) {
    uint32_t key = sv.warm_key(i, nc);
    if (key == 0xffffffffu) continue;
    uint32_t h = wslot[i];
    if (h >= WH || S.warm_tab[wbase + h] != key || wwin[h] != sv.warm_rank(i, nc)) continue;
    float4 v = sv.warm_value(i, nc);
    uint32_t* vo = S.warm_tab + 2u * WH + (wbase + h) * 4u;
    vo[0] = __float_as_uint(v.x); vo[1] = __float_as_uint(v.y); vo[2] = __float_as_uint(v.z); vo[3] = __float_as_uint(v.w);
  }
  // Integrate (wgsl.js:3768-3828). The reference copies qd and damps the floating bases in two
  // unsynchronised loops; here the copy completes before the damping.
  if (S.PATCH == 1u) {
    for (uint32_t b = tid; b < S.NB; b += nt) { S.ppos[b] = S.pos[b]; S.prot[b] = S.rot[b]; }
    tm.sync();
  }
  for (uint32_t b = tid; b < S.NB; b += nt) {
    if (sv.bkind((int)b) != 1u) continue;
    f3 v = v3(sv.tw[b * 2u]), w = v3(sv.tw[b * 2u + 1u]);
    float damp = (sv.bflags((int)b) & 1u) != 0u ? 1.0f : 1.0f - S.sf[S.SF_BODY + b * 8u + 3u].w * P.dt;
    S.lv[b] = mf4(v, 0.0f);
    S.av[b] = mf4(w * damp, 0.0f);
    if (S.VELITERS > 0u) {
      f3 s2[2];
      sv.snap_tw((int)b, s2);
      v = s2[0];
      w = s2[1];
    }
    if (asleep(b)) {  // a sleeping body stays put at rest (wgsl.js:3779)
      S.lv[b] = make_float4(0, 0, 0, 0);
      S.av[b] = make_float4(0, 0, 0, 0);
      continue;
    }
    f3 c = v3(S.pos[b]) + v * P.dt;
    float4 q = S.rot[b];
    q = nrm4(add4(q, scale4(0.5f * P.dt, qmul(mf4(w, 0.0f), q))));
    S.pos[b] = mf4(c, 0.0f);
    S.rot[b] = q;
  }
  for (uint32_t i = tid; i < S.ND; i += nt) {
    A[S.A_QD + i] = sv.aqd[i];
    if (S.VELITERS > 0u) sv.aqd[i] = A[S.A_SNAP + S.NB * 8u + i];
  }
  tm.sync();
  for (uint32_t l = tid; l < S.NL; l += nt) {
    if (sv.ar.ltype(l) != 4u || sv.ar.lparent(l) >= 0) continue;
    float k = 1.0f - S.sf[S.SF_BODY + (uint32_t)sv.ar.lbody(l) * 8u + 3u].w * P.dt;
    uint32_t d = sv.ar.ldof(l);
    A[S.A_QD + d + 3u] *= k; A[S.A_QD + d + 4u] *= k; A[S.A_QD + d + 5u] *= k;
  }
  tm.sync();
  // Joint integration of link l (wgsl.js:3797-3826).
  auto integrate_link = [&](uint32_t l) {
    float* Q = A + S.A_Q;
    const float* aqd = sv.aqd;
    uint32_t qs = sv.ar.lqs(l), d = sv.ar.ldof(l), t = sv.ar.ltype(l);
    if (t == 1u || t == 0u || t == 6u)
      for (uint32_t r = 0; r < sv.ar.lndof(l); r++) Q[qs + r] += aqd[d + r] * P.dt;
    if (t == 2u) {
      f3 w = mf3(aqd[d], aqd[d + 1u], aqd[d + 2u]);
      float4 q = make_float4(Q[qs], Q[qs + 1], Q[qs + 2], Q[qs + 3]);
      q = nrm4(add4(q, scale4(0.5f * P.dt, qmul(mf4(w, 0.0f), q))));
      Q[qs] = q.x; Q[qs + 1] = q.y; Q[qs + 2] = q.z; Q[qs + 3] = q.w;
    }
    if (t == 4u) {
      for (uint32_t c = 0; c < 3u; c++) Q[qs + c] += aqd[d + c] * P.dt;
      f3 w = mf3(aqd[d + 3u], aqd[d + 4u], aqd[d + 5u]);
      float4 q = make_float4(Q[qs + 3], Q[qs + 4], Q[qs + 5], Q[qs + 6]);
      q = nrm4(add4(q, scale4(0.5f * P.dt, qmul(mf4(w, 0.0f), q))));
      Q[qs + 3] = q.x; Q[qs + 4] = q.y; Q[qs + 5] = q.z; Q[qs + 6] = q.w;
    }
  };
  auto store_link_pose = [&](uint32_t l) {
    uint32_t b = (uint32_t)sv.ar.lbody(l);
    S.pos[b] = mf4(sv.ar.ld3(sv.ar.lo(l) + L_COM), 0.0f);
    S.rot[b] = sv.ar.link_rot(l);
  };
  if (S.NA <= (nt >> 5u)) {
    // Few articulations: a warp each; the links' joint updates and body poses are independent,
    // the FK runs across lanes (fk_warp).
    const uint32_t lane = tid & 31u;
    for (uint32_t a = tid >> 5u; a < S.NA; a += nt >> 5u) {
      uint4 ai = sv.ar.info(a);
      for (uint32_t k = lane; k < ai.y; k += 32u) integrate_link(ai.x + k);
      __syncwarp();
      sv.ar.fk_warp(a, lane);
      for (uint32_t k = lane; k < ai.y; k += 32u) store_link_pose(ai.x + k);
      __syncwarp();
    }
  } else {
    for (uint32_t a = tid; a < S.NA; a += nt) {
      uint4 ai = sv.ar.info(a);
      for (uint32_t k = 0; k < ai.y; k++) integrate_link(ai.x + k);
      sv.ar.fk(a);
      for (uint32_t k = 0; k < ai.y; k++) store_link_pose(ai.x + k);
    }
  }
  // Friction anchors: advance and store for the next substep (wgsl.js:3832-3878).
  if (S.PATCH == 1u) {
    tm.sync();
    const uint32_t AH = S.AH, ab = 10u * WH + (1u - P.parity) * AH, AVb = 10u * WH + 2u * AH;
    const float keep_frac = (float)(1.0 - 1e-5);
    for (uint32_t i = tid; i < nc; i += nt) {
      uint32_t o = i * S.ROWS;
      const float4* rows = S.rows;
      const uint32_t PO = S.PO;
      if (rows[o + PO].w != 2.0f) continue;
      uint32_t pair = __float_as_uint(rows[o + PO + 3u].w);
      int a = (int)(pair & 0xffffu) - 1, b = (int)(pair >> 16u) - 1;
      f3 fra = v3(rows[o + PO]), frb = v3(rows[o + PO + 1u]);
      uint32_t k = f2u(rows[o + PO + 1u].w);
      float4 ex = rows[o + PO + 2u];
      float lim = ex.w;
      if (lim <= 0.0f) continue;
      f3 n = v3(rows[o]), t1 = v3(rows[o + 1u]), t2 = v3(rows[o + 2u]);
      f3 ta[2], tb[2];
      sv.load_tw(a, ta);
      sv.load_tw(b, tb);
      if (S.VELITERS > 0u) { sv.snap_tw(a, ta); sv.snap_tw(b, tb); }
      f3 vrel = (tb[0] + cross(tb[1], frb)) - (ta[0] + cross(ta[1], fra));
      float4 lam = rows[o + 6u];
      f3 lt = t1 * lam.y + t2 * lam.z;
      float r = fmx(fmn(sv.bradius(a), sv.bradius(b)), 1e-4f);
      if (len(lt) >= keep_frac * lim && dot(vrel, lt) < (((-lim) * 1e-5f) * r) / P.dt) continue;
      float4 qa = make_float4(0, 0, 0, 1);
      f3 ca = sp3(0.0f);
      if (a >= 0) { qa = S.rot[a]; ca = v3(S.pos[a]); }
      f3 ll = v3(rows[o + PO + 3u]);
      f3 x = ca + qrot(qa, ll);
      f3 e = (v3(ex) + sv.body_motion(b, x)) - sv.body_motion(a, x);
      e -= n * dot(n, e);
      f3 el = qinv(qa, e);
      uint32_t hk = max(mix32(pair * 2u + k), 1u);
      uint32_t h = hk % AH;
      for (uint32_t probe = 0; probe < 32u; probe++) {
        uint32_t old = atomicCAS(&S.warm_tab[ab + h], 0u, hk);
        if (old == 0u) {
          uint32_t* vo = S.warm_tab + AVb + ((1u - P.parity) * AH + h) * AVN_S;
          f3 il = qinv(qa, lt), nl_ = qinv(qa, n);
          vo[11] = __float_as_uint(nl_.x); vo[12] = __float_as_uint(nl_.y); vo[13] = __float_as_uint(nl_.z);
          vo[8] = __float_as_uint(il.x); vo[9] = __float_as_uint(il.y); vo[10] = __float_as_uint(il.z);
          vo[0] = pair; vo[1] = k;
          vo[2] = __float_as_uint(ll.x); vo[3] = __float_as_uint(ll.y); vo[4] = __float_as_uint(ll.z);
          vo[5] = __float_as_uint(el.x); vo[6] = __float_as_uint(el.y); vo[7] = __float_as_uint(el.z);
          break;
        }
        h = (h + 1u) % AH;
      }
    }
  }
  if (tid == 0u) {
    uint32_t* st = S.stats;
    st[1] = max(st[1], S.counters[1]);
    st[2] = max(st[2], ncol);
    st[3] = max(st[3], nu);
    st[4] = max(st[4], S.counters[0]);
    st[5] = S.counters[1];
    st[6] = ncol;
    st[7] = max(st[7], S.sched[S.S_META + 3u]);
    st[8] = S.sched[S.S_META + 5u];
    S.counters[0] = 0u;
    S.counters[1] = 0u;
  }
  if (staged_links) {
    tm.sync();
    for (uint32_t i = tid; i < S.NL * LBLK; i += nt) S.art[S.A_LINK + i] = lb[i];
  }
}

}  // namespace steel
