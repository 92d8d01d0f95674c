// Test infrastructure: the oracle's articulated torsional/rolling friction cone
// (wgsl.js:2655-2930), the angular block (t1, t2, spin, roll1, roll2) of a contact that touches an
// articulation, solved in coefficient-normalized impulses over the elliptic or pyramidal cone.
#pragma once
#include <cmath>
#include "omath.h"

namespace orc {

// Cone norm of coefficient-normalized impulses y = (t1, t2, spin, roll1, roll2): the ball (elliptic
// cone) or the sum of the group norms |(t1, t2)| + |spin| + |(roll1, roll2)| (pyramidal cone).
static inline float cone_norm5(const float* y, bool pyr) {
  if (pyr) return (std::sqrt(y[0] * y[0] + y[1] * y[1]) + std::fabs(y[2])) + std::sqrt(y[3] * y[3] + y[4] * y[4]);
  float s = 0.0f;
  for (int k = 0; k < 5; k++) s += y[k] * y[k];
  return std::sqrt(s);
}
static inline float ball_norm5(const float* y) {
  float s = 0.0f;
  for (int k = 0; k < 5; k++) s += y[k] * y[k];
  return std::sqrt(s);
}

// Projection onto the cone. Pyramid: onto sum_g w_g |y_g| <= load over the groups (t1, t2), (spin),
// (roll1, roll2) by the group soft threshold theta (the largest (partial weighted sum - load) /
// partial squared weights over the groups taken in decreasing |y_g| / w_g), then a final rescale.
static inline void cone_project5(float* y, float w0, float w1, float w2, float load, bool pyr) {
  if (!pyr) {
    const float n = ball_norm5(y);
    if (n > load) {
      const float s = load / n;
      for (int k = 0; k < 5; k++) y[k] *= s;
    }
    return;
  }
  const float w[3] = {w0, w1, w2};
  const float nm[3] = {std::sqrt(y[0] * y[0] + y[1] * y[1]), std::fabs(y[2]), std::sqrt(y[3] * y[3] + y[4] * y[4])};
  if ((w[0] * nm[0] + w[1] * nm[1]) + w[2] * nm[2] <= load) return;
  int ord[3] = {0, 1, 2};
  for (int i = 0; i < 2; i++)
    for (int j = i + 1; j < 3; j++)
      if (nm[ord[j]] * w[ord[i]] > nm[ord[i]] * w[ord[j]]) { const int t = ord[i]; ord[i] = ord[j]; ord[j] = t; }
  float theta = 0.0f, lin = 0.0f, quad = 0.0f;
  for (int i = 0; i < 3; i++) {
    const int g = ord[i];
    lin += w[g] * nm[g];
    quad += w[g] * w[g];
    theta = fmaxf_(theta, (lin - load) / quad);
  }
  float total = 0.0f;
  for (int g = 0; g < 3; g++) {
    const float sc = nm[g] > 0.0f ? fmaxf_(nm[g] - theta * w[g], 0.0f) / nm[g] : 0.0f;
    if (g == 0) { y[0] *= sc; y[1] *= sc; }
    else if (g == 1) { y[2] *= sc; }
    else { y[3] *= sc; y[4] *= sc; }
    total += (w[g] * nm[g]) * sc;
  }
  if (total > load) {
    const float s = load / total;
    for (int k = 0; k < 5; k++) y[k] *= s;
  }
}

static inline bool live5(const float* H, const bool* act, int k) { return act[k] && H[k * 5 + k] > 0.0f; }

// Cholesky L L' = H + alpha I over the live rows (dead rows get a unit pivot); false when a pivot
// is not above 1e-6 of its diagonal.
static inline bool factor5(const float* H, const bool* act, float alpha, float* L) {
  for (int k = 0; k < 5; k++) {
    const bool lk = live5(H, act, k);
    for (int l = 0; l <= k; l++) {
      float v = (lk && live5(H, act, l)) ? H[k * 5 + l] : 0.0f;
      if (k == l) v = lk ? v + alpha : 1.0f;
      for (int m = 0; m < l; m++) v -= L[k * 5 + m] * L[l * 5 + m];
      if (k == l) {
        const float ref = lk ? H[k * 5 + k] + alpha : 1.0f;
        if (!(v > 1e-6f * ref)) return false;
        L[k * 5 + k] = std::sqrt(v);
      } else {
        L[k * 5 + l] = v / L[l * 5 + l];
      }
    }
  }
  return true;
}
static inline void lower5(const float* L, float* x) {
  for (int k = 0; k < 5; k++) {
    for (int m = 0; m < k; m++) x[k] -= L[k * 5 + m] * x[m];
    x[k] /= L[k * 5 + k];
  }
}
static inline void upper5(const float* L, float* x) {
  for (int k = 4; k >= 0; k--) {
    for (int m = k + 1; m < 5; m++) x[k] -= L[m * 5 + k] * x[m];
    x[k] /= L[k * 5 + k];
  }
}

struct Ball5 {
  float y[5];
  bool ok, interior;
};

// Trust-region step y = -(H + alpha I)^-1 c on the ball |y| <= load (More-Sorensen): alpha by a
// safeguarded Newton iteration on 1 / |y(alpha)| inside the bracket [lo, hi], starting at 0
// (an interior minimizer ends it). ok when |y| met the boundary to 1e-5 or the minimizer is inside.
static Ball5 cholesky_ball5(const float* H, const float* c, const bool* act, float load) {
  Ball5 r;
  float b[5], L[25];
  float cn = 0.0f;
  for (int k = 0; k < 5; k++) {
    b[k] = live5(H, act, k) ? c[k] : 0.0f;
    cn += b[k] * b[k];
    r.y[k] = 0.0f;
  }
  cn = std::sqrt(cn);
  r.interior = !(cn > 0.0f);
  r.ok = true;
  if (!(load > 0.0f && cn > 0.0f)) return r;
  r.ok = false;
  float lo = 0.0f, hi = cn / load, alpha = 0.0f;
  for (int it = 0; it < 40; it++) {
    float nx = -1.0f;
    if (factor5(H, act, alpha, L)) {
      for (int k = 0; k < 5; k++) r.y[k] = -b[k];
      lower5(L, r.y);
      upper5(L, r.y);
      const float n = ball_norm5(r.y);
      if (alpha == 0.0f && n <= load) {
        r.interior = true;
        r.ok = true;
        return r;
      }
      if (std::fabs(n - load) <= 1e-5f * load) {
        r.ok = true;
        break;
      }
      if (n < load) hi = alpha;
      else lo = alpha;
      float w[5];
      for (int k = 0; k < 5; k++) w[k] = r.y[k];
      lower5(L, w);
      float wn = 0.0f;
      for (int k = 0; k < 5; k++) wn += w[k] * w[k];
      nx = alpha + (((n * n) / wn) * (n - load)) / load;
    } else {
      lo = alpha;
    }
    if (hi - lo <= 1e-4f * hi) break;
    alpha = (nx > lo && nx < hi) ? nx : (lo > 0.0f ? std::sqrt(lo * hi) : 1e-3f * hi);
  }
  const float n = ball_norm5(r.y);
  if (n > load) {
    const float s = load / n;
    for (int k = 0; k < 5; k++) r.y[k] *= s;
  }
  return r;
}

// The ball step; when dependent rows defeat the factorization, a proximal term
// 0.5 rho (y - center / scale)' diag(H) (y - center / scale) with rho = 1e-5, raised tenfold up to
// seven times, until the ball step converges to a finite answer.
static Ball5 trust_region5(const float* H, const float* c, const bool* act, float load, const float* center,
                          const float* scale) {
  const Ball5 first = cholesky_ball5(H, c, act, load);
  if (first.ok) return first;
  float ce[5];
  for (int k = 0; k < 5; k++) ce[k] = (act[k] && scale[k] > 0.0f) ? center[k] / scale[k] : 0.0f;
  float rho = 1e-5f;
  for (int it = 0; it < 7; it++) {
    float K[25], g[5];
    for (int k = 0; k < 25; k++) K[k] = H[k];
    for (int k = 0; k < 5; k++) {
      const float wt = live5(H, act, k) ? rho * H[k * 5 + k] : 0.0f;
      K[k * 5 + k] += wt;
      g[k] = c[k] - wt * ce[k];
    }
    rho *= 10.0f;
    const Ball5 t = cholesky_ball5(K, g, act, load);
    if (!t.ok) continue;
    bool fin = true;
    for (int k = 0; k < 5; k++) fin = fin && std::fabs(t.y[k]) < 3.0e38f;
    if (fin) return t;
  }
  return first;
}

// Pyramid face: accelerated projected gradient (FISTA with restart on ascent, step 1 / the largest
// live absolute row sum) from y0, in coordinates scaled per group by the root of the group's
// largest live diagonal; at most 64 steps, stopping at a group residual of 1e-5 load.
static void pyr_descend5(const float* H, const float* c, const bool* act, float load, const float* y0, float* y) {
  float s[5], w[3];
  for (int g = 0; g < 3; g++) {
    const int f = g == 0 ? 0 : (g == 1 ? 2 : 3), n = g == 1 ? 1 : 2;
    float cv = 0.0f;
    for (int k = f; k < f + n; k++) cv = fmaxf_(cv, act[k] ? H[k * 5 + k] : 0.0f);
    const float sc = cv > 0.0f ? std::sqrt(cv) : 1.0f;
    w[g] = 1.0f / sc;
    for (int k = f; k < f + n; k++) s[k] = sc;
  }
  float Hu[25], cu[5], u[5], z[5];
  float lip = 0.0f;
  for (int k = 0; k < 5; k++) {
    float rs = 0.0f;
    for (int l = 0; l < 5; l++) {
      Hu[k * 5 + l] = H[k * 5 + l] / (s[k] * s[l]);
      rs += std::fabs(Hu[k * 5 + l]);
    }
    lip = fmaxf_(lip, act[k] ? rs : 0.0f);
    cu[k] = c[k] / s[k];
    u[k] = y0[k] * s[k];
  }
  cone_project5(u, w[0], w[1], w[2], load, true);
  for (int k = 0; k < 5; k++) z[k] = u[k];
  float mom = 1.0f;
  for (int it = 0; it < 64 && lip > 0.0f; it++) {
    float nx[5];
    for (int k = 0; k < 5; k++) {
      float gr = cu[k];
      for (int l = 0; l < 5; l++) gr += Hu[k * 5 + l] * z[l];
      nx[k] = act[k] ? z[k] - gr / lip : 0.0f;
    }
    cone_project5(nx, w[0], w[1], w[2], load, true);
    const float e0 = nx[0] - z[0], e1 = nx[1] - z[1], e3 = nx[3] - z[3], e4 = nx[4] - z[4];
    const float r0 = std::sqrt(e0 * e0 + e1 * e1) * w[0];
    const float r1 = std::fabs(nx[2] - z[2]) * w[1];
    const float r2 = std::sqrt(e3 * e3 + e4 * e4) * w[2];
    const float res = fmaxf_(r0, fmaxf_(r1, r2));
    float asc = 0.0f;
    for (int k = 0; k < 5; k++) asc += (z[k] - nx[k]) * (nx[k] - u[k]);
    if (asc > 0.0f) mom = 1.0f;
    const float nm = 0.5f * (1.0f + std::sqrt(1.0f + (4.0f * mom) * mom));
    const float bl = (mom - 1.0f) / nm;
    for (int k = 0; k < 5; k++) {
      z[k] = nx[k] + bl * (nx[k] - u[k]);
      u[k] = nx[k];
    }
    mom = nm;
    if (res <= 1e-5f * load) break;
  }
  for (int k = 0; k < 5; k++) y[k] = u[k] / s[k];
}

// One visit of an articulated contact's angular block (t1, t2, spin, roll1, roll2): H0 the rows'
// 5x5 response, g0 their velocity residual, mu_in the row coefficients, lam the current impulses,
// load_in the normal load. Creep compliance F_CREEP / (mu^2 load) softens the three angular rows;
// the minimizer over the cone in y = lambda / mu (stick when the ball step is interior), relaxed by
// omega, is reached by an exact line search from the current impulses moved into the cone.
static void ell_block5(const float* H0, const float* g0, const float* mu_in, const float* lam, float load_in, bool pyr,
                      float creep, float omega, float* out) {
  const float load = fmaxf_(load_in, 0.0f);
  float mu[5], H[25], gr[5];
  for (int k = 0; k < 25; k++) H[k] = H0[k];
  for (int k = 0; k < 5; k++) gr[k] = g0[k];
  float big = 0.0f;
  for (int k = 0; k < 5; k++) {
    mu[k] = fmaxf_(mu_in[k], 0.0f);
    big = fmaxf_(big, H[k * 5 + k]);
  }
  bool act[5];
  float comp[5];
  for (int k = 0; k < 5; k++) {
    act[k] = mu[k] > 0.0f && H[k * 5 + k] > 1e-12f * big;
    comp[k] = (k >= 2 && act[k] && load > 0.0f) ? creep / ((mu[k] * mu[k]) * load) : 0.0f;
    H[k * 5 + k] += comp[k];
    gr[k] += comp[k] * lam[k];
  }
  float y0[5], c[5], y[5];
  for (int k = 0; k < 5; k++) {
    y0[k] = act[k] ? lam[k] / mu[k] : 0.0f;
    gr[k] = act[k] ? gr[k] * mu[k] : 0.0f;
    for (int l = 0; l < 5; l++) H[k * 5 + l] *= mu[k] * mu[l];
  }
  for (int k = 0; k < 5; k++) {
    float v = gr[k];
    for (int l = 0; l < 5; l++) v -= H[k * 5 + l] * y0[l];
    c[k] = act[k] ? v : 0.0f;
  }
  const Ball5 tr = trust_region5(H, c, act, load, lam, mu_in);
  for (int k = 0; k < 5; k++) y[k] = tr.y[k];
  const bool stick = tr.interior && cone_norm5(y, pyr) <= load;
  if (!stick) {
    if (pyr) {
      // On the face, sum_g |y_g| <= load equals sum_g |y_g|^2 / t_g <= load^2 at t_g = |y_g| / sum |y|;
      // alternating the weighted ball step with that t converges to the face optimum.
      pyr_descend5(H, c, act, load, y0, y);
      for (int it = 0; it < 8; it++) {
        const float n0 = std::sqrt(y[0] * y[0] + y[1] * y[1]), n1 = std::fabs(y[2]), n2 = std::sqrt(y[3] * y[3] + y[4] * y[4]);
        const float tot = (n0 + n1) + n2;
        if (!(tot > 0.0f)) break;
        const float q0 = std::sqrt(n0 / tot), q1 = std::sqrt(n1 / tot), q2 = std::sqrt(n2 / tot);
        const float r[5] = {q0, q0, q1, q2, q2};
        float cr[5], Hu[25];
        for (int k = 0; k < 5; k++) {
          cr[k] = r[k] * c[k];
          for (int l = 0; l < 5; l++) Hu[k * 5 + l] = (r[k] * r[l]) * H[k * 5 + l];
        }
        const Ball5 t = trust_region5(Hu, cr, act, load, y, r);
        for (int k = 0; k < 5; k++) y[k] = t.y[k] * r[k];
      }
    }
    cone_project5(y, 1.0f, 1.0f, 1.0f, load, pyr);
  }
  float stp[5], shift[5];
  for (int k = 0; k < 5; k++) stp[k] = lam[k] + omega * (mu[k] * y[k] - lam[k]);
  if (omega != 1.0f) {
    for (int k = 0; k < 5; k++) y[k] = act[k] ? stp[k] / mu_in[k] : 0.0f;
    cone_project5(y, 1.0f, 1.0f, 1.0f, load, pyr);
    for (int k = 0; k < 5; k++) stp[k] = mu[k] * y[k];
  }
  for (int k = 0; k < 5; k++) y[k] = act[k] ? lam[k] / mu_in[k] : 0.0f;
  cone_project5(y, 1.0f, 1.0f, 1.0f, load, pyr);
  for (int k = 0; k < 5; k++) {
    const float b = mu[k] * y[k];
    shift[k] = b - lam[k];
    stp[k] -= b;
  }
  float slope = 0.0f, curv = 0.0f;
  for (int k = 0; k < 5; k++) {
    float hs = 0.0f, hp = 0.0f;
    for (int l = 0; l < 5; l++) {
      hs += H0[k * 5 + l] * shift[l];
      hp += H0[k * 5 + l] * stp[l];
    }
    slope += stp[k] * ((g0[k] + hs) + comp[k] * (lam[k] + shift[k]));
    curv += stp[k] * (hp + comp[k] * stp[k]);
  }
  const float t = slope < 0.0f ? (curv > -slope ? (-slope) / curv : 1.0f) : 0.0f;
  for (int k = 0; k < 5; k++) out[k] = (lam[k] + shift[k]) + (t > 0.0f ? t * stp[k] : 0.0f);
}

}  // namespace orc
