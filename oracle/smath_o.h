// Test infrastructure: the oracle's sin / cos / atan2 (float in, float out).
//
// ORACLE ONLY. WGSL leaves sin/cos/atan2 precision to the implementation, so the
// oracle defines them: evaluated in IEEE double from published series, then
// rounded once to float.
//   sin/cos: Cody-Waite style reduction by pi/2 (k = nearest integer of x*2/pi,
//            r = x - k*pi/2 in double), then the Taylor series of sin and cos on
//            |r| <= pi/4 to degree 21/20 (truncation error < 1e-19).
//   atan:    two argument halvings atan(t) = 2 atan(t / (1 + sqrt(1 + t^2))),
//            then the Taylor series of atan to degree 41 on |t| <= tan(pi/16).
//   atan2:   quadrant fix-up of atan(y/x) (or pi/2 - atan(x/y) when |y| > |x|).
// Built without FMA contraction, so every run and every build agree.
#pragma once
#include <cmath>

namespace orc {

static inline double o_sin_poly(double r) {
  double r2 = r * r, t = r, s = r;
  for (int n = 1; n <= 10; n++) { t = -t * r2 / (double)((2 * n) * (2 * n + 1)); s = s + t; }
  return s;
}
static inline double o_cos_poly(double r) {
  double r2 = r * r, t = 1.0, s = 1.0;
  for (int n = 1; n <= 10; n++) { t = -t * r2 / (double)((2 * n - 1) * (2 * n)); s = s + t; }
  return s;
}
static inline void o_reduce(double x, double* r, int* q) {
  const double half_pi = 1.5707963267948966;
  double k = std::nearbyint(x * 0.6366197723675814);
  *r = x - k * half_pi;
  long long kk = (long long)k;
  *q = (int)(((kk % 4) + 4) % 4);
}
static inline float sin_o(float xf) {
  double r; int q; o_reduce((double)xf, &r, &q);
  double v = (q == 0) ? o_sin_poly(r) : (q == 1) ? o_cos_poly(r) : (q == 2) ? -o_sin_poly(r) : -o_cos_poly(r);
  return (float)v;
}
static inline float cos_o(float xf) {
  double r; int q; o_reduce((double)xf, &r, &q);
  double v = (q == 0) ? o_cos_poly(r) : (q == 1) ? -o_sin_poly(r) : (q == 2) ? -o_cos_poly(r) : o_sin_poly(r);
  return (float)v;
}
static inline double o_atan_small(double t) {
  double t2 = t * t, p = t, s = t;
  for (int n = 1; n <= 20; n++) { p = -p * t2; s = s + p / (double)(2 * n + 1); }
  return s;
}
static inline double o_atan(double t) {  // |t| <= 1
  double a = t / (1.0 + std::sqrt(1.0 + t * t));
  double b = a / (1.0 + std::sqrt(1.0 + a * a));
  return 4.0 * o_atan_small(b);
}
static inline float atan2_o(float yf, float xf) {
  double y = yf, x = xf;
  const double pi = 3.141592653589793;
  if (x == 0.0 && y == 0.0) return (float)(std::signbit(x) ? (std::signbit(y) ? -pi : pi) : (std::signbit(y) ? -0.0 : 0.0));
  double v;
  if (std::fabs(y) <= std::fabs(x)) {
    v = o_atan(y / x);
    if (x < 0.0) v = (y < 0.0 || (y == 0.0 && std::signbit(y))) ? v - pi : v + pi;
  } else {
    v = (y > 0.0 ? pi / 2 : -pi / 2) - o_atan(x / y);
  }
  return (float)v;
}

}  // namespace orc
