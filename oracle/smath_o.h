// Test infrastructure: the oracle's sin / cos / atan2 (float in, float out).
//
// ORACLE ONLY. WGSL leaves sin/cos/atan2 precision to the implementation, so the
// oracle defines them: evaluated in IEEE double from published series, then
// rounded once to float.
//   sin/cos: Cody-Waite style reduction by pi/2 (k = nearest integer of x*2/pi,
//            r = x - k*pi/2 in double), then the Taylor series of sin and cos on
//            |r| <= pi/4 to degree 21/20 (truncation error < 1e-19), in Horner form with
//            the coefficients (-1)^n/(2n+1)! and (-1)^n/(2n)! as their nearest doubles.
//   atan:    two argument halvings atan(t) = 2 atan(t / (1 + sqrt(1 + t^2))),
//            then the Taylor series of atan to degree 41 on |t| <= tan(pi/16), Horner form
//            with the coefficients (-1)^n/(2n+1) as their nearest doubles.
//   atan2:   quadrant fix-up of atan(y/x) (or pi/2 - atan(x/y) when |y| > |x|).
// Built without FMA contraction, so every run and every build agree.
#pragma once
#include <cmath>

namespace orc {

static inline double o_sin_poly(double r) {
  double r2 = r * r;
  double q = -0x1.5555555555555p-3 + r2 * (0x1.1111111111111p-7 + r2 * (-0x1.a01a01a01a01ap-13 + r2 * (0x1.71de3a556c734p-19 + r2 * (-0x1.ae64567f544e4p-26 + r2 * (0x1.6124613a86d09p-33 + r2 * (-0x1.ae7f3e733b81fp-41 + r2 * (0x1.952c77030ad4ap-49 + r2 * (-0x1.2f49b46814157p-57 + r2 * (0x1.71b8ef6dcf572p-66)))))))));
  return r + (r * r2) * q;
}
static inline double o_cos_poly(double r) {
  double r2 = r * r;
  double q = -0x1.0000000000000p-1 + r2 * (0x1.5555555555555p-5 + r2 * (-0x1.6c16c16c16c17p-10 + r2 * (0x1.a01a01a01a01ap-16 + r2 * (-0x1.27e4fb7789f5cp-22 + r2 * (0x1.1eed8eff8d898p-29 + r2 * (-0x1.93974a8c07c9dp-37 + r2 * (0x1.ae7f3e733b81fp-45 + r2 * (-0x1.6827863b97d97p-53 + r2 * (0x1.e542ba4020225p-62)))))))));
  return 1.0 + r2 * q;
}
static inline void o_reduce(double x, double* r, int* q) {
  const double half_pi = 1.5707963267948966;
  double k = std::nearbyint(x * 0.6366197723675814);
  *r = x - k * half_pi;
  *q = (int)((long long)k & 3);
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
  double t2 = t * t;
  double q = -0x1.5555555555555p-2 + t2 * (0x1.999999999999ap-3 + t2 * (-0x1.2492492492492p-3 + t2 * (0x1.c71c71c71c71cp-4 + t2 * (-0x1.745d1745d1746p-4 + t2 * (0x1.3b13b13b13b14p-4 + t2 * (-0x1.1111111111111p-4 + t2 * (0x1.e1e1e1e1e1e1ep-5 + t2 * (-0x1.af286bca1af28p-5 + t2 * (0x1.8618618618618p-5 + t2 * (-0x1.642c8590b2164p-5 + t2 * (0x1.47ae147ae147bp-5 + t2 * (-0x1.2f684bda12f68p-5 + t2 * (0x1.1a7b9611a7b96p-5 + t2 * (-0x1.0842108421084p-5 + t2 * (0x1.f07c1f07c1f08p-6 + t2 * (-0x1.d41d41d41d41dp-6 + t2 * (0x1.bacf914c1bad0p-6 + t2 * (-0x1.a41a41a41a41ap-6 + t2 * (0x1.8f9c18f9c18fap-6)))))))))))))))))));
  return t + (t * t2) * q;
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
