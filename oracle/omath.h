// Test infrastructure: the CPU oracle's float32 vector math.
//
// ORACLE ONLY. Nothing in the product (steel_webgpu_b200/) may include this file.
//
// WGSL leaves the evaluation order of dot/length/normalize/mat*vec and the
// precision of inverseSqrt/sin/cos to the implementation. The oracle pins them
// to IEEE-exact float32 operations in a fixed order, built without FMA
// contraction (-ffp-contract=off):
//   dot(a,b)      = (a.x*b.x + a.y*b.y) + a.z*b.z
//   length(v)     = sqrt(dot(v,v))
//   normalize(v)  = v / length(v)              (component-wise division)
//   inverseSqrt(x)= 1 / sqrt(x)
//   m * v         = (m[0]*v.x + m[1]*v.y) + m[2]*v.z   (m column-major)
//   mix(a,b,t)    = a*(1-t) + b*t               (WGSL spec form)
// sin/cos/atan2 come from smath_o.h (a restatement of published methods).
#pragma once
#include <cmath>
#include <cstdint>
#include <cstring>

#ifndef ORC_F64
typedef float f32_t;  // IEEE binary32 at the buffer boundary (o_f64.h keeps it when float is widened)
#endif

namespace orc {

struct v2 { float x, y; };
struct v3 { float x, y, z; };
struct v4 { float x, y, z, w; };
struct u4 { uint32_t x, y, z, w; };
struct m3 { v3 c[3]; };  // column-major, as WGSL mat3x3f

static inline v2 mk2(float x, float y) { return {x, y}; }
static inline v3 mk3(float x, float y, float z) { return {x, y, z}; }
static inline v3 splat3(float s) { return {s, s, s}; }
static inline v4 mk4(float x, float y, float z, float w) { return {x, y, z, w}; }
static inline v4 mk4(v3 a, float w) { return {a.x, a.y, a.z, w}; }
static inline v4 mk4(float x, v3 a) { return {x, a.x, a.y, a.z}; }
static inline v3 xyz(v4 a) { return {a.x, a.y, a.z}; }

static inline v2 operator+(v2 a, v2 b) { return {a.x + b.x, a.y + b.y}; }
static inline v2 operator-(v2 a, v2 b) { return {a.x - b.x, a.y - b.y}; }
static inline v2 operator*(v2 a, float s) { return {a.x * s, a.y * s}; }
static inline v2 operator*(float s, v2 a) { return {s * a.x, s * a.y}; }
static inline v2 operator/(v2 a, float s) { return {a.x / s, a.y / s}; }
static inline float dot(v2 a, v2 b) { return a.x * b.x + a.y * b.y; }
static inline float length(v2 a) { return std::sqrt(dot(a, a)); }
static inline v2 normalize(v2 a) { float l = length(a); return {a.x / l, a.y / l}; }

static inline v3 operator+(v3 a, v3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
static inline v3 operator-(v3 a, v3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
static inline v3 operator-(v3 a) { return {-a.x, -a.y, -a.z}; }
static inline v3 operator*(v3 a, float s) { return {a.x * s, a.y * s, a.z * s}; }
static inline v3 operator*(float s, v3 a) { return {s * a.x, s * a.y, s * a.z}; }
static inline v3 operator*(v3 a, v3 b) { return {a.x * b.x, a.y * b.y, a.z * b.z}; }
static inline v3 operator/(v3 a, float s) { return {a.x / s, a.y / s, a.z / s}; }
static inline v3& operator+=(v3& a, v3 b) { a = a + b; return a; }
static inline v3& operator-=(v3& a, v3 b) { a = a - b; return a; }
static inline v3& operator/=(v3& a, float s) { a = a / s; return a; }
static inline float dot(v3 a, v3 b) { return (a.x * b.x + a.y * b.y) + a.z * b.z; }
static inline v3 cross(v3 a, v3 b) { return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
static inline float length(v3 a) { return std::sqrt(dot(a, a)); }
static inline v3 normalize(v3 a) { float l = length(a); return {a.x / l, a.y / l, a.z / l}; }
static inline v3 vabs(v3 a) { return {std::fabs(a.x), std::fabs(a.y), std::fabs(a.z)}; }
static inline float at(v3 a, int k) { return k == 0 ? a.x : (k == 1 ? a.y : a.z); }
static inline void setat(v3& a, int k, float v) { if (k == 0) a.x = v; else if (k == 1) a.y = v; else a.z = v; }
static inline bool any_ne0(v3 a) { return a.x != 0.0f || a.y != 0.0f || a.z != 0.0f; }

static inline v4 operator+(v4 a, v4 b) { return {a.x + b.x, a.y + b.y, a.z + b.z, a.w + b.w}; }
static inline v4 operator-(v4 a, v4 b) { return {a.x - b.x, a.y - b.y, a.z - b.z, a.w - b.w}; }
static inline v4 operator-(v4 a) { return {-a.x, -a.y, -a.z, -a.w}; }
static inline v4 operator*(v4 a, float s) { return {a.x * s, a.y * s, a.z * s, a.w * s}; }
static inline v4 operator*(float s, v4 a) { return {s * a.x, s * a.y, s * a.z, s * a.w}; }
static inline v4 operator/(v4 a, float s) { return {a.x / s, a.y / s, a.z / s, a.w / s}; }
static inline float dot(v4 a, v4 b) { return ((a.x * b.x + a.y * b.y) + a.z * b.z) + a.w * b.w; }
static inline float length(v4 a) { return std::sqrt(dot(a, a)); }
static inline v4 normalize(v4 a) { float l = length(a); return {a.x / l, a.y / l, a.z / l, a.w / l}; }

static inline float fminf_(float a, float b) { return b < a ? b : a; }
static inline float fmaxf_(float a, float b) { return b > a ? b : a; }
static inline float clampf(float x, float lo, float hi) { return fminf_(fmaxf_(x, lo), hi); }
static inline float inverse_sqrt(float x) { return 1.0f / std::sqrt(x); }
static inline float mixf(float a, float b, float t) { return a * (1.0f - t) + b * t; }

// WGSL float -> integer conversions: truncate toward zero, then clamp to the range.
static inline uint32_t f2u(float f) {
  if (!(f > 0.0f)) return 0u;
  if (f >= 4294967296.0f) return 0xffffffffu;
  return (uint32_t)f;
}
static inline int32_t f2i(float f) {
  if (f != f) return 0;
  if (f >= 2147483648.0f) return 0x7fffffff;
  if (f <= -2147483648.0f) return (int32_t)0x80000000u;
  return (int32_t)f;
}
#ifndef ORC_F64
static inline uint32_t fbits(float f) { uint32_t u; std::memcpy(&u, &f, 4); return u; }
static inline float bitsf(uint32_t u) { float f; std::memcpy(&f, &u, 4); return f; }
#else
// All-FP64 instance: a word carrying u32 bits holds the binary32 value of those bits.
static inline uint32_t fbits(double d) { f32_t f = (f32_t)d; uint32_t u; std::memcpy(&u, &f, 4); return u; }
static inline double bitsf(uint32_t u) { f32_t f; std::memcpy(&f, &u, 4); return (double)f; }
#endif

// Matrices (column-major).
static inline m3 mcols(v3 a, v3 b, v3 c) { return {{a, b, c}}; }
static inline v3 mul(const m3& m, v3 v) { return (m.c[0] * v.x + m.c[1] * v.y) + m.c[2] * v.z; }
static inline m3 transpose(const m3& m) {
  return mcols(mk3(m.c[0].x, m.c[1].x, m.c[2].x), mk3(m.c[0].y, m.c[1].y, m.c[2].y), mk3(m.c[0].z, m.c[1].z, m.c[2].z));
}
static inline m3 mul(const m3& a, const m3& b) { return mcols(mul(a, b.c[0]), mul(a, b.c[1]), mul(a, b.c[2])); }
static inline m3 madd(const m3& a, const m3& b) { return mcols(a.c[0] + b.c[0], a.c[1] + b.c[1], a.c[2] + b.c[2]); }
static inline m3 msub(const m3& a, const m3& b) { return mcols(a.c[0] - b.c[0], a.c[1] - b.c[1], a.c[2] - b.c[2]); }
static inline m3 mscale(const m3& a, float s) { return mcols(a.c[0] * s, a.c[1] * s, a.c[2] * s); }
static inline m3 mscale(float s, const m3& a) { return mcols(s * a.c[0], s * a.c[1], s * a.c[2]); }

// Quaternions (x, y, z, w), wgsl.js:48-60.
static inline v3 qrot(v4 q, v3 v) {
  v3 u = xyz(q); float s = q.w;
  return ((2.0f * dot(u, v)) * u + (s * s - dot(u, u)) * v) + (2.0f * s) * cross(u, v);
}
static inline v3 qinvrot(v4 q, v3 v) { return qrot(mk4(-xyz(q), q.w), v); }
static inline v4 qmul(v4 a, v4 b) {
  v3 v = (a.w * xyz(b) + b.w * xyz(a)) + cross(xyz(a), xyz(b));
  return mk4(v, a.w * b.w - dot(xyz(a), xyz(b)));
}
static inline v4 qconj(v4 q) { return mk4(-q.x, -q.y, -q.z, q.w); }
static inline m3 qmat(v4 q) { return mcols(qrot(q, mk3(1, 0, 0)), qrot(q, mk3(0, 1, 0)), qrot(q, mk3(0, 0, 1))); }
static inline uint32_t hash_u32(uint32_t x) {
  x ^= x >> 16; x *= 0x7feb352du; x ^= x >> 15; x *= 0x846ca68bu; x ^= x >> 16;
  return x;
}

}  // namespace orc
