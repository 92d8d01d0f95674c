// Device-side vector math, scene descriptor and per-substep parameters.
//
// Every float expression here is evaluated as written, one IEEE-rounded step at a
// time: the library is built with --fmad=false (no contraction), -prec-div and
// -prec-sqrt (correctly rounded division and square root), and no fast math. The
// evaluation order of the reference's WGSL built-ins that WGSL leaves open is fixed:
//   dot(a,b)       = (a.x*b.x + a.y*b.y) + a.z*b.z
//   length(v)      = sqrt(dot(v,v)),  normalize(v) = v / length(v)
//   inverseSqrt(x) = 1 / sqrt(x)
//   m * v          = (m[0]*v.x + m[1]*v.y) + m[2]*v.z   (m column-major)
// so that a run is reproducible bit for bit across launches, batch sizes and GPUs.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#define SD static __device__ __forceinline__
#define SHD static __host__ __device__ __forceinline__

namespace steel {

struct f2 { float x, y; };
struct f3 { float x, y, z; };
struct m3 { f3 c[3]; };

SHD f2 mf2(float x, float y) { return {x, y}; }
SHD f3 mf3(float x, float y, float z) { return {x, y, z}; }
SHD f3 sp3(float s) { return {s, s, s}; }
SHD float4 mf4(float x, float y, float z, float w) { return make_float4(x, y, z, w); }
SHD float4 mf4(f3 a, float w) { return make_float4(a.x, a.y, a.z, w); }
SHD float4 mf4(float x, f3 a) { return make_float4(x, a.x, a.y, a.z); }
SHD f3 v3(float4 a) { return {a.x, a.y, a.z}; }

SHD f2 operator+(f2 a, f2 b) { return {a.x + b.x, a.y + b.y}; }
SHD f2 operator-(f2 a, f2 b) { return {a.x - b.x, a.y - b.y}; }
SHD f2 operator*(f2 a, float s) { return {a.x * s, a.y * s}; }
SHD f2 operator*(float s, f2 a) { return {s * a.x, s * a.y}; }
SHD f2 operator/(f2 a, float s) { return {a.x / s, a.y / s}; }
SHD float dot(f2 a, f2 b) { return a.x * b.x + a.y * b.y; }
SHD float len(f2 a) { return sqrtf(dot(a, a)); }
SHD f2 nrm(f2 a) { float l = len(a); return {a.x / l, a.y / l}; }

SHD f3 operator+(f3 a, f3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
SHD f3 operator-(f3 a, f3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
SHD f3 operator-(f3 a) { return {-a.x, -a.y, -a.z}; }
SHD f3 operator*(f3 a, float s) { return {a.x * s, a.y * s, a.z * s}; }
SHD f3 operator*(float s, f3 a) { return {s * a.x, s * a.y, s * a.z}; }
SHD f3 operator/(f3 a, float s) { return {a.x / s, a.y / s, a.z / s}; }
SHD f3& operator+=(f3& a, f3 b) { a = a + b; return a; }
SHD f3& operator-=(f3& a, f3 b) { a = a - b; return a; }
SHD float dot(f3 a, f3 b) { return (a.x * b.x + a.y * b.y) + a.z * b.z; }
SHD f3 cross(f3 a, f3 b) { return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
SHD float len(f3 a) { return sqrtf(dot(a, a)); }
SHD f3 nrm(f3 a) { float l = len(a); return {a.x / l, a.y / l, a.z / l}; }
SHD f3 vabs(f3 a) { return {fabsf(a.x), fabsf(a.y), fabsf(a.z)}; }
SHD float comp(f3 a, int k) { return k == 0 ? a.x : (k == 1 ? a.y : a.z); }
SHD void setc(f3& a, int k, float v) { if (k == 0) a.x = v; else if (k == 1) a.y = v; else a.z = v; }
SHD bool nonzero(f3 a) { return a.x != 0.0f || a.y != 0.0f || a.z != 0.0f; }

SHD float4 add4(float4 a, float4 b) { return make_float4(a.x + b.x, a.y + b.y, a.z + b.z, a.w + b.w); }
SHD float4 scale4(float s, float4 a) { return make_float4(s * a.x, s * a.y, s * a.z, s * a.w); }
SHD float dot4(float4 a, float4 b) { return ((a.x * b.x + a.y * b.y) + a.z * b.z) + a.w * b.w; }
SHD float4 nrm4(float4 a) { float l = sqrtf(dot4(a, a)); return make_float4(a.x / l, a.y / l, a.z / l, a.w / l); }
SHD float4 neg4(float4 a) { return make_float4(-a.x, -a.y, -a.z, -a.w); }

SHD float fmn(float a, float b) { return b < a ? b : a; }
SHD float fmx(float a, float b) { return b > a ? b : a; }
SHD float clmp(float x, float lo, float hi) { return fmn(fmx(x, lo), hi); }
SHD float rsq(float x) { return 1.0f / sqrtf(x); }

// Float -> integer as WGSL converts: truncate toward zero, clamp to the range.
SHD uint32_t f2u(float f) {
  if (!(f > 0.0f)) return 0u;
  if (f >= 4294967296.0f) return 0xffffffffu;
  return (uint32_t)f;
}
SHD int32_t f2i(float f) {
  if (f != f) return 0;
  if (f >= 2147483648.0f) return 0x7fffffff;
  if (f <= -2147483648.0f) return (int32_t)0x80000000u;
  return (int32_t)f;
}
SD uint32_t fbits(float f) { return __float_as_uint(f); }
SD float ubits(uint32_t u) { return __uint_as_float(u); }

SHD m3 mcols(f3 a, f3 b, f3 c) { m3 m; m.c[0] = a; m.c[1] = b; m.c[2] = c; return m; }
SHD f3 mul(const m3& m, f3 v) { return (m.c[0] * v.x + m.c[1] * v.y) + m.c[2] * v.z; }
SHD m3 tr(const m3& m) {
  return mcols(mf3(m.c[0].x, m.c[1].x, m.c[2].x), mf3(m.c[0].y, m.c[1].y, m.c[2].y), mf3(m.c[0].z, m.c[1].z, m.c[2].z));
}
SHD m3 mul(const m3& a, const m3& b) { return mcols(mul(a, b.c[0]), mul(a, b.c[1]), mul(a, b.c[2])); }
SHD m3 madd(const m3& a, const m3& b) { return mcols(a.c[0] + b.c[0], a.c[1] + b.c[1], a.c[2] + b.c[2]); }
SHD m3 msub(const m3& a, const m3& b) { return mcols(a.c[0] - b.c[0], a.c[1] - b.c[1], a.c[2] - b.c[2]); }
SHD m3 mscl(float s, const m3& a) { return mcols(s * a.c[0], s * a.c[1], s * a.c[2]); }

// Quaternions (x, y, z, w).
SHD f3 qrot(float4 q, f3 v) {
  f3 u = v3(q);
  float s = q.w;
  return ((2.0f * dot(u, v)) * u + (s * s - dot(u, u)) * v) + (2.0f * s) * cross(u, v);
}
SHD f3 qinv(float4 q, f3 v) { return qrot(make_float4(-q.x, -q.y, -q.z, q.w), v); }
SHD float4 qmul(float4 a, float4 b) {
  f3 v = (a.w * v3(b) + b.w * v3(a)) + cross(v3(a), v3(b));
  return mf4(v, a.w * b.w - dot(v3(a), v3(b)));
}
SHD float4 qconj(float4 q) { return make_float4(-q.x, -q.y, -q.z, q.w); }
SHD m3 qmat(float4 q) { return mcols(qrot(q, mf3(1, 0, 0)), qrot(q, mf3(0, 1, 0)), qrot(q, mf3(0, 0, 1))); }
SHD uint32_t mix32(uint32_t x) {
  x ^= x >> 16; x *= 0x7feb352du; x ^= x >> 15; x *= 0x846ca68bu; x ^= x >> 16;
  return x;
}

// sin, cos and atan2 for float arguments, computed in double and rounded once:
// reduction by pi/2 (nearest multiple), then the Taylor series of sin/cos on
// |r| <= pi/4 to degree 21/20; atan by two half-angle reductions
// t -> t / (1 + sqrt(1 + t^2)) followed by its Taylor series to degree 41.
// Series are evaluated in Horner form; the coefficients (-1)^n/(2n+1)!, (-1)^n/(2n)! and
// (-1)^n/(2n+1) are written as their nearest doubles (hexadecimal literals).
SHD double ser_sin(double r) {
  double r2 = r * r;
  double q = -0x1.5555555555555p-3 + r2 * (0x1.1111111111111p-7 + r2 * (-0x1.a01a01a01a01ap-13 + r2 * (0x1.71de3a556c734p-19 + r2 * (-0x1.ae64567f544e4p-26 + r2 * (0x1.6124613a86d09p-33 + r2 * (-0x1.ae7f3e733b81fp-41 + r2 * (0x1.952c77030ad4ap-49 + r2 * (-0x1.2f49b46814157p-57 + r2 * (0x1.71b8ef6dcf572p-66)))))))));
  return r + (r * r2) * q;
}
SHD double ser_cos(double r) {
  double r2 = r * r;
  double q = -0x1.0000000000000p-1 + r2 * (0x1.5555555555555p-5 + r2 * (-0x1.6c16c16c16c17p-10 + r2 * (0x1.a01a01a01a01ap-16 + r2 * (-0x1.27e4fb7789f5cp-22 + r2 * (0x1.1eed8eff8d898p-29 + r2 * (-0x1.93974a8c07c9dp-37 + r2 * (0x1.ae7f3e733b81fp-45 + r2 * (-0x1.6827863b97d97p-53 + r2 * (0x1.e542ba4020225p-62)))))))));
  return 1.0 + r2 * q;
}
SHD void quadrant(double x, double* r, int* q) {
  double k = nearbyint(x * 0.6366197723675814);
  *r = x - k * 1.5707963267948966;
  *q = (int)((long long)k & 3);
}
SHD float fsin(float xf) {
  double r; int q; quadrant((double)xf, &r, &q);
  double v = q == 0 ? ser_sin(r) : q == 1 ? ser_cos(r) : q == 2 ? -ser_sin(r) : -ser_cos(r);
  return (float)v;
}
SHD float fcos(float xf) {
  double r; int q; quadrant((double)xf, &r, &q);
  double v = q == 0 ? ser_cos(r) : q == 1 ? -ser_sin(r) : q == 2 ? -ser_cos(r) : ser_sin(r);
  return (float)v;
}
SHD double ser_atan(double t) {
  double t2 = t * t;
  double q = -0x1.5555555555555p-2 + t2 * (0x1.999999999999ap-3 + t2 * (-0x1.2492492492492p-3 + t2 * (0x1.c71c71c71c71cp-4 + t2 * (-0x1.745d1745d1746p-4 + t2 * (0x1.3b13b13b13b14p-4 + t2 * (-0x1.1111111111111p-4 + t2 * (0x1.e1e1e1e1e1e1ep-5 + t2 * (-0x1.af286bca1af28p-5 + t2 * (0x1.8618618618618p-5 + t2 * (-0x1.642c8590b2164p-5 + t2 * (0x1.47ae147ae147bp-5 + t2 * (-0x1.2f684bda12f68p-5 + t2 * (0x1.1a7b9611a7b96p-5 + t2 * (-0x1.0842108421084p-5 + t2 * (0x1.f07c1f07c1f08p-6 + t2 * (-0x1.d41d41d41d41dp-6 + t2 * (0x1.bacf914c1bad0p-6 + t2 * (-0x1.a41a41a41a41ap-6 + t2 * (0x1.8f9c18f9c18fap-6)))))))))))))))))));
  return t + (t * t2) * q;
}
SHD double atan_unit(double t) {
  double a = t / (1.0 + sqrt(1.0 + t * t));
  double b = a / (1.0 + sqrt(1.0 + a * a));
  return 4.0 * ser_atan(b);
}
SHD float fatan2(float yf, float xf) {
  double y = yf, x = xf;
  const double pi = 3.141592653589793;
  if (x == 0.0 && y == 0.0) return (float)(signbit(x) ? (signbit(y) ? -pi : pi) : (signbit(y) ? -0.0 : 0.0));
  double v;
  if (fabs(y) <= fabs(x)) {
    v = atan_unit(y / x);
    if (x < 0.0) v = (y < 0.0 || (y == 0.0 && signbit(y))) ? v - pi : v + pi;
  } else {
    v = (y > 0.0 ? pi / 2 : -pi / 2) - atan_unit(x / y);
  }
  return (float)v;
}

// View of an array that no kernel writes while it runs (the scene's static data): element reads
// go through the read-only data path, so the compiler may issue them ahead of stores.
template <class T>
struct RO {
  const T* p;
  __device__ __forceinline__ T operator[](size_t i) const { return __ldg(p + i); }
  __host__ __device__ RO operator+(size_t i) const { return RO{p + i}; }
};

// Per-substep parameters (the reference's 112-byte Params uniform, wgsl.js:34-45).
struct Params {
  float dt; uint32_t substep, parity, iterations;
  float phase, frame_dt, beta, max_depen;
  float4 gravity;
  float warm_scale; uint32_t path_frames, driven, integral_count;
  float reg; uint32_t pad[3];
};

// One scene of a batch: static data in the reference's packed format (statF/statU and the
// offsets its packer computed), the dynamic state, scratch and capacities. Offsets are in
// elements of the array they index.
struct SceneDev {
  // static, reference format
  RO<float4> sf;                     // static scene data, read-only in every kernel
  RO<uint32_t> su;
  uint32_t SF_BODY, SF_SHAPE, SF_HAABB, SF_VERTS, SF_FPLANE, SF_LINK, SF_DOF, SF_PATH, SF_LOOP, SF_MIMIC, SF_CTRL;
  uint32_t SU_HULL, SU_FACE, SU_FV, SU_HEDGE, SU_EDGE, SU_ART, SU_ACON, SU_FILTER;
  // counts
  uint32_t NB, NS, NA, NL, ND, NQ, NDA, JM, MAXPATH, MAXLP, NLOOP, NMIMIC;
  // solver flags and constants
  uint32_t PATCH, EXTRA, SHARED, FSHARED, REST, FSTART, TGT_HELD, CTRL_KIND, CTRL_A, CTRL_B, VLIM_FREE, VLIM_ON, ART_F64, SLEEP, NEST, MO, TORS, TO, COMPL, CO, VELITERS, JFL,
      DRIVE_ROWS, FUSE_VLIM, VEL_DRIVE_ACTIVE, FMODE, FMO, ANG, ANG_ART, EO, PYRAMID, CTI, LONGEST_FIRST;
  uint32_t FRICTION_COMBINE, RESTITUTION_COMBINE, NCOLW, NCOL;
  float F_ANCHOR_BETA, F_CFM, F_OMEGA, F_SPEC, F_GAP_GATE, F_FGAP, F_FSCALE, F_REST_SPEED, F_FR_MUT, F_FR_MUR;
  float F_BP_CELL, F_JL_GAP, F_JL_SPEED, F_VLIM_FRAC, F_SLEEP_LIN, F_SLEEP_ANG, F_SLEEP_TIME, F_CREEP;
  // writeParams inputs
  double fps;
  uint32_t substeps, iterations, target_frames, driven, integral_count, user_targets;
  float beta, warm, reg, gx, gy, gz;
  // capacities (per scene)
  uint32_t MAXP, MAXC, MAXU, WH, AH, MAXDENSE, ROWS, PO, DHDR, DPS;
  // state
  float4 *pos, *rot, *ppos, *prot;  // body COM pose and previous pose [NB]
  float4 *lv, *av;                   // body COM twist [NB]
  float4 *spos, *srot, *alo, *ahi;   // shape pose and AABB [NS]
  float* art;                        // articulation buffer (A_* layout)
  uint32_t A_Q, A_QD, A_QDH, A_INT, A_TGT, A_TGTV, A_LIM, A_DRV, A_JF, A_BF, A_FRIC, A_HINV, A_LINK, A_VLG, A_AVL, A_LG,
      A_RL, A_RLN, A_ULOAD, A_DENSE, A_SLP, A_SNAP, A_JFL;
  uint32_t* counters;                // [0] pairs, [1] contacts
  uint32_t* stats;                   // SimStats words (sim.js:822-834)
  Params* params;                    // this substep's parameters
  float4* craw;                      // narrowphase contacts: 5 float4 per record, then MAXC shape-mu entries
  float4* con;                       // sorted contacts (same layout)
  uint4* ckeys;                      // sort scratch [MAXC]
  float4* rows;                      // row records [MAXC * ROWS]
  float4* slots;                     // slot table [MAXC * 2]
  uint32_t* warm_tab;                // warm table: 10*WH + 30*AH words
  uint32_t* sched;                   // scheduling arrays, offsets below
  uint32_t S_UNITOF, S_DSLOT, S_CORDER, S_UKEY, S_USTART0, S_USIZE, S_USTART, S_RK0, S_RK1, S_RK2, S_BPC, S_LEAD,
      S_KEEP, S_SLOT, S_KEPT, S_ROWOF, S_RUNIT, S_RCON, S_PCOL, S_PORD, S_CSTART, S_META, S_WWIN, S_WSLOT, S_WMASK,
      S_WCOUNT, S_LINKHIT, S_JSPLIT, S_UF, S_UFF, S_UTP, S_DSTART, S_DOFF, S_DLIST, S_BSTART, S_BPOS, S_BREADY,
      S_BLIST, S_RKEY, S_RFLAG, S_WL;
  float* tscr;                       // per-thread scratch slices (path temporaries), TSCR floats each
  uint32_t TSCR;
  uint32_t TSCR_T;                   // threads the scratch has slices for
  float4 *tw, *imp;                  // solve: body twists and link impulses [NB * 2]
  uint32_t stage;                    // shared-memory staging: bit 0 link blocks (prepare, solve),
                                     // bit 1 twists, impulses and qd (solve)
  float* aqd;                        // solve: generalized velocities [ND]
  uint32_t scene_index;
};

}  // namespace steel
