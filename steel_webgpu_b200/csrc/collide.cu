// Collision kernels of one substep: parameters, shape poses/AABBs, broadphase, narrowphase and
// the canonical contact sort.
//
// Reference behaviour followed (packages/steel-webgpu/src/wgsl.js):
//   shapes  wgsl.js:117-150   broad  wgsl.js:154-177   narrow wgsl.js:182-1217
//   csort   wgsl.js:3899-3982 (canonical order (pair, feature, point-bit hash, raw index))
// B200 layout: shape tiles of a scene are tested by one block from shared memory; candidate
// pairs of every scene of the batch go to one compacted list (warp-aggregated atomics); the
// narrowphase runs one warp per pair with shuffle reductions over faces, edge pairs and
// support points; each scene's contacts are sorted by one block.
#include <cooperative_groups.h>

#include <algorithm>
#include <map>
#include <mutex>

#include "batch.cuh"
#include "contact_key.cuh"

namespace steel {

// --------------------------------------------------------------------------------------------
// Per-substep parameters (sim.js:625-639): one thread per scene.
__global__ void k_params(BatchDev B, uint32_t substep) {
  uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s == 0u) { B.pair_count[0] = 0u; B.pair_count[1] = 0u; }
  if (s >= B.nscenes || B.active[s] == 0u) return;
  const SceneDev& S = B.scenes[s];
  Params P;
  double dt = 1.0 / S.fps / (double)S.substeps;
  P.dt = (float)dt;
  P.substep = substep;
  P.parity = (uint32_t)((B.substep_count[s] + substep) % 2ull);
  P.iterations = S.iterations;
  P.phase = (float)B.phase[s];
  P.frame_dt = (float)(1.0 / S.fps);
  P.beta = S.beta;
  P.max_depen = 2.0f;
  P.gravity = make_float4(S.gx, S.gy, S.gz, 0.0f);
  P.warm_scale = S.warm;
  P.path_frames = S.target_frames;
  P.driven = S.user_targets ? 0u : S.driven;
  P.integral_count = S.integral_count;
  P.reg = S.reg;
  P.pad[0] = P.pad[1] = P.pad[2] = 0u;
  *S.params = P;
}
// Frame end (sim.js:674-678): advance the clocks.
__global__ void k_frame_end(BatchDev B) {
  uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= B.nscenes || B.active[s] == 0u) return;
  B.phase[s] += 1.0 / B.scenes[s].fps;
  B.substep_count[s] += (unsigned long long)B.scenes[s].substeps;
}

// --------------------------------------------------------------------------------------------
// Shape world poses and AABBs (wgsl.js:117-150): one thread per shape of the batch.
__global__ void k_shapes(BatchDev B) {
  uint32_t g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= B.nshapes || B.active[B.shape_scene[g]] == 0u) return;
  const SceneDev& S = B.scenes[B.shape_scene[g]];
  uint32_t s = B.shape_local[g];
  RO<float4> sf = S.sf + S.SF_SHAPE + s * 7u;
  float4 r0 = sf[0];
  int body = f2i(r0.x);
  uint32_t hull = f2u(r0.y);
  f3 bp = sp3(0.0f);
  float4 bq = make_float4(0, 0, 0, 1);
  if (body >= 0) {
    f3 c = v3(S.pos[body]);
    bq = S.rot[body];
    bp = c - qrot(bq, v3(S.sf[S.SF_BODY + (uint32_t)body * 8u + 1u]));
  }
  f3 spp = bp + qrot(bq, v3(sf[1]));
  float4 sq = nrm4(qmul(bq, sf[2]));
  S.spos[s] = mf4(spp, 0.0f);
  S.srot[s] = sq;
  if (sf[3].x == 4.0f) {
    S.alo[s] = make_float4(-1e6f, -1e6f, -1e6f, 0.0f);
    S.ahi[s] = make_float4(1e6f, 1e6f, 1e6f, 0.0f);
    return;
  }
  f3 hc = v3(S.sf[S.SF_HAABB + hull * 2u]);
  f3 hh = v3(S.sf[S.SF_HAABB + hull * 2u + 1u]);
  m3 m = qmat(sq);
  f3 c = spp + mul(m, hc);
  f3 e = ((vabs(m.c[0]) * hh.x + vabs(m.c[1]) * hh.y) + vabs(m.c[2]) * hh.z) + sp3(r0.w);
  S.alo[s] = mf4(c - e, 0.0f);
  S.ahi[s] = mf4(c + e, 0.0f);
}

// --------------------------------------------------------------------------------------------
// Broadphase (wgsl.js:154-177): the reference's all-pairs test with its filter rules, one block
// per 32x32 shape tile of a scene, tile data staged in shared memory. Hits are compacted by
// warp ballots into the batch's pair list; the per-scene count keeps the reference's capacity
// semantics (a scene keeps its first MAXP candidate pairs).
struct TileShape { float4 lo, hi; int body; uint32_t fixed; };

__global__ void __launch_bounds__(256) k_broad(BatchDev B) {
  __shared__ TileShape ti_[BROAD_TILE], tj_[BROAD_TILE];
  uint4 job = B.tiles[blockIdx.x];
  if (B.active[job.x] == 0u) return;
  const SceneDev& S = B.scenes[job.x];
  const uint32_t i0 = job.y * BROAD_TILE, j0 = job.z * BROAD_TILE;
  const uint32_t t = threadIdx.x;
  if (t < 2u * BROAD_TILE) {
    uint32_t k = t % BROAD_TILE;
    uint32_t s = (t < BROAD_TILE ? i0 : j0) + k;
    TileShape ts;
    ts.body = -2;
    ts.fixed = 1u;
    ts.lo = ts.hi = make_float4(0, 0, 0, 0);
    if (s < S.NS) {
      int b = f2i(S.sf[S.SF_SHAPE + s * 7u].x);
      ts.body = b;
      bool fx = b < 0;
      if (!fx) {
        float4 br = S.sf[S.SF_BODY + (uint32_t)b * 8u];
        fx = f2u(br.y) == 3u || (f2u(S.sf[S.SF_BODY + (uint32_t)b * 8u + 7u].w) & 1u) != 0u;
      }
      ts.fixed = fx ? 1u : 0u;
      ts.lo = S.alo[s];
      ts.hi = S.ahi[s];
    }
    if (t < BROAD_TILE) ti_[k] = ts; else tj_[k] = ts;
  }
  __syncthreads();
  const uint32_t lane = t & 31u;
  for (uint32_t q = t; q < BROAD_TILE * BROAD_TILE; q += blockDim.x) {
    uint32_t a = q / BROAD_TILE, b = q % BROAD_TILE;
    uint32_t i = i0 + a, j = j0 + b;
    bool hit = false;
    if (i < S.NS && j < S.NS && i < j) {
      const TileShape& A = ti_[a];
      const TileShape& Bs = tj_[b];
      hit = A.body != Bs.body && !(A.body < 0 && Bs.body < 0) && !(A.fixed && Bs.fixed);
      if (hit) {
        uint32_t k = i * S.NS + j;
        hit = (S.su[S.SU_FILTER + (k >> 5u)] & (1u << (k & 31u))) == 0u;
      }
      if (hit) {
        hit = !(A.lo.x > Bs.hi.x || A.lo.y > Bs.hi.y || A.lo.z > Bs.hi.z || Bs.lo.x > A.hi.x ||
                Bs.lo.y > A.hi.y || Bs.lo.z > A.hi.z);
      }
    }
    uint32_t mask = __ballot_sync(0xffffffffu, hit);
    if (mask == 0u) continue;
    uint32_t nhit = __popc(mask), rank = __popc(mask & ((1u << lane) - 1u));
    uint32_t leader = __ffs(mask) - 1u;
    uint32_t sbase = 0u, gbase = 0u;
    if (lane == leader) {
      sbase = atomicAdd(&S.counters[0], nhit);
      uint32_t keep = sbase >= S.MAXP ? 0u : min(nhit, S.MAXP - sbase);
      gbase = keep ? atomicAdd(B.pair_count, keep) : 0u;
    }
    sbase = __shfl_sync(0xffffffffu, sbase, leader);
    gbase = __shfl_sync(0xffffffffu, gbase, leader);
    if (hit && sbase + rank < S.MAXP) B.pairs[gbase + rank] = make_uint4(job.x, i, j, 0u);
  }
}

// --------------------------------------------------------------------------------------------
// Narrowphase (wgsl.js:182-1217): one warp per candidate pair.
static constexpr uint32_t GT_PLANE = 1u, GT_SPHERE = 3u, GT_CAPSULE = 4u, GT_CYL = 6u, GT_BOX = 7u, GT_CONE = 9u,
                          GT_CONVEX = 10u;
static constexpr float MEPS = 1e-5f;
static constexpr float COS_TILT = 0.9993908270190958f;
static constexpr float SIN_TILT = 0.03489949670250097f;
static constexpr float COS_DEEP = 0.9999984769132877f;
static constexpr float WITNESS_TOL = 1e-3f;
static constexpr float SAT_TIE = 1e-5f;
__constant__ float PENTX[5] = {1.0f, 0.30901699437494745f, -0.8090169943749473f, -0.8090169943749476f,
                               0.30901699437494723f};
__constant__ float PENTY[5] = {0.0f, 0.9510565162951535f, 0.5877852522924732f, -0.587785252292473f,
                               -0.9510565162951536f};

struct FaceQ { float sep; uint32_t face; };
struct EdgeQ { float sep; f3 axis, a0, a1, b0, b1; uint32_t id; };
struct SegQ { float d2; f3 ps, ph; uint32_t face, kind; };
struct Geo { uint32_t t; f3 s; uint32_t h; };

// Index of the first lane holding the best value (max or min): the reference's lane-0 scan
// "rsep[k] > rsep[b]" over the 32 lanes, as a butterfly over (value, lane).
SD uint32_t best_lane(float v, bool want_max) {
  uint32_t lane = threadIdx.x & 31u;
  float bv = v;
  uint32_t bl = lane;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    float ov = __shfl_xor_sync(0xffffffffu, bv, o);
    uint32_t ol = __shfl_xor_sync(0xffffffffu, bl, o);
    bool take = want_max ? (ov > bv || (ov == bv && ol < bl)) : (ov < bv || (ov == bv && ol < bl));
    if (take) { bv = ov; bl = ol; }
  }
  return bl;
}
SD f3 shfl3(f3 v, uint32_t src) {
  return mf3(__shfl_sync(0xffffffffu, v.x, src), __shfl_sync(0xffffffffu, v.y, src), __shfl_sync(0xffffffffu, v.z, src));
}

// Serial narrowphase work that k_narrow hands to k_narrow_jobs: the routine and its argument
// values, stored bit for bit in a record of NJOB_WORDS words (word 0 the routine, word 1 the
// scene). The routines run one per thread there instead of on lane 0 of a warp.
enum : uint32_t { J_PLANE_CONVEX = 1u, J_PLANE = 2u, J_PRIM = 3u, J_CAPSULE = 4u, J_SEGFACE = 5u, J_SAT = 6u, J_MPR = 7u };
struct JobW {
  uint32_t w[NJOB_WORDS];
  uint32_t n = 2u;
  __device__ void u(uint32_t x) { w[n++] = x; }
  __device__ void f(float x) { w[n++] = __float_as_uint(x); }
  __device__ void v(f3 x) { f(x.x); f(x.y); f(x.z); }
  __device__ void q(float4 x) { f(x.x); f(x.y); f(x.z); f(x.w); }
  __device__ void fq(FaceQ x) { f(x.sep); u(x.face); }
  __device__ void eq(const EdgeQ& x) { f(x.sep); v(x.axis); v(x.a0); v(x.a1); v(x.b0); v(x.b1); u(x.id); }
};
struct JobR {
  uint32_t w[NJOB_WORDS];
  uint32_t n = 2u;
  __device__ explicit JobR(const uint4* p) {
#pragma unroll
    for (uint32_t k = 0; k < NJOB_WORDS / 4u; k++) {
      uint4 x = p[k];
      w[4u * k] = x.x; w[4u * k + 1u] = x.y; w[4u * k + 2u] = x.z; w[4u * k + 3u] = x.w;
    }
  }
  __device__ uint32_t u() { return w[n++]; }
  __device__ float f() { return __uint_as_float(w[n++]); }
  __device__ f3 v() { float x = f(), y = f(), z = f(); return mf3(x, y, z); }
  __device__ float4 q() { float x = f(), y = f(), z = f(), ww = f(); return make_float4(x, y, z, ww); }
  __device__ FaceQ fq() { float sp = f(); uint32_t fc = u(); return FaceQ{sp, fc}; }
  __device__ EdgeQ eq() {
    EdgeQ e;
    e.sep = f(); e.axis = v(); e.a0 = v(); e.a1 = v(); e.b0 = v(); e.b1 = v(); e.id = u();
    return e;
  }
};

// Warp-aggregated counter increment: the lanes that reach it together and share `label` (the
// counter's scene) take consecutive slots with one atomic by their first lane. Works in divergent
// code (the coalesced group of the calling lanes).
SD uint32_t warp_agg_inc(uint32_t* ctr, uint32_t label) {
  namespace cg = cooperative_groups;
  cg::coalesced_group g = cg::coalesced_threads();
  cg::coalesced_group same = cg::labeled_partition(g, label);
  uint32_t base = 0u;
  if (same.thread_rank() == 0u) base = atomicAdd(ctr, same.size());
  return same.shfl(base, 0u) + same.thread_rank();
}

// Per-warp shared scratch of the edge query: the Gauss-map arcs of up to EDGE_MAX edges of each hull.
constexpr uint32_t EDGE_MAX = 32u;
constexpr uint32_t EDGE_SCRATCH = 2u * 9u * EDGE_MAX;  // floats per warp

struct Narrow {
  const SceneDev& S;
  uint32_t lane;
  const BatchDev* B;  // job list of the batch
  uint32_t scene;
  float* ew;          // this warp's edge scratch in shared memory (k_narrow), or null
  __device__ Narrow(const SceneDev& s, const BatchDev* b, uint32_t sc, float* edge_scratch = nullptr)
      : S(s), lane(threadIdx.x & 31u), B(b), scene(sc), ew(edge_scratch) {}

  // Appends a job (lane 0 of k_narrow). Each pair adds at most one, so the list holds pair_cap.
  __device__ void defer(uint32_t kind, JobW& j) const {
    uint32_t slot = warp_agg_inc(B->pair_count + 1, 0u);
    if (slot >= B->pair_cap) { atomicCAS(B->error, 0u, (uint32_t)ERR_JOB_CAPACITY); return; }
    j.w[0] = kind;
    j.w[1] = scene;
    uint4* dst = B->jobs + (size_t)slot * (NJOB_WORDS / 4u);
    for (uint32_t k = 0; 4u * k < j.n; k++) dst[k] = make_uint4(j.w[4u * k], j.w[4u * k + 1u], j.w[4u * k + 2u], j.w[4u * k + 3u]);
  }
  __device__ void defer_capsule(uint32_t c, uint32_t h, f3 pc, float4 qc, f3 wp, float4 wq, f3 wc, f3 wh, f3 nh,
                                float thresh) const {
    JobW j;
    j.u(c); j.u(h); j.v(pc); j.q(qc); j.v(wp); j.q(wq); j.v(wc); j.v(wh); j.v(nh); j.f(thresh);
    defer(J_CAPSULE, j);
  }
  __device__ void defer_segface(uint32_t hs, uint32_t ps, uint32_t h, uint32_t f, f3 e0, f3 e1, float r, f3 wp,
                                float4 wq, float thresh, bool flip) const {
    JobW j;
    j.u(hs); j.u(ps); j.u(h); j.u(f); j.v(e0); j.v(e1); j.f(r); j.v(wp); j.q(wq); j.f(thresh); j.u(flip ? 1u : 0u);
    defer(J_SEGFACE, j);
  }
  __device__ void defer_sat(uint32_t sa, uint32_t sb, uint32_t ha, uint32_t hb, f3 pa, float4 qa, float4 rBA, f3 tBA,
                            float thresh, FaceQ fa, FaceQ fb, const EdgeQ& eq) const {
    JobW j;
    j.u(sa); j.u(sb); j.u(ha); j.u(hb); j.v(pa); j.q(qa); j.q(rBA); j.v(tBA); j.f(thresh); j.fq(fa); j.fq(fb); j.eq(eq);
    defer(J_SAT, j);
  }
  // Runs one job (k_narrow_jobs, one per thread).
  __device__ void run_job(JobR& r) const {
    const uint32_t kind = r.w[0];
    if (kind == J_PLANE_CONVEX || kind == J_PLANE || kind == J_PRIM) {
      uint32_t sa = r.u(), sb = r.u();
      f3 pa = r.v(); float4 qa = r.q(); f3 pb = r.v(); float4 qb = r.q(); float thresh = r.f();
      if (kind == J_PLANE_CONVEX) plane_convex(sa, sb, pa, qa, pb, qb, thresh);
      else if (kind == J_PLANE) plane_contacts(sa, sb, pa, qa, pb, qb, thresh);
      else prim_prim(sa, sb, pa, qa, pb, qb, thresh);
    } else if (kind == J_CAPSULE) {
      uint32_t c = r.u(), h = r.u();
      f3 pc = r.v(); float4 qc = r.q(); f3 wp = r.v(); float4 wq = r.q(); f3 wc = r.v(); f3 wh = r.v(); f3 nh = r.v();
      float thresh = r.f();
      capsule_generic(c, h, pc, qc, wp, wq, wc, wh, nh, thresh);
    } else if (kind == J_SEGFACE) {
      uint32_t hs = r.u(), ps = r.u(), h = r.u(), f = r.u();
      f3 e0 = r.v(); f3 e1 = r.v(); float rad = r.f(); f3 wp = r.v(); float4 wq = r.q(); float thresh = r.f();
      bool flip = r.u() != 0u;
      seg_on_face(hs, ps, h, f, e0, e1, rad, wp, wq, thresh, flip);
    } else if (kind == J_SAT || kind == J_MPR) {
      uint32_t sa = r.u(), sb = r.u(), ha = r.u(), hb = r.u();
      f3 pa = r.v(); float4 qa = r.q(); float4 rBA = r.q(); f3 tBA = r.v(); float thresh = r.f();
      if (kind == J_SAT) {
        FaceQ fa = r.fq(), fb = r.fq();
        EdgeQ eq = r.eq();
        sat_generic(sa, sb, ha, hb, pa, qa, rBA, tBA, thresh, fa, fb, eq);
      } else {
        f3 n = r.v();
        mpr_generic(sa, sb, ha, hb, pa, qa, rBA, tBA, thresh, n);
      }
    }
  }

  __device__ f3 hv(uint32_t h, uint32_t i) const { return v3(S.sf[S.SF_VERTS + S.su[S.SU_HULL + h * 4u] + i]); }
  __device__ uint32_t hnv(uint32_t h) const { return S.su[S.SU_HULL + h * 4u + 1u]; }
  __device__ uint32_t hfo(uint32_t h) const { return S.su[S.SU_HULL + h * 4u + 2u]; }
  __device__ uint32_t hnf(uint32_t h) const { return S.su[S.SU_HULL + h * 4u + 3u]; }
  __device__ float4 fplane(uint32_t f) const { return S.sf[S.SF_FPLANE + f]; }
  __device__ uint32_t fstart(uint32_t f) const { return S.su[S.SU_FACE + f * 2u]; }
  __device__ uint32_t fcount(uint32_t f) const { return S.su[S.SU_FACE + f * 2u + 1u]; }
  __device__ uint32_t fvert(uint32_t k) const { return S.su[S.SU_FV + k]; }
  __device__ uint32_t hne(uint32_t h) const { return S.su[S.SU_HEDGE + h * 2u + 1u]; }
  __device__ uint4 hedge(uint32_t h, uint32_t k) const {
    RO<uint32_t> e = S.su + S.SU_EDGE + (S.su[S.SU_HEDGE + h * 2u] + k) * 4u;
    return make_uint4(e[0], e[1], e[2], e[3]);
  }
  __device__ float4 shp(uint32_t s, uint32_t k) const { return S.sf[S.SF_SHAPE + s * 7u + k]; }
  __device__ uint32_t geo_type(uint32_t s) const { return f2u(shp(s, 6).x); }
  __device__ uint32_t body_kind(int b) const { return f2u(S.sf[S.SF_BODY + (uint32_t)b * 8u].y); }

  // --- warp-cooperative queries ---
  __device__ __noinline__ FaceQ face_query(uint32_t ha, uint32_t hb, float4 rq, f3 t) const {
    FaceQ best{-1e30f, 0u};
    uint32_t fo = hfo(ha), nf = hnf(ha), nv = hnv(hb);
    for (uint32_t f = lane; f < nf; f += 32u) {
      float4 pl = fplane(fo + f);
      f3 nb = qinv(rq, v3(pl));
      float m = 1e30f;
      for (uint32_t v = 0; v < nv; v++) m = fmn(m, dot(nb, hv(hb, v)));
      float s = (m + dot(v3(pl), t)) - pl.w;
      if (s > best.sep) best = FaceQ{s, f};
    }
    uint32_t w = best_lane(best.sep, true);
    return FaceQ{__shfl_sync(0xffffffffu, best.sep, w), __shfl_sync(0xffffffffu, best.face, w)};
  }
  __device__ float support_min(uint32_t h, f3 n) const {
    float m = 1e30f;
    for (uint32_t v = 0; v < hnv(h); v++) m = fmn(m, dot(n, hv(h, v)));
    return m;
  }
  __device__ float support_max(uint32_t h, f3 n) const {
    float m = -1e30f;
    for (uint32_t v = 0; v < hnv(h); v++) m = fmx(m, dot(n, hv(h, v)));
    return m;
  }
  __device__ __noinline__ EdgeQ edge_query_strided(uint32_t ha, uint32_t hb, float4 rq, f3 t) const {
    EdgeQ best{-1e30f, sp3(0), sp3(0), sp3(0), sp3(0), sp3(0), 0u};
    uint32_t foa = hfo(ha), fob = hfo(hb);
    f3 cena = v3(S.sf[S.SF_HAABB + ha * 2u]);
    f3 cenb = qrot(rq, v3(S.sf[S.SF_HAABB + hb * 2u])) + t;
    uint32_t nea = hne(ha), neb = hne(hb);
    for (uint32_t k = lane; k < nea * neb; k += 32u) {
      uint4 ea_ = hedge(ha, k / neb), eb_ = hedge(hb, k % neb);
      f3 a = v3(fplane(foa + ea_.z)), b = v3(fplane(foa + ea_.w));
      f3 c = -qrot(rq, v3(fplane(fob + eb_.z))), d = -qrot(rq, v3(fplane(fob + eb_.w)));
      f3 bxa = cross(b, a), dxc = cross(d, c);
      float cba = dot(c, bxa), dba = dot(d, bxa), adc = dot(a, dxc), bdc = dot(b, dxc);
      if (cba * dba > 1e-3f || adc * bdc > 1e-3f || cba * bdc < -1e-3f) continue;
      f3 a0 = hv(ha, ea_.x), a1 = hv(ha, ea_.y);
      f3 ea = a1 - a0;
      f3 b0 = qrot(rq, hv(hb, eb_.x)) + t, b1 = qrot(rq, hv(hb, eb_.y)) + t;
      f3 ax = cross(ea, b1 - b0);
      float l = len(ax);
      if (l < (1e-6f * len(ea)) * len(b1 - b0)) continue;
      ax = ax / l;
      if (dot(ax, cenb - cena) < 0.0f) ax = -ax;
      float amax = support_max(ha, ax);
      float bmin = dot(ax, t) + support_min(hb, qinv(rq, ax));
      float s = bmin - amax;
      float tol = 1e-4f + 1e-3f * (len(ea) + len(b1 - b0));
      if (dot(ax, a0) < amax - tol || dot(ax, a1) < amax - tol || dot(ax, b0) > bmin + tol || dot(ax, b1) > bmin + tol)
        continue;
      if (s > best.sep) best = EdgeQ{s, ax, a0, a1, b0, b1, (ea_.x << 24u) ^ (ea_.y << 16u) ^ (eb_.x << 8u) ^ eb_.y};
    }
    uint32_t w = best_lane(best.sep, true);
    EdgeQ r;
    r.sep = __shfl_sync(0xffffffffu, best.sep, w);
    r.axis = shfl3(best.axis, w); r.a0 = shfl3(best.a0, w); r.a1 = shfl3(best.a1, w);
    r.b0 = shfl3(best.b0, w); r.b1 = shfl3(best.b1, w);
    r.id = __shfl_sync(0xffffffffu, best.id, w);
    return r;
  }
  // Edge-pair axes (wgsl.js edge query). The lane-strided scan (pair k on lane k mod 32, pairs in
  // increasing k, the first maximum per lane, then the lowest lane among equal maxima) recomputes
  // both edges' Gauss-map arcs for every pair and runs the support scans of the few pairs that
  // pass the Gauss-map test one lane at a time. Here each edge's arcs (its two face normals and
  // their cross product; B's negated and rotated into A's frame) are computed once, into the
  // warp's shared scratch; pass 1 runs the test over all pairs, 32 per round, from the scratch,
  // keeping each round's ballot in a register; pass 2 hands the surviving pairs to the lanes in
  // order, so the support scans run side by side. Every value is computed by the same operations,
  // and the winner is the same pair: the largest separation, ties broken by the strided scan's
  // order (the lowest k mod 32, then the lowest k). Hulls with more than EDGE_MAX edges or 256
  // edge pairs use the strided scan.
  static constexpr uint32_t EDGE_ROUNDS = 8u;
  __device__ __noinline__ EdgeQ edge_query(uint32_t ha, uint32_t hb, float4 rq, f3 t) const {
    const uint32_t nea = hne(ha), neb = hne(hb), n = nea * neb;
    if (ew == nullptr || n > 32u * EDGE_ROUNDS || nea > EDGE_MAX || neb > EDGE_MAX) return edge_query_strided(ha, hb, rq, t);
    if (n == 0u) return EdgeQ{-1e30f, sp3(0), sp3(0), sp3(0), sp3(0), sp3(0), 0u};
    float* EA = ew;                    // [component][edge]: a, b, b x a
    float* EB = ew + 9u * EDGE_MAX;    // c, d, d x c
    if (lane < nea) {
      const uint32_t foa = hfo(ha);
      const uint4 e = hedge(ha, lane);
      const f3 a = v3(fplane(foa + e.z)), b = v3(fplane(foa + e.w));
      const f3 bxa = cross(b, a);
      const float w[9] = {a.x, a.y, a.z, b.x, b.y, b.z, bxa.x, bxa.y, bxa.z};
#pragma unroll
      for (uint32_t c = 0; c < 9u; c++) EA[c * EDGE_MAX + lane] = w[c];
    }
    if (lane < neb) {
      const uint32_t fob = hfo(hb);
      const uint4 e = hedge(hb, lane);
      const f3 c = -qrot(rq, v3(fplane(fob + e.z))), d = -qrot(rq, v3(fplane(fob + e.w)));
      const f3 dxc = cross(d, c);
      const float w[9] = {c.x, c.y, c.z, d.x, d.y, d.z, dxc.x, dxc.y, dxc.z};
#pragma unroll
      for (uint32_t k = 0; k < 9u; k++) EB[k * EDGE_MAX + lane] = w[k];
    }
    __syncwarp();
    uint32_t pass[EDGE_ROUNDS];
    uint32_t total = 0u;
    uint32_t ia = lane / neb, ib = lane % neb;  // pair k = 32 r + lane: A's edge k / neb, B's edge k % neb
    const uint32_t step_a = 32u / neb, step_b = 32u % neb;
#pragma unroll
    for (uint32_t r = 0; r < EDGE_ROUNDS; r++) {
      const uint32_t k = r * 32u + lane;
      if (r * 32u < n) {
        bool meet = false;
        if (k < n) {
          const f3 a = mf3(EA[ia], EA[EDGE_MAX + ia], EA[2u * EDGE_MAX + ia]);
          const f3 b = mf3(EA[3u * EDGE_MAX + ia], EA[4u * EDGE_MAX + ia], EA[5u * EDGE_MAX + ia]);
          const f3 bxa = mf3(EA[6u * EDGE_MAX + ia], EA[7u * EDGE_MAX + ia], EA[8u * EDGE_MAX + ia]);
          const f3 c = mf3(EB[ib], EB[EDGE_MAX + ib], EB[2u * EDGE_MAX + ib]);
          const f3 d = mf3(EB[3u * EDGE_MAX + ib], EB[4u * EDGE_MAX + ib], EB[5u * EDGE_MAX + ib]);
          const f3 dxc = mf3(EB[6u * EDGE_MAX + ib], EB[7u * EDGE_MAX + ib], EB[8u * EDGE_MAX + ib]);
          const float cba = dot(c, bxa), dba = dot(d, bxa), adc = dot(a, dxc), bdc = dot(b, dxc);
          meet = !(cba * dba > 1e-3f || adc * bdc > 1e-3f || cba * bdc < -1e-3f);
        }
        pass[r] = __ballot_sync(0xffffffffu, meet);
      } else {
        pass[r] = 0u;
      }
      total += __popc(pass[r]);
      ia += step_a;
      ib += step_b;
      if (ib >= neb) { ib -= neb; ia++; }
    }
    __syncwarp();  // the scratch is free for the next pair once every lane has read it
    EdgeQ best{-1e30f, sp3(0), sp3(0), sp3(0), sp3(0), sp3(0), 0u};
    uint32_t bkey = 0xffffffffu;
    const f3 cena = v3(S.sf[S.SF_HAABB + ha * 2u]);
    const f3 cenb = qrot(rq, v3(S.sf[S.SF_HAABB + hb * 2u])) + t;
    for (uint32_t j = lane; j < total; j += 32u) {
      uint32_t rem = j, k = 0u;
#pragma unroll
      for (uint32_t r = 0; r < EDGE_ROUNDS; r++) {
        const uint32_t c = __popc(pass[r]);
        if (rem < c) {  // the rem-th set bit of this round's ballot
          uint32_t m = pass[r];
          for (uint32_t i = 0; i < rem; i++) m &= m - 1u;
          k = r * 32u + (uint32_t)(__ffs(m) - 1);
          break;
        }
        rem -= c;
      }
      uint4 ea_ = hedge(ha, k / neb), eb_ = hedge(hb, k % neb);
      f3 a0 = hv(ha, ea_.x), a1 = hv(ha, ea_.y);
      f3 ea = a1 - a0;
      f3 b0 = qrot(rq, hv(hb, eb_.x)) + t, b1 = qrot(rq, hv(hb, eb_.y)) + t;
      f3 ax = cross(ea, b1 - b0);
      float l = len(ax);
      if (l < (1e-6f * len(ea)) * len(b1 - b0)) continue;
      ax = ax / l;
      if (dot(ax, cenb - cena) < 0.0f) ax = -ax;
      float amax = support_max(ha, ax);
      float bmin = dot(ax, t) + support_min(hb, qinv(rq, ax));
      float s = bmin - amax;
      float tol = 1e-4f + 1e-3f * (len(ea) + len(b1 - b0));
      if (dot(ax, a0) < amax - tol || dot(ax, a1) < amax - tol || dot(ax, b0) > bmin + tol || dot(ax, b1) > bmin + tol)
        continue;
      const uint32_t key = ((k & 31u) << 8u) | (k >> 5u);
      if (s > -1e30f && (s > best.sep || (s == best.sep && key < bkey))) {
        best = EdgeQ{s, ax, a0, a1, b0, b1, (ea_.x << 24u) ^ (ea_.y << 16u) ^ (eb_.x << 8u) ^ eb_.y};
        bkey = key;
      }
    }
    float bv = best.sep;
    uint32_t bk = bkey, w = lane;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      const float ov = __shfl_xor_sync(0xffffffffu, bv, o);
      const uint32_t ok = __shfl_xor_sync(0xffffffffu, bk, o), ow = __shfl_xor_sync(0xffffffffu, w, o);
      if (ov > bv || (ov == bv && (ok < bk || (ok == bk && ow < w)))) { bv = ov; bk = ok; w = ow; }
    }
    EdgeQ r;
    r.sep = __shfl_sync(0xffffffffu, best.sep, w);
    r.axis = shfl3(best.axis, w); r.a0 = shfl3(best.a0, w); r.a1 = shfl3(best.a1, w);
    r.b0 = shfl3(best.b0, w); r.b1 = shfl3(best.b1, w);
    r.id = __shfl_sync(0xffffffffu, best.id, w);
    return r;
  }
  // Support point of hull h along d: per-lane strided scan, then the first lane with the maximum.
  __device__ f3 sup_lane(uint32_t h, f3 d) const {
    float best = -1e30f;
    f3 bp = sp3(0.0f);
    uint32_t nv = hnv(h);
    for (uint32_t v = lane; v < nv; v += 32u) {
      f3 x = hv(h, v);
      float s = dot(d, x);
      if (s > best) { best = s; bp = x; }
    }
    uint32_t w = best_lane(best, true);
    return shfl3(bp, w);
  }
  __device__ f3 sup_md(uint32_t ha, uint32_t hb, float4 rq, f3 t, float r, f3 d) const {
    f3 sb = qrot(rq, sup_lane(hb, qinv(rq, d))) + t;
    f3 sa = sup_lane(ha, -d);
    return (sb - sa) + (2.0f * r) * nrm(d);
  }
  // MPR (wgsl.js:342-389), every lane computes the same values.
  __device__ float4 mpr(uint32_t ha, uint32_t hb, float4 rq, f3 t, float r) const {
    const float4 none = make_float4(0.0f, 0.0f, 1.0f, -1.0f);
    f3 v0 = (qrot(rq, v3(S.sf[S.SF_HAABB + hb * 2u])) + t) - v3(S.sf[S.SF_HAABB + ha * 2u]);
    if (dot(v0, v0) < 1e-14f) v0 = mf3(1e-5f, 0.0f, 0.0f);
    f3 n = -v0;
    f3 v1 = sup_md(ha, hb, rq, t, r, n);
    if (dot(v1, n) <= 0.0f) return none;
    n = cross(v1, v0);
    if (dot(n, n) < 1e-14f) { f3 nn = nrm(v1 - v0); return mf4(nn, dot(v1, nn)); }
    f3 v2 = sup_md(ha, hb, rq, t, r, n);
    if (dot(v2, n) <= 0.0f) return none;
    n = cross(v1 - v0, v2 - v0);
    if (dot(n, v0) > 0.0f) { f3 tmp = v1; v1 = v2; v2 = tmp; n = -n; }
    f3 w3 = sp3(0.0f);
    bool found = false;
    for (uint32_t i = 0; i < 32u; i++) {
      w3 = sup_md(ha, hb, rq, t, r, n);
      if (dot(w3, n) <= 0.0f) return none;
      if (dot(cross(v1, w3), v0) < 0.0f) { v2 = w3; n = cross(v1 - v0, w3 - v0); continue; }
      if (dot(cross(w3, v2), v0) < 0.0f) { v1 = w3; n = cross(w3 - v0, v2 - v0); continue; }
      found = true;
      break;
    }
    if (!found) return none;
    for (uint32_t i = 0; i < 32u; i++) {
      n = cross(v2 - v1, w3 - v1);
      float ln = len(n);
      if (ln < 1e-12f) break;
      n = n / ln;
      if (dot(n, v1 - v0) < 0.0f) n = -n;
      f3 w4 = sup_md(ha, hb, rq, t, r, n);
      float d1 = dot(n, v1);
      if (dot(w4, n) - d1 < 1e-6f || i == 31u) {
        if (d1 < 0.0f) return none;
        return mf4(n, d1);
      }
      if (dot(w4, n) < 0.0f) return none;
      f3 c = cross(w4, v0);
      if (dot(v1, c) > 0.0f) { if (dot(v2, c) > 0.0f) v1 = w4; else w3 = w4; }
      else { if (dot(w3, c) > 0.0f) v2 = w4; else v1 = w4; }
    }
    float d1 = dot(n, v1);
    if (d1 < 0.0f) return none;
    return mf4(n, d1);
  }
  __device__ FaceQ face_query_seg(uint32_t h, f3 e0, f3 e1, float r) const {
    FaceQ best{-1e30f, 0u};
    uint32_t fo = hfo(h);
    for (uint32_t f = lane; f < hnf(h); f += 32u) {
      float4 pl = fplane(fo + f);
      float s = (fmn(dot(v3(pl), e0), dot(v3(pl), e1)) - pl.w) - r;
      if (s > best.sep) best = FaceQ{s, f};
    }
    uint32_t w = best_lane(best.sep, true);
    return FaceQ{__shfl_sync(0xffffffffu, best.sep, w), __shfl_sync(0xffffffffu, best.face, w)};
  }
  __device__ bool seg_hits_hull(uint32_t h, f3 e0, f3 e1) const {
    float t0 = 0.0f, t1 = 1.0f;
    for (uint32_t f = 0; f < hnf(h); f++) {
      float4 pl = fplane(hfo(h) + f);
      float d0 = dot(v3(pl), e0) - pl.w, d1 = dot(v3(pl), e1) - pl.w;
      if (d0 > 0.0f && d1 > 0.0f) return false;
      if (d0 > 0.0f) t0 = fmx(t0, d0 / (d0 - d1));
      else if (d1 > 0.0f) t1 = fmn(t1, d0 / (d0 - d1));
    }
    return t0 <= t1;
  }
  static __device__ void closest_seg(f3 a0, f3 a1, f3 b0, f3 b1, f3 out[2]) {
    f3 d1 = a1 - a0, d2 = b1 - b0, r = a0 - b0;
    float a = dot(d1, d1), e = dot(d2, d2), f = dot(d2, r);
    float s = 0.0f, t = 0.0f;
    if (a <= 1e-12f && e <= 1e-12f) { out[0] = a0; out[1] = b0; return; }
    if (a <= 1e-12f) {
      t = clmp(f / e, 0.0f, 1.0f);
    } else {
      float c = dot(d1, r);
      if (e <= 1e-12f) {
        s = clmp(-c / a, 0.0f, 1.0f);
      } else {
        float b = dot(d1, d2), den = a * e - b * b;
        if (den > 1e-12f) s = clmp((b * f - c * e) / den, 0.0f, 1.0f);
        t = (b * s + f) / e;
        if (t < 0.0f) { t = 0.0f; s = clmp(-c / a, 0.0f, 1.0f); }
        else if (t > 1.0f) { t = 1.0f; s = clmp((b - c) / a, 0.0f, 1.0f); }
      }
    }
    out[0] = a0 + d1 * s;
    out[1] = b0 + d2 * t;
  }
  __device__ SegQ seg_hull_query(uint32_t h, f3 e0, f3 e1) const {
    SegQ best{1e30f, sp3(0), sp3(0), 0u, 1u};
    uint32_t fo = hfo(h);
    for (uint32_t f = lane; f < hnf(h); f += 32u) {
      float4 pl = fplane(fo + f);
      uint32_t sr = fstart(fo + f), cr = fcount(fo + f);
      bool in0 = dot(v3(pl), e0) > pl.w, in1 = dot(v3(pl), e1) > pl.w;
      for (uint32_t k = 0; k < cr; k++) {
        f3 r0 = hv(h, fvert(sr + k)), r1 = hv(h, fvert(sr + (k + 1u) % cr));
        f3 out = cross(r1 - r0, v3(pl));
        if (dot(e0 - r0, out) > 0.0f) in0 = false;
        if (dot(e1 - r0, out) > 0.0f) in1 = false;
        f3 c[2];
        closest_seg(e0, e1, r0, r1, c);
        float d2 = dot(c[0] - c[1], c[0] - c[1]);
        if (d2 < best.d2) best = SegQ{d2, c[0], c[1], f, 1u};
      }
      if (in0) { float sd = dot(v3(pl), e0) - pl.w; if (sd * sd <= best.d2 * 1.0001f) best = SegQ{sd * sd, e0, e0 - v3(pl) * sd, f, 0u}; }
      if (in1) { float sd = dot(v3(pl), e1) - pl.w; if (sd * sd <= best.d2 * 1.0001f) best = SegQ{sd * sd, e1, e1 - v3(pl) * sd, f, 0u}; }
    }
    uint32_t w = best_lane(best.d2, false);
    SegQ r;
    r.d2 = __shfl_sync(0xffffffffu, best.d2, w);
    r.ps = shfl3(best.ps, w); r.ph = shfl3(best.ph, w);
    r.face = __shfl_sync(0xffffffffu, best.face, w);
    r.kind = __shfl_sync(0xffffffffu, best.kind, w);
    return r;
  }

  // --- lane-0 work ---
  static __device__ float combine(float a, float b, uint32_t mode) {
    if (mode == 1u) return fmn(a, b);
    if (mode == 2u) return a * b;
    if (mode == 3u) return fmx(a, b);
    return 0.5f * (a + b);
  }
  // emit (wgsl.js:269-307)
  __device__ __noinline__ void emit(uint32_t sa, uint32_t sb, f3 p, f3 n, float phi, uint32_t key) const {
    float4 A0 = shp(sa, 0), B0 = shp(sb, 0);
    int ba = f2i(A0.x), bb = f2i(B0.x);
    float4 ma = shp(sa, 4), mb = shp(sb, 4);
    float mu = combine(A0.z, B0.z, S.FRICTION_COMBINE);
    bool art_c = (ba >= 0 && body_kind(ba) >= 2u) || (bb >= 0 && body_kind(bb) >= 2u);
    float mt = 0.0f, mr = 0.0f;
    if (art_c) {
      if (S.ANG_ART == 1u) {
        mt = combine(ma.y, mb.y, S.FRICTION_COMBINE);
        mr = combine(ma.z, mb.z, S.FRICTION_COMBINE);
      }
    } else {
      mt = fmx(ma.w >= 4.0f ? ma.y : 0.0f, mb.w >= 4.0f ? mb.y : 0.0f);
      mr = fmx(ma.w >= 6.0f ? ma.z : 0.0f, mb.w >= 6.0f ? mb.z : 0.0f);
      if (S.F_FR_MUT >= 0.0f) mt = S.F_FR_MUT;
      if (S.F_FR_MUR >= 0.0f) mr = S.F_FR_MUR;
    }
    float trd = art_c ? fmx(shp(sa, 3).w, shp(sb, 3).w) : 0.0f;
    f3 mat = mf3(combine(clmp(ma.x, 0.0f, 1.0f), clmp(mb.x, 0.0f, 1.0f), S.RESTITUTION_COMBINE), mt, mr);
    int a = ba, b = bb;
    f3 nn = n;
    float smx = A0.z, smy = B0.z;
    if (a > b) { a = bb; b = ba; nn = -n; float tt = smx; smx = smy; smy = tt; }
    uint32_t k = warp_agg_inc(&S.counters[1], S.scene_index);
    if (k >= S.MAXC) return;
    float4* rec = S.craw + k * 5u;
    S.craw[S.MAXC * 5u + k] = make_float4(smx, smy, 0.0f, 0.0f);
    rec[0] = mf4(p, phi);
    rec[1] = mf4(nn, mu);
    rec[2] = make_float4((float)a, (float)b, (float)(key & 0xffffu), (float)(key >> 16u));
    rec[3] = mf4(mat, trd);
    float4 A5 = shp(sa, 5), B5 = shp(sb, 5);
    float kc = (A5.x > 0.0f && B5.x > 0.0f) ? (A5.x * B5.x) / (A5.x + B5.x) : 0.0f;
    float ga = A5.z, gb = B5.z;
    if (ba > bb) { float tt = ga; ga = gb; gb = tt; }
    rec[4] = make_float4(kc, A5.y + B5.y, ga, gb);
  }
  static __device__ void sphere_sphere(f3 p1, float r1, f3 p2, float r2, float4 out[2]) {
    f3 dv = p2 - p1;
    float l = len(dv);
    f3 n = l == 0.0f ? mf3(1.0f, 0.0f, 0.0f) : dv / l;
    float d = l - (r1 + r2);
    out[0] = mf4(p1 + n * (r1 + 0.5f * d), d);
    out[1] = mf4(n, 0.0f);
  }
  __device__ __noinline__ void prim_prim(uint32_t sa, uint32_t sb, f3 pa, float4 qa, f3 pb, float4 qb, float thresh) const {
    float4 A = shp(sa, 6), Bq = shp(sb, 6);
    f3 ua = qrot(qa, mf3(0.0f, 0.0f, A.z)), ub = qrot(qb, mf3(0.0f, 0.0f, Bq.z));
    uint32_t base = mix32(sa * 7919u + sb * 104729u);
    float4 c[2][2];
    c[0][0] = c[0][1] = c[1][0] = c[1][1] = make_float4(0, 0, 0, 0);
    uint32_t nc = 1u;
    if (f2u(A.x) == GT_SPHERE) {
      f3 a = pb - ub, ab = (pb + ub) - a;
      sphere_sphere(pa, A.y, a + clmp(dot(pa - a, ab) / (dot(ab, ab) + 1e-6f), 0.0f, 1.0f) * ab, Bq.y, c[0]);
    } else {
      f3 dif = pa - pb;
      float ma = dot(ua, ua), mb = -dot(ua, ub), mc = dot(ub, ub);
      float u = -dot(ua, dif), v = dot(ub, dif);
      float det = ma * mc - mb * mb;
      if (fabsf(det) >= 1e-15f) {
        float inv_det = 1.0f / det;
        float x1 = (mc * u - mb * v) * inv_det, x2 = (ma * v - mb * u) * inv_det;
        if (x1 > 1.0f) { x1 = 1.0f; x2 = (v - mb) / mc; } else if (x1 < -1.0f) { x1 = -1.0f; x2 = (v + mb) / mc; }
        if (x2 > 1.0f) { x2 = 1.0f; x1 = clmp((u - mb) / ma, -1.0f, 1.0f); }
        else if (x2 < -1.0f) { x2 = -1.0f; x1 = clmp((u + mb) / ma, -1.0f, 1.0f); }
        sphere_sphere(pa + ua * x1, A.y, pb + ub * x2, Bq.y, c[0]);
      } else {
        sphere_sphere(pa + ua, A.y, pb + ub * clmp((v - mb) / mc, -1.0f, 1.0f), Bq.y, c[0]);
        sphere_sphere(pa - ua, A.y, pb + ub * clmp((v + mb) / mc, -1.0f, 1.0f), Bq.y, c[1]);
        c[1][1] = c[0][1];
        nc = 2u;
      }
    }
    for (uint32_t i = 0; i < nc; i++)
      if (c[i][0].w <= thresh) emit(sa, sb, v3(c[i][0]), v3(c[0][1]), c[i][0].w, mix32(base ^ (i * 977u + 13u)));
  }
  __device__ __noinline__ void plane_contacts(uint32_t pl, uint32_t os, f3 pp, float4 pq, f3 op, float4 oq, float thresh) const {
    f3 n = qrot(pq, mf3(0.0f, 0.0f, 1.0f));
    uint32_t sa = pl, sb = os;
    uint32_t base = mix32(sa * 7919u + sb * 104729u);
    float4 g = shp(os, 6);
    uint32_t gt = f2u(g.x);
    float d[4] = {1e30f, 1e30f, 1e30f, 1e30f};
    f3 x[4];
    for (int k = 0; k < 4; k++) x[k] = sp3(0.0f);
    uint32_t nc = 0u;
    if (gt == GT_SPHERE || gt == GT_CAPSULE) {
      f3 u = qrot(oq, mf3(0.0f, 0.0f, g.z));
      uint32_t cnt = gt == GT_SPHERE ? 1u : 2u;
      for (uint32_t i = 0; i < cnt; i++) {
        f3 e = op + (i == 1u ? -u : u);
        d[i] = dot(n, e - pp) - g.y;
        x[i] = e - n * (g.y + 0.5f * d[i]);
      }
      nc = cnt;
    } else if (gt == GT_BOX) {
      float cd0 = dot(op - pp, n);
      uint32_t worst = 0u;
      m3 rot = qmat(oq);
      for (uint32_t i = 0; i < 8u; i++) {
        f3 c = mul(rot, mf3((i & 1u) ? g.y : -g.y, (i & 2u) ? g.z : -g.z, (i & 4u) ? g.w : -g.w));
        float cd = cd0 + dot(n, c);
        if (cd > thresh) continue;
        f3 cp = (c + op) - (0.5f * n) * cd;
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
      f3 ax = qrot(oq, mf3(0.0f, 0.0f, 1.0f));
      float dna = dot(n, ax);
      if (dna > 0.0f) { ax = -ax; dna = -dna; }
      f3 cap = op + ax * g.z;
      f3 pa = -n + ax * dna;
      float l2 = dot(pa, pa);
      bool has = l2 > 1e-10f;
      if (has) pa = pa * (1.0f / sqrtf(l2));
      bool flat = -dna >= 0.9238795325112867f;
      f3 pf = sp3(0.0f);
      if (flat || !has) {
        f3 rf = mf3(1.0f, 0.0f, 0.0f);
        if (fabsf(dot(ax, rf)) > 0.9f) rf = mf3(0.0f, 1.0f, 0.0f);
        pf = nrm(rf - ax * dot(ax, rf));
      }
      f3 dp = has ? pa : pf;
      f3 dpt = cap + dp * g.y;
      d[0] = dot(dpt - pp, n);
      x[0] = dpt - n * (d[0] * 0.5f);
      nc = 1u;
      float mt = 0.01f * fmx(g.y, g.z);
      f3 cand[3];
      uint32_t ncand = 0u;
      if (flat) {
        f3 u = pf * g.y, v = cross(ax, pf) * g.y;
        cand[0] = cap + u;
        cand[1] = (cap - 0.5f * u) + 0.8660254f * v;
        cand[2] = (cap - 0.5f * u) - 0.8660254f * v;
        ncand = 3u;
      } else {
        f3 u = dp * g.y, v = cross(ax, dp) * g.y;
        cand[0] = (op - ax * g.z) + u;
        float dpv = dot((cap + v) - pp, n), dnv = dot((cap - v) - pp, n);
        cand[1] = dpv <= dnv ? cap + v : cap - v;
        ncand = 2u;
      }
      for (uint32_t k = 0; k < ncand; k++) {
        float dk = dot(cand[k] - pp, n);
        f3 pk = cand[k] - n * (dk * 0.5f);
        if (nc < 4u && dot(pk - x[0], pk - x[0]) > mt * mt) { d[nc] = dk; x[nc] = pk; nc++; }
      }
    }
    for (uint32_t i = 0; i < nc; i++)
      if (d[i] <= thresh) emit(sa, sb, x[i], n, d[i], mix32(base ^ (i + 7u)));
  }
  __device__ __noinline__ void seg_on_face(uint32_t hs, uint32_t ps, uint32_t h, uint32_t f, f3 e0, f3 e1, float r, f3 wp,
                              float4 wq, float thresh, bool flip) const {
    float4 pl = fplane(hfo(h) + f);
    float t0 = 0.0f, t1 = 1.0f;
    uint32_t sr = fstart(hfo(h) + f), cr = fcount(hfo(h) + f);
    for (uint32_t k = 0; k < cr; k++) {
      f3 r0 = hv(h, fvert(sr + k)), r1 = hv(h, fvert(sr + (k + 1u) % cr));
      f3 out = cross(r1 - r0, v3(pl));
      float d0 = dot(e0 - r0, out), d1 = dot(e1 - r0, out);
      if (d0 > 0.0f && d1 > 0.0f) { t0 = 2.0f; break; }
      if (d0 > 0.0f) t0 = fmx(t0, d0 / (d0 - d1));
      if (d1 > 0.0f) t1 = fmn(t1, d0 / (d0 - d1));
    }
    float ts[2] = {t0, t1};
    uint32_t n = 2u;
    if (t0 > t1) { ts[0] = dot(v3(pl), e0) <= dot(v3(pl), e1) ? 0.0f : 1.0f; n = 1u; }
    else if (t1 - t0 < 1e-4f || len(e1 - e0) < 1e-7f) n = 1u;
    f3 nw = qrot(wq, v3(pl));
    uint32_t sa = flip ? ps : hs, sb = flip ? hs : ps;
    uint32_t base = mix32(sa * 7919u + sb * 104729u);
    for (uint32_t i = 0; i < n; i++) {
      f3 x = e0 + (e1 - e0) * ts[i];
      float sd = dot(v3(pl), x) - pl.w;
      float phi = sd - r;
      if (phi > thresh) continue;
      f3 mid = x - v3(pl) * (0.5f * (sd + r));
      emit(sa, sb, wp + qrot(wq, mid), flip ? -nw : nw, phi, mix32(base ^ (f * 131u + i * 7u + 3u)));
    }
  }

  // Newton's generic convex manifold (wgsl.js:644-977).
  __device__ Geo geo(uint32_t s) const {
    float4 g = shp(s, 6);
    Geo r{f2u(g.x), mf3(g.y, g.z, g.w), f2u(shp(s, 0).y)};
    if (r.t == GT_SPHERE || r.t == GT_CAPSULE) r.s.x = 1e-4f;
    return r;
  }
  __device__ f3 gsup(const Geo& g, f3 d) const {
    if (g.t == GT_BOX) {
      float th = 1e-10f * fmx(fabsf(d.x), fmx(fabsf(d.y), fabsf(d.z)));
      return mf3(d.x >= -th ? g.s.x : -g.s.x, d.y >= -th ? g.s.y : -g.s.y, d.z >= -th ? g.s.z : -g.s.z);
    }
    if (g.t == GT_SPHERE || g.t == GT_CAPSULE) {
      float l2 = dot(d, d);
      f3 p = (l2 > 1e-12f ? d * rsq(l2) : mf3(1.0f, 0.0f, 0.0f)) * g.s.x;
      if (g.t == GT_CAPSULE) p.z = p.z + (d.z >= 0.0f ? g.s.y : -g.s.y);
      return p;
    }
    if (g.t == GT_CYL) {
      f3 xy = mf3(d.x, d.y, 0.0f);
      float l2 = dot(xy, xy);
      f3 p = l2 > 1e-12f ? (xy * rsq(l2)) * g.s.x : mf3(g.s.x, 0.0f, 0.0f);
      if (d.z > 0.0f) p.z = g.s.y; else if (d.z < 0.0f) p.z = -g.s.y;
      return p;
    }
    float best = -1e10f;
    f3 bp = sp3(0.0f);
    for (uint32_t v = 0; v < hnv(g.h); v++) {
      f3 x = hv(g.h, v);
      float s = dot(x, d);
      if (s > best) { best = s; bp = x; }
    }
    return bp;
  }
  __device__ f3 fsup(const Geo& g, f3 d, f3 n) const {
    f3 p = gsup(g, d);
    if ((g.t == GT_CAPSULE || (g.t == GT_CYL && g.s.z == 0.0f)) && fabsf(n.z) <= 1e-4f) {
      f3 rad = nrm(mf3(n.x, n.y, 0.0f)) * g.s.x;
      p = mf3(rad.x, rad.y, d.z >= 0.0f ? g.s.y : -g.s.y);
    }
    return p;
  }
  __device__ bool plane_supporting(const Geo& g, f3 dir, float d) const {
    float off = dot(dir, gsup(g, dir)) + d;
    return off * off <= (MEPS * MEPS) * dot(dir, dir);
  }
  struct Trk { f3 r, p, n; float a2; bool np; };
  static __device__ Trk trk_add(Trk t, f3 x, uint32_t id, bool chk) {
    Trk o = t;
    if (id == 0u) { o.r = x; o.a2 = 0.0f; o.n = sp3(0.0f); o.np = false; }
    else if (id == 1u) { o.p = x; }
    else {
      if (chk && o.a2 > 0.0f) { float off = dot(o.n, x - o.r); if (off * off > (MEPS * MEPS) * o.a2) o.np = true; }
      f3 c = cross(o.p - o.r, x - o.r);
      float a2 = dot(c, c);
      if (a2 > o.a2) { o.a2 = a2; o.n = c; }
      o.p = x;
    }
    return o;
  }
  static __device__ bool trk_anchor(const Trk& t, f3 x) {
    float off = dot(t.n, x - t.r);
    return !t.np && off * off <= (MEPS * MEPS) * t.a2;
  }
  struct Proj { float d; f3 n; };
  static __device__ f3 line_proj_n(f3 dir, f3 rn) {
    f3 nn = cross(cross(dir, rn), dir);
    float l = len(nn);
    return l > 1e-12f ? nn * (1.0f / l) : rn;
  }
  static __device__ void make_proj(const Trk& ta, f3 pa, const Trk& tb, f3 pb, f3 n, Proj out[2]) {
    Proj A{0.0f, sp3(0.0f)}, Bp{0.0f, sp3(0.0f)};
    if (ta.a2 == 0.0f && tb.a2 == 0.0f) {
      A.n = line_proj_n(ta.p - ta.r, n); A.d = -dot(0.5f * (ta.r + ta.p), A.n);
      Bp.n = line_proj_n(tb.p - tb.r, n); Bp.d = -dot(0.5f * (tb.r + tb.p), Bp.n);
      out[0] = A; out[1] = Bp;
      return;
    }
    if (ta.a2 > 0.0f) { A.n = ta.n * (1.0f / sqrtf(fmx(1e-12f, ta.a2))); A.d = -dot(pa, A.n); }
    if (tb.a2 > 0.0f) { Bp.n = tb.n * (1.0f / sqrtf(fmx(1e-12f, tb.a2))); Bp.d = -dot(pb, Bp.n); }
    if (ta.a2 == 0.0f) { A.n = line_proj_n(ta.p - ta.r, Bp.n); A.d = -dot(0.5f * (ta.r + ta.p), A.n); }
    if (tb.a2 == 0.0f) { Bp.n = line_proj_n(tb.p - tb.r, A.n); Bp.d = -dot(0.5f * (tb.r + tb.p), Bp.n); }
    out[0] = A; out[1] = Bp;
  }
  static __device__ f3 proj_on(const Proj& pr, f3 x, f3 n) {
    float den = dot(n, pr.n);
    if (fabsf(den) < 1e-12f) return x;
    return x + n * (-(dot(x, pr.n) + pr.d) / den);
  }
  static __device__ float sarea(f2 a, f2 b, f2 q) { return (b.x - a.x) * (q.y - a.y) - (b.y - a.y) * (q.x - a.x); }
  static __device__ bool add_nodup(f2* arr, int cnt, f2 v) {
    if (cnt > 0) { f2 d = arr[0] - v; if (dot(d, d) < MEPS * MEPS) return false; }
    if (cnt > 1) { f2 d = arr[cnt - 1] - v; if (dot(d, d) < MEPS * MEPS) return false; }
    arr[cnt] = v;
    return true;
  }
  static __device__ int trim_in_place(f2 s0, f2 s1, f2* lp, int cnt0) {
    int cnt = cnt0;
    if (cnt < 3) return cnt;
    f2 ia = mf2(0, 0), ib = mf2(0, 0);
    int ca = -1, cb = -1;
    bool keep = false;
    bool prev_out = sarea(s0, s1, lp[0]) <= 0.0f;
    for (int i = 0; i < cnt; i++) {
      int nx = (i + 1) % cnt;
      bool out = sarea(s0, s1, lp[nx]) <= 0.0f;
      if (out != prev_out) {
        f2 a = lp[i], b = lp[nx];
        float sa = sarea(s0, s1, a), sb = sarea(s0, s1, b);
        float t = fabsf(sa) / fabsf(sa - sb);
        f2 x = (1.0f - t) * a + t * b;
        if (ca < 0) { ca = i; keep = !prev_out; ia = x; } else { cb = i; ib = x; }
      }
      prev_out = out;
    }
    if (ca >= 0 && cb >= 0) {
      int li = -1, ncnt = cnt, i = 0;
      for (int guard = 0; guard < 24 && i < cnt; guard++) {
        if (keep) { li++; lp[li] = lp[i]; }
        if (i == ca || i == cb) {
          f2 pt = i == ca ? ia : ib;
          if (li == i && !keep) {
            li++;
            for (int k = min(ncnt, 9); k > li; k--) lp[k] = lp[k - 1];
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
  static __device__ int trim_all(f2* tp, int tn, f2* lp, int ln) {
    if (tn <= 1) return min(1, ln);
    if (tn == 2 || ln == 2) {
      f2 st = lp[0], en = lp[1];
      if (tn == 2) { st = tp[0]; en = tp[1]; }
      f2 dir = en - st;
      float l2 = dot(dir, dir);
      if (l2 <= MEPS * MEPS) return 0;
      float lo = 0.0f, hi = 1.0f;
      if (tn == 2 && ln == 2) {
        f2 os = lp[0], od = lp[1] - os;
        float cr = dir.x * od.y - dir.y * od.x;
        if (fabsf(cr) > 1e-6f * sqrtf(l2 * dot(od, od))) return 0;
        float t0 = dot(os - st, dir) / l2, t1 = dot(lp[1] - st, dir) / l2;
        lo = fmx(lo, fmn(t0, t1));
        hi = fmn(hi, fmx(t0, t1));
      } else {
        bool useLoop = tn == 2;
        int pc = useLoop ? ln : tn;
        for (int i = 0; i < pc; i++) {
          f2 e0 = useLoop ? lp[i] : tp[i];
          f2 e1 = useLoop ? lp[(i + 1) % pc] : tp[(i + 1) % pc];
          float a = sarea(e0, e1, st), b = sarea(e0, e1, en);
          if (a < 0.0f && b < 0.0f) return 0;
          if (a < 0.0f) lo = fmx(lo, a / (a - b));
          else if (b < 0.0f) hi = fmn(hi, a / (a - b));
        }
      }
      if (hi <= lo) return 0;
      lp[0] = st + lo * dir;
      lp[1] = st + hi * dir;
      return 2;
    }
    int c = ln;
    f2 t0 = tp[0];
    for (int i = 0; i < tn; i++) {
      f2 s1 = (i == tn - 1) ? t0 : tp[i + 1];
      c = trim_in_place(tp[i], s1, lp, c);
    }
    return c;
  }
  static __device__ int remove_zero_edges(f2* lp, int cnt) {
    if (cnt < 2) return 0;
    int w = 0;
    for (int r = 1; r < cnt; r++) {
      f2 d = lp[r] - lp[w];
      if (dot(d, d) > MEPS * MEPS) { w++; lp[w] = lp[r]; }
    }
    int n = w + 1;
    if (w > 0) { f2 d = lp[w] - lp[0]; if (dot(d, d) < MEPS * MEPS) n = w; }
    return n < 2 ? 0 : n;
  }
  static __device__ void calipers(const f2* h, int n, int out[4]) {
    int p1 = 0, p3 = 1;
    f2 d0 = h[0] - h[1];
    float md = dot(d0, d0);
    const float te = 1e-3f;
    int j = 1;
    for (int i = 0; i < n; i++) {
      f2 hi = h[i], hi1 = h[(i + 1) % n];
      for (int g = 0; g < 16; g++) {
        if (sarea(hi, hi1, h[(j + 1) % n]) > sarea(hi, hi1, h[j])) j = (j + 1) % n; else break;
      }
      f2 hj = h[j];
      f2 a = hi - hj;
      if (dot(a, a) > md * (1.0f + te)) { md = dot(a, a); p1 = i; p3 = j; }
      f2 b = hi1 - hj;
      if (dot(b, b) > md * (1.0f + te)) { md = dot(b, b); p1 = (i + 1) % n; p3 = j; }
    }
    int p2 = 0, p4 = 0;
    float m1 = 0.0f, m2 = 0.0f;
    f2 q1 = h[p1], q3 = h[p3];
    for (int i = 0; i < n; i++) {
      float ar = sarea(q1, q3, h[i]);
      if (ar > m1 * (1.0f + te)) { m1 = ar; p2 = i; }
      else if (-ar > m2 * (1.0f + te)) { m2 = -ar; p4 = i; }
    }
    out[0] = p1; out[1] = p2; out[2] = p3; out[3] = p4;
  }
  static __device__ void onb(f3 n, f3 out[2]) {
    if (n.z < 0.0f) {
      float a = 1.0f / (1.0f - n.z), b = (n.x * n.y) * a;
      out[0] = mf3(1.0f - (n.x * n.x) * a, -b, n.x);
      out[1] = mf3(b, (n.y * n.y) * a - 1.0f, -n.y);
      return;
    }
    float a = 1.0f / (1.0f + n.z), b = (-n.x * n.y) * a;
    out[0] = mf3(1.0f - (n.x * n.x) * a, b, -n.x);
    out[1] = mf3(b, 1.0f - (n.y * n.y) * a, -n.y);
  }
  static __device__ bool planar_geo(const Geo& g) { return g.t == GT_BOX || g.t == GT_CONVEX; }
  static __device__ bool is_discrete(uint32_t t) { return t == GT_BOX || t == GT_CONVEX || t == GT_PLANE; }

  // build_manifold + gen_run (wgsl.js:875-977)
  __device__ __noinline__ void gen_run(uint32_t sa, uint32_t sb, const Geo& ga, const Geo& gb, f3 pa, float4 qa, float4 rq, f3 rt,
                          f3 wa, f3 wb, f3 n, float thresh) const {
    f3 mp[5];
    float md[5];
    uint32_t mn = 0u;
    {
      f3 fna = n;
      if (ga.t == GT_CYL && gb.t == GT_CYL && ga.s.z == 0.0f && gb.s.z == 0.0f) {
        f3 axb = qrot(rq, mf3(0.0f, 0.0f, 1.0f));
        f3 ro = mf3(rt.x, rt.y, 0.0f);
        if (axb.x * axb.x + axb.y * axb.y <= 1e-12f && fabsf(rt.z) < ga.s.y + gb.s.y && dot(ro, ro) > 1e-20f) {
          f3 rn = nrm(ro);
          if (dot(n, rn) >= COS_TILT) fna = rn;
        }
      }
      f3 tb[2];
      onb(n, tb);
      bool pla = planar_geo(ga), plb = planar_geo(gb);
      f3 center = 0.5f * (wa + wb);
      f2 A[10], Bv[10];
      for (int k = 0; k < 10; k++) { A[k] = mf2(0, 0); Bv[k] = mf2(0, 0); }
      int ac = 0, bc = 0;
      Trk ta{sp3(0), sp3(0), sp3(0), 0.0f, false};
      Trk tbk = ta;
      f3 lnb = qinv(rq, -n), lfb = qinv(rq, -fna);
      f3 lta = qinv(rq, -tb[0]), ltb = qinv(rq, -tb[1]);
      for (uint32_t e = 0; e < 5u; e++) {
        f2 cs = mf2(PENTX[e], PENTY[e]) * SIN_TILT;
        f3 x = fsup(ga, (n * COS_TILT + cs.x * tb[0]) + cs.y * tb[1], fna);
        f3 xa = x - center;
        if (add_nodup(A, ac, mf2(dot(tb[0], xa), dot(tb[1], xa)))) { ac++; ta = trk_add(ta, x, (uint32_t)(ac - 1), pla); }
        f3 y = qrot(rq, fsup(gb, (lnb * COS_TILT + cs.x * lta) + cs.y * ltb, lfb)) + rt;
        f3 yb = y - center;
        if (add_nodup(Bv, bc, mf2(dot(tb[0], yb), dot(tb[1], yb)))) { bc++; tbk = trk_add(tbk, y, (uint32_t)(bc - 1), plb); }
      }
      uint32_t cnt = 0u;
      float ndot = 0.0f;
      if (ac >= 2 && bc >= 2 && !(pla && !trk_anchor(ta, wa)) && !(plb && !trk_anchor(tbk, wb))) {
        Proj pr[2];
        make_proj(ta, wa, tbk, wb, n, pr);
        bool ok = fabsf(dot(n, pr[0].n)) >= COS_TILT && fabsf(dot(n, pr[1].n)) >= COS_TILT;
        if (ok && pla && (ta.a2 == 0.0f || dot(cross(n, pr[0].n), cross(n, pr[0].n)) > 0.0f)) {
          bool flip = dot(pr[0].n, n) < 0.0f;
          ok = plane_supporting(ga, flip ? -pr[0].n : pr[0].n, flip ? -pr[0].d : pr[0].d);
        }
        if (ok && plb && (tbk.a2 == 0.0f || dot(cross(n, pr[1].n), cross(n, pr[1].n)) > 0.0f)) {
          bool flip = dot(pr[1].n, n) > 0.0f;
          f3 db = flip ? -pr[1].n : pr[1].n;
          float dd = flip ? -pr[1].d : pr[1].d;
          ok = plane_supporting(gb, qinv(rq, db), dd + dot(db, rt));
        }
        if (ok) {
          ndot = fabsf(dot(pr[0].n, pr[1].n));
          int lc = remove_zero_edges(Bv, trim_all(A, ac, Bv, bc));
          if (lc > 1) {
            int idx[4] = {0, 1, 2, 3};
            if (lc > 4) { calipers(Bv, lc, idx); lc = 4; }
            for (int i = 0; i < lc; i++) {
              f2 q = Bv[idx[i]];
              f3 plp = (q.x * tb[0] + q.y * tb[1]) + center;
              f3 a = proj_on(pr[0], plp, n), b = proj_on(pr[1], plp, n);
              mp[cnt] = 0.5f * (a + b);
              md[cnt] = dot(b - a, n);
              cnt++;
            }
          } else {
            ndot = 0.0f;
          }
        }
      }
      if (ndot < COS_DEEP || cnt == 0u) {
        mp[cnt] = 0.5f * (wa + wb);
        md[cnt] = dot(wb - wa, n);
        cnt++;
      }
      mn = cnt;
    }
    f3 nw = qrot(qa, n);
    float ra = (ga.t == GT_SPHERE || ga.t == GT_CAPSULE) ? shp(sa, 6).y : 0.0f;
    float rb = (gb.t == GT_SPHERE || gb.t == GT_CAPSULE) ? shp(sb, 6).y : 0.0f;
    bool axA = ga.t == GT_CYL || ga.t == GT_CONE, axB = gb.t == GT_CYL || gb.t == GT_CONE;
    bool roll = false;
    f3 rpos = sp3(0.0f), rn = sp3(0.0f);
    if ((is_discrete(ga.t) && axB) || (is_discrete(gb.t) && axA)) {
      bool onB = is_discrete(ga.t) && axB;
      f3 ax = onB ? qrot(qmul(qa, rq), mf3(0.0f, 0.0f, 1.0f)) : qrot(qa, mf3(0.0f, 0.0f, 1.0f));
      f3 an = onB ? nw : -nw;
      if (fabsf(dot(ax, an)) <= SIN_TILT) {
        roll = true;
        rpos = onB ? pa + qrot(qa, rt) : pa;
        rn = nrm(cross(ax, an));
      }
    }
    uint32_t base = mix32(sa * 7919u + sb * 104729u);
    for (uint32_t i = 0; i < mn; i++) {
      f3 p = ((pa + qrot(qa, mp[i])) + nw * (0.5f * ra)) - nw * (0.5f * rb);
      float d = (md[i] - ra) - rb;
      if (roll) p = p - rn * dot(p - rpos, rn);
      if (d > thresh) continue;
      emit(sa, sb, p, nw, d, mix32(base ^ (i * 0x9e3779b1u + 0x51u)));
    }
  }
  __device__ float hull_out(uint32_t h, f3 x) const {
    float m = -1e30f;
    for (uint32_t f = 0; f < hnf(h); f++) { float4 pl = fplane(hfo(h) + f); m = fmx(m, dot(v3(pl), x) - pl.w); }
    return m;
  }
  __device__ f3 ray_face(uint32_t h, f3 o, f3 n, f3 s) const {
    float best = -2.0f;
    float4 pl = make_float4(0, 0, 0, 0);
    for (uint32_t f = 0; f < hnf(h); f++) {
      float4 q = fplane(hfo(h) + f);
      if (dot(v3(q), n) > best) { best = dot(v3(q), n); pl = q; }
    }
    f3 x = o + n * ((pl.w - dot(v3(pl), o)) / dot(v3(pl), n));
    if (fabsf(dot(x - s, n)) > WITNESS_TOL) return o + n * dot(s - o, n);
    return x;
  }
  __device__ void sup_witness(const Geo& ga, const Geo& gb, float4 rq, f3 rt, f3 n, bool refA, f3 out[2]) const {
    f3 sA = gsup(ga, n);
    f3 lb = gsup(gb, qinv(rq, -n));
    f3 sB = qrot(rq, lb) + rt;
    f3 wb0 = ray_face(ga.h, sB, n, sA), wb1 = sB;
    f3 wa0 = sA, wa1 = qrot(rq, ray_face(gb.h, qinv(rq, sA - rt), qinv(rq, -n), lb)) + rt;
    float ob = fmx(hull_out(ga.h, wb0), hull_out(gb.h, qinv(rq, wb1 - rt)));
    float oa = fmx(hull_out(ga.h, wa0), hull_out(gb.h, qinv(rq, wa1 - rt)));
    if ((refA && !(oa < ob - 1e-6f)) || (!refA && ob < oa - 1e-6f)) { out[0] = wb0; out[1] = wb1; return; }
    out[0] = wa0; out[1] = wa1;
  }
  __device__ __noinline__ void sat_generic(uint32_t sa, uint32_t sb, uint32_t ha, uint32_t hb, f3 pa, float4 qa, float4 rBA, f3 tBA,
                              float thresh, FaceQ fa, FaceQ fb, const EdgeQ& eq) const {
    Geo ga = geo(sa), gb = geo(sb);
    if (eq.sep > fmx(fa.sep, fb.sep) + SAT_TIE) {
      f3 c[2];
      closest_seg(eq.a0, eq.a1, eq.b0, eq.b1, c);
      gen_run(sa, sb, ga, gb, pa, qa, rBA, tBA, c[0], c[1], eq.axis, thresh);
      return;
    }
    bool refA = !(fb.sep > fa.sep + SAT_TIE);
    f3 n = refA ? v3(fplane(hfo(ha) + fa.face)) : -qrot(rBA, v3(fplane(hfo(hb) + fb.face)));
    f3 w[2];
    sup_witness(ga, gb, rBA, tBA, n, refA, w);
    gen_run(sa, sb, ga, gb, pa, qa, rBA, tBA, w[0], w[1], n, thresh);
  }
  __device__ __noinline__ void plane_convex(uint32_t sa, uint32_t sb, f3 pa, float4 qa, f3 pb, float4 qb, float thresh) const {
    Geo gb = geo(sb);
    f3 nw = qrot(qa, mf3(0.0f, 0.0f, 1.0f));
    float L = 10.0f * (len(v3(S.sf[S.SF_HAABB + gb.h * 2u])) + len(v3(S.sf[S.SF_HAABB + gb.h * 2u + 1u])));
    f3 c = pb - nw * (dot(pb - pa, nw) + L);
    float4 rq = qmul(qconj(qa), qb);
    f3 rt = qinv(qa, pb - c);
    f3 n = mf3(0.0f, 0.0f, 1.0f);
    f3 wb = qrot(rq, gsup(gb, qinv(rq, -n))) + rt;
    float sep = wb.z - L;
    if (sep > thresh) return;
    gen_run(sa, sb, Geo{GT_BOX, mf3(L, L, L), 0u}, gb, c, qa, rq, rt, wb - n * sep, wb, n, thresh);
  }
  __device__ __noinline__ void capsule_generic(uint32_t c, uint32_t h, f3 pc, float4 qc, f3 wp, float4 wq, f3 wc, f3 wh, f3 nh,
                                  float thresh) const {
    if (dot(wh - wc, nh) - shp(c, 6).y > thresh) return;
    float4 rq = qmul(qconj(qc), wq);
    f3 rt = qinv(qc, wp - pc);
    gen_run(c, h, geo(c), geo(h), pc, qc, rq, rt, qrot(rq, wc) + rt, qrot(rq, wh) + rt, qrot(rq, nh), thresh);
  }
  __device__ __noinline__ void mpr_generic(uint32_t sa, uint32_t sb, uint32_t ha, uint32_t hb, f3 pa, float4 qa, float4 rBA, f3 tBA,
                              float thresh, f3 n) const {
    float alA = -2.0f;
    for (uint32_t f = 0; f < hnf(ha); f++) alA = fmx(alA, dot(v3(fplane(hfo(ha) + f)), n));
    float alB = -2.0f;
    for (uint32_t f = 0; f < hnf(hb); f++) alB = fmx(alB, -dot(qrot(rBA, v3(fplane(hfo(hb) + f))), n));
    Geo ga = geo(sa), gb = geo(sb);
    f3 w[2];
    sup_witness(ga, gb, rBA, tBA, n, alA >= alB, w);
    gen_run(sa, sb, ga, gb, pa, qa, rBA, tBA, w[0], w[1], n, thresh);
  }

  // narrow_pair (wgsl.js:1072-1195): all lanes enter; the serial paths become jobs of lane 0.
  __device__ void pair(uint32_t p0, uint32_t p1) const {
    bool swp = geo_type(p0) > geo_type(p1);
    uint32_t sa = swp ? p1 : p0, sb = swp ? p0 : p1;
    uint32_t ha = f2u(shp(sa, 0).y), hb = f2u(shp(sb, 0).y);
    f3 pa = v3(S.spos[sa]);
    float4 qa = S.srot[sa];
    f3 pb = v3(S.spos[sb]);
    float4 qb = S.srot[sb];
    float thresh = fmn(shp(sa, 0).w + shp(sb, 0).w, S.F_GAP_GATE);
    float4 rBA = qmul(qconj(qa), qb);
    f3 tBA = qinv(qa, pb - pa);
    float4 rAB = qconj(rBA);
    f3 tAB = qinv(qb, pa - pb);
    float4 ka = shp(sa, 3), kb = shp(sb, 3);
    if (ka.x == 4.0f || kb.x == 4.0f) {
      if (lane == 0u) {
        JobW j;
        j.u(sa); j.u(sb); j.v(pa); j.q(qa); j.v(pb); j.q(qb); j.f(thresh);
        defer(geo_type(sb) == GT_CONVEX ? J_PLANE_CONVEX : J_PLANE, j);
      }
      return;
    }
    if (ka.x != 0.0f && kb.x != 0.0f) {
      if (lane == 0u) {
        JobW j;
        j.u(sa); j.u(sb); j.v(pa); j.q(qa); j.v(pb); j.q(qb); j.f(thresh);
        defer(J_PRIM, j);
      }
      return;
    }
    if (ka.x != 0.0f || kb.x != 0.0f) {
      bool flip = ka.x != 0.0f;
      uint32_t hs = flip ? sb : sa, ps = flip ? sa : sb;
      uint32_t h = flip ? hb : ha;
      float4 pr = flip ? ka : kb;
      float4 rq = flip ? rAB : rBA;
      f3 rt = flip ? tAB : tBA;
      f3 u = qrot(rq, mf3(0.0f, 0.0f, pr.z));
      f3 e0 = rt - u, e1 = rt + u;
      FaceQ fq = face_query_seg(h, e0, e1, pr.y);
      if (fq.sep > thresh) return;
      f3 wp = flip ? pb : pa;
      float4 wq = flip ? qb : qa;
      if (fq.sep + pr.y > 1e-6f || (pr.x == 2.0f && !seg_hits_hull(h, e0, e1))) {
        SegQ q = seg_hull_query(h, e0, e1);
        if (lane != 0u) return;
        if (pr.x == 2.0f) {
          float d = sqrtf(q.d2);
          if (d >= 1e-9f) {
            f3 nh = (q.ph - q.ps) / d;
            defer_capsule(ps, hs, flip ? pa : pb, flip ? qa : qb, wp, wq, q.ps + nh * 1e-4f, q.ph, nh, thresh);
          }
        } else {
          float d = sqrtf(q.d2);
          float phi = d - pr.y;
          f3 n = (q.ps - q.ph) / fmx(d, 1e-9f);
          if (phi > thresh || d < 1e-9f) {
          } else if (dot(n, v3(fplane(hfo(h) + fq.face))) > 0.999f) {
            defer_segface(hs, ps, h, fq.face, e0, e1, pr.y, wp, wq, thresh, flip);
          } else {
            uint32_t sa2 = flip ? ps : hs, sb2 = flip ? hs : ps;
            f3 nw = qrot(wq, n);
            uint32_t key = mix32(mix32(sa2 * 7919u + sb2 * 104729u) ^ (q.face * 131u + q.kind * 17u + 0x9e37u));
            emit(sa2, sb2, wp + qrot(wq, q.ph + n * (0.5f * phi)), flip ? -nw : nw, phi, key);
          }
        }
        return;
      }
      if (lane != 0u) return;
      if (pr.x == 2.0f) {
        float4 pl = fplane(hfo(h) + fq.face);
        f3 x = dot(v3(pl), e0) <= dot(v3(pl), e1) ? e0 : e1;
        defer_capsule(ps, hs, flip ? pa : pb, flip ? qa : qb, wp, wq, x - v3(pl) * 1e-4f,
                      x - v3(pl) * (dot(v3(pl), x) - pl.w), -v3(pl), thresh);
      } else {
        defer_segface(hs, ps, h, fq.face, e0, e1, pr.y, wp, wq, thresh, flip);
      }
      return;
    }
    FaceQ fa = face_query(ha, hb, rBA, tBA);
    if (fa.sep > thresh) return;
    FaceQ fb = face_query(hb, ha, rAB, tAB);
    if (fb.sep > thresh) return;
    EdgeQ none{-1e30f, sp3(0), sp3(0), sp3(0), sp3(0), sp3(0), 0u};
    bool small = hnv(ha) <= 16u && hnv(hb) <= 16u;
    if (!small) {
      float4 m = mpr(ha, hb, rBA, tBA, 0.5f * thresh);
      if (lane == 0u && m.w >= 0.0f) {
        f3 n = -v3(m);
        float sep = (dot(n, tBA) + support_min(hb, qinv(rBA, n))) - support_max(ha, n);
        if (fmx(fa.sep, fb.sep) > sep + 1e-4f) {
          defer_sat(sa, sb, ha, hb, pa, qa, rBA, tBA, thresh, fa, fb, none);
        } else {
          JobW j;
          j.u(sa); j.u(sb); j.u(ha); j.u(hb); j.v(pa); j.q(qa); j.q(rBA); j.v(tBA); j.f(thresh); j.v(n);
          defer(J_MPR, j);
        }
      }
      return;
    }
    EdgeQ eq = edge_query(ha, hb, rBA, tBA);
    if (eq.sep > thresh) return;
    if (lane == 0u) defer_sat(sa, sb, ha, hb, pa, qa, rBA, tBA, thresh, fa, fb, eq);
  }
};

__global__ void __launch_bounds__(NARROW_WARPS * 32, 3) k_narrow(BatchDev B) {
  __shared__ float edge_scratch[NARROW_WARPS * EDGE_SCRATCH];
  uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5u;
  uint32_t nwarps = (gridDim.x * blockDim.x) >> 5u;
  uint32_t total = *B.pair_count;
  float* ew = edge_scratch + (threadIdx.x >> 5u) * EDGE_SCRATCH;
  for (uint32_t g = warp; g < total; g += nwarps) {
    uint4 pr = B.pairs[g];
    Narrow N(B.scenes[pr.x], &B, pr.x, ew);
    N.pair(pr.y, pr.z);
    __syncwarp();
  }
}

// The jobs k_narrow deferred, one per thread (grid-stride over blocks of NARROW_JOB_THREADS
// jobs). Each block first orders its jobs by kind (a counting sort in shared memory), so a warp's
// threads mostly run the same routine. The order within a kind follows shared-memory atomics;
// jobs only append contacts, whose order the canonical sort fixes.
__global__ void __launch_bounds__(NARROW_JOB_THREADS, 4) k_narrow_jobs(BatchDev B) {
  constexpr uint32_t KINDS = 8u;  // job kinds are 1..7
  __shared__ uint32_t start[KINDS];
  __shared__ uint32_t order[NARROW_JOB_THREADS];
  const uint32_t total = min(B.pair_count[1], B.pair_cap);
  const uint32_t tid = threadIdx.x;
  for (uint32_t base = blockIdx.x * NARROW_JOB_THREADS; base < total; base += gridDim.x * NARROW_JOB_THREADS) {
    const uint32_t j = base + tid;
    if (tid < KINDS) start[tid] = 0u;
    __syncthreads();
    uint32_t kind = 0u, pos = 0u;
    if (j < total) {
      kind = min(B.jobs[(size_t)j * (NJOB_WORDS / 4u)].x, KINDS - 1u);
      pos = atomicAdd(&start[kind], 1u);
    }
    __syncthreads();
    if (tid == 0u) {
      uint32_t acc = 0u;
      for (uint32_t k = 0; k < KINDS; k++) { uint32_t c = start[k]; start[k] = acc; acc += c; }
    }
    __syncthreads();
    if (j < total) order[start[kind] + pos] = j;
    __syncthreads();
    if (tid < min(NARROW_JOB_THREADS, total - base)) {
      JobR r(B.jobs + (size_t)order[tid] * (NJOB_WORDS / 4u));
      const uint32_t scene = r.w[1];
      Narrow N(B.scenes[scene], &B, scene);
      N.run_job(r);
    }
    __syncthreads();
  }
}

// --------------------------------------------------------------------------------------------
// Canonical contact sort (wgsl.js:3899-3982): key (pair, feature key, point-bit hash, raw index).
// Scenes whose padded keys fit the shared array sort there, one block per scene, with a bitonic
// network; larger scenes are left to the device-wide radix sort below.
__global__ void __launch_bounds__(SORT_THREADS) k_csort(BatchDev B, uint32_t smem_keys) {
  extern __shared__ uint4 sk[];
  const uint32_t scene = B.order[blockIdx.x];
  if (B.active[scene] == 0u) return;
  const SceneDev& S = B.scenes[scene];
  uint32_t nc = min(S.counters[1], S.MAXC);
  if (nc == 0u) return;
  uint32_t n2 = 1u;
  while (n2 < nc) n2 <<= 1u;
  if (n2 > smem_keys) return;  // the radix sort's scene
  uint4* keys = sk;
  for (uint32_t q = threadIdx.x; q < n2; q += blockDim.x)
    keys[q] = q < nc ? contact_key(S.craw, q) : make_uint4(0xffffffffu, 0xffffffffu, 0xffffffffu, 0xffffffffu);
  __syncthreads();
  for (uint32_t k = 2u; k <= n2; k <<= 1u) {
    for (uint32_t j = k >> 1u; j > 0u; j >>= 1u) {
      for (uint32_t q = threadIdx.x; q < n2 / 2u; q += blockDim.x) {
        uint32_t i = 2u * j * (q / j) + q % j, l = i + j;
        uint4 a = keys[i], b = keys[l];
        if (key_gt(a, b) == ((i & k) == 0u)) { keys[i] = b; keys[l] = a; }
      }
      __syncthreads();
    }
  }
  for (uint32_t i = threadIdx.x; i < nc; i += blockDim.x) {
    uint32_t c = keys[i].w;
#pragma unroll
    for (uint32_t q = 0; q < 5u; q++) S.con[i * 5u + q] = S.craw[c * 5u + q];
    S.con[S.MAXC * 5u + i] = S.craw[S.MAXC * 5u + c];
  }
}

// --- device-wide radix sort of one large scene's contact keys ----------------------------------
// Digit d (0 = least significant) of a key: byte d % 4 of word d / 4 counted from the hash.
SD uint32_t rs_digit(const uint4& k, uint32_t d) {
  const uint32_t w = d >> 2u;
  const uint32_t word = w == 0u ? k.z : (w == 1u ? k.y : k.x);
  return (word >> (8u * (d & 3u))) & 255u;
}
// The scene's contact count; `here` when this sort (not k_csort's shared array) handles it.
SD uint32_t rs_count(const BatchDev& B, const RadixDev& R, uint32_t smem_keys, bool& here) {
  const SceneDev& S = B.scenes[R.scene];
  const uint32_t nc = min(S.counters[1], S.MAXC);
  uint32_t n2 = 1u;
  while (n2 < nc) n2 <<= 1u;
  here = B.active[R.scene] != 0u && n2 > smem_keys;
  return nc;
}
// Whether digit d leaves the order as it is (one bucket holds every key), decided by the whole
// block from the key histogram (RS_THREADS == 256 buckets, one per thread).
SD bool rs_trivial(const RadixDev& R, uint32_t d, uint32_t nc) {
  return __syncthreads_or(R.hist[d * 256u + threadIdx.x] == nc) != 0;
}
// Index of the buffer that holds the keys before digit d: the non-trivial digits below d flip it.
SD uint32_t rs_source(const RadixDev& R, uint32_t d, uint32_t nc) {
  uint32_t cur = 0u;
  for (uint32_t e = 0; e < d; e++) cur ^= rs_trivial(R, e, nc) ? 0u : 1u;
  return cur;
}

__global__ void k_rsort_clear(RadixDev R) {
  const uint32_t n = RS_DIGITS * R.tiles * 256u;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) R.status[i] = 0u;
  if (blockIdx.x == 0u) {
    for (uint32_t i = threadIdx.x; i < RS_DIGITS * 256u; i += blockDim.x) R.hist[i] = 0u;
    if (threadIdx.x < RS_DIGITS) R.ctr[threadIdx.x] = 0u;
  }
}

// Keys of one tile into keys[0], and their bucket counts for every digit into the histogram.
__global__ void __launch_bounds__(RS_THREADS) k_rsort_init(BatchDev B, RadixDev R, uint32_t smem_keys) {
  __shared__ uint32_t h[RS_DIGITS * 256u];
  bool here;
  const uint32_t nc = rs_count(B, R, smem_keys, here);
  if (!here || blockIdx.x * RS_TILE >= nc) return;
  const SceneDev& S = B.scenes[R.scene];
  for (uint32_t i = threadIdx.x; i < RS_DIGITS * 256u; i += RS_THREADS) h[i] = 0u;
  __syncthreads();
  for (uint32_t r = 0; r < RS_ITEMS; r++) {
    const uint32_t i = blockIdx.x * RS_TILE + r * RS_THREADS + threadIdx.x;
    if (i >= nc) break;
    const uint4 k = contact_key(S.craw, i);
    R.keys[0][i] = k;
#pragma unroll
    for (uint32_t d = 0; d < RS_DIGITS; d++) atomicAdd(&h[d * 256u + rs_digit(k, d)], 1u);
  }
  __syncthreads();
  for (uint32_t i = threadIdx.x; i < RS_DIGITS * 256u; i += RS_THREADS)
    if (h[i]) atomicAdd(&R.hist[i], h[i]);
}

// One stable pass over digit d. A block takes the next tile ticket, ranks its keys within the tile
// (tile order = raw order within the tile: round, then warp, then lane), publishes its bucket
// counts, sums the counts of the tiles before it (decoupled look-back, bounded polls) and
// scatters every key to bucket start + preceding tiles' keys in that bucket + its rank.
__global__ void __launch_bounds__(RS_THREADS) k_rsort_pass(BatchDev B, RadixDev R, uint32_t d, uint32_t smem_keys) {
  __shared__ uint32_t warp_cnt[RS_THREADS / 32u][256];
  __shared__ uint32_t warp_off[RS_THREADS / 32u][256];
  __shared__ uint32_t tile_cnt[256];
  __shared__ uint32_t dst_off[256];
  __shared__ uint32_t wsum[RS_THREADS / 32u];
  __shared__ uint32_t ticket;
  bool here;
  const uint32_t nc = rs_count(B, R, smem_keys, here);
  const uint32_t ntiles = (nc + RS_TILE - 1u) / RS_TILE;
  if (!here || blockIdx.x >= ntiles) return;
  const uint32_t tid = threadIdx.x, lane = tid & 31u, warp = tid >> 5u;
  const uint32_t cur = rs_source(R, d, nc);
  if (rs_trivial(R, d, nc)) return;
  if (tid == 0u) ticket = atomicAdd(&R.ctr[d], 1u);
  for (uint32_t w = 0; w < RS_THREADS / 32u; w++) warp_cnt[w][tid] = 0u;
  tile_cnt[tid] = 0u;
  __syncthreads();
  const uint32_t t = ticket;
  if (t >= ntiles) {  // more tickets than tiles: the counters were not cleared
    if (tid == 0u) atomicCAS(B.error, 0u, (uint32_t)ERR_SORT_TIMEOUT);
    return;
  }
  const uint4* src = cur ? R.keys[1] : R.keys[0];
  uint4* dst = cur ? R.keys[0] : R.keys[1];
  uint4 k[RS_ITEMS];
  uint32_t rank[RS_ITEMS];
  const uint32_t lt = (1u << lane) - 1u;
#pragma unroll
  for (uint32_t r = 0; r < RS_ITEMS; r++) {
    const uint32_t i = t * RS_TILE + r * RS_THREADS + tid;
    const bool valid = i < nc;
    k[r] = valid ? src[i] : make_uint4(0u, 0u, 0u, 0u);
    const uint32_t dig = valid ? rs_digit(k[r], d) : 256u;
    const uint32_t peers = __match_any_sync(0xffffffffu, dig);
    const uint32_t below = __popc(peers & lt);
    if (valid && below == 0u) warp_cnt[warp][dig] = __popc(peers);
    __syncthreads();
    // Bucket tid: offsets of each warp's keys after the earlier rounds and warps.
    uint32_t run = tile_cnt[tid];
#pragma unroll
    for (uint32_t w = 0; w < RS_THREADS / 32u; w++) {
      const uint32_t c = warp_cnt[w][tid];
      warp_off[w][tid] = run;
      run += c;
      warp_cnt[w][tid] = 0u;
    }
    tile_cnt[tid] = run;
    __syncthreads();
    rank[r] = valid ? warp_off[warp][dig] + below : 0u;
  }
  // Publish this tile's counts (tile 0: already the inclusive prefix), then look back.
  const uint32_t cnt = tile_cnt[tid];
  volatile uint32_t* st = R.status + ((size_t)d * R.tiles) * 256u;
  st[(size_t)t * 256u + tid] = (t == 0u ? 2u << 30 : 1u << 30) | cnt;
  uint32_t excl = 0u;
  if (t > 0u) {
    uint32_t p = t - 1u;
    for (;;) {
      uint32_t w = 0u, polls = 0u;
      do { w = st[(size_t)p * 256u + tid]; } while ((w >> 30) == 0u && ++polls < RS_SPIN_LIMIT);
      if ((w >> 30) == 0u) {
        atomicCAS(B.error, 0u, (uint32_t)ERR_SORT_TIMEOUT);
        break;
      }
      excl += w & 0x3fffffffu;
      if ((w >> 30) == 2u || p == 0u) break;
      p--;
    }
    st[(size_t)t * 256u + tid] = (2u << 30) | (excl + cnt);
  }
  // Bucket starts over all keys (exclusive scan of the digit's histogram).
  const uint32_t hv = R.hist[d * 256u + tid];
  uint32_t incl = hv;
#pragma unroll
  for (uint32_t o = 1; o < 32u; o <<= 1u) {
    const uint32_t v = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += v;
  }
  if (lane == 31u) wsum[warp] = incl;
  __syncthreads();
  uint32_t wbase = 0u;
  for (uint32_t w = 0; w < warp; w++) wbase += wsum[w];
  dst_off[tid] = wbase + incl - hv + excl;
  __syncthreads();
#pragma unroll
  for (uint32_t r = 0; r < RS_ITEMS; r++) {
    const uint32_t i = t * RS_TILE + r * RS_THREADS + tid;
    if (i >= nc) continue;
    const uint32_t j = dst_off[rs_digit(k[r], d)] + rank[r];
    if (j < nc) dst[j] = k[r];
    else atomicCAS(B.error, 0u, (uint32_t)ERR_SORT_TIMEOUT);  // inconsistent counts: never write past nc
  }
}

// The records in sorted order: contact i of the output is raw contact keys[i].w.
__global__ void __launch_bounds__(RS_THREADS) k_rsort_gather(BatchDev B, RadixDev R, uint32_t smem_keys) {
  bool here;
  const uint32_t nc = rs_count(B, R, smem_keys, here);
  if (!here || blockIdx.x * RS_THREADS >= nc) return;
  const SceneDev& S = B.scenes[R.scene];
  const uint4* keys = rs_source(R, RS_DIGITS, nc) ? R.keys[1] : R.keys[0];
  for (uint32_t i = blockIdx.x * RS_THREADS + threadIdx.x; i < nc; i += gridDim.x * RS_THREADS) {
    const uint32_t c = keys[i].w;
    if (c >= nc) {
      atomicCAS(B.error, 0u, (uint32_t)ERR_SORT_TIMEOUT);
      continue;
    }
#pragma unroll
    for (uint32_t q = 0; q < 5u; q++) S.con[i * 5u + q] = S.craw[c * 5u + q];
    S.con[S.MAXC * 5u + i] = S.craw[S.MAXC * 5u + c];
  }
}

// --------------------------------------------------------------------------------------------
void launch_params(const BatchDev& b, uint32_t substep, cudaStream_t st) {
  k_params<<<(b.nscenes + 127) / 128, 128, 0, st>>>(b, substep);
}
void launch_frame_end(const BatchDev& b, cudaStream_t st) {
  k_frame_end<<<(b.nscenes + 127) / 128, 128, 0, st>>>(b);
}
// Packed joint targets -> each scene's A_TGT (one block per scene); the targets replace the
// scene's recorded trajectory from now on (sim.js:720).
__global__ void k_scatter_targets(BatchDev B, const float* packed, const uint64_t* offsets) {
  SceneDev& S = B.scenes[blockIdx.x];
  const float* src = packed + offsets[blockIdx.x];
  for (uint32_t d = threadIdx.x; d < S.ND; d += blockDim.x) S.art[S.A_TGT + d] = src[d];
  if (threadIdx.x == 0 && S.ND) S.user_targets = 1u;
}
// Each scene's body poses -> one packed array (one block per scene), COM position then quaternion.
__global__ void k_gather_poses(BatchDev B, float* packed, const uint64_t* offsets) {
  const SceneDev& S = B.scenes[blockIdx.x];
  float4* dst = reinterpret_cast<float4*>(packed + offsets[blockIdx.x]);
  for (uint32_t b = threadIdx.x; b < S.NB; b += blockDim.x) { dst[2 * b] = S.pos[b]; dst[2 * b + 1] = S.rot[b]; }
}
// One scene's body poses -> a caller's device buffer of BodyPose records (COM vec4, quaternion vec4).
__global__ void k_copy_poses(const float4* __restrict__ pos, const float4* __restrict__ rot, uint32_t nb,
                             float4* __restrict__ dst) {
  for (uint32_t b = blockIdx.x * blockDim.x + threadIdx.x; b < nb; b += gridDim.x * blockDim.x) {
    dst[2 * b] = pos[b];
    dst[2 * b + 1] = rot[b];
  }
}
void launch_copy_poses(const float4* pos, const float4* rot, uint32_t nb, float4* dst, cudaStream_t st) {
  k_copy_poses<<<std::max<uint32_t>(1u, std::min<uint32_t>((nb + 255u) / 256u, 592u)), 256, 0, st>>>(pos, rot, nb, dst);
}
void launch_scatter_targets(const BatchDev& b, const float* packed, const uint64_t* offsets, cudaStream_t st) {
  k_scatter_targets<<<b.nscenes, 128, 0, st>>>(b, packed, offsets);
}
void launch_gather_poses(const BatchDev& b, float* packed, const uint64_t* offsets, cudaStream_t st) {
  k_gather_poses<<<b.nscenes, 128, 0, st>>>(b, packed, offsets);
}
// Prepare / solve launches and their shared-memory configuration, by the batch's block size.
#define STEEL_BY_BLOCK(threads, call)         \
  switch (threads) {                          \
    case 32: call(32); break;                 \
    case 64: call(64); break;                 \
    case 256: call(256); break;               \
    case 512: call(512); break;               \
    default: call(128); break;                \
  }
// A kernel's largest dynamic shared memory is an attribute of the function for the whole process,
// not of a batch: every batch needs it at least as large as its own launches, so it only grows.
namespace {
std::mutex g_smem_mu;
std::map<std::pair<int, int>, size_t> g_smem_max;  // (kernel set, block size) -> bytes set so far
size_t grow_smem(int set, uint32_t threads, size_t bytes) {
  std::lock_guard<std::mutex> lock(g_smem_mu);
  size_t& m = g_smem_max[{set, (int)threads}];
  m = std::max(m, bytes);
  return m;
}
}  // namespace
cudaError_t configure_prepare(uint32_t threads, size_t smem_bytes) {
  cudaError_t e = cudaSuccess;
  const size_t bytes = grow_smem(0, threads, smem_bytes);
#define STEEL_CALL(N) e = configure_prepare_t<N>(bytes)
  STEEL_BY_BLOCK(threads, STEEL_CALL)
#undef STEEL_CALL
  return e;
}
cudaError_t configure_solve(uint32_t threads, size_t smem_bytes) {
  cudaError_t e = cudaSuccess;
  const size_t bytes = grow_smem(1, threads, smem_bytes);
#define STEEL_CALL(N) e = configure_solve_t<N>(bytes)
  STEEL_BY_BLOCK(threads, STEEL_CALL)
#undef STEEL_CALL
  return e;
}
void launch_prepare(const BatchDev& b, cudaStream_t st) {
#define STEEL_CALL(N) launch_prepare_t<N>(b, st)
  STEEL_BY_BLOCK(b.block_threads, STEEL_CALL)
#undef STEEL_CALL
}
void launch_solve(const BatchDev& b, cudaStream_t st) {
#define STEEL_CALL(N) launch_solve_t<N>(b, st)
  STEEL_BY_BLOCK(b.block_threads, STEEL_CALL)
#undef STEEL_CALL
}
int solve_team_blocks_per_sm(uint32_t threads, size_t smem_bytes) {
  int n = 0;
#define STEEL_CALL(N) n = solve_team_blocks_per_sm_t<N>(smem_bytes)
  STEEL_BY_BLOCK(threads, STEEL_CALL)
#undef STEEL_CALL
  return n;
}
int prepare_team_blocks_per_sm(uint32_t threads, size_t smem_bytes) {
  int n = 0;
#define STEEL_CALL(N) n = prepare_team_blocks_per_sm_t<N>(smem_bytes)
  STEEL_BY_BLOCK(threads, STEEL_CALL)
#undef STEEL_CALL
  return n;
}
#undef STEEL_BY_BLOCK
// Each scene's shared-memory staging flags (SceneDev::stage) from a packed array, one per scene.
__global__ void k_set_stage(BatchDev B, const uint32_t* stage) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < B.nscenes) B.scenes[i].stage = stage[i];
}
void launch_set_stage(const BatchDev& b, const uint32_t* stage, cudaStream_t st) {
  k_set_stage<<<(b.nscenes + 127) / 128, 128, 0, st>>>(b, stage);
}
void launch_shapes(const BatchDev& b, cudaStream_t st) {
  if (b.nshapes) k_shapes<<<(b.nshapes + 127) / 128, 128, 0, st>>>(b);
}
void launch_broad(const BatchDev& b, cudaStream_t st) {
  if (b.ntiles) k_broad<<<b.ntiles, 256, 0, st>>>(b);
}
// Resident narrowphase blocks per SM (the persistent grid is this times the SM count).
int narrow_blocks_per_sm() {
  int n = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_narrow, NARROW_WARPS * 32, 0) != cudaSuccess || n < 1) n = 1;
  return n;
}
void launch_narrow(const BatchDev& b, uint32_t narrow_blocks, cudaStream_t st) {
  k_narrow<<<narrow_blocks, NARROW_WARPS * 32, 0, st>>>(b);
  k_narrow_jobs<<<narrow_blocks * 2u, NARROW_JOB_THREADS, 0, st>>>(b);
}
cudaError_t configure_sort(size_t smem_keys) {
  const size_t bytes = grow_smem(2, SORT_THREADS, smem_keys * sizeof(uint4));
  return cudaFuncSetAttribute(k_csort, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
}
void launch_csort(const BatchDev& b, size_t smem_keys, const RadixDev* radix, uint32_t nradix, cudaStream_t st) {
  k_csort<<<b.nlaunch, SORT_THREADS, smem_keys * sizeof(uint4), st>>>(b, (uint32_t)smem_keys);
  for (uint32_t k = 0; k < nradix; k++) {
    const RadixDev& R = radix[k];
    const uint32_t sk = (uint32_t)smem_keys;
    k_rsort_clear<<<std::min<uint32_t>(R.tiles * 4u, 592u), 256, 0, st>>>(R);
    k_rsort_init<<<R.tiles, RS_THREADS, 0, st>>>(b, R, sk);
    for (uint32_t d = 0; d < RS_DIGITS; d++) k_rsort_pass<<<R.tiles, RS_THREADS, 0, st>>>(b, R, d, sk);
    k_rsort_gather<<<std::min<uint32_t>(R.tiles * RS_ITEMS, 1184u), RS_THREADS, 0, st>>>(b, R, sk);
  }
}

}  // namespace steel
