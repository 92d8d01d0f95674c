// Convex hull of a point cloud on the host, the hull SceneBuilder.addConvexHull stores for a
// hull shape (packages/steel-webgpu/src/builder.js:61-173): faces are outward planes n . x = d with
// their vertices counter-clockwise about n, coplanar triangles merged into one polygon.
//
// The method is quickhull in double precision. Its steps are the ones the reference's builder
// takes, in the same order, because the packed scene depends on the hull's vertex and face order
// (statF's hull, face and edge tables, sim.js:180-209): the same initial simplex (the lowest-x
// point, the point farthest from it, the point farthest from their line, the point farthest from
// their plane; first of equals), the same assignment of each point to the face it lies farthest
// above, the same choice of the next face (the first live face of the list with points above it)
// and apex (its farthest point), the visible region found breadth first across shared edges, new
// faces made along the horizon in the order it was found, then the coplanar flood fill and each
// polygon's boundary by a monotone chain on the plane. Only the data structures are this file's
// own: faces in an index-stable array, directed edges in a hash map, point lists as vectors.
//
// Euclidean norms are computed as the correctly rounded square root of the exactly summed squares
// (Dekker's exact products with fma, Knuth's two-sum, one Newton step on the double-double sum),
// so a norm is the nearest double to the true value except in rare near-halfway cases.
#include "hull.h"

#include <algorithm>
#include <cmath>
#include <unordered_map>

namespace steel {
namespace hull {
namespace {

struct V3 {
  double x, y, z;
};
V3 sub(const V3& a, const V3& b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
V3 add(const V3& a, const V3& b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
V3 scale(const V3& a, double s) { return {a.x * s, a.y * s, a.z * s}; }
double dot(const V3& a, const V3& b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
V3 cross(const V3& a, const V3& b) { return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }

// |a|: sum of squares as an unevaluated pair hi + lo (exact products by fma, exact sums by two-sum),
// then sqrt(hi) corrected by one Newton step on hi + lo.
double norm(const V3& a) {
  double hi = 0.0, lo = 0.0;
  for (double c : {a.x, a.y, a.z}) {
    const double p = c * c, pe = std::fma(c, c, -p);  // c^2 = p + pe exactly
    const double s = hi + p, bb = s - hi, se = (hi - (s - bb)) + (p - bb);  // hi + p = s + se exactly
    hi = s;
    lo += se + pe;
  }
  const double s = hi + lo;
  const double e = lo - (s - hi);
  if (s <= 0.0) return 0.0;
  const double r = std::sqrt(s);
  const double rem = std::fma(-r, r, s) + e;  // (s + e) - r^2
  return r + rem / (2.0 * r);
}

constexpr int64_t K = 1048576;  // directed edge (a, b) -> a * K + b

struct Face {
  int v[3];
  V3 n;
  double d;
  bool alive = false, vis = false;
  int group = -1;
  std::vector<int> out;  // points above this face, assigned to it
};

}  // namespace

bool convex_hull(const double* pts, uint32_t count, Hull& out, std::string& err) {
  // Distinct points, first occurrence kept, in input order.
  std::vector<V3> P;
  {
    struct H {
      size_t operator()(const V3& p) const {  // equal values hash alike (+0.0 for -0.0)
        const double x = p.x + 0.0, y = p.y + 0.0, z = p.z + 0.0;
        uint64_t a, b, c;
        std::memcpy(&a, &x, 8); std::memcpy(&b, &y, 8); std::memcpy(&c, &z, 8);
        return (size_t)(a * 0x9E3779B97F4A7C15ull ^ (b + 0x632BE59BD9B4E019ull) * 0xC2B2AE3D27D4EB4Full ^ c);
      }
    };
    struct E {
      bool operator()(const V3& p, const V3& q) const { return p.x == q.x && p.y == q.y && p.z == q.z; }
    };
    std::unordered_map<V3, int, H, E> seen;
    for (uint32_t i = 0; i < count; i++) {
      const V3 p{pts[3 * i], pts[3 * i + 1], pts[3 * i + 2]};
      if (seen.emplace(p, (int)P.size()).second) P.push_back(p);
    }
  }
  const int np = (int)P.size();
  if (np < 4) { err = "a convex hull needs at least 4 distinct points"; return false; }
  V3 lo{INFINITY, INFINITY, INFINITY}, hi{-INFINITY, -INFINITY, -INFINITY};
  for (const V3& p : P) {
    lo = {std::min(lo.x, p.x), std::min(lo.y, p.y), std::min(lo.z, p.z)};
    hi = {std::max(hi.x, p.x), std::max(hi.y, p.y), std::max(hi.z, p.z)};
  }
  const double eps = 1e-7 * std::max(norm(sub(hi, lo)), 1e-12);
  int i0 = 0;
  for (int i = 1; i < np; i++)
    if (P[i].x < P[i0].x) i0 = i;
  auto farthest = [&](auto dist, double* best_d) {
    int best = -1;
    double bd = -1.0;
    for (int i = 0; i < np; i++) {
      const double d = dist(P[i]);
      if (d > bd) { bd = d; best = i; }
    }
    *best_d = bd;
    return best;
  };
  double dd;
  const int i1 = farthest([&](const V3& p) { return norm(sub(p, P[i0])); }, &dd);
  const V3 e = sub(P[i1], P[i0]);
  const int i2 = farthest([&](const V3& p) { return norm(cross(e, sub(p, P[i0]))) / norm(e); }, &dd);
  if (dd <= eps) { err = "convex hull points are collinear"; return false; }
  const V3 n0 = cross(e, sub(P[i2], P[i0]));
  const int i3 = farthest([&](const V3& p) { return std::fabs(dot(n0, sub(p, P[i0]))) / norm(n0); }, &dd);
  if (dd <= eps) { err = "convex hull points are coplanar"; return false; }
  const V3 center = scale(add(add(P[i0], P[i1]), add(P[i2], P[i3])), 0.25);

  std::vector<Face> F;
  F.reserve(4 * (size_t)np);
  std::unordered_map<int64_t, int> edges;
  auto plane = [&](int a, int b, int c, V3* n, double* d) {
    V3 m = cross(sub(P[b], P[a]), sub(P[c], P[a]));
    m = scale(m, 1.0 / norm(m));
    *n = m;
    *d = dot(m, P[a]);
  };
  auto make = [&](int a, int b, int c) {
    Face f;
    f.v[0] = a; f.v[1] = b; f.v[2] = c;
    plane(a, b, c, &f.n, &f.d);
    f.alive = true;
    const int id = (int)F.size();
    F.push_back(std::move(f));
    for (int k = 0; k < 3; k++) edges[(int64_t)F[id].v[k] * K + F[id].v[(k + 1) % 3]] = id;
    return id;
  };
  auto make_oriented = [&](int a, int b, int c) {  // outward: the simplex's center below the plane
    V3 n; double d;
    plane(a, b, c, &n, &d);
    return dot(n, center) - d > 0.0 ? make(a, c, b) : make(a, b, c);
  };
  std::vector<int> faces = {make_oriented(i0, i1, i2), make_oriented(i0, i1, i3), make_oriented(i0, i2, i3),
                            make_oriented(i1, i2, i3)};
  auto assign = [&](const std::vector<int>& points, const std::vector<int>& cands) {
    for (int i : points) {
      int best = -1;
      double bd = eps;
      for (int f : cands) {
        const double d = dot(F[f].n, P[i]) - F[f].d;
        if (d > bd) { bd = d; best = f; }
      }
      if (best >= 0) F[best].out.push_back(i);
    }
  };
  {
    std::vector<int> rest;
    for (int i = 0; i < np; i++)
      if (i != i0 && i != i1 && i != i2 && i != i3) rest.push_back(i);
    assign(rest, faces);
  }
  std::vector<int> visible, orphans, fresh, next;
  std::vector<std::pair<int, int>> horizon;
  for (int guard = 0; guard < 4 * np + 16; guard++) {
    int f0 = -1;
    for (int f : faces)
      if (F[f].alive && !F[f].out.empty()) { f0 = f; break; }
    if (f0 < 0) break;
    int p = F[f0].out[0];
    double pd = -INFINITY;
    for (int i : F[f0].out) {
      const double d = dot(F[f0].n, P[i]) - F[f0].d;
      if (d > pd) { pd = d; p = i; }
    }
    F[f0].vis = true;
    visible.assign(1, f0);
    horizon.clear();
    for (size_t k = 0; k < visible.size(); k++) {
      const int f = visible[k];
      for (int s = 0; s < 3; s++) {
        const int a = F[f].v[s], b = F[f].v[(s + 1) % 3];
        const auto it = edges.find((int64_t)b * K + a);
        if (it == edges.end()) continue;
        const int nb = it->second;
        if (F[nb].vis) continue;
        if (dot(F[nb].n, P[p]) - F[nb].d > eps) {
          F[nb].vis = true;
          visible.push_back(nb);
        } else {
          horizon.push_back({a, b});
        }
      }
    }
    orphans.clear();
    for (int f : visible) {
      F[f].alive = false;
      for (int k = 0; k < 3; k++) {
        const auto it = edges.find((int64_t)F[f].v[k] * K + F[f].v[(k + 1) % 3]);
        if (it != edges.end() && it->second == f) edges.erase(it);
      }
      for (int i : F[f].out)
        if (i != p) orphans.push_back(i);
    }
    fresh.clear();
    for (const auto& ab : horizon)
      if (edges.find((int64_t)ab.first * K + ab.second) == edges.end()) fresh.push_back(make(ab.first, ab.second, p));
    assign(orphans, fresh);
    next.clear();
    for (int f : faces)
      if (F[f].alive) next.push_back(f);
    next.insert(next.end(), fresh.begin(), fresh.end());
    faces.swap(next);
  }

  // Connected coplanar triangles into polygons: a depth-first flood fill across shared edges.
  struct Plane {
    V3 n;
    double d;
    std::vector<int> ids;  // vertices in first-visit order
  };
  std::vector<Plane> planes;
  std::vector<char> in_plane((size_t)np, 0);
  std::vector<int> stack;
  for (int f : faces) {
    if (F[f].group >= 0) continue;
    const int g_id = (int)planes.size();
    planes.push_back(Plane{F[f].n, F[f].d, {}});
    Plane& pl = planes.back();
    F[f].group = g_id;
    stack.assign(1, f);
    while (!stack.empty()) {
      const int g = stack.back();
      stack.pop_back();
      for (int v : F[g].v)
        if (!in_plane[v]) { in_plane[v] = 1; pl.ids.push_back(v); }
      for (int k = 0; k < 3; k++) {
        const auto it = edges.find((int64_t)F[g].v[(k + 1) % 3] * K + F[g].v[k]);
        if (it == edges.end()) continue;
        const int nb = it->second;
        if (F[nb].group >= 0 || !(dot(F[nb].n, pl.n) > 0.0)) continue;
        bool flat = true;
        for (int v : F[nb].v) flat = flat && std::fabs(dot(pl.n, P[v]) - pl.d) <= 10.0 * eps;
        if (!flat) continue;
        F[nb].group = g_id;
        stack.push_back(nb);
      }
    }
    for (int v : pl.ids) in_plane[v] = 0;
  }

  // Each polygon's boundary: the 2-D convex hull of its vertices on the plane (monotone chain over
  // the points sorted by their plane coordinates, turns of at most eps^2 dropped), counter-
  // clockwise about the normal.
  struct Q {
    int id;
    double u, w;
  };
  auto turn = [](const Q& o, const Q& a, const Q& b) { return (a.u - o.u) * (b.w - o.w) - (a.w - o.w) * (b.u - o.u); };
  auto half = [&](const std::vector<Q>& lst, std::vector<int>& loop) {
    std::vector<Q> h;
    for (const Q& q : lst) {
      while (h.size() >= 2 && turn(h[h.size() - 2], h[h.size() - 1], q) <= eps * eps) h.pop_back();
      h.push_back(q);
    }
    h.pop_back();
    for (const Q& q : h) loop.push_back(q.id);
  };
  struct Loop {
    V3 n;
    double d;
    std::vector<int> ids;
  };
  std::vector<Loop> loops;
  for (const Plane& pl : planes) {
    V3 c{0.0, 0.0, 0.0};
    for (int i : pl.ids) c = add(c, P[i]);
    c = scale(c, 1.0 / (double)pl.ids.size());
    const V3 ref = std::fabs(pl.n.x) < 0.9 ? V3{1.0, 0.0, 0.0} : V3{0.0, 1.0, 0.0};
    V3 u = cross(pl.n, ref);
    u = scale(u, 1.0 / norm(u));
    const V3 w = cross(pl.n, u);
    std::vector<Q> q;
    for (int i : pl.ids) q.push_back(Q{i, dot(sub(P[i], c), u), dot(sub(P[i], c), w)});
    std::stable_sort(q.begin(), q.end(), [](const Q& a, const Q& b) { return a.u != b.u ? a.u < b.u : a.w < b.w; });
    Loop lp{pl.n, pl.d, {}};
    half(q, lp.ids);
    std::reverse(q.begin(), q.end());
    half(q, lp.ids);
    if (lp.ids.size() >= 3) loops.push_back(std::move(lp));
  }
  std::vector<int> remap((size_t)np, -1);
  for (const Loop& lp : loops)
    for (int v : lp.ids) remap[v] = 0;
  out = Hull{};
  for (int v = 0; v < np; v++) {
    if (remap[v] < 0) continue;
    remap[v] = (int)(out.verts.size() / 3);
    out.verts.insert(out.verts.end(), {P[v].x, P[v].y, P[v].z});
  }
  out.face_start.push_back(0);
  for (const Loop& lp : loops) {
    out.planes.insert(out.planes.end(), {lp.n.x, lp.n.y, lp.n.z, lp.d});
    for (int v : lp.ids) out.face_verts.push_back((uint32_t)remap[v]);
    out.face_start.push_back((uint32_t)out.face_verts.size());
  }
  return true;
}

}  // namespace hull
}  // namespace steel
