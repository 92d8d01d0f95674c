// Convex hull of a point cloud on the host (SceneBuilder.addConvexHull, builder.js:61-173).
#pragma once
#include <cstdint>
#include <cstring>
#include <string>
#include <vector>

namespace steel {
namespace hull {

// verts: the hull's vertices (x, y, z), in increasing order of their index among the distinct
// input points; planes: per face the outward unit normal and offset d (n . x = d); face_start:
// offsets into face_verts (one more than the faces); face_verts: each face's vertices, counter-
// clockwise about its normal.
struct Hull {
  std::vector<double> verts, planes;
  std::vector<uint32_t> face_start, face_verts;
};
// pts: count points (x, y, z). False with a message for fewer than 4 distinct points, or
// collinear or coplanar points.
bool convex_hull(const double* pts, uint32_t count, Hull& out, std::string& err);

}  // namespace hull
}  // namespace steel
