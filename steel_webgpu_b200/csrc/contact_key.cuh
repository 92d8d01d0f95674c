// Key of the canonical contact order (wgsl.js:3899-3982): (pair, feature key, point-bit hash, raw
// index), compared lexicographically. Raw contact records are 5 vec4 each; record 2 carries the
// two shape indices and the two feature ids.
#pragma once
#include "common.cuh"

namespace steel {

SD bool key_gt(uint4 a, uint4 b) {
  if (a.x != b.x) return a.x > b.x;
  if (a.y != b.y) return a.y > b.y;
  if (a.z != b.z) return a.z > b.z;
  return a.w > b.w;
}
SD uint4 contact_key(const float4* craw, uint32_t c) {
  float4 p = craw[c * 5u], m = craw[c * 5u + 2u];
  uint32_t pair = (uint32_t)(f2i(m.x) + 1) | ((uint32_t)(f2i(m.y) + 1) << 16u);
  uint32_t feat = f2u(m.z) | (f2u(m.w) << 16u);
  uint32_t bits = mix32(mix32(mix32(fbits(p.x)) ^ fbits(p.y)) ^ fbits(p.z)) ^ fbits(p.w);
  return make_uint4(pair, feat, bits, c);
}

}  // namespace steel
