// Host shim for the del-geo C++ headers that del-splat's CUDA kernels
// include (TEST ONLY).  The del-geo crate is absent from the reference tree,
// so every function here forwards to this oracle's restatement in
// oracle/del_geo_restated.h; it exists only so that the reference's own
// kernel sources compile for the host unchanged.
#pragma once
#include <array>
#include <cmath>
#include <cstdint>
#include "../../del_geo_restated.h"

namespace aabb2 {
// scaled about its centre
inline cuda::std::array<float, 4> scale(const float* a, float s) {
  const float cx = (a[0] + a[2]) * 0.5f, cy = (a[1] + a[3]) * 0.5f;
  const float hx = (a[2] - a[0]) * 0.5f * s, hy = (a[3] - a[1]) * 0.5f * s;
  return {cx - hx, cy - hy, cx + hx, cy + hy};
}
inline cuda::std::array<float, 4> translate(const float* a, const float* t) {
  return {a[0] + t[0], a[1] + t[1], a[2] + t[0], a[3] + t[1]};
}
// inclusive on every side
inline bool is_inlcude_point(const float* a, const float* p) {
  return a[0] <= p[0] && p[0] <= a[2] && a[1] <= p[1] && p[1] <= a[3];
}
inline cuda::std::array<float, 4> from_point(const float* p, float r) {
  return {p[0] - r, p[1] - r, p[0] + r, p[1] + r};
}
}  // namespace aabb2
