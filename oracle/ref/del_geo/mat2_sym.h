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

namespace mat2_sym {
inline cuda::std::array<float, 3> projected_spd_mat3(const float* p, const float* quat, const float* scale) {
  cuda::std::array<float, 3> abc;
  dsplat_geo::projected_spd_mat3(p, quat, scale, abc.data());
  return abc;
}
inline cuda::std::array<float, 3> safe_inverse_preserve_positive_definiteness(const float* s, float eps) {
  cuda::std::array<float, 3> inv;
  dsplat_geo::safe_inverse_spd(s, eps, inv.data());
  return inv;
}
// bounding box of the ellipse x^T K x = 1 about the origin
inline cuda::std::array<float, 4> aabb2(const float* k) {
  const float det = k[0] * k[2] - k[1] * k[1];
  const float ex = std::sqrt(k[2] / det), ey = std::sqrt(k[0] / det);
  return {-ex, -ey, ex, ey};
}
inline float mult_vec_from_both_sides(const float* m, const float* b, const float* c) {
  return dsplat_geo::mult_vec_from_both_sides(m, b, c);
}
}  // namespace mat2_sym
