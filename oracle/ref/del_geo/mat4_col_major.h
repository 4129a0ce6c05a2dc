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

namespace mat4_col_major {
inline cuda::std::array<float, 9> jacobian_transform(const float* t, const float* p) {
  cuda::std::array<float, 9> j;
  dsplat_geo::jacobian_transform(t, p, j.data());
  return j;
}
inline cuda::std::array<float, 3> transform_homogeneous(const float* t, const float* p) {
  cuda::std::array<float, 3> q;
  dsplat_geo::transform_homogeneous(t, p, q.data());
  return q;
}
}  // namespace mat4_col_major

namespace mat3_col_major {
// try_inverse(..).value() as splat_circle.cu:30 uses it
struct Inverse3 {
  cuda::std::array<float, 9> m;
  cuda::std::array<float, 9> value() const { return m; }
};
inline Inverse3 try_inverse(const float* a) {
  Inverse3 r;
  dsplat_geo::mat3_inverse(a, r.m.data());
  return r;
}
}  // namespace mat3_col_major

namespace vec3 {
inline float norm(const float* v) { return dsplat_geo::norm3(v); }
}  // namespace vec3
