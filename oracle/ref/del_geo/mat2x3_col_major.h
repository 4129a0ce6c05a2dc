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

namespace mat2x3_col_major {
inline cuda::std::array<float, 6> transform_ndc2pix(uint32_t w, uint32_t h) {
  cuda::std::array<float, 6> n;
  dsplat_geo::transform_ndc2pix(int(w), int(h), n.data());
  return n;
}
inline cuda::std::array<float, 6> mult_mat3_col_major(const float* a, const float* b) {
  cuda::std::array<float, 6> r;
  dsplat_geo::mult_2x3_3x3(a, b, r.data());
  return r;
}
inline cuda::std::array<float, 2> mult_vec3(const float* a, const float* v) {
  return {a[0] * v[0] + a[2] * v[1] + a[4] * v[2], a[1] * v[0] + a[3] * v[1] + a[5] * v[2]};
}
}  // namespace mat2x3_col_major
