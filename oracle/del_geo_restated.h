// del_geo_restated.h -- the del-geo helpers that del-splat's projection
// calls, restated from their mathematical definitions (TEST ONLY).
//
// The del-geo crate (and its C++ headers) is not part of the del-splat tree
// (path dependency ../del-geo; the deploy pins 0.1.32/0.1.33 are commented
// out), so these definitions are this oracle's, not upstream's: "parity
// unpinned" for the helpers themselves.  oracle.cpp uses them for its own
// projection, and oracle/ref/del_geo/*.h expose them under del-geo's names so
// that the reference's own kernels (splat_gauss.cu, splat_circle.cu) compile
// for the host around them -- which pins how the reference composes them.
#pragma once
#include <cmath>

namespace dsplat_geo {

// M is a column-major 4x4 (M[i + 4*j] = row i, col j).
template <class T>
inline void transform_homogeneous(const T* m, const T* p, T* out) {
  T x = m[0] * p[0] + m[4] * p[1] + m[8] * p[2] + m[12];
  T y = m[1] * p[0] + m[5] * p[1] + m[9] * p[2] + m[13];
  T z = m[2] * p[0] + m[6] * p[1] + m[10] * p[2] + m[14];
  T w = m[3] * p[0] + m[7] * p[1] + m[11] * p[2] + m[15];
  out[0] = x / w;
  out[1] = y / w;
  out[2] = z / w;
}

// d(transform_homogeneous)/dp, 3x3 column-major: J[i + 3*j] = d ndc_i / d p_j.
template <class T>
inline void jacobian_transform(const T* t, const T* p, T* J) {
  T a[3];
  a[0] = t[0] * p[0] + t[4] * p[1] + t[8] * p[2] + t[12];
  a[1] = t[1] * p[0] + t[5] * p[1] + t[9] * p[2] + t[13];
  a[2] = t[2] * p[0] + t[6] * p[1] + t[10] * p[2] + t[14];
  T b = t[3] * p[0] + t[7] * p[1] + t[11] * p[2] + t[15];
  T ee = T(1) / b;
  T ee2 = ee * ee;
  for (int j = 0; j < 3; ++j)
    for (int i = 0; i < 3; ++i)
      J[i + 3 * j] = t[i + 4 * j] * ee - a[i] * t[3 + 4 * j] * ee2;
}

// ndc -> pixel as a 2x3 column-major affine map (third column = translation).
template <class T>
inline void transform_ndc2pix(int w, int h, T* n) {
  n[0] = T(0.5) * T(w);
  n[1] = T(0);
  n[2] = T(0);
  n[3] = T(-0.5) * T(h);
  n[4] = T(0.5) * T(w);
  n[5] = T(0.5) * T(h);
}

// (2x3) * (3x3), column-major.  Used with the ndc->pixel map exactly as the
// reference composes it (splat_gauss.cu:28), i.e. including the third column.
template <class T>
inline void mult_2x3_3x3(const T* a, const T* b, T* r) {
  for (int j = 0; j < 3; ++j)
    for (int i = 0; i < 2; ++i)
      r[i + 2 * j] = a[i] * b[0 + 3 * j] + a[i + 2] * b[1 + 3 * j] +
                     a[i + 4] * b[2 + 3 * j];
}

// unit quaternion (x, y, z, w) -> 3x3 rotation, column-major.
template <class T>
inline void quat_to_mat3(const T* q, T* r) {
  T x2 = q[0] * q[0] * T(2), y2 = q[1] * q[1] * T(2), z2 = q[2] * q[2] * T(2);
  T xy = q[0] * q[1] * T(2), yz = q[1] * q[2] * T(2), zx = q[2] * q[0] * T(2);
  T xw = q[0] * q[3] * T(2), yw = q[1] * q[3] * T(2), zw = q[2] * q[3] * T(2);
  r[0] = T(1) - y2 - z2; r[1] = xy + zw;          r[2] = zx - yw;
  r[3] = xy - zw;          r[4] = T(1) - z2 - x2; r[5] = yz + xw;
  r[6] = zx + yw;          r[7] = yz - xw;          r[8] = T(1) - x2 - y2;
}

// symmetric 2x2 (a, b, c) = P R diag(d)^2 R^T P^T
template <class T>
inline void projected_spd_mat3(const T* p, const T* q, const T* d, T* abc) {
  T r[9], pr[6];
  quat_to_mat3(q, r);
  mult_2x3_3x3(p, r, pr);
  T dd0 = d[0] * d[0], dd1 = d[1] * d[1], dd2 = d[2] * d[2];
  abc[0] = pr[0] * pr[0] * dd0 + pr[2] * pr[2] * dd1 + pr[4] * pr[4] * dd2;
  abc[1] = pr[0] * pr[1] * dd0 + pr[2] * pr[3] * dd1 + pr[4] * pr[5] * dd2;
  abc[2] = pr[1] * pr[1] * dd0 + pr[3] * pr[3] * dd1 + pr[5] * pr[5] * dd2;
}

// Inverse of a symmetric 2x2 whose eigenvalues are clamped from below at eps.
// Only +, -, *, /, sqrt are used so that the GPU can reproduce it exactly.
template <class T>
inline void safe_inverse_spd(const T* s, T eps, T* inv) {
  T a = s[0], b = s[1], c = s[2];
  T hm = (a + c) * T(0.5);
  T hd = (a - c) * T(0.5);
  T r = std::sqrt(hd * hd + b * b);
  T l2 = hm - r;
  if (l2 >= eps) {
    T det = a * c - b * b;
    T di = T(1) / det;
    inv[0] = c * di;
    inv[1] = -b * di;
    inv[2] = a * di;
    return;
  }
  T l1 = hm + r;
  T l1c = l1 > eps ? l1 : eps;
  T l2c = eps;
  if (r > T(0)) {
    T r2 = r + r;
    T pa = (a - l2) / r2, pb = b / r2, pc = (c - l2) / r2;
    inv[0] = pa / l1c + (T(1) - pa) / l2c;
    inv[1] = pb / l1c - pb / l2c;
    inv[2] = pc / l1c + (T(1) - pc) / l2c;
  } else {
    inv[0] = T(1) / l2c;
    inv[1] = T(0);
    inv[2] = T(1) / l2c;
  }
}

// Half extents of the ellipse x^T K x = 1, scaled by 3 (3-sigma box).
template <class T>
inline void conic_half_extent3(const T* k, T* hx, T* hy) {
  T det = k[0] * k[2] - k[1] * k[1];
  T ex = std::sqrt(k[2] / det);
  T ey = std::sqrt(k[0] / det);
  *hx = T(3) * ex;
  *hy = T(3) * ey;
}

// 3x3 inverse via the adjugate, column-major in and out.  The entries are
// written even for a singular matrix (then infinite or NaN, as 1/det makes
// them); the return value says whether det != 0.
template <class T>
inline bool mat3_inverse(const T* m, T* inv) {
  T a = m[0], d = m[1], g = m[2], b = m[3], e = m[4], hh = m[5], c = m[6],
    f = m[7], k = m[8];
  T co0 = e * k - f * hh, co1 = f * g - d * k, co2 = d * hh - e * g;
  T det = a * co0 + b * co1 + c * co2;
  T inv_det = T(1) / det;
  inv[0] = co0 * inv_det;
  inv[1] = co1 * inv_det;
  inv[2] = co2 * inv_det;
  inv[3] = (c * hh - b * k) * inv_det;
  inv[4] = (a * k - c * g) * inv_det;
  inv[5] = (b * g - a * hh) * inv_det;
  inv[6] = (b * f - c * e) * inv_det;
  inv[7] = (c * d - a * f) * inv_det;
  inv[8] = (a * e - b * d) * inv_det;
  return det != T(0);
}

template <class T>
inline T norm3(const T* v) {
  return std::sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
}

// b^T M c for a symmetric 2x2 M = (m0, m1; m1, m2), in the order
// m0 b0 c0 + m1 (b0 c1 + b1 c0) + m2 b1 c1, left to right.
template <class T>
inline T mult_vec_from_both_sides(const T* m, const T* b, const T* c) {
  return m[0] * b[0] * c[0] + m[1] * (b[0] * c[1] + b[1] * c[0]) + m[2] * b[1] * c[1];
}

}  // namespace dsplat_geo
