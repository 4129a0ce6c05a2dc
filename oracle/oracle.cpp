// oracle.cpp -- CPU restatement of del-splat's splatting path (TEST ONLY).
//
// This file is the checker for the CUDA implementation.  It is loaded only by
// tests/, __graft_entry__.smoke() and bench.py's CPU arms.  It is compiled
// with -ffp-contract=off and without fast-math so that the FP32 stages whose
// results become integer keys (projection -> AABB -> tile span -> key bits)
// follow IEEE single precision operation by operation; the CUDA projection
// kernels are compiled with -fmad=false and perform the same operations in
// the same order, which makes tile counts, keys and permutations bit-exact.
//
// Reference files restated (paths relative to the del-splat repository):
//   del-splat-cpu/src/pnt2xyz.rs:51-96          project_gauss
//   del-splat-cuda-kernels/cuda/splat_gauss.cu:10-53   splat3_to_splat2
//   del-splat-cpu/src/splat_sphere.rs:51-87     circle projection
//   del-splat-cuda-kernels/cuda/splat_circle.cu:7-41   (same, GPU)
//   del-splat-cpu/src/tile_acceleration.rs:3-58 tile2pnt (count, prefix, stable sort)
//   del-splat-cuda-kernels/cuda/tile_acceleration.h:15-86 tile span + key bits
//   del-splat-cuda-kernels/cuda/splat_gauss.cu:56-109  tiled front-to-back blend
//   del-splat-cpu/src/pnt2pixxyndcz.rs:42-100   naive blend (global depth sort)
//   del-splat-cuda-kernels/cuda/splat_circle.cu:93-132 tiled circle painter
//   del-splat-cpu/examples/cpu_splat_sphere_ply.rs:101-118 (CPU twin)
//   del-splat-cpu/src/pnt2pixxyndcz.rs:1-40     point painter (sorted overwrite)
//
// The geometry helpers (mat4 homogeneous transform and its Jacobian, the
// ndc->pixel 2x3 map, quaternion->rotation, projected covariance, the
// positive-definite safe inverse and the ellipse bounding box) come from the
// del-geo crate, which is not part of the reference tree; they are restated
// from their mathematical definitions (the crate is unpinned upstream: path
// dependency ../del-geo, deploy pins 0.1.32/0.1.33 commented out).
#include "oracle.h"
#include "del_geo_restated.h"

#include <algorithm>
#include <parallel/algorithm>
#include <cmath>
#include <cstring>
#include <numeric>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

using namespace dsplat_geo;

struct Proj {
  float px, py, ndcz;
  float conic[3];
  float aabb[4];
};

// splat_gauss.cu:10-53 / pnt2xyz.rs:51-96 (scale is the linear std-dev).
inline void project_one(const float* xyz, const float* q, const float* s,
                        const float* mvp, int w, int h, Proj* o) {
  float J[9], n[6], P[6], ndc[3], sig[3];
  jacobian_transform(mvp, xyz, J);
  transform_ndc2pix(w, h, n);
  mult_2x3_3x3(n, J, P);
  transform_homogeneous(mvp, xyz, ndc);
  o->px = n[0] * ndc[0] + n[2] * ndc[1] + n[4] * 1.f;
  o->py = n[1] * ndc[0] + n[3] * ndc[1] + n[5] * 1.f;
  o->ndcz = ndc[2];
  projected_spd_mat3(P, q, s, sig);
  safe_inverse_spd(sig, 1.0e-5f, o->conic);
  float hx, hy;
  conic_half_extent3(o->conic, &hx, &hy);
  o->aabb[0] = o->px - hx;
  o->aabb[1] = o->py - hy;
  o->aabb[2] = o->px + hx;
  o->aabb[3] = o->py + hy;
}

// tile_acceleration.h:22-31: [floor(min/ts), floor(max/ts)+1) clipped to grid.
inline void tile_span(const float* aabb, int tile_w, int tile_h, int ts,
                      int* x0, int* y0, int* x1, int* y1) {
  const float tsf = float(ts);
  auto lo = [&](float a, int lim) {
    float f = std::floor(a / tsf);
    return (f >= 0.f) ? (f < float(lim) ? int(f) : lim) : 0;
  };
  auto hi = [&](float a, int lim) {
    float f = std::floor(a / tsf);
    return (f >= 0.f) ? (f < float(lim) ? int(f) + 1 : lim) : 0;
  };
  *x0 = lo(aabb[0], tile_w);
  *y0 = lo(aabb[1], tile_h);
  *x1 = hi(aabb[2], tile_w);
  *y1 = hi(aabb[3], tile_h);
  if (*x1 < *x0) *x1 = *x0;
  if (*y1 < *y0) *y1 = *y0;
}

// tile_acceleration.h:43-46: depth bits = bits(max(ndc_z + 1, 0)).
inline uint32_t depth_bits(float ndcz) {
  float zp1 = ndcz + 1.f;
  if (zp1 <= 0.f) zp1 = 0.f;
  uint32_t u;
  std::memcpy(&u, &zp1, 4);
  return u;
}


// exp(x) correctly rounded to float: e^x evaluated in double and rounded
// once.  glibc's double exp is accurate to well under one double ulp, and
// (float)exp((double)x) equals (float)expl(x) for every float x checked in
// [-110, 0], so this is the float nearest to e^x.  The CUDA kernels'
// expf_cr is held to it bit for bit (tests/test_gpu_parity.py).
inline float cr_expf(float x) { return float(std::exp(double(x))); }

// The blend's arithmetic, del-splat-cpu's pnt2pixxyndcz.rs:86-93 (the same
// expressions as splat_gauss.cu:96-106) in f32 with no contraction:
//   q = A dx dx + B (dx dy + dy dx) + C dy dy   (mat2_sym::mult_vec_from_both_sides,
//       left-to-right as written; the del-geo crate itself is absent)
//   e = exp(-0.5 q) * opacity;  e_out = T e;  rgb += c * e_out (per channel);
//   T *= 1 - e;  alpha_sum += e_out;  stop once alpha_sum > 0.999
// Modes (bit flags):
//   kBlendLibmExp  -- exp is the C library's expf (glibc), as in
//                     del-splat-cpu's `f32::exp` and the CUDA kernel
//                     compiled for the host; default: cr_expf.
//   kBlendCudaStop -- the stop test of splat_gauss.cu:105, `alpha_sum >
//                     0.999` compared in double (= alpha_sum >= 0.999f);
//                     default: del-splat-cpu's f32 `alpha_sum > 0.999f`.
constexpr int kBlendLibmExp = 1, kBlendCudaStop = 2;

inline float quad_form(const float* m, float dx, float dy) {
  const float d[2] = {dx, dy};
  return mult_vec_from_both_sides(m, d, d);
}

inline float blend_exp(float x, int mode) {
  return (mode & kBlendLibmExp) ? ::expf(x) : cr_expf(x);
}

inline bool blend_stop(float alpha_sum, int mode) {
  return (mode & kBlendCudaStop) ? (double(alpha_sum) > 0.999) : (alpha_sum > 0.999f);
}

inline bool in_aabb(const float* a, float x, float y) {
  return a[0] <= x && x <= a[2] && a[1] <= y && y <= a[3];
}

// Real spherical harmonics up to degree 3 (standard normalisation constants).
constexpr double kC0 = 0.28209479177387814;
constexpr double kC1 = 0.4886025119029199;
constexpr double kC2[5] = {1.0925484305920792, -1.0925484305920792,
                           0.31539156525252005, -1.0925484305920792,
                           0.5462742152960396};
constexpr double kC3[7] = {-0.5900435899266435, 2.890611442640554,
                           -0.4570457994644658, 0.3731763325901154,
                           -0.4570457994644658, 1.445305721320277,
                           -0.5900435899266435};

template <class T>
inline void sh_basis(int deg, T x, T y, T z, T* b) {
  b[0] = T(kC0);
  if (deg < 1) return;
  b[1] = -T(kC1) * y;
  b[2] = T(kC1) * z;
  b[3] = -T(kC1) * x;
  if (deg < 2) return;
  T xx = x * x, yy = y * y, zz = z * z, xy = x * y, yz = y * z, xz = x * z;
  b[4] = T(kC2[0]) * xy;
  b[5] = T(kC2[1]) * yz;
  b[6] = T(kC2[2]) * (T(2) * zz - xx - yy);
  b[7] = T(kC2[3]) * xz;
  b[8] = T(kC2[4]) * (xx - yy);
  if (deg < 3) return;
  b[9] = T(kC3[0]) * y * (T(3) * xx - yy);
  b[10] = T(kC3[1]) * xy * z;
  b[11] = T(kC3[2]) * y * (T(4) * zz - xx - yy);
  b[12] = T(kC3[3]) * z * (T(2) * zz - T(3) * xx - T(3) * yy);
  b[13] = T(kC3[4]) * x * (T(4) * zz - xx - yy);
  b[14] = T(kC3[5]) * z * (xx - yy);
  b[15] = T(kC3[6]) * x * (xx - T(3) * yy);
}

// d basis / d (x, y, z) for each coefficient: db[k*3 + axis]
template <class T>
inline void sh_basis_grad(int deg, T x, T y, T z, T* db) {
  for (int k = 0; k < 48; ++k) db[k] = T(0);
  if (deg < 1) return;
  db[1 * 3 + 1] = -T(kC1);
  db[2 * 3 + 2] = T(kC1);
  db[3 * 3 + 0] = -T(kC1);
  if (deg < 2) return;
  T xx = x * x, yy = y * y, zz = z * z;
  db[4 * 3 + 0] = T(kC2[0]) * y;
  db[4 * 3 + 1] = T(kC2[0]) * x;
  db[5 * 3 + 1] = T(kC2[1]) * z;
  db[5 * 3 + 2] = T(kC2[1]) * y;
  db[6 * 3 + 0] = -T(2) * T(kC2[2]) * x;
  db[6 * 3 + 1] = -T(2) * T(kC2[2]) * y;
  db[6 * 3 + 2] = T(4) * T(kC2[2]) * z;
  db[7 * 3 + 0] = T(kC2[3]) * z;
  db[7 * 3 + 2] = T(kC2[3]) * x;
  db[8 * 3 + 0] = T(2) * T(kC2[4]) * x;
  db[8 * 3 + 1] = -T(2) * T(kC2[4]) * y;
  if (deg < 3) return;
  db[9 * 3 + 0] = T(kC3[0]) * T(6) * x * y;
  db[9 * 3 + 1] = T(kC3[0]) * (T(3) * xx - T(3) * yy);
  db[10 * 3 + 0] = T(kC3[1]) * y * z;
  db[10 * 3 + 1] = T(kC3[1]) * x * z;
  db[10 * 3 + 2] = T(kC3[1]) * x * y;
  db[11 * 3 + 0] = T(kC3[2]) * (-T(2) * x * y);
  db[11 * 3 + 1] = T(kC3[2]) * (T(4) * zz - xx - T(3) * yy);
  db[11 * 3 + 2] = T(kC3[2]) * (T(8) * y * z);
  db[12 * 3 + 0] = T(kC3[3]) * (-T(6) * x * z);
  db[12 * 3 + 1] = T(kC3[3]) * (-T(6) * y * z);
  db[12 * 3 + 2] = T(kC3[3]) * (T(6) * zz - T(3) * xx - T(3) * yy);
  db[13 * 3 + 0] = T(kC3[4]) * (T(4) * zz - T(3) * xx - yy);
  db[13 * 3 + 1] = T(kC3[4]) * (-T(2) * x * y);
  db[13 * 3 + 2] = T(kC3[4]) * (T(8) * x * z);
  db[14 * 3 + 0] = T(kC3[5]) * (T(2) * x * z);
  db[14 * 3 + 1] = T(kC3[5]) * (-T(2) * y * z);
  db[14 * 3 + 2] = T(kC3[5]) * (xx - yy);
  db[15 * 3 + 0] = T(kC3[6]) * (T(3) * xx - T(3) * yy);
  db[15 * 3 + 1] = T(kC3[6]) * (-T(6) * x * y);
}

inline int sh_count(int deg) { return deg < 0 ? 1 : (deg + 1) * (deg + 1); }

// Colour of one Gaussian: sh_deg < 0 -> RGB passthrough, else SH + 0.5 clamped at 0.
template <class T>
inline void eval_color(int sh_deg, const T* mean, const T* campos,
                       const float* coef, T* rgb, T* raw = nullptr) {
  if (sh_deg < 0) {
    for (int c = 0; c < 3; ++c) {
      rgb[c] = T(coef[c]);
      if (raw) raw[c] = rgb[c];
    }
    return;
  }
  T d[3] = {mean[0] - campos[0], mean[1] - campos[1], mean[2] - campos[2]};
  T nrm = std::sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
  T x = d[0] / nrm, y = d[1] / nrm, z = d[2] / nrm;
  T b[16];
  sh_basis(sh_deg, x, y, z, b);
  const int K = sh_count(sh_deg);
  for (int c = 0; c < 3; ++c) {
    T acc = T(0);
    for (int k = 0; k < K; ++k) acc += b[k] * T(coef[k * 3 + c]);
    acc += T(0.5);
    if (raw) raw[c] = acc;
    rgb[c] = acc > T(0) ? acc : T(0);
  }
}

}  // namespace

// cr_expf elementwise (checks of the CUDA expf_cr); threaded.
extern "C" void orc_expf_cr(int64_t n, const float* x, float* out) {
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < n; ++i) out[i] = cr_expf(x[i]);
}

// ============================================================================
// Reference forward path (FP32)
// ============================================================================
extern "C" void orc_gauss_project(int64_t n, const float* xyz,
                                  const float* quat, const float* scale,
                                  const float* mvp, int w, int h, float* xyd,
                                  float* conic, float* aabb) {
  for (int64_t i = 0; i < n; ++i) {
    Proj p;
    project_one(xyz + 3 * i, quat + 4 * i, scale + 3 * i, mvp, w, h, &p);
    xyd[3 * i + 0] = p.px;
    xyd[3 * i + 1] = p.py;
    xyd[3 * i + 2] = p.ndcz;
    for (int k = 0; k < 3; ++k) conic[3 * i + k] = p.conic[k];
    for (int k = 0; k < 4; ++k) aabb[4 * i + k] = p.aabb[k];
  }
}

// splat_circle.cu:7-41 / splat_sphere.rs:51-87
extern "C" void orc_circle_project(int64_t n, const float* xyz,
                                   const float* mvp, int w, int h,
                                   float radius, float* xyd, float* rad) {
  for (int64_t i = 0; i < n; ++i) {
    const float* p = xyz + 3 * i;
    float q[3];
    transform_homogeneous(mvp, p, q);
    float r0 = (q[0] + 1.f) * 0.5f * float(w);
    float r1 = (1.f - q[1]) * 0.5f * float(h);
    float J[9];
    jacobian_transform(mvp, p, J);
    float inv[9];
    mat3_inverse(J, inv);
    float nx = norm3(inv), ny = norm3(inv + 3);
    float rx = (1.f / nx) * 0.5f * float(w) * radius;
    float ry = (1.f / ny) * 0.5f * float(h) * radius;
    xyd[3 * i + 0] = r0;
    xyd[3 * i + 1] = r1;
    xyd[3 * i + 2] = q[2];
    rad[i] = 0.5f * (rx + ry);
  }
}

// aabb2::from_point(xy, r) (splat_circle.cu:61, tile_acceleration.rs:189)
extern "C" void orc_circle_aabb(int64_t n, const float* xyd, const float* rad,
                                float* aabb) {
  for (int64_t i = 0; i < n; ++i) {
    float x = xyd[3 * i], y = xyd[3 * i + 1], r = rad[i];
    aabb[4 * i + 0] = x - r;
    aabb[4 * i + 1] = y - r;
    aabb[4 * i + 2] = x + r;
    aabb[4 * i + 3] = y + r;
  }
}

// tile_acceleration.rs:110-127: per-tile counts then inclusive prefix into
// tile2idx[1..T]; returns the pair count P = tile2idx[T].
extern "C" uint64_t orc_tile2pnt_count(int64_t n, const float* aabb,
                                       int tile_w, int tile_h, int ts,
                                       uint32_t* tile2idx) {
  const int64_t T = int64_t(tile_w) * tile_h;
  std::fill(tile2idx, tile2idx + T + 1, 0u);
  for (int64_t i = 0; i < n; ++i) {
    int x0, y0, x1, y1;
    tile_span(aabb + 4 * i, tile_w, tile_h, ts, &x0, &y0, &x1, &y1);
    for (int ix = x0; ix < x1; ++ix)
      for (int iy = y0; iy < y1; ++iy) tile2idx[int64_t(iy) * tile_w + ix + 1] += 1;
  }
  for (int64_t t = 0; t < T; ++t) tile2idx[t + 1] += tile2idx[t];
  return tile2idx[T];
}

// tile_acceleration.rs:128-153: emit (tile, depth) per overlapped tile in
// point order, then a stable sort by (tile, depth).
extern "C" void orc_tile2pnt_fill(int64_t n, const float* aabb,
                                  const float* xyd, int tile_w, int tile_h,
                                  int ts, const uint32_t* tile2idx,
                                  uint32_t* idx2pnt, uint64_t* keys) {
  const int64_t T = int64_t(tile_w) * tile_h;
  const uint64_t P = tile2idx[T];
  // (key, point) pairs in emission order; a point appears at most once per
  // tile and is emitted in index order, so the reference's stable sort by
  // key equals a sort by (key, point), done here in parallel
  struct KV {
    uint64_t k;
    uint32_t v;
    bool operator<(const KV& o) const { return k < o.k || (k == o.k && v < o.v); }
  };
  std::vector<KV> kv;
  kv.reserve(P);
  for (int64_t i = 0; i < n; ++i) {
    int x0, y0, x1, y1;
    tile_span(aabb + 4 * i, tile_w, tile_h, ts, &x0, &y0, &x1, &y1);
    uint32_t zb = depth_bits(xyd[3 * i + 2]);
    for (int ix = x0; ix < x1; ++ix)
      for (int iy = y0; iy < y1; ++iy) {
        uint64_t tile = uint64_t(iy) * tile_w + ix;
        kv.push_back(KV{(tile << 32) | zb, uint32_t(i)});
      }
  }
  __gnu_parallel::sort(kv.begin(), kv.end());
  for (uint64_t j = 0; j < kv.size() && j < P; ++j) {
    idx2pnt[j] = kv[j].v;
    if (keys) keys[j] = kv[j].k;
  }
}

// splat_gauss.cu:56-109, one pixel.  Returns the absolute list position at
// which the walk stopped (the break position, or the list start).
namespace {
inline int32_t blend_pixel(int ix, int iy, uint32_t start, uint32_t end,
                           const uint32_t* idx2pnt, const float* xyd,
                           const float* conic, const float* aabb,
                           const float* opacity, const float* rgb, float* out,
                           float* outT, int mode) {
  const float tx = float(ix) + 0.5f, ty = float(iy) + 0.5f;
  float asum = 0.f, occ = 1.f;
  float c0 = out[0], c1 = out[1], c2 = out[2];
  int32_t last = int32_t(start);
  for (uint32_t pos = end; pos-- > start;) {
    const uint32_t g = idx2pnt[pos];
    if (!in_aabb(aabb + 4 * g, tx, ty)) continue;
    const float dx = tx - xyd[3 * g], dy = ty - xyd[3 * g + 1];
    const float e = blend_exp(-0.5f * quad_form(conic + 3 * g, dx, dy), mode) * opacity[g];
    const float eo = occ * e;
    c0 += rgb[3 * g + 0] * eo;
    c1 += rgb[3 * g + 1] * eo;
    c2 += rgb[3 * g + 2] * eo;
    occ *= 1.f - e;
    asum += eo;
    if (blend_stop(asum, mode)) {
      last = int32_t(pos);
      break;
    }
  }
  out[0] = c0;
  out[1] = c1;
  out[2] = c2;
  *outT = occ;
  return last;
}
}  // namespace

extern "C" void orc_gauss_rasterize_tiled_mode(
    int w, int h, int ts, const uint32_t* tile2idx, const uint32_t* idx2pnt,
    const float* xyd, const float* conic, const float* aabb,
    const float* opacity, const float* rgb, float* pix_rgb, float* pix_T,
    int32_t* pix_last, int nthreads, int mode) {
  const int tw = (w + ts - 1) / ts;
#pragma omp parallel for schedule(dynamic, 1) num_threads(nthreads > 0 ? nthreads : 1) collapse(2)
  for (int iy = 0; iy < h; ++iy)
    for (int ix = 0; ix < w; ++ix) {
      const int t = (iy / ts) * tw + (ix / ts);
      const int64_t pix = int64_t(iy) * w + ix;
      float T;
      int32_t last = blend_pixel(ix, iy, tile2idx[t], tile2idx[t + 1], idx2pnt,
                                 xyd, conic, aabb, opacity, rgb,
                                 pix_rgb + 3 * pix, &T, mode);
      if (pix_T) pix_T[pix] = T;
      if (pix_last) pix_last[pix] = last;
    }
}

extern "C" void orc_gauss_rasterize_tiled(
    int w, int h, int ts, const uint32_t* tile2idx, const uint32_t* idx2pnt,
    const float* xyd, const float* conic, const float* aabb,
    const float* opacity, const float* rgb, float* pix_rgb, float* pix_T,
    int32_t* pix_last, int nthreads) {
  orc_gauss_rasterize_tiled_mode(w, h, ts, tile2idx, idx2pnt, xyd, conic, aabb,
                                 opacity, rgb, pix_rgb, pix_T, pix_last,
                                 nthreads, 0);
}

// pnt2pixxyndcz.rs:42-100: global stable sort by ndc_z+1, clip |ndc_z| >= 1.
extern "C" void orc_gauss_render_naive_mode(int64_t n, const float* xyd,
                                            const float* conic, const float* aabb,
                                            const float* opacity, const float* rgb,
                                            int w, int h, float* pix_rgb, int mode) {
  std::vector<uint32_t> ord(n);
  std::iota(ord.begin(), ord.end(), 0u);
  std::stable_sort(ord.begin(), ord.end(), [&](uint32_t a, uint32_t b) {
    return xyd[3 * a + 2] + 1.f < xyd[3 * b + 2] + 1.f;
  });
#pragma omp parallel for schedule(dynamic, 4)
  for (int iy = 0; iy < h; ++iy)
    for (int ix = 0; ix < w; ++ix) {
      const float tx = float(ix) + 0.5f, ty = float(iy) + 0.5f;
      float asum = 0.f, occ = 1.f;
      float* o = pix_rgb + 3 * (int64_t(iy) * w + ix);
      for (int64_t j = n; j-- > 0;) {
        const uint32_t g = ord[j];
        const float z = xyd[3 * g + 2];
        if (z <= -1.f || z >= 1.f) continue;
        if (!in_aabb(aabb + 4 * g, tx, ty)) continue;
        const float dx = tx - xyd[3 * g], dy = ty - xyd[3 * g + 1];
        const float e = blend_exp(-0.5f * quad_form(conic + 3 * g, dx, dy), mode) * opacity[g];
        const float eo = occ * e;
        o[0] += rgb[3 * g + 0] * eo;
        o[1] += rgb[3 * g + 1] * eo;
        o[2] += rgb[3 * g + 2] * eo;
        occ *= 1.f - e;
        asum += eo;
        if (blend_stop(asum, mode)) break;
      }
    }
}

extern "C" void orc_gauss_render_naive(int64_t n, const float* xyd,
                                       const float* conic, const float* aabb,
                                       const float* opacity, const float* rgb,
                                       int w, int h, float* pix_rgb) {
  orc_gauss_render_naive_mode(n, xyd, conic, aabb, opacity, rgb, w, h, pix_rgb, 0);
}

// splat_circle.cu:93-132: ascending walk, the last covering entry wins.
extern "C" void orc_circle_splat_tiled(int w, int h, int ts,
                                       const uint32_t* tile2idx,
                                       const uint32_t* idx2pnt,
                                       const float* xyd, const float* rad,
                                       int32_t* winner) {
  const int tw = (w + ts - 1) / ts;
  for (int iy = 0; iy < h; ++iy)
    for (int ix = 0; ix < w; ++ix) {
      const int t = (iy / ts) * tw + (ix / ts);
      const float px = float(ix) + 0.5f, py = float(iy) + 0.5f;
      int32_t win = -1;
      for (uint32_t pos = tile2idx[t]; pos < tile2idx[t + 1]; ++pos) {
        const uint32_t g = idx2pnt[pos];
        const float dx = xyd[3 * g] - px, dy = xyd[3 * g + 1] - py;
        const float dist = std::sqrt(dx * dx + dy * dy);
        if (dist > rad[g]) continue;
        win = int32_t(g);
      }
      winner[int64_t(iy) * w + ix] = win;
    }
}

// pnt2pixxyndcz.rs:1-40: stable sort by ndc_z+1, skip |ndc_z| >= 1, then
// overwrite.  `as usize` saturates: negative/NaN -> 0.
extern "C" void orc_point_render_sort_depth(int64_t n, const float* xyd, int w,
                                            int h, int32_t* winner) {
  std::vector<uint32_t> ord;
  ord.reserve(n);
  for (int64_t i = 0; i < n; ++i)
    if (!std::isnan(xyd[3 * i + 2])) ord.push_back(uint32_t(i));
  std::stable_sort(ord.begin(), ord.end(), [&](uint32_t a, uint32_t b) {
    return xyd[3 * a + 2] + 1.f < xyd[3 * b + 2] + 1.f;
  });
  std::fill(winner, winner + int64_t(w) * h, -1);
  for (uint32_t g : ord) {
    const float z = xyd[3 * g + 2];
    if (z <= -1.f || z >= 1.f) continue;
    const float x = xyd[3 * g], y = xyd[3 * g + 1];
    int64_t ix, iy;
    if (!(x >= 0.f)) ix = 0; else if (x >= float(w)) continue; else ix = int64_t(x);
    if (!(y >= 0.f)) iy = 0; else if (y >= float(h)) continue; else iy = int64_t(y);
    if (ix >= w || iy >= h) continue;
    winner[iy * w + ix] = int32_t(g);
  }
}

// ============================================================================
// Differentiable path: FP32 mirror of the fused projection kernel.
// ============================================================================
namespace {
inline void normalize_quat(const float* q, float* qn) {
  float nrm = std::sqrt(q[0] * q[0] + q[1] * q[1] + q[2] * q[2] + q[3] * q[3]);
  qn[0] = q[0] / nrm;
  qn[1] = q[1] / nrm;
  qn[2] = q[2] / nrm;
  qn[3] = q[3] / nrm;
}
}  // namespace

extern "C" void orc_sh_eval(int64_t n, const float* means, const float* colors,
                            int sh_deg, const float* campos, float* rgb) {
  const int K = sh_count(sh_deg);
  for (int64_t i = 0; i < n; ++i)
    eval_color<float>(sh_deg, means + 3 * i, campos, colors + 3 * K * i,
                      rgb + 3 * i);
}

extern "C" void orc_fused_project(int64_t n, const float* means,
                                  const float* log_scales, const float* quats,
                                  const float* colors, int sh_deg,
                                  const float* mvp, const float* campos, int w,
                                  int h, float* xyd, float* conic, float* aabb,
                                  float* rgb) {
  const int K = sh_count(sh_deg);
  for (int64_t i = 0; i < n; ++i) {
    float s[3] = {cr_expf(log_scales[3 * i]), cr_expf(log_scales[3 * i + 1]),
                  cr_expf(log_scales[3 * i + 2])};
    float qn[4];
    normalize_quat(quats + 4 * i, qn);
    Proj p;
    project_one(means + 3 * i, qn, s, mvp, w, h, &p);
    xyd[3 * i + 0] = p.px;
    xyd[3 * i + 1] = p.py;
    xyd[3 * i + 2] = p.ndcz;
    for (int k = 0; k < 3; ++k) conic[3 * i + k] = p.conic[k];
    for (int k = 0; k < 4; ++k) aabb[4 * i + k] = p.aabb[k];
    if (rgb)
      eval_color<float>(sh_deg, means + 3 * i, campos, colors + 3 * K * i,
                        rgb + 3 * i);
  }
}

// ============================================================================
// Gradient oracle.  Generic over the scalar type: double for the FD-checked
// analytic gradient, float for the timed CPU baseline.
// ============================================================================
namespace {

template <class T>
struct G2 {  // per-Gaussian 2D state of one view
  T px, py, ca, cb, cc, op, col[3];
};

template <class T>
struct Params {  // a scalar view of the parameters with one optional override
  const orc64_scene* s;
  int kind = -1;
  int64_t gauss = -1;
  int comp = -1;
  T delta = T(0);
  T get(int k, int64_t g, int c, const float* arr, int stride) const {
    T v = T(arr[g * stride + c]);
    if (k == kind && g == gauss && c == comp) v += delta;
    return v;
  }
};

template <class T>
void project_gauss_T(const Params<T>& P, int64_t g, G2<T>* o, T* raw_col) {
  const orc64_scene* s = P.s;
  T M[16];
  for (int i = 0; i < 16; ++i) M[i] = T(s->mvp[i]);
  T p[3], ls[3], q[4];
  for (int c = 0; c < 3; ++c) p[c] = P.get(0, g, c, s->means, 3);
  for (int c = 0; c < 3; ++c) ls[c] = P.get(1, g, c, s->log_scales, 3);
  for (int c = 0; c < 4; ++c) q[c] = P.get(2, g, c, s->quats, 4);
  T sc[3] = {std::exp(ls[0]), std::exp(ls[1]), std::exp(ls[2])};
  T nrm = std::sqrt(q[0] * q[0] + q[1] * q[1] + q[2] * q[2] + q[3] * q[3]);
  T qn[4] = {q[0] / nrm, q[1] / nrm, q[2] / nrm, q[3] / nrm};
  T J[9], N[6], Pm[6], ndc[3], sig[3], con[3];
  jacobian_transform(M, p, J);
  transform_ndc2pix(s->w, s->h, N);
  mult_2x3_3x3(N, J, Pm);
  transform_homogeneous(M, p, ndc);
  o->px = N[0] * ndc[0] + N[2] * ndc[1] + N[4];
  o->py = N[1] * ndc[0] + N[3] * ndc[1] + N[5];
  projected_spd_mat3(Pm, qn, sc, sig);
  safe_inverse_spd(sig, T(1.0e-5), con);
  o->ca = con[0];
  o->cb = con[1];
  o->cc = con[2];
  o->op = P.get(3, g, 0, s->opacity, 1);
  const int K = sh_count(s->sh_deg);
  // colour coefficients with the override applied
  float coef[48];
  for (int k = 0; k < 3 * K; ++k) coef[k] = s->colors[g * 3 * K + k];
  T cam[3] = {T(s->campos[0]), T(s->campos[1]), T(s->campos[2])};
  if (P.kind == 4 && P.gauss == g) {
    // apply the perturbation in T precision on a local copy
    T tmp[48];
    for (int k = 0; k < 3 * K; ++k) tmp[k] = T(coef[k]);
    tmp[P.comp] += P.delta;
    if (s->sh_deg < 0) {
      for (int c = 0; c < 3; ++c) {
        o->col[c] = tmp[c];
        if (raw_col) raw_col[c] = tmp[c];
      }
    } else {
      T d[3] = {p[0] - cam[0], p[1] - cam[1], p[2] - cam[2]};
      T dn = std::sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
      T b[16];
      sh_basis(s->sh_deg, d[0] / dn, d[1] / dn, d[2] / dn, b);
      for (int c = 0; c < 3; ++c) {
        T acc = T(0);
        for (int k = 0; k < K; ++k) acc += b[k] * tmp[k * 3 + c];
        acc += T(0.5);
        if (raw_col) raw_col[c] = acc;
        o->col[c] = acc > T(0) ? acc : T(0);
      }
    }
    return;
  }
  eval_color<T>(s->sh_deg, p, cam, coef, o->col, raw_col);
}

template <class T>
struct Contrib {
  uint32_t g;
  T dx, dy, G, e, Tb;  // Tb: transmittance before this Gaussian
};

// Forward of one pixel with frozen structure; appends contributions.
template <class T>
T pixel_forward(const orc64_scene* s, const std::vector<G2<T>>& g2, int ix,
                int iy, uint32_t start, uint32_t end, int32_t last, T* C,
                std::vector<Contrib<T>>* rec) {
  const float tx = float(ix) + 0.5f, ty = float(iy) + 0.5f;
  T occ = T(1);
  C[0] = C[1] = C[2] = T(0);
  if (last < int32_t(start)) last = int32_t(start);
  for (uint32_t pos = end; pos-- > uint32_t(last);) {
    const uint32_t g = s->idx2pnt[pos];
    if (!in_aabb(s->aabb + 4 * g, tx, ty)) continue;
    const G2<T>& a = g2[g];
    const T dx = T(tx) - a.px, dy = T(ty) - a.py;
    const T q = a.ca * dx * dx + a.cb * (dx * dy + dy * dx) + a.cc * dy * dy;
    const T G = std::exp(T(-0.5) * q);
    const T e = G * a.op;
    const T eo = occ * e;
    for (int c = 0; c < 3; ++c) C[c] += a.col[c] * eo;
    if (rec) rec->push_back({g, dx, dy, G, e, occ});
    occ *= T(1) - e;
  }
  return occ;
}

template <class T>
void compute_g2(const orc64_scene* s, const Params<T>& P,
                std::vector<G2<T>>* g2, std::vector<T>* raw) {
  g2->resize(s->n);
  if (raw) raw->resize(3 * s->n);
  for (int64_t g = 0; g < s->n; ++g)
    project_gauss_T<T>(P, g, &(*g2)[g], raw ? raw->data() + 3 * g : nullptr);
}

template <class T>
T loss_T(const orc64_scene* s, const Params<T>& P, const uint8_t* tile_mask,
         double* pix_rgb) {
  std::vector<G2<T>> g2;
  compute_g2<T>(s, P, &g2, nullptr);
  const int tw = (s->w + s->ts - 1) / s->ts;
  T loss = T(0);
  for (int iy = 0; iy < s->h; ++iy)
    for (int ix = 0; ix < s->w; ++ix) {
      const int t = (iy / s->ts) * tw + (ix / s->ts);
      if (tile_mask && !tile_mask[t]) continue;
      const int64_t pix = int64_t(iy) * s->w + ix;
      T C[3];
      pixel_forward<T>(s, g2, ix, iy, s->tile2idx[t], s->tile2idx[t + 1],
                       s->pix_last[pix], C, nullptr);
      for (int c = 0; c < 3; ++c) {
        if (pix_rgb) pix_rgb[3 * pix + c] = double(C[c]);
        T d = C[c] - T(s->target[3 * pix + c]);
        loss += d * d;
      }
    }
  return loss;
}

// Back-to-front accumulation of the 2D gradients of one pixel: the
// transmittance is rebuilt from the final value (T_i = T_{i+1} / (1 - e_i)),
// exactly the scheme of the CUDA backward rasteriser.
template <class T>
void pixel_backward(const orc64_scene* s, const std::vector<G2<T>>& g2, int ix,
                    int iy, uint32_t start, uint32_t end, int32_t last,
                    const T* dC, T Tfinal, T* g2grad /* [N,9] */) {
  const float tx = float(ix) + 0.5f, ty = float(iy) + 0.5f;
  if (last < int32_t(start)) last = int32_t(start);
  T Tcur = Tfinal;
  T acc[3] = {T(0), T(0), T(0)};
  for (uint32_t pos = uint32_t(last); pos < end; ++pos) {
    const uint32_t g = s->idx2pnt[pos];
    if (!in_aabb(s->aabb + 4 * g, tx, ty)) continue;
    const G2<T>& a = g2[g];
    const T dx = T(tx) - a.px, dy = T(ty) - a.py;
    const T q = a.ca * dx * dx + a.cb * (dx * dy + dy * dx) + a.cc * dy * dy;
    const T G = std::exp(T(-0.5) * q);
    const T e = G * a.op;
    const T om = T(1) - e;
    Tcur = Tcur / om;  // transmittance in front of this Gaussian
    const T w = e * Tcur;
    T dLde = T(0);
    for (int c = 0; c < 3; ++c) {
      dLde += dC[c] * (a.col[c] * Tcur - acc[c] / om);
      acc[c] += a.col[c] * w;
    }
    T* gg = g2grad + 9 * int64_t(g);
    gg[6] += w * dC[0];
    gg[7] += w * dC[1];
    gg[8] += w * dC[2];
    gg[5] += G * dLde;
    const T dLdq = dLde * a.op * G * T(-0.5);
    gg[2] += dLdq * dx * dx;
    gg[3] += dLdq * T(2) * dx * dy;
    gg[4] += dLdq * dy * dy;
    gg[0] += -dLdq * (T(2) * a.ca * dx + T(2) * a.cb * dy);
    gg[1] += -dLdq * (T(2) * a.cb * dx + T(2) * a.cc * dy);
  }
}

// Chain rule from the per-Gaussian 2D gradients (px, py, A, B, C, op, r, g, b)
// back to the parameters.  Mirrors the CUDA projection backward.
template <class T>
void project_backward_one(const orc64_scene* s, int64_t gi, const T* gg,
                          T* gm, T* gls, T* gq, T* gop, T* gcol) {
  T M[16];
  for (int i = 0; i < 16; ++i) M[i] = T(s->mvp[i]);
  T p[3], ls[3], q[4];
  for (int c = 0; c < 3; ++c) p[c] = T(s->means[3 * gi + c]);
  for (int c = 0; c < 3; ++c) ls[c] = T(s->log_scales[3 * gi + c]);
  for (int c = 0; c < 4; ++c) q[c] = T(s->quats[4 * gi + c]);
  T sc[3] = {std::exp(ls[0]), std::exp(ls[1]), std::exp(ls[2])};
  T nrm = std::sqrt(q[0] * q[0] + q[1] * q[1] + q[2] * q[2] + q[3] * q[3]);
  T qn[4] = {q[0] / nrm, q[1] / nrm, q[2] / nrm, q[3] / nrm};
  T a[3], w;
  a[0] = M[0] * p[0] + M[4] * p[1] + M[8] * p[2] + M[12];
  a[1] = M[1] * p[0] + M[5] * p[1] + M[9] * p[2] + M[13];
  a[2] = M[2] * p[0] + M[6] * p[1] + M[10] * p[2] + M[14];
  w = M[3] * p[0] + M[7] * p[1] + M[11] * p[2] + M[15];
  T J[9], N[6], Pm[6], R[9], PR[6];
  jacobian_transform(M, p, J);
  transform_ndc2pix(s->w, s->h, N);
  mult_2x3_3x3(N, J, Pm);
  quat_to_mat3(qn, R);
  mult_2x3_3x3(Pm, R, PR);
  T dd[3] = {sc[0] * sc[0], sc[1] * sc[1], sc[2] * sc[2]};
  T sa = PR[0] * PR[0] * dd[0] + PR[2] * PR[2] * dd[1] + PR[4] * PR[4] * dd[2];
  T sb = PR[0] * PR[1] * dd[0] + PR[2] * PR[3] * dd[1] + PR[4] * PR[5] * dd[2];
  T scc = PR[1] * PR[1] * dd[0] + PR[3] * PR[3] * dd[1] + PR[5] * PR[5] * dd[2];
  // conic = (scc, -sb, sa) / det
  T det = sa * scc - sb * sb;
  T id2 = T(1) / (det * det);
  const T gA = gg[2], gB = gg[3], gC = gg[4];
  T dsa = (-scc * scc * gA + sb * scc * gB - sb * sb * gC) * id2;
  T dsb = (T(2) * sb * scc * gA - (sa * scc + sb * sb) * gB + T(2) * sa * sb * gC) * id2;
  T dsc = (-sb * sb * gA + sa * sb * gB - sa * sa * gC) * id2;
  // sigma = sum_k dd_k PR[:,k] PR[:,k]^T
  T dPR[6];
  for (int k = 0; k < 3; ++k) {
    const T u = PR[2 * k], v = PR[2 * k + 1];
    dPR[2 * k] = dd[k] * (T(2) * u * dsa + v * dsb);
    dPR[2 * k + 1] = dd[k] * (u * dsb + T(2) * v * dsc);
    const T ddd = u * u * dsa + u * v * dsb + v * v * dsc;
    gls[k] += ddd * T(2) * dd[k];  // d(s^2)/d(ls) = 2 s^2
  }
  // PR = Pm R : dPm[i][k] = sum_j dPR[i][j] R[k][j]; dR[k][j] = sum_i Pm[i][k] dPR[i][j]
  T dP[6], dR[9];
  for (int i = 0; i < 2; ++i)
    for (int k = 0; k < 3; ++k) {
      T acc = T(0);
      for (int j = 0; j < 3; ++j) acc += dPR[i + 2 * j] * R[k + 3 * j];
      dP[i + 2 * k] = acc;
    }
  for (int k = 0; k < 3; ++k)
    for (int j = 0; j < 3; ++j)
      dR[k + 3 * j] = Pm[0 + 2 * k] * dPR[0 + 2 * j] + Pm[1 + 2 * k] * dPR[1 + 2 * j];
  // rotation from the unit quaternion (x, y, z, w); R_ij stored at R[i + 3j]
  {
    const T x = qn[0], y = qn[1], z = qn[2], ww = qn[3];
    auto G_ = [&](int i, int j) { return dR[i + 3 * j]; };
    T dqx = G_(1, 0) * 2 * y + G_(2, 0) * 2 * z + G_(0, 1) * 2 * y - G_(1, 1) * 4 * x +
            G_(2, 1) * 2 * ww + G_(0, 2) * 2 * z - G_(1, 2) * 2 * ww - G_(2, 2) * 4 * x;
    T dqy = -G_(0, 0) * 4 * y + G_(1, 0) * 2 * x - G_(2, 0) * 2 * ww + G_(0, 1) * 2 * x +
            G_(2, 1) * 2 * z + G_(0, 2) * 2 * ww + G_(1, 2) * 2 * z - G_(2, 2) * 4 * y;
    T dqz = -G_(0, 0) * 4 * z + G_(1, 0) * 2 * ww + G_(2, 0) * 2 * x - G_(0, 1) * 2 * ww -
            G_(1, 1) * 4 * z + G_(2, 1) * 2 * y + G_(0, 2) * 2 * x + G_(1, 2) * 2 * y;
    T dqw = G_(1, 0) * 2 * z - G_(2, 0) * 2 * y - G_(0, 1) * 2 * z + G_(2, 1) * 2 * x +
            G_(0, 2) * 2 * y - G_(1, 2) * 2 * x;
    T dqn[4] = {dqx, dqy, dqz, dqw};
    T dot = dqn[0] * qn[0] + dqn[1] * qn[1] + dqn[2] * qn[2] + dqn[3] * qn[3];
    for (int c = 0; c < 4; ++c) gq[c] += (dqn[c] - qn[c] * dot) / nrm;
  }
  // Pm = N J (N includes the translation column, as the reference composes it)
  T dJ[9];
  for (int j = 0; j < 3; ++j) {
    dJ[0 + 3 * j] = N[0] * dP[0 + 2 * j];
    dJ[1 + 3 * j] = N[3] * dP[1 + 2 * j];
    dJ[2 + 3 * j] = N[4] * dP[0 + 2 * j] + N[5] * dP[1 + 2 * j];
  }
  // pixel centre
  for (int m = 0; m < 3; ++m) gm[m] += gg[0] * N[0] * J[0 + 3 * m] + gg[1] * N[3] * J[1 + 3 * m];
  // J[i][j] = M[i][j]/w - a_i M[3][j]/w^2
  {
    const T iw = T(1) / w, iw2 = iw * iw, iw3 = iw2 * iw;
    for (int m = 0; m < 3; ++m) {
      T acc = T(0);
      for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
          const T d = -M[i + 4 * j] * M[3 + 4 * m] * iw2 - M[i + 4 * m] * M[3 + 4 * j] * iw2 +
                      T(2) * a[i] * M[3 + 4 * j] * M[3 + 4 * m] * iw3;
          acc += dJ[i + 3 * j] * d;
        }
      gm[m] += acc;
    }
  }
  *gop += gg[5];
  // colour
  const int K = sh_count(s->sh_deg);
  const T* dcol = gg + 6;
  if (s->sh_deg < 0) {
    for (int c = 0; c < 3; ++c) gcol[c] += dcol[c];
  } else {
    T cam[3] = {T(s->campos[0]), T(s->campos[1]), T(s->campos[2])};
    T d[3] = {p[0] - cam[0], p[1] - cam[1], p[2] - cam[2]};
    T dn = std::sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
    T x = d[0] / dn, y = d[1] / dn, z = d[2] / dn;
    T b[16], db[48];
    sh_basis(s->sh_deg, x, y, z, b);
    sh_basis_grad(s->sh_deg, x, y, z, db);
    T draw[3];
    const float* coef = s->colors + gi * 3 * K;
    for (int c = 0; c < 3; ++c) {
      T acc = T(0);
      for (int k = 0; k < K; ++k) acc += b[k] * T(coef[k * 3 + c]);
      acc += T(0.5);
      draw[c] = acc > T(0) ? dcol[c] : T(0);
    }
    T dn3[3] = {T(0), T(0), T(0)};
    for (int k = 0; k < K; ++k) {
      T gk = T(0);
      for (int c = 0; c < 3; ++c) {
        gcol[k * 3 + c] += b[k] * draw[c];
        gk += T(coef[k * 3 + c]) * draw[c];
      }
      for (int ax = 0; ax < 3; ++ax) dn3[ax] += gk * db[k * 3 + ax];
    }
    T nn[3] = {x, y, z};
    T dot = dn3[0] * nn[0] + dn3[1] * nn[1] + dn3[2] * nn[2];
    for (int m = 0; m < 3; ++m) gm[m] += (dn3[m] - nn[m] * dot) / dn;
  }
}

template <class T>
T backward_T(const orc64_scene* s, int nthreads, T* gm, T* gls, T* gq, T* gop,
             T* gcol, std::vector<T>* pix_rgb_out) {
  Params<T> P;
  P.s = s;
  std::vector<G2<T>> g2;
  compute_g2<T>(s, P, &g2, nullptr);
  const int tw = (s->w + s->ts - 1) / s->ts;
  const int th = (s->h + s->ts - 1) / s->ts;
  const int64_t n = s->n;
  int nt = nthreads > 0 ? nthreads : 1;
  std::vector<std::vector<T>> part(nt, std::vector<T>());
  T loss = T(0);
  if (pix_rgb_out) pix_rgb_out->assign(3 * int64_t(s->w) * s->h, T(0));
#pragma omp parallel num_threads(nt) reduction(+ : loss)
  {
    int tid = 0;
#ifdef _OPENMP
    tid = omp_get_thread_num();
#endif
    std::vector<T>& gg = part[tid];
    gg.assign(9 * n, T(0));
#pragma omp for schedule(dynamic, 1)
    for (int t = 0; t < tw * th; ++t) {
      const int tx0 = (t % tw) * s->ts, ty0 = (t / tw) * s->ts;
      for (int iy = ty0; iy < std::min(ty0 + s->ts, s->h); ++iy)
        for (int ix = tx0; ix < std::min(tx0 + s->ts, s->w); ++ix) {
          const int64_t pix = int64_t(iy) * s->w + ix;
          T C[3];
          T Tf = pixel_forward<T>(s, g2, ix, iy, s->tile2idx[t],
                                  s->tile2idx[t + 1], s->pix_last[pix], C,
                                  nullptr);
          T dC[3];
          for (int c = 0; c < 3; ++c) {
            T d = C[c] - T(s->target[3 * pix + c]);
            loss += d * d;
            dC[c] = T(2) * d;
            if (pix_rgb_out) (*pix_rgb_out)[3 * pix + c] = C[c];
          }
          pixel_backward<T>(s, g2, ix, iy, s->tile2idx[t], s->tile2idx[t + 1],
                            s->pix_last[pix], dC, Tf, gg.data());
        }
    }
  }
  std::vector<T> tot(9 * n, T(0));
  for (int k = 0; k < nt; ++k)
    if (!part[k].empty())
      for (int64_t i = 0; i < 9 * n; ++i) tot[i] += part[k][i];
  const int K = sh_count(s->sh_deg);
#pragma omp parallel for num_threads(nt) schedule(static)
  for (int64_t g = 0; g < n; ++g)
    project_backward_one<T>(s, g, tot.data() + 9 * g, gm + 3 * g, gls + 3 * g,
                            gq + 4 * g, gop + g, gcol + 3 * K * g);
  return loss;
}

}  // namespace

extern "C" double orc64_loss(const orc64_scene* s, const uint8_t* tile_mask,
                             double* pix_rgb) {
  Params<double> P;
  P.s = s;
  return loss_T<double>(s, P, tile_mask, pix_rgb);
}

extern "C" double orc64_backward(const orc64_scene* s, double* g_means,
                                 double* g_log_scales, double* g_quats,
                                 double* g_opacity, double* g_colors) {
  const int K = sh_count(s->sh_deg);
  std::fill(g_means, g_means + 3 * s->n, 0.0);
  std::fill(g_log_scales, g_log_scales + 3 * s->n, 0.0);
  std::fill(g_quats, g_quats + 4 * s->n, 0.0);
  std::fill(g_opacity, g_opacity + s->n, 0.0);
  std::fill(g_colors, g_colors + 3 * K * s->n, 0.0);
  int nt = 1;
#ifdef _OPENMP
  nt = omp_get_max_threads();
#endif
  return backward_T<double>(s, nt, g_means, g_log_scales, g_quats, g_opacity,
                            g_colors, nullptr);
}

extern "C" double orc64_fd(const orc64_scene* s, int kind, int64_t gauss,
                           int comp, double h) {
  const int tw = (s->w + s->ts - 1) / s->ts;
  const int th = (s->h + s->ts - 1) / s->ts;
  std::vector<uint8_t> mask(size_t(tw) * th, 0);
  for (int t = 0; t < tw * th; ++t)
    for (uint32_t pos = s->tile2idx[t]; pos < s->tile2idx[t + 1]; ++pos)
      if (s->idx2pnt[pos] == uint32_t(gauss)) {
        mask[t] = 1;
        break;
      }
  Params<double> P;
  P.s = s;
  P.kind = kind;
  P.gauss = gauss;
  P.comp = comp;
  P.delta = h;
  double lp = loss_T<double>(s, P, mask.data(), nullptr);
  P.delta = -h;
  double lm = loss_T<double>(s, P, mask.data(), nullptr);
  return (lp - lm) / (2.0 * h);
}

extern "C" uint64_t orc_cpu_fwd_bwd(const orc64_scene* s, int nthreads,
                                    float* pix_rgb, float* g_means,
                                    float* g_log_scales, float* g_quats,
                                    float* g_opacity, float* g_colors) {
  // Full FP32 CPU pipeline for one view: fused projection, tile lists,
  // forward blend (stop positions), backward.  The scene's structure fields
  // are ignored and rebuilt here.
  const int64_t n = s->n;
  const int K = sh_count(s->sh_deg);
  const int tw = (s->w + s->ts - 1) / s->ts;
  const int th = (s->h + s->ts - 1) / s->ts;
  std::vector<float> xyd(3 * n), con(3 * n), aabb(4 * n), rgb(3 * n), op(n);
  int nt = nthreads > 0 ? nthreads : 1;
#pragma omp parallel for num_threads(nt) schedule(static)
  for (int64_t i = 0; i < n; ++i)
    orc_fused_project(1, s->means + 3 * i, s->log_scales + 3 * i,
                      s->quats + 4 * i, s->colors + 3 * K * i, s->sh_deg,
                      s->mvp, s->campos, s->w, s->h, &xyd[3 * i], &con[3 * i],
                      &aabb[4 * i], &rgb[3 * i]);
  std::vector<uint32_t> tile2idx(size_t(tw) * th + 1);
  uint64_t P = orc_tile2pnt_count(n, aabb.data(), tw, th, s->ts, tile2idx.data());
  std::vector<uint32_t> idx2pnt(P);
  orc_tile2pnt_fill(n, aabb.data(), xyd.data(), tw, th, s->ts, tile2idx.data(),
                    idx2pnt.data(), nullptr);
  std::vector<float> T(int64_t(s->w) * s->h);
  std::vector<int32_t> last(int64_t(s->w) * s->h);
  std::fill(pix_rgb, pix_rgb + 3 * int64_t(s->w) * s->h, 0.f);
  orc_gauss_rasterize_tiled(s->w, s->h, s->ts, tile2idx.data(), idx2pnt.data(),
                            xyd.data(), con.data(), aabb.data(), s->opacity,
                            rgb.data(), pix_rgb, T.data(), last.data(), nt);
  orc64_scene s2 = *s;
  s2.tile2idx = tile2idx.data();
  s2.idx2pnt = idx2pnt.data();
  s2.pix_last = last.data();
  s2.aabb = aabb.data();
  std::fill(g_means, g_means + 3 * n, 0.f);
  std::fill(g_log_scales, g_log_scales + 3 * n, 0.f);
  std::fill(g_quats, g_quats + 4 * n, 0.f);
  std::fill(g_opacity, g_opacity + n, 0.f);
  std::fill(g_colors, g_colors + 3 * K * n, 0.f);
  backward_T<float>(&s2, nt, g_means, g_log_scales, g_quats, g_opacity,
                    g_colors, nullptr);
  return P;
}
