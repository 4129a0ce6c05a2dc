// project.cu -- per-Gaussian / per-point projection kernels.
//
// Built with -fmad=false: every FP32 operation below is a separately rounded
// IEEE operation performed in the order written, the same order as the CPU
// oracle (oracle/oracle.cpp).  That makes pixel centres, conics and 3-sigma
// boxes -- and therefore tile spans and sort keys -- bit-identical between
// the GPU and the oracle.
//
// Reference counterparts (del-splat):
//   k_gauss_project_ref   del-splat-cuda-kernels/cuda/splat_gauss.cu:10-53
//                         (CPU twin del-splat-cpu/src/pnt2xyz.rs:51-96)
//   k_circle_project_ref  del-splat-cuda-kernels/cuda/splat_circle.cu:7-41
//   k_prep_tiles          tile_acceleration.h:15-86 (span + key), with the
//                         per-point counts of count_splat_in_tile
//   k_fused_project       no counterpart: quaternion + log-scale + SH, all
//                         views of a batch per parameter read.
#include "common.cuh"

namespace dsplat {
namespace {

// mat4_col_major::transform_homogeneous
__device__ __forceinline__ void transform_homogeneous(const float* m, const float* p, float* out) {
  float x = m[0] * p[0] + m[4] * p[1] + m[8] * p[2] + m[12];
  float y = m[1] * p[0] + m[5] * p[1] + m[9] * p[2] + m[13];
  float z = m[2] * p[0] + m[6] * p[1] + m[10] * p[2] + m[14];
  float w = m[3] * p[0] + m[7] * p[1] + m[11] * p[2] + m[15];
  out[0] = x / w;
  out[1] = y / w;
  out[2] = z / w;
}

// mat4_col_major::jacobian_transform, J[i + 3*j] = d ndc_i / d p_j
__device__ __forceinline__ void jacobian_transform(const float* t, const float* p, float* J) {
  float a[3];
  a[0] = t[0] * p[0] + t[4] * p[1] + t[8] * p[2] + t[12];
  a[1] = t[1] * p[0] + t[5] * p[1] + t[9] * p[2] + t[13];
  a[2] = t[2] * p[0] + t[6] * p[1] + t[10] * p[2] + t[14];
  float b = t[3] * p[0] + t[7] * p[1] + t[11] * p[2] + t[15];
  float ee = 1.f / b;
  float ee2 = ee * ee;
#pragma unroll
  for (int j = 0; j < 3; ++j)
#pragma unroll
    for (int i = 0; i < 3; ++i) J[i + 3 * j] = t[i + 4 * j] * ee - a[i] * t[3 + 4 * j] * ee2;
}

__device__ __forceinline__ void transform_ndc2pix(int w, int h, float* n) {
  n[0] = 0.5f * float(w);
  n[1] = 0.f;
  n[2] = 0.f;
  n[3] = -0.5f * float(h);
  n[4] = 0.5f * float(w);
  n[5] = 0.5f * float(h);
}

__device__ __forceinline__ void mult_2x3_3x3(const float* a, const float* b, float* r) {
#pragma unroll
  for (int j = 0; j < 3; ++j)
#pragma unroll
    for (int i = 0; i < 2; ++i)
      r[i + 2 * j] = a[i] * b[0 + 3 * j] + a[i + 2] * b[1 + 3 * j] + a[i + 4] * b[2 + 3 * j];
}

__device__ __forceinline__ void quat_to_mat3(const float* q, float* r) {
  float x2 = q[0] * q[0] * 2.f, y2 = q[1] * q[1] * 2.f, z2 = q[2] * q[2] * 2.f;
  float xy = q[0] * q[1] * 2.f, yz = q[1] * q[2] * 2.f, zx = q[2] * q[0] * 2.f;
  float xw = q[0] * q[3] * 2.f, yw = q[1] * q[3] * 2.f, zw = q[2] * q[3] * 2.f;
  r[0] = 1.f - y2 - z2;
  r[1] = xy + zw;
  r[2] = zx - yw;
  r[3] = xy - zw;
  r[4] = 1.f - z2 - x2;
  r[5] = yz + xw;
  r[6] = zx + yw;
  r[7] = yz - xw;
  r[8] = 1.f - x2 - y2;
}

// mat2_sym::projected_spd_mat3 with the rotation already expanded
__device__ __forceinline__ void projected_spd(const float* p, const float* r, const float* d, float* abc) {
  float pr[6];
  mult_2x3_3x3(p, r, pr);
  float dd0 = d[0] * d[0], dd1 = d[1] * d[1], dd2 = d[2] * d[2];
  abc[0] = pr[0] * pr[0] * dd0 + pr[2] * pr[2] * dd1 + pr[4] * pr[4] * dd2;
  abc[1] = pr[0] * pr[1] * dd0 + pr[2] * pr[3] * dd1 + pr[4] * pr[5] * dd2;
  abc[2] = pr[1] * pr[1] * dd0 + pr[3] * pr[3] * dd1 + pr[5] * pr[5] * dd2;
}

// mat2_sym::safe_inverse_preserve_positive_definiteness(abc, 1e-5): inverse
// of the symmetric 2x2 with eigenvalues clamped below at eps.
__device__ __forceinline__ void safe_inverse_spd(const float* s, float eps, float* inv) {
  float a = s[0], b = s[1], c = s[2];
  float hm = (a + c) * 0.5f;
  float hd = (a - c) * 0.5f;
  float r = sqrtf(hd * hd + b * b);
  float l2 = hm - r;
  if (l2 >= eps) {
    float det = a * c - b * b;
    float di = 1.f / det;
    inv[0] = c * di;
    inv[1] = -b * di;
    inv[2] = a * di;
    return;
  }
  float l1 = hm + r;
  float l1c = l1 > eps ? l1 : eps;
  float l2c = eps;
  if (r > 0.f) {
    float r2 = r + r;
    float pa = (a - l2) / r2, pb = b / r2, pc = (c - l2) / r2;
    inv[0] = pa / l1c + (1.f - pa) / l2c;
    inv[1] = pb / l1c - pb / l2c;
    inv[2] = pc / l1c + (1.f - pc) / l2c;
  } else {
    inv[0] = 1.f / l2c;
    inv[1] = 0.f;
    inv[2] = 1.f / l2c;
  }
}

// mat2_sym::aabb2 scaled by 3 (aabb2::scale(.., 3)): 3-sigma half extents
__device__ __forceinline__ void conic_half_extent3(const float* k, float* hx, float* hy) {
  float det = k[0] * k[2] - k[1] * k[1];
  float ex = sqrtf(k[2] / det);
  float ey = sqrtf(k[0] / det);
  *hx = 3.f * ex;
  *hy = 3.f * ey;
}

struct Proj {
  float px, py, ndcz, conic[3], hx, hy;
};

__device__ __forceinline__ void project_core(const float* xyz, const float* rot, const float* s,
                                             const float* mvp, int w, int h, Proj* o) {
  float J[9], n[6], P[6], ndc[3], sig[3];
  jacobian_transform(mvp, xyz, J);
  transform_ndc2pix(w, h, n);
  mult_2x3_3x3(n, J, P);
  transform_homogeneous(mvp, xyz, ndc);
  o->px = n[0] * ndc[0] + n[2] * ndc[1] + n[4] * 1.f;
  o->py = n[1] * ndc[0] + n[3] * ndc[1] + n[5] * 1.f;
  o->ndcz = ndc[2];
  projected_spd(P, rot, s, sig);
  safe_inverse_spd(sig, 1.0e-5f, o->conic);
  conic_half_extent3(o->conic, &o->hx, &o->hy);
}

// Real SH basis up to degree 3; expression trees identical to the oracle.
__device__ __forceinline__ void sh_basis(int deg, float x, float y, float z, float* b) {
  b[0] = 0.28209479177387814f;
  if (deg < 1) return;
  b[1] = -0.4886025119029199f * y;
  b[2] = 0.4886025119029199f * z;
  b[3] = -0.4886025119029199f * x;
  if (deg < 2) return;
  float xx = x * x, yy = y * y, zz = z * z, xy = x * y, yz = y * z, xz = x * z;
  b[4] = 1.0925484305920792f * xy;
  b[5] = -1.0925484305920792f * yz;
  b[6] = 0.31539156525252005f * (2.f * zz - xx - yy);
  b[7] = -1.0925484305920792f * xz;
  b[8] = 0.5462742152960396f * (xx - yy);
  if (deg < 3) return;
  b[9] = -0.5900435899266435f * y * (3.f * xx - yy);
  b[10] = 2.890611442640554f * xy * z;
  b[11] = -0.4570457994644658f * y * (4.f * zz - xx - yy);
  b[12] = 0.3731763325901154f * z * (2.f * zz - 3.f * xx - 3.f * yy);
  b[13] = -0.4570457994644658f * x * (4.f * zz - xx - yy);
  b[14] = 1.445305721320277f * z * (xx - yy);
  b[15] = -0.5900435899266435f * x * (xx - 3.f * yy);
}

}  // namespace

// ---------------------------------------------------------------------------
// splat_gauss.cu:10-53 -- AoS in, AoS out (pnt2pixxydepth, pnt2pixconvinv,
// pnt2pixaabb).  `scale` is the linear standard deviation, `quat` (x,y,z,w)
// is used as given.
// ---------------------------------------------------------------------------
__global__ void k_gauss_project_ref(uint32_t n, const float* __restrict__ xyz,
                                    const float* __restrict__ quat, const float* __restrict__ scale,
                                    const float* __restrict__ mvp_g, int w, int h,
                                    float* __restrict__ xyd, float* __restrict__ conic,
                                    float* __restrict__ aabb) {
  __shared__ float mvp[16];
  if (threadIdx.x < 16) mvp[threadIdx.x] = mvp_g[threadIdx.x];
  __syncthreads();
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  float p[3] = {xyz[3 * i], xyz[3 * i + 1], xyz[3 * i + 2]};
  float q[4] = {quat[4 * i], quat[4 * i + 1], quat[4 * i + 2], quat[4 * i + 3]};
  float s[3] = {scale[3 * i], scale[3 * i + 1], scale[3 * i + 2]};
  float r[9];
  quat_to_mat3(q, r);
  Proj o;
  project_core(p, r, s, mvp, w, h, &o);
  xyd[3 * i] = o.px;
  xyd[3 * i + 1] = o.py;
  xyd[3 * i + 2] = o.ndcz;
  conic[3 * i] = o.conic[0];
  conic[3 * i + 1] = o.conic[1];
  conic[3 * i + 2] = o.conic[2];
  aabb[4 * i] = o.px - o.hx;
  aabb[4 * i + 1] = o.py - o.hy;
  aabb[4 * i + 2] = o.px + o.hx;
  aabb[4 * i + 3] = o.py + o.hy;
}

// ---------------------------------------------------------------------------
// splat_circle.cu:7-41 -- pixel centre + pixel radius of a world-space sphere
// ---------------------------------------------------------------------------
__global__ void k_circle_project_ref(uint32_t n, const float* __restrict__ xyz,
                                     const float* __restrict__ mvp_g, int w, int h, float radius,
                                     float* __restrict__ xyd, float* __restrict__ rad) {
  __shared__ float mvp[16];
  if (threadIdx.x < 16) mvp[threadIdx.x] = mvp_g[threadIdx.x];
  __syncthreads();
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  float p[3] = {xyz[3 * i], xyz[3 * i + 1], xyz[3 * i + 2]};
  float q[3];
  transform_homogeneous(mvp, p, q);
  float r0 = (q[0] + 1.f) * 0.5f * float(w);
  float r1 = (1.f - q[1]) * 0.5f * float(h);
  float J[9];
  jacobian_transform(mvp, p, J);
  float a = J[0], d = J[1], g = J[2], b = J[3], e = J[4], hh = J[5], c = J[6], f = J[7], k = J[8];
  float co0 = e * k - f * hh, co1 = f * g - d * k, co2 = d * hh - e * g;
  float det = a * co0 + b * co1 + c * co2;
  float inv_det = 1.f / det;
  float inv0 = co0 * inv_det, inv1 = co1 * inv_det, inv2 = co2 * inv_det;
  float inv3 = (c * hh - b * k) * inv_det;
  float inv4 = (a * k - c * g) * inv_det;
  float inv5 = (b * g - a * hh) * inv_det;
  float nx = sqrtf(inv0 * inv0 + inv1 * inv1 + inv2 * inv2);
  float ny = sqrtf(inv3 * inv3 + inv4 * inv4 + inv5 * inv5);
  float rx = (1.f / nx) * 0.5f * float(w) * radius;
  float ry = (1.f / ny) * 0.5f * float(h) * radius;
  xyd[3 * i] = r0;
  xyd[3 * i + 1] = r1;
  xyd[3 * i + 2] = q[2];
  rad[i] = 0.5f * (rx + ry);
}

// ---------------------------------------------------------------------------
// Tile span, depth key and pair count per point from an AABB source:
//   aabb != nullptr : Gaussian boxes [N,4] (pnt2pixaabb)
//   aabb == nullptr : circles, box = centre +- rad (aabb2::from_point)
// ---------------------------------------------------------------------------
__global__ void k_prep_tiles(uint32_t n, const float* __restrict__ xyd, const float* __restrict__ aabb,
                             const float* __restrict__ rad, int ts, int tile_w, int tile_h,
                             uint2* __restrict__ rect, uint32_t* __restrict__ dkey,
                             uint32_t* __restrict__ cnt) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  float a0, a1, a2, a3;
  if (aabb) {
    a0 = aabb[4 * i];
    a1 = aabb[4 * i + 1];
    a2 = aabb[4 * i + 2];
    a3 = aabb[4 * i + 3];
  } else {
    const float x = xyd[3 * i], y = xyd[3 * i + 1], r = rad[i];
    a0 = x - r;
    a1 = y - r;
    a2 = x + r;
    a3 = y + r;
  }
  const float tsf = tile_inv(ts);
  int x0 = tile_lo(a0, tsf, tile_w), y0 = tile_lo(a1, tsf, tile_h);
  int x1 = tile_hi(a2, tsf, tile_w), y1 = tile_hi(a3, tsf, tile_h);
  if (x1 < x0) x1 = x0;
  if (y1 < y0) y1 = y0;
  const uint32_t c = uint32_t(x1 - x0) * uint32_t(y1 - y0);
  rect[i] = pack_rect(x0, y0, x1, y1);
  cnt[i] = c;
  dkey[i] = c ? depth_bits(xyd[3 * i + 2]) : 0xffffffffu;
}

// ---------------------------------------------------------------------------
// Fused projection for a batch of views.  One thread per Gaussian reads its
// parameters once and writes, for every view v:
//   rec[v*N+g]   3 x float4 = (px, py, A, B) (C, opacity, r, g) (b, hx, hy, ndcz)
//   rect[v*N+g]  packed tile span, cnt[v*N+g] = #tiles (cnt nullable)
//   dkey[v*Npad+g] depth key bits(max(ndc_z+1,0)); 0xffffffff when no tile
// sh_deg < 0: colors are RGB [N,3]; else SH coefficients [N,(deg+1)^2,3].
// ---------------------------------------------------------------------------
constexpr int kProjThreads = 128;
constexpr int kProjStride = 49;  // 48 coefficients + 1 pad (odd stride: conflict-free rows)

__global__ void __launch_bounds__(kProjThreads) k_fused_project(
    uint32_t n, uint32_t npad, int sh_deg, const float* __restrict__ means,
    const float* __restrict__ log_scales, const float* __restrict__ quats,
    const float* __restrict__ opacity, const float* __restrict__ colors, const ViewBatch b,
    float4* __restrict__ rec, uint2* __restrict__ rect, uint32_t* __restrict__ dkey,
    uint32_t* __restrict__ cnt) {
  // the block's colour rows (128 Gaussians x 3K floats, contiguous) are
  // loaded coalesced into shared memory, padded to an odd stride
  __shared__ float crow[kProjThreads * kProjStride];
  const int K = sh_deg < 0 ? 1 : (sh_deg + 1) * (sh_deg + 1);
  const int C = 3 * K;
  const uint32_t g0 = blockIdx.x * kProjThreads;
  const uint32_t cnt_blk = n > g0 ? min(uint32_t(kProjThreads), n - g0) : 0u;
  for (uint32_t i = threadIdx.x; i < cnt_blk * uint32_t(C); i += kProjThreads)
    crow[(i / C) * kProjStride + (i % C)] = colors[size_t(g0) * C + i];
  __syncthreads();
  const uint32_t g = g0 + threadIdx.x;
  if (g >= n) return;
  const float p[3] = {means[3 * g], means[3 * g + 1], means[3 * g + 2]};
  const float s[3] = {expf_cr(log_scales[3 * g]), expf_cr(log_scales[3 * g + 1]),
                      expf_cr(log_scales[3 * g + 2])};
  const float q[4] = {quats[4 * g], quats[4 * g + 1], quats[4 * g + 2], quats[4 * g + 3]};
  const float nrm = sqrtf(q[0] * q[0] + q[1] * q[1] + q[2] * q[2] + q[3] * q[3]);
  const float qn[4] = {q[0] / nrm, q[1] / nrm, q[2] / nrm, q[3] / nrm};
  float r[9];
  quat_to_mat3(qn, r);
  const float op = opacity[g];
  const float* coef = crow + threadIdx.x * kProjStride;  // read per view from shared memory
  const float tsf = tile_inv(b.ts);
  for (int v = 0; v < b.num_views; ++v) {
    const ViewDev& vd = b.v[v];
    Proj o;
    project_core(p, r, s, vd.mvp, vd.w, vd.h, &o);
    float col[3];
    if (sh_deg < 0) {
      col[0] = coef[0];
      col[1] = coef[1];
      col[2] = coef[2];
    } else {
      const float d0 = p[0] - vd.campos[0], d1 = p[1] - vd.campos[1], d2 = p[2] - vd.campos[2];
      const float dn = sqrtf(d0 * d0 + d1 * d1 + d2 * d2);
      float bs[16];
      sh_basis(sh_deg, d0 / dn, d1 / dn, d2 / dn, bs);
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        float acc = 0.f;
#pragma unroll
        for (int k = 0; k < 16; ++k)
          if (k < K) acc += bs[k] * coef[k * 3 + c];
        acc += 0.5f;
        col[c] = acc > 0.f ? acc : 0.f;
      }
    }
    const float a0 = o.px - o.hx, a1 = o.py - o.hy, a2 = o.px + o.hx, a3 = o.py + o.hy;
    int x0 = tile_lo(a0, tsf, vd.tile_w), y0 = tile_lo(a1, tsf, vd.tile_h);
    int x1 = tile_hi(a2, tsf, vd.tile_w), y1 = tile_hi(a3, tsf, vd.tile_h);
    if (x1 < x0) x1 = x0;
    if (y1 < y0) y1 = y0;
    const uint32_t c = uint32_t(x1 - x0) * uint32_t(y1 - y0);
    const size_t o_idx = size_t(v) * n + g;
    if (c) {  // only points with tiles are ever read back (list entries)
      rec[3 * o_idx + 0] = make_float4(o.px, o.py, o.conic[0], o.conic[1]);
      rec[3 * o_idx + 1] = make_float4(o.conic[2], op, col[0], col[1]);
      rec[3 * o_idx + 2] = make_float4(col[2], o.hx, o.hy, o.ndcz);
    }
    rect[o_idx] = pack_rect(x0, y0, x1, y1);
    if (cnt) cnt[o_idx] = c;
    dkey[size_t(v) * npad + g] = c ? depth_bits(o.ndcz) : 0xffffffffu;
  }
}

}  // namespace dsplat
