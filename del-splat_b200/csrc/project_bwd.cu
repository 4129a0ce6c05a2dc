// project_bwd.cu -- backward of the fused projection (no reference
// counterpart; the reference has no gradient code).
//
// Two kernels, one thread per Gaussian each, looping over the views of the
// batch with the next view's 2D gradient prefetched: k_project_bwd_geom
// carries the geometry chain (mean through the projection, log-scale,
// quaternion, opacity), k_project_bwd_colour the SH coefficients and the part
// of the mean gradient that flows through the SH view direction.  The colour
// kernel stages its block's coefficients through shared memory, so the
// [N, K, 3] parameter rows are read and written with coalesced accesses.
// Both add into the caller's gradient buffers (so a per-view loop
// accumulates naturally).
//
// Forward recomputed here (all column-major, M = world->NDC):
//   a = M[0:3]·[p,1], w = M[3]·[p,1], ndc = a/w,
//   J_ij = M_ij/w - a_i M_3j / w^2            (d ndc / d p)
//   P = N J with N = [[W/2, 0, W/2], [0, -H/2, H/2]]   (the reference composes
//       the full 2x3 ndc->pixel map with J, translation column included)
//   Sigma = (P R) diag(s^2) (P R)^T, conic = Sigma^-1, s = exp(log_scale),
//   R = R(q/|q|), colour = max(SH(dir) + 0.5, 0), dir = (p - campos)/|..|
#include "common.cuh"

namespace dsplat {
namespace {

// Real SH basis b[0..K) at unit direction (x, y, z), same constants and sign
// convention as the forward.
__device__ __forceinline__ void sh_basis(int deg, float x, float y, float z, float* b) {
  const float C0 = 0.28209479177387814f, C1 = 0.4886025119029199f;
  b[0] = C0;
  if (deg < 1) return;
  b[1] = -C1 * y;
  b[2] = C1 * z;
  b[3] = -C1 * x;
  if (deg < 2) return;
  const float C20 = 1.0925484305920792f, C21 = -1.0925484305920792f, C22 = 0.31539156525252005f,
              C23 = -1.0925484305920792f, C24 = 0.5462742152960396f;
  const float xx = x * x, yy = y * y, zz = z * z, xy = x * y, yz = y * z, xz = x * z;
  b[4] = C20 * xy;
  b[5] = C21 * yz;
  b[6] = C22 * (2.f * zz - xx - yy);
  b[7] = C23 * xz;
  b[8] = C24 * (xx - yy);
  if (deg < 3) return;
  const float C30 = -0.5900435899266435f, C31 = 2.890611442640554f, C32 = -0.4570457994644658f,
              C33 = 0.3731763325901154f, C34 = -0.4570457994644658f, C35 = 1.445305721320277f,
              C36 = -0.5900435899266435f;
  b[9] = C30 * y * (3.f * xx - yy);
  b[10] = C31 * xy * z;
  b[11] = C32 * y * (4.f * zz - xx - yy);
  b[12] = C33 * z * (2.f * zz - 3.f * xx - 3.f * yy);
  b[13] = C34 * x * (4.f * zz - xx - yy);
  b[14] = C35 * z * (xx - yy);
  b[15] = C36 * x * (xx - 3.f * yy);
}

// dv = sum_k w_k grad b_k(x, y, z)
__device__ __forceinline__ void sh_weighted_grad(int deg, float x, float y, float z, const float* w, float* dv) {
  dv[0] = dv[1] = dv[2] = 0.f;
  if (deg < 1) return;
  const float C1 = 0.4886025119029199f;
  dv[1] += -C1 * w[1];
  dv[2] += C1 * w[2];
  dv[0] += -C1 * w[3];
  if (deg < 2) return;
  const float C20 = 1.0925484305920792f, C21 = -1.0925484305920792f, C22 = 0.31539156525252005f,
              C23 = -1.0925484305920792f, C24 = 0.5462742152960396f;
  dv[0] += C20 * y * w[4] - 2.f * C22 * x * w[6] + C23 * z * w[7] + 2.f * C24 * x * w[8];
  dv[1] += C20 * x * w[4] + C21 * z * w[5] - 2.f * C22 * y * w[6] - 2.f * C24 * y * w[8];
  dv[2] += C21 * y * w[5] + 4.f * C22 * z * w[6] + C23 * x * w[7];
  if (deg < 3) return;
  const float C30 = -0.5900435899266435f, C31 = 2.890611442640554f, C32 = -0.4570457994644658f,
              C33 = 0.3731763325901154f, C34 = -0.4570457994644658f, C35 = 1.445305721320277f,
              C36 = -0.5900435899266435f;
  const float xx = x * x, yy = y * y, zz = z * z;
  dv[0] += C30 * 6.f * x * y * w[9] + C31 * y * z * w[10] + C32 * (-2.f * x * y) * w[11] +
           C33 * (-6.f * x * z) * w[12] + C34 * (4.f * zz - 3.f * xx - yy) * w[13] + C35 * (2.f * x * z) * w[14] +
           C36 * (3.f * xx - 3.f * yy) * w[15];
  dv[1] += C30 * (3.f * xx - 3.f * yy) * w[9] + C31 * x * z * w[10] + C32 * (4.f * zz - xx - 3.f * yy) * w[11] +
           C33 * (-6.f * y * z) * w[12] + C34 * (-2.f * x * y) * w[13] + C35 * (-2.f * y * z) * w[14] +
           C36 * (-6.f * x * y) * w[15];
  dv[2] += C31 * x * y * w[10] + C32 * (8.f * y * z) * w[11] + C33 * (6.f * zz - 3.f * xx - 3.f * yy) * w[12] +
           C34 * (8.f * x * z) * w[13] + C35 * (xx - yy) * w[14];
}

// Geometry contributions of one view: out[0..2] d mean, out[3..5] d s^2,
// out[6..14] d R (column-major), out[15] d opacity.
__device__ __forceinline__ void geometry_view(const float* p, const float* dd, const float* R, const float* M,
                                              float vw, float vh, float4 g0, float2 g1, float* out) {
  float a[3];
  a[0] = M[0] * p[0] + M[4] * p[1] + M[8] * p[2] + M[12];
  a[1] = M[1] * p[0] + M[5] * p[1] + M[9] * p[2] + M[13];
  a[2] = M[2] * p[0] + M[6] * p[1] + M[10] * p[2] + M[14];
  const float w = M[3] * p[0] + M[7] * p[1] + M[11] * p[2] + M[15];
  const float iw = 1.f / w, iw2 = iw * iw, iw3 = iw2 * iw;
  float J[9];
#pragma unroll
  for (int j = 0; j < 3; ++j)
#pragma unroll
    for (int i = 0; i < 3; ++i) J[i + 3 * j] = M[i + 4 * j] * iw - a[i] * M[3 + 4 * j] * iw2;
  const float N0 = 0.5f * vw, N3 = -0.5f * vh, N4 = 0.5f * vw, N5 = 0.5f * vh;
  float P[6];
#pragma unroll
  for (int j = 0; j < 3; ++j) {
    P[0 + 2 * j] = N0 * J[0 + 3 * j] + N4 * J[2 + 3 * j];
    P[1 + 2 * j] = N3 * J[1 + 3 * j] + N5 * J[2 + 3 * j];
  }
  float PR[6];
#pragma unroll
  for (int j = 0; j < 3; ++j)
#pragma unroll
    for (int i = 0; i < 2; ++i)
      PR[i + 2 * j] = P[i] * R[3 * j] + P[i + 2] * R[1 + 3 * j] + P[i + 4] * R[2 + 3 * j];
  const float sa = PR[0] * PR[0] * dd[0] + PR[2] * PR[2] * dd[1] + PR[4] * PR[4] * dd[2];
  const float sb = PR[0] * PR[1] * dd[0] + PR[2] * PR[3] * dd[1] + PR[4] * PR[5] * dd[2];
  const float sc = PR[1] * PR[1] * dd[0] + PR[3] * PR[3] * dd[1] + PR[5] * PR[5] * dd[2];
  const float det = sa * sc - sb * sb;
  const float id2 = 1.f / (det * det);
  const float gA = g0.z, gB = g0.w, gC = g1.x;
  const float dsa = (-sc * sc * gA + sb * sc * gB - sb * sb * gC) * id2;
  const float dsb = (2.f * sb * sc * gA - (sa * sc + sb * sb) * gB + 2.f * sa * sb * gC) * id2;
  const float dsc = (-sb * sb * gA + sa * sb * gB - sa * sa * gC) * id2;
  float dPR[6];
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    const float u = PR[2 * k], vv = PR[2 * k + 1];
    dPR[2 * k] = dd[k] * (2.f * u * dsa + vv * dsb);
    dPR[2 * k + 1] = dd[k] * (u * dsb + 2.f * vv * dsc);
    out[3 + k] = u * u * dsa + u * vv * dsb + vv * vv * dsc;
  }
  float dP[6];
#pragma unroll
  for (int i = 0; i < 2; ++i)
#pragma unroll
    for (int k = 0; k < 3; ++k)
      dP[i + 2 * k] = dPR[i] * R[k] + dPR[i + 2] * R[k + 3] + dPR[i + 4] * R[k + 6];
#pragma unroll
  for (int k = 0; k < 3; ++k)
#pragma unroll
    for (int j = 0; j < 3; ++j) out[6 + k + 3 * j] = P[2 * k] * dPR[2 * j] + P[1 + 2 * k] * dPR[1 + 2 * j];
  float dJ[9];
#pragma unroll
  for (int j = 0; j < 3; ++j) {
    dJ[0 + 3 * j] = N0 * dP[2 * j];
    dJ[1 + 3 * j] = N3 * dP[1 + 2 * j];
    dJ[2 + 3 * j] = N4 * dP[2 * j] + N5 * dP[1 + 2 * j];
  }
  // sum_ij dJ_ij dJ_ij/dp_m with dJ_ij/dp_m = -(M_ij M_3m + M_im M_3j)/w^2
  // + 2 a_i M_3j M_3m / w^3, contracted once:
  //   S1 = sum_ij dJ_ij M_ij, u_i = sum_j dJ_ij M_3j, S3 = sum_i a_i u_i
  float S1 = 0.f, u[3];
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    u[i] = 0.f;
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      S1 += dJ[i + 3 * j] * M[i + 4 * j];
      u[i] += dJ[i + 3 * j] * M[3 + 4 * j];
    }
  }
  const float S3 = a[0] * u[0] + a[1] * u[1] + a[2] * u[2];
#pragma unroll
  for (int m = 0; m < 3; ++m) {
    const float M3m = M[3 + 4 * m];
    out[m] = g0.x * N0 * J[0 + 3 * m] + g0.y * N3 * J[1 + 3 * m] - M3m * S1 * iw2 -
             (u[0] * M[4 * m] + u[1] * M[1 + 4 * m] + u[2] * M[2 + 4 * m]) * iw2 + 2.f * M3m * S3 * iw3;
  }
  out[15] = g1.y;
}

}  // namespace

__global__ void __launch_bounds__(128) k_project_bwd_geom(uint32_t n, const float* __restrict__ means,
                                                          const float* __restrict__ log_scales,
                                                          const float* __restrict__ quats, const ViewBatch b,
                                                          float4* __restrict__ grad2d,
                                                          float* __restrict__ g_means, float* __restrict__ g_ls,
                                                          float* __restrict__ g_quats, float* __restrict__ g_op) {
  const uint32_t g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= n) return;
  const float p[3] = {means[3 * g], means[3 * g + 1], means[3 * g + 2]};
  const float s[3] = {expf_cr(log_scales[3 * g]), expf_cr(log_scales[3 * g + 1]), expf_cr(log_scales[3 * g + 2])};
  const float dd[3] = {s[0] * s[0], s[1] * s[1], s[2] * s[2]};
  const float q[4] = {quats[4 * g], quats[4 * g + 1], quats[4 * g + 2], quats[4 * g + 3]};
  const float nrm = sqrtf(q[0] * q[0] + q[1] * q[1] + q[2] * q[2] + q[3] * q[3]);
  const float qn[4] = {q[0] / nrm, q[1] / nrm, q[2] / nrm, q[3] / nrm};
  float R[9];
  {
    const float x = qn[0], y = qn[1], z = qn[2], ww = qn[3];
    R[0] = 1.f - 2.f * (y * y + z * z);
    R[1] = 2.f * (x * y + z * ww);
    R[2] = 2.f * (x * z - y * ww);
    R[3] = 2.f * (x * y - z * ww);
    R[4] = 1.f - 2.f * (x * x + z * z);
    R[5] = 2.f * (y * z + x * ww);
    R[6] = 2.f * (x * z + y * ww);
    R[7] = 2.f * (y * z - x * ww);
    R[8] = 1.f - 2.f * (x * x + y * y);
  }
  float acc[16];
#pragma unroll
  for (int k = 0; k < 16; ++k) acc[k] = 0.f;
  float4 n0 = grad2d[3 * size_t(g)];
  float2 n1 = *reinterpret_cast<const float2*>(grad2d + 3 * size_t(g) + 1);
  for (int v = 0; v < b.num_views; ++v) {
    const float4 g0 = n0;
    const float2 g1 = n1;
    if (v + 1 < b.num_views) {  // prefetch the next view's record
      const float4* gp = grad2d + 3 * (size_t(v + 1) * n + g);
      n0 = gp[0];
      n1 = *reinterpret_cast<const float2*>(gp + 1);
    }
    if (g0.x == 0.f && g0.y == 0.f && g0.z == 0.f && g0.w == 0.f && g1.x == 0.f && g1.y == 0.f) continue;
    {  // consumed: leave the record's geometry part zero for the next backward
      float4* gp = grad2d + 3 * (size_t(v) * n + g);
      gp[0] = make_float4(0.f, 0.f, 0.f, 0.f);
      *reinterpret_cast<float2*>(gp + 1) = make_float2(0.f, 0.f);
    }
    float c[16];
    geometry_view(p, dd, R, b.v[v].mvp, float(b.v[v].w), float(b.v[v].h), g0, g1, c);
#pragma unroll
    for (int k = 0; k < 16; ++k) acc[k] += c[k];
  }
  // rotation -> unit quaternion -> raw quaternion
  float dq[4];
  {
    const float x = qn[0], y = qn[1], z = qn[2], ww = qn[3];
    auto GR = [&](int i, int j) { return acc[6 + i + 3 * j]; };
    const float dqx = GR(1, 0) * 2.f * y + GR(2, 0) * 2.f * z + GR(0, 1) * 2.f * y - GR(1, 1) * 4.f * x +
                      GR(2, 1) * 2.f * ww + GR(0, 2) * 2.f * z - GR(1, 2) * 2.f * ww - GR(2, 2) * 4.f * x;
    const float dqy = -GR(0, 0) * 4.f * y + GR(1, 0) * 2.f * x - GR(2, 0) * 2.f * ww + GR(0, 1) * 2.f * x +
                      GR(2, 1) * 2.f * z + GR(0, 2) * 2.f * ww + GR(1, 2) * 2.f * z - GR(2, 2) * 4.f * y;
    const float dqz = -GR(0, 0) * 4.f * z + GR(1, 0) * 2.f * ww + GR(2, 0) * 2.f * x - GR(0, 1) * 2.f * ww -
                      GR(1, 1) * 4.f * z + GR(2, 1) * 2.f * y + GR(0, 2) * 2.f * x + GR(1, 2) * 2.f * y;
    const float dqw = GR(1, 0) * 2.f * z - GR(2, 0) * 2.f * y - GR(0, 1) * 2.f * z + GR(2, 1) * 2.f * x +
                      GR(0, 2) * 2.f * y - GR(1, 2) * 2.f * x;
    const float dot = dqx * x + dqy * y + dqz * z + dqw * ww;
    dq[0] = (dqx - x * dot) / nrm;
    dq[1] = (dqy - y * dot) / nrm;
    dq[2] = (dqz - z * dot) / nrm;
    dq[3] = (dqw - ww * dot) / nrm;
  }
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    g_means[3 * g + c] += acc[c];
    g_ls[3 * g + c] += acc[3 + c] * 2.f * dd[c];
  }
#pragma unroll
  for (int c = 0; c < 4; ++c) g_quats[4 * g + c] += dq[c];
  g_op[g] += acc[15];
}

// dL/d coef_kc = sum_v b_k(dir_v) dL/dcolour_vc (zero where the forward
// clamped the colour), and the mean gradient through
// dir_v = (p - campos_v) / |p - campos_v|.  The block's coefficient rows
// (128 Gaussians x 3K floats, contiguous) pass through shared memory with a
// padded row stride so that per-thread reads are conflict-free.
constexpr int kColThreads = 128;
constexpr int kColStride = 49;  // 48 coefficients + 1 pad (odd stride: no bank conflicts)

__global__ void __launch_bounds__(kColThreads) k_project_bwd_colour(uint32_t n, int sh_deg,
                                                                    const float* __restrict__ means,
                                                                    const float* __restrict__ colors,
                                                                    const ViewBatch b,
                                                                    float4* __restrict__ grad2d,
                                                                    float* __restrict__ g_means,
                                                                    float* __restrict__ g_col,
                                                                    unsigned long long* __restrict__ clean_tag,
                                                                    unsigned long long tag) {
  __shared__ float rows[kColThreads * kColStride];
  const int K = sh_deg < 0 ? 1 : (sh_deg + 1) * (sh_deg + 1);
  const int C = 3 * K;
  const uint32_t g0 = blockIdx.x * kColThreads;
  const uint32_t cnt = min(uint32_t(kColThreads), n - g0);
  for (uint32_t i = threadIdx.x; i < cnt * uint32_t(C); i += kColThreads)
    rows[(i / C) * kColStride + (i % C)] = colors[size_t(g0) * C + i];
  __syncthreads();
  const uint32_t g = g0 + threadIdx.x;
  const bool live = threadIdx.x < cnt;
  const float* coef = rows + threadIdx.x * kColStride;  // coef[3k + c]
  float gcol[48];
#pragma unroll
  for (int j = 0; j < 48; ++j) gcol[j] = 0.f;
  if (live) {
    float* gflat = reinterpret_cast<float*>(grad2d);
    const float p[3] = {means[3 * g], means[3 * g + 1], means[3 * g + 2]};
    float gm[3] = {0.f, 0.f, 0.f};
    const float* r0 = gflat + 12 * size_t(g) + 6;
    float nd0 = r0[0], nd1 = r0[1], nd2 = r0[2];
    for (int v = 0; v < b.num_views; ++v) {
      const float dc[3] = {nd0, nd1, nd2};
      if (v + 1 < b.num_views) {  // prefetch the next view's colour gradient
        const float* r = gflat + 12 * (size_t(v + 1) * n + g) + 6;
        nd0 = r[0];
        nd1 = r[1];
        nd2 = r[2];
      }
      if (dc[0] == 0.f && dc[1] == 0.f && dc[2] == 0.f) continue;
      {  // consumed: leave the record's colour part zero for the next backward
        float* r = gflat + 12 * (size_t(v) * n + g) + 6;
        r[0] = 0.f;
        r[1] = 0.f;
        r[2] = 0.f;
      }
      if (sh_deg < 0) {
        gcol[0] += dc[0];
        gcol[1] += dc[1];
        gcol[2] += dc[2];
        continue;
      }
      const ViewDev& vd = b.v[v];
      const float d0 = p[0] - vd.campos[0], d1 = p[1] - vd.campos[1], d2 = p[2] - vd.campos[2];
      const float dn = sqrtf(d0 * d0 + d1 * d1 + d2 * d2);
      const float x = d0 / dn, y = d1 / dn, z = d2 / dn;
      float bs[16];
      sh_basis(sh_deg, x, y, z, bs);
      float draw[3];
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        float col = 0.f;
#pragma unroll
        for (int k = 0; k < 16; ++k)
          if (k < K) col += bs[k] * coef[3 * k + c];
        draw[c] = col + 0.5f > 0.f ? dc[c] : 0.f;
      }
      float w[16];  // w_k = sum_c coef_kc draw_c
#pragma unroll
      for (int k = 0; k < 16; ++k) {
        w[k] = 0.f;
        if (k < K) {
#pragma unroll
          for (int c = 0; c < 3; ++c) {
            gcol[3 * k + c] += bs[k] * draw[c];
            w[k] += coef[3 * k + c] * draw[c];
          }
        }
      }
      float dv[3];
      sh_weighted_grad(sh_deg, x, y, z, w, dv);
      const float dot = dv[0] * x + dv[1] * y + dv[2] * z;
      gm[0] += (dv[0] - x * dot) / dn;
      gm[1] += (dv[1] - y * dot) / dn;
      gm[2] += (dv[2] - z * dot) / dn;
    }
    if (sh_deg >= 0) {
#pragma unroll
      for (int c = 0; c < 3; ++c) g_means[3 * g + c] += gm[c];
    }
  }
  __syncthreads();
  float* mine = rows + threadIdx.x * kColStride;
#pragma unroll
  for (int j = 0; j < 48; ++j)
    if (j < C) mine[j] = gcol[j];
  __syncthreads();
  for (uint32_t i = threadIdx.x; i < cnt * uint32_t(C); i += kColThreads)
    g_col[size_t(g0) * C + i] += rows[(i / C) * kColStride + (i % C)];
  // after this kernel and k_project_bwd_geom every record is zero again
  if (blockIdx.x == 0 && threadIdx.x == 0) *clean_tag = tag;
}

// Clears grad2d unless the tag says it is already all zero (the previous
// backward on this layout consumed it).  Blocks only read the tag; the
// colour kernel of the same backward writes it.
__global__ void k_prepare_grad2d(const unsigned long long* __restrict__ clean_tag, unsigned long long tag,
                                 float4* __restrict__ grad2d, size_t count) {
  if (*clean_tag == tag) return;
  for (size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < count; i += size_t(gridDim.x) * blockDim.x)
    grad2d[i] = make_float4(0.f, 0.f, 0.f, 0.f);
}

// Adam (Kingma & Ba 2015), bias-corrected, in place: config-4 training step.
__global__ void k_adam(size_t n, float* __restrict__ p, const float* __restrict__ g, float* __restrict__ m,
                       float* __restrict__ v, float lr, float b1, float b2, float eps, float bc1, float bc2) {
  const size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float gi = g[i];
  const float mi = b1 * m[i] + (1.f - b1) * gi;
  const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
  m[i] = mi;
  v[i] = vi;
  p[i] -= lr * (mi / bc1) / (sqrtf(vi / bc2) + eps);
}

// Fused Adam over the five parameter tensors of a Gaussian scene (one
// launch), with the step count kept on the device so that a captured graph
// replays correctly: every block reads t = *step + 1 and k_adam_step_inc
// stores it after the update.  The update is torch.optim.Adam's (no weight
// decay, no amsgrad), in its order: m += (1-b1)(g - m); v = v b2 + (1-b2) g^2;
// p -= (lr / (1 - b1^t)) m / (sqrt(v) / sqrt(1 - b2^t) + eps), with the
// hyper-parameters and bias corrections formed in double and rounded to
// float as torch rounds its Python scalars.  The opacity tensor is then kept
// in [0, kOpacityMax]: the blend needs alpha < 1 (the backward rebuilds T in
// front of an entry as T / (1 - alpha)).
constexpr float kOpacityMax = 0.999f;

// One Adam element update (the order above); CLAMP keeps the result in
// [0, kOpacityMax].
template <bool CLAMP>
__device__ __forceinline__ void adam_elem(float& p, float g, float& m, float& v, float step_size, float bc2_sqrt,
                                          float w1, float b2f, float w2, float epsf) {
  m = m + w1 * (g - m);
  v = v * b2f + w2 * (g * g);
  const float denom = sqrtf(v) / bc2_sqrt + epsf;
  p = p - step_size * (m / denom);
  if (CLAMP) p = fminf(fmaxf(p, 0.f), kOpacityMax);
}

// One tensor of the scene: 16-byte vectors when its four arrays allow them
// (the same element operations), the rest element by element.
template <bool CLAMP>
__device__ __forceinline__ void adam_tensor(float* __restrict__ p, const float* __restrict__ g, float* __restrict__ m,
                                            float* __restrict__ v, size_t n, float step_size, float bc2_sqrt,
                                            float w1, float b2f, float w2, float epsf) {
  const size_t tid = size_t(blockIdx.x) * blockDim.x + threadIdx.x, stride = size_t(gridDim.x) * blockDim.x;
  size_t head = 0;
  const bool vec = ((reinterpret_cast<uintptr_t>(p) | reinterpret_cast<uintptr_t>(g) |
                     reinterpret_cast<uintptr_t>(m) | reinterpret_cast<uintptr_t>(v)) & 15u) == 0;
  if (vec) {
    const size_t n4 = n / 4;
    float4* p4 = reinterpret_cast<float4*>(p);
    const float4* g4 = reinterpret_cast<const float4*>(g);
    float4* m4 = reinterpret_cast<float4*>(m);
    float4* v4 = reinterpret_cast<float4*>(v);
    for (size_t i = tid; i < n4; i += stride) {
      float4 pp = p4[i], mm = m4[i], vv = v4[i];
      const float4 gg = __ldg(g4 + i);
      adam_elem<CLAMP>(pp.x, gg.x, mm.x, vv.x, step_size, bc2_sqrt, w1, b2f, w2, epsf);
      adam_elem<CLAMP>(pp.y, gg.y, mm.y, vv.y, step_size, bc2_sqrt, w1, b2f, w2, epsf);
      adam_elem<CLAMP>(pp.z, gg.z, mm.z, vv.z, step_size, bc2_sqrt, w1, b2f, w2, epsf);
      adam_elem<CLAMP>(pp.w, gg.w, mm.w, vv.w, step_size, bc2_sqrt, w1, b2f, w2, epsf);
      p4[i] = pp;
      m4[i] = mm;
      v4[i] = vv;
    }
    head = n4 * 4;
  }
  for (size_t i = head + tid; i < n; i += stride) {
    float pp = p[i], mm = m[i], vv = v[i];
    adam_elem<CLAMP>(pp, g[i], mm, vv, step_size, bc2_sqrt, w1, b2f, w2, epsf);
    p[i] = pp;
    m[i] = mm;
    v[i] = vv;
  }
}

__global__ void __launch_bounds__(256) k_adam_fused(AdamSeg seg, double lr, double b1, double b2, double eps,
                                                    const int32_t* __restrict__ step) {
  __shared__ float coef[2];
  if (threadIdx.x == 0) {  // bias corrections once per block
    const double t = double(*step + 1);
    coef[0] = float(lr / (1.0 - pow(b1, t)));
    coef[1] = float(sqrt(1.0 - pow(b2, t)));
  }
  __syncthreads();
  const float step_size = coef[0], bc2_sqrt = coef[1];
  const float w1 = float(1.0 - b1), b2f = float(b2), w2 = float(1.0 - b2), epsf = float(eps);
  size_t begin = 0;
#pragma unroll
  for (int k = 0; k < 5; ++k) {
    const size_t n = seg.end[k] - begin;
    if (k == 3)
      adam_tensor<true>(seg.p[k], seg.g[k], seg.m[k], seg.v[k], n, step_size, bc2_sqrt, w1, b2f, w2, epsf);
    else
      adam_tensor<false>(seg.p[k], seg.g[k], seg.m[k], seg.v[k], n, step_size, bc2_sqrt, w1, b2f, w2, epsf);
    begin = seg.end[k];
  }
}

__global__ void k_adam_step_inc(int32_t* step) {
  if (threadIdx.x == 0 && blockIdx.x == 0) *step += 1;
}

}  // namespace dsplat
