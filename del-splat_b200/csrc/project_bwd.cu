// project_bwd.cu -- backward of the fused projection (no reference
// counterpart; the reference has no gradient code).
//
// One thread per Gaussian reads its parameters once, loops over the views of
// the batch, pulls the per-view 2D gradient (d px, d py, d conic, d opacity,
// d rgb) written by the backward rasteriser and accumulates the parameter
// gradients in registers; it then adds them into the caller's gradient
// buffers (so a per-view loop accumulates naturally).
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

__device__ __forceinline__ void sh_basis_and_grad(int deg, float x, float y, float z, float* b, float* db) {
#pragma unroll
  for (int k = 0; k < 48; ++k) db[k] = 0.f;
  const float C0 = 0.28209479177387814f, C1 = 0.4886025119029199f;
  b[0] = C0;
  if (deg < 1) return;
  b[1] = -C1 * y;
  b[2] = C1 * z;
  b[3] = -C1 * x;
  db[1 * 3 + 1] = -C1;
  db[2 * 3 + 2] = C1;
  db[3 * 3 + 0] = -C1;
  if (deg < 2) return;
  const float C20 = 1.0925484305920792f, C21 = -1.0925484305920792f, C22 = 0.31539156525252005f,
              C23 = -1.0925484305920792f, C24 = 0.5462742152960396f;
  const float xx = x * x, yy = y * y, zz = z * z, xy = x * y, yz = y * z, xz = x * z;
  b[4] = C20 * xy;
  b[5] = C21 * yz;
  b[6] = C22 * (2.f * zz - xx - yy);
  b[7] = C23 * xz;
  b[8] = C24 * (xx - yy);
  db[4 * 3 + 0] = C20 * y;
  db[4 * 3 + 1] = C20 * x;
  db[5 * 3 + 1] = C21 * z;
  db[5 * 3 + 2] = C21 * y;
  db[6 * 3 + 0] = -2.f * C22 * x;
  db[6 * 3 + 1] = -2.f * C22 * y;
  db[6 * 3 + 2] = 4.f * C22 * z;
  db[7 * 3 + 0] = C23 * z;
  db[7 * 3 + 2] = C23 * x;
  db[8 * 3 + 0] = 2.f * C24 * x;
  db[8 * 3 + 1] = -2.f * C24 * y;
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
  db[9 * 3 + 0] = C30 * 6.f * x * y;
  db[9 * 3 + 1] = C30 * (3.f * xx - 3.f * yy);
  db[10 * 3 + 0] = C31 * y * z;
  db[10 * 3 + 1] = C31 * x * z;
  db[10 * 3 + 2] = C31 * x * y;
  db[11 * 3 + 0] = C32 * (-2.f * x * y);
  db[11 * 3 + 1] = C32 * (4.f * zz - xx - 3.f * yy);
  db[11 * 3 + 2] = C32 * (8.f * y * z);
  db[12 * 3 + 0] = C33 * (-6.f * x * z);
  db[12 * 3 + 1] = C33 * (-6.f * y * z);
  db[12 * 3 + 2] = C33 * (6.f * zz - 3.f * xx - 3.f * yy);
  db[13 * 3 + 0] = C34 * (4.f * zz - 3.f * xx - yy);
  db[13 * 3 + 1] = C34 * (-2.f * x * y);
  db[13 * 3 + 2] = C34 * (8.f * x * z);
  db[14 * 3 + 0] = C35 * (2.f * x * z);
  db[14 * 3 + 1] = C35 * (-2.f * y * z);
  db[14 * 3 + 2] = C35 * (xx - yy);
  db[15 * 3 + 0] = C36 * (3.f * xx - 3.f * yy);
  db[15 * 3 + 1] = C36 * (-6.f * x * y);
}

}  // namespace

__global__ void __launch_bounds__(128) k_project_bwd(uint32_t n, int sh_deg, const float* __restrict__ means,
                                                     const float* __restrict__ log_scales,
                                                     const float* __restrict__ quats,
                                                     const float* __restrict__ colors, const ViewBatch b,
                                                     const float4* __restrict__ grad2d, float* __restrict__ g_means,
                                                     float* __restrict__ g_ls, float* __restrict__ g_quats,
                                                     float* __restrict__ g_op, float* __restrict__ g_col) {
  const uint32_t g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= n) return;
  const float p[3] = {means[3 * g], means[3 * g + 1], means[3 * g + 2]};
  const float s[3] = {dexp(log_scales[3 * g]), dexp(log_scales[3 * g + 1]), dexp(log_scales[3 * g + 2])};
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
  const int K = sh_deg < 0 ? 1 : (sh_deg + 1) * (sh_deg + 1);
  float coef[48];
#pragma unroll
  for (int k = 0; k < 48; ++k) coef[k] = k < 3 * K ? colors[size_t(g) * 3 * K + k] : 0.f;
  float gm[3] = {0.f, 0.f, 0.f}, gs2[3] = {0.f, 0.f, 0.f}, gR[9], gop = 0.f, gcol[48];
#pragma unroll
  for (int k = 0; k < 9; ++k) gR[k] = 0.f;
#pragma unroll
  for (int k = 0; k < 48; ++k) gcol[k] = 0.f;

  for (int v = 0; v < b.num_views; ++v) {
    const float4* gp = grad2d + 3 * (size_t(v) * n + g);
    const float4 g0 = gp[0], g1 = gp[1];
    const float gbl = gp[2].x;
    if (g0.x == 0.f && g0.y == 0.f && g0.z == 0.f && g0.w == 0.f && g1.x == 0.f && g1.y == 0.f && g1.z == 0.f &&
        g1.w == 0.f && gbl == 0.f)
      continue;
    const ViewDev& vd = b.v[v];
    const float* M = vd.mvp;
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
    const float N0 = 0.5f * float(vd.w), N3 = -0.5f * float(vd.h), N4 = 0.5f * float(vd.w), N5 = 0.5f * float(vd.h);
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
      gs2[k] += u * u * dsa + u * vv * dsb + vv * vv * dsc;
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
      for (int j = 0; j < 3; ++j) gR[k + 3 * j] += P[2 * k] * dPR[2 * j] + P[1 + 2 * k] * dPR[1 + 2 * j];
    float dJ[9];
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      dJ[0 + 3 * j] = N0 * dP[2 * j];
      dJ[1 + 3 * j] = N3 * dP[1 + 2 * j];
      dJ[2 + 3 * j] = N4 * dP[2 * j] + N5 * dP[1 + 2 * j];
    }
#pragma unroll
    for (int m = 0; m < 3; ++m) {
      float acc = g0.x * N0 * J[0 + 3 * m] + g0.y * N3 * J[1 + 3 * m];
#pragma unroll
      for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) {
          const float d = -M[i + 4 * j] * M[3 + 4 * m] * iw2 - M[i + 4 * m] * M[3 + 4 * j] * iw2 +
                          2.f * a[i] * M[3 + 4 * j] * M[3 + 4 * m] * iw3;
          acc += dJ[i + 3 * j] * d;
        }
      gm[m] += acc;
    }
    gop += g1.y;
    const float dcol[3] = {g1.z, g1.w, gbl};
    if (sh_deg < 0) {
      gcol[0] += dcol[0];
      gcol[1] += dcol[1];
      gcol[2] += dcol[2];
    } else {
      const float d0 = p[0] - vd.campos[0], d1 = p[1] - vd.campos[1], d2 = p[2] - vd.campos[2];
      const float dn = sqrtf(d0 * d0 + d1 * d1 + d2 * d2);
      const float x = d0 / dn, y = d1 / dn, z = d2 / dn;
      float bs[16], db[48];
      sh_basis_and_grad(sh_deg, x, y, z, bs, db);
      float draw[3];
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        float acc = 0.f;
#pragma unroll
        for (int k = 0; k < 16; ++k)
          if (k < K) acc += bs[k] * coef[k * 3 + c];
        draw[c] = acc + 0.5f > 0.f ? dcol[c] : 0.f;
      }
      float dn3[3] = {0.f, 0.f, 0.f};
#pragma unroll
      for (int k = 0; k < 16; ++k) {
        if (k < K) {
          float gk = 0.f;
#pragma unroll
          for (int c = 0; c < 3; ++c) {
            gcol[k * 3 + c] += bs[k] * draw[c];
            gk += coef[k * 3 + c] * draw[c];
          }
          dn3[0] += gk * db[k * 3];
          dn3[1] += gk * db[k * 3 + 1];
          dn3[2] += gk * db[k * 3 + 2];
        }
      }
      const float dot = dn3[0] * x + dn3[1] * y + dn3[2] * z;
      gm[0] += (dn3[0] - x * dot) / dn;
      gm[1] += (dn3[1] - y * dot) / dn;
      gm[2] += (dn3[2] - z * dot) / dn;
    }
  }
  // rotation -> unit quaternion -> raw quaternion
  float dq[4];
  {
    const float x = qn[0], y = qn[1], z = qn[2], ww = qn[3];
    auto G = [&](int i, int j) { return gR[i + 3 * j]; };
    const float dqx = G(1, 0) * 2.f * y + G(2, 0) * 2.f * z + G(0, 1) * 2.f * y - G(1, 1) * 4.f * x +
                      G(2, 1) * 2.f * ww + G(0, 2) * 2.f * z - G(1, 2) * 2.f * ww - G(2, 2) * 4.f * x;
    const float dqy = -G(0, 0) * 4.f * y + G(1, 0) * 2.f * x - G(2, 0) * 2.f * ww + G(0, 1) * 2.f * x +
                      G(2, 1) * 2.f * z + G(0, 2) * 2.f * ww + G(1, 2) * 2.f * z - G(2, 2) * 4.f * y;
    const float dqz = -G(0, 0) * 4.f * z + G(1, 0) * 2.f * ww + G(2, 0) * 2.f * x - G(0, 1) * 2.f * ww -
                      G(1, 1) * 4.f * z + G(2, 1) * 2.f * y + G(0, 2) * 2.f * x + G(1, 2) * 2.f * y;
    const float dqw = G(1, 0) * 2.f * z - G(2, 0) * 2.f * y - G(0, 1) * 2.f * z + G(2, 1) * 2.f * x +
                      G(0, 2) * 2.f * y - G(1, 2) * 2.f * x;
    const float dot = dqx * x + dqy * y + dqz * z + dqw * ww;
    dq[0] = (dqx - x * dot) / nrm;
    dq[1] = (dqy - y * dot) / nrm;
    dq[2] = (dqz - z * dot) / nrm;
    dq[3] = (dqw - ww * dot) / nrm;
  }
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    g_means[3 * g + c] += gm[c];
    g_ls[3 * g + c] += gs2[c] * 2.f * dd[c];
  }
#pragma unroll
  for (int c = 0; c < 4; ++c) g_quats[4 * g + c] += dq[c];
  g_op[g] += gop;
#pragma unroll
  for (int k = 0; k < 48; ++k)
    if (k < 3 * K) g_col[size_t(g) * 3 * K + k] += gcol[k];
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

}  // namespace dsplat
