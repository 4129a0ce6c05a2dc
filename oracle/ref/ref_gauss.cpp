// ref_gauss.cpp -- runs the reference's splat_gauss.cu on the CPU (TEST ONLY).
// The source is #included from the del-splat tree given by -I at build time
// (oracle/ref/Makefile); nothing is copied.  Its del-geo includes resolve to
// oracle/ref/del_geo/ (the oracle's restatement of the absent crate).
//
//   splat_gauss.cu:10-53   splat3_to_splat2            (projection)
//   splat_gauss.cu:56-109  rasterize_splat_using_tile  (front-to-back blend)
//
// On the host, `expf` is the C library's and `alpha_sum > 0.999` compares in
// double exactly as written; with -ffp-contract=off nothing is fused, so the
// blend performs del-splat-cpu's f32 operations (pnt2pixxyndcz.rs:86-93)
// apart from that double stop test.
#define DSPLAT_SHIM_INTERNAL
#define splat3_to_splat2 gauss_splat3_to_splat2
#define count_splat_in_tile gauss_count_splat_in_tile
#define fill_index_info gauss_fill_index_info
#define rasterize_splat_using_tile gauss_rasterize_splat_using_tile
#include "cuda_host_shim.h"

#include "splat_gauss.cu"

extern "C" {

void ref_gauss_project(uint32_t n, const float* xyz, const float* quat, const float* scale, const float* mvp,
                       uint32_t w, uint32_t h, float* xyd, float* conic, float* aabb) {
  blockDim = {1, 1, 1};
  threadIdx = {0, 0, 0};
  for (uint32_t i = 0; i < n; ++i) {
    blockIdx = {i, 0, 0};
    splat3_to_splat2(n, xyd, conic, aabb, xyz, quat, scale, mvp, w, h);
  }
}

// pix2rgb accumulates (the caller zeroes it, as del-splat-cudarc does).
void ref_gauss_rasterize(uint32_t w, uint32_t h, float* pix2rgb, const float* xyd, const float* conic,
                         const float* aabb, const float* opacity, const float* rgb, uint32_t ts,
                         const uint32_t* tile2idx, const uint32_t* idx2pnt) {
  const uint32_t tw = (w + ts - 1) / ts, th = (h + ts - 1) / ts;
#pragma omp parallel for schedule(dynamic, 4)
  for (int64_t iy = 0; iy < int64_t(h); ++iy) {
    blockDim = {1, 1, 1};
    threadIdx = {0, 0, 0};
    for (uint32_t ix = 0; ix < w; ++ix) {
      blockIdx = {ix, uint32_t(iy), 0};
      rasterize_splat_using_tile(w, h, pix2rgb, xyd, conic, aabb, opacity, rgb, tw, th, ts, tile2idx, idx2pnt);
    }
  }
}

}  // extern "C"
