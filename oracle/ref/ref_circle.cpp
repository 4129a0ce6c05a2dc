// ref_circle.cpp -- runs the reference's splat_circle.cu on the CPU (TEST
// ONLY).  The source is #included from the del-splat tree given by -I at
// build time (oracle/ref/Makefile); nothing is copied.
//
//   splat_circle.cu:7-41    splat3_to_splat2            (circle projection)
//   splat_circle.cu:93-132  rasterize_splat_using_tile  (last covering entry wins)
#define DSPLAT_SHIM_INTERNAL
#define splat3_to_splat2 circle_splat3_to_splat2
#define count_splat_in_tile circle_count_splat_in_tile
#define fill_index_info circle_fill_index_info
#define rasterize_splat_using_tile circle_rasterize_splat_using_tile
#include "cuda_host_shim.h"

#include "splat_circle.cu"

extern "C" {

void ref_circle_project(uint32_t n, const float* xyz, const float* mvp, uint32_t w, uint32_t h, float radius,
                        float* xyd, float* rad) {
  blockDim = {1, 1, 1};
  threadIdx = {0, 0, 0};
  for (uint32_t i = 0; i < n; ++i) {
    blockIdx = {i, 0, 0};
    splat3_to_splat2(n, xyz, xyd, rad, mvp, w, h, radius);
  }
}

void ref_circle_rasterize(uint32_t w, uint32_t h, float* pix2rgb, uint32_t ts, const uint32_t* tile2idx,
                          const uint32_t* idx2pnt, const float* xyd, const float* rad, const float* rgb) {
  const uint32_t tw = (w + ts - 1) / ts, th = (h + ts - 1) / ts;
#pragma omp parallel for schedule(dynamic, 4)
  for (int64_t iy = 0; iy < int64_t(h); ++iy) {
    blockDim = {1, 1, 1};
    threadIdx = {0, 0, 0};
    for (uint32_t ix = 0; ix < w; ++ix) {
      blockIdx = {ix, uint32_t(iy), 0};
      rasterize_splat_using_tile(w, h, pix2rgb, tw, th, ts, tile2idx, idx2pnt, xyd, rad, rgb);
    }
  }
}

}  // extern "C"
