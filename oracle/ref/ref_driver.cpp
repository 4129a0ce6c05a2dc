// ref_driver.cpp -- runs the reference's own CUDA device code serially on the
// CPU (TEST ONLY).  The reference sources are #included from the del-splat
// tree given by -I at build time (oracle/ref/Makefile); nothing is copied.
//
//   tile_acceleration.h:15-52  fill_index_info  (key = tile<<32 | bits(max(z+1,0)))
//   tile_acceleration.h:54-86  count_splat_in_tile
//   splat_point.cu:1-74        rasterize_zbuffer + ztest_and_write_color
//
// The scan and the stable radix sort that the reference takes from the
// (absent) del-cudarc-sys crate are done here with std::partial_sum and
// std::stable_sort, which is what an LSD radix sort of (key, value) produces.
#include "cuda_host_shim.h"

thread_local dsplat_shim_dim3 threadIdx, blockIdx, blockDim;

#include "tile_acceleration.h"
#include "splat_point.cu"

#include <algorithm>
#include <numeric>
#include <vector>

extern "C" {

// tile counts (count_splat_in_tile) + exclusive scan -> tile2idx[T+1]; returns P
uint64_t ref_tiles_count(int64_t n, const float* aabb, uint32_t tile_w,
                         uint32_t tile_h, uint32_t ts, uint32_t* tile2idx) {
  const uint64_t T = uint64_t(tile_w) * tile_h;
  std::vector<uint32_t> tile2ind(T + 1, 0), pnt2ind(n + 1, 0);
  for (int64_t i = 0; i < n; ++i) {
    const cuda::std::array<float, 4> a{aabb[4 * i], aabb[4 * i + 1],
                                       aabb[4 * i + 2], aabb[4 * i + 3]};
    tile_acceleration::count_splat_in_tile(int(i), a, tile2ind.data(),
                                           pnt2ind.data(), tile_w, tile_h, ts);
  }
  tile2idx[0] = 0;
  for (uint64_t t = 0; t < T; ++t) tile2idx[t + 1] = tile2idx[t] + tile2ind[t];
  return tile2idx[T];
}

// fill_index_info over an exclusive scan of per-point counts, then a stable
// sort by the 64-bit key.
void ref_tiles_fill(int64_t n, const float* aabb, const float* xyd,
                    uint32_t tile_w, uint32_t tile_h, uint32_t ts,
                    uint32_t* idx2pnt, uint64_t* keys) {
  const uint64_t T = uint64_t(tile_w) * tile_h;
  std::vector<uint32_t> tile2ind(T + 1, 0), pnt2ind(n + 1, 0), pnt2idx(n + 1, 0);
  for (int64_t i = 0; i < n; ++i) {
    const cuda::std::array<float, 4> a{aabb[4 * i], aabb[4 * i + 1],
                                       aabb[4 * i + 2], aabb[4 * i + 3]};
    tile_acceleration::count_splat_in_tile(int(i), a, tile2ind.data(),
                                           pnt2ind.data(), tile_w, tile_h, ts);
  }
  for (int64_t i = 0; i < n; ++i) pnt2idx[i + 1] = pnt2idx[i] + pnt2ind[i];
  const uint64_t P = pnt2idx[n];
  std::vector<uint64_t> k(P);
  std::vector<uint32_t> v(P);
  for (int64_t i = 0; i < n; ++i) {
    const cuda::std::array<float, 4> a{aabb[4 * i], aabb[4 * i + 1],
                                       aabb[4 * i + 2], aabb[4 * i + 3]};
    tile_acceleration::fill_index_info(int(i), a, xyd[3 * i + 2],
                                       pnt2idx.data(), k.data(), v.data(),
                                       tile_w, tile_h, ts);
  }
  std::vector<uint64_t> ord(P);
  std::iota(ord.begin(), ord.end(), 0);
  std::stable_sort(ord.begin(), ord.end(),
                   [&](uint64_t a, uint64_t b) { return k[a] < k[b]; });
  for (uint64_t j = 0; j < P; ++j) {
    idx2pnt[j] = v[ord[j]];
    if (keys) keys[j] = k[ord[j]];
  }
}

// rasterize_zbuffer for every point in index order; pix2unitdepth must be
// pre-filled with FLT_MAX by the caller (dlpack splat_point.rs:87).
void ref_point_zbuffer(uint32_t n, const float* xyd, const float* rgb,
                       float* pix2unitdepth, float* pix2rgb, int w, int h) {
  blockDim = {1, 1, 1};
  threadIdx = {0, 0, 0};
  for (uint32_t i = 0; i < n; ++i) {
    blockIdx = {i, 0, 0};
    rasterize_zbuffer(n, xyd, rgb, pix2unitdepth, pix2rgb, w, h);
  }
}

}  // extern "C"
