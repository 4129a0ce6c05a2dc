// zbuffer.cu -- point and circle splatting through a packed 64-bit z-buffer.
//
// Every pixel keeps the minimum of a 64-bit key; the high word orders by depth
// (nearest wins) and the low word, 0xFFFFFFFE - index, makes the larger point
// index win a depth tie.  One atomicMin per covered pixel, then a resolve pass
// gathers the winner's colour.  This is deterministic, unlike the reference's
// CAS loop followed by an unordered colour store (splat_point.cu:14-45), and
// it reproduces the reference's sequential painters exactly:
//
//  * points (del-splat-cpu/src/pnt2pixxyndcz.rs:1-40, render_pix_sort_depth):
//    stable sort by ndc_z+1, skip ndc_z <= -1 or >= 1, overwrite -> the
//    nearest (largest ndc_z+1) wins, ties -> larger index; pixel = Rust
//    `as usize` truncation (negative / NaN -> 0).  High word: ~bits(z+1).
//  * circles (del-splat-cuda-kernels/cuda/splat_circle.cu:93-132 over the
//    tile lists of tile_acceleration.h): ascending (tile, bits(max(z+1,0)),
//    index) walk, covered iff sqrt(dx^2+dy^2) <= rad, last writer wins ->
//    largest depth bits, ties -> larger index, restricted to circles listed
//    in the pixel's tile.  High word: ~bits(max(z+1,0)).
//
// The all-ones key means "no point"; it can never be produced (low word <=
// 0xFFFFFFFE).
#include <cfloat>
#include <cstdio>

#include "common.cuh"

namespace dsplat {

constexpr uint64_t kEmpty = ~0ull;

__global__ void k_fill_u64(uint64_t* __restrict__ p, size_t n, uint64_t v) {
  const size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i < n) p[i] = v;
}

__global__ void k_point_zbuf(uint32_t n, const float* __restrict__ xyd, int w, int h, uint64_t* __restrict__ zbuf) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float z = xyd[3 * i + 2];
  if (!(z > -1.f && z < 1.f)) return;
  const float x = xyd[3 * i], y = xyd[3 * i + 1];
  int ix, iy;
  if (!(x >= 0.f)) ix = 0;
  else if (x >= float(w)) return;
  else ix = int(x);
  if (!(y >= 0.f)) iy = 0;
  else if (y >= float(h)) return;
  else iy = int(y);
  const uint32_t hi = ~__float_as_uint(fa(z, 1.f));
  const uint64_t key = (uint64_t(hi) << 32) | uint64_t(0xFFFFFFFEu - i);
  atomicMin(reinterpret_cast<unsigned long long*>(zbuf + size_t(iy) * w + ix), (unsigned long long)key);
}

// rgb / unit depth of the winner (splat_point.cu:66: unitdepth computed in
// double: 1 - (ndcz + 1) * 0.5); empty pixels: rgb untouched, depth FLT_MAX.
__global__ void k_point_resolve(size_t npix, const uint64_t* __restrict__ zbuf, const float* __restrict__ xyd,
                                const float* __restrict__ rgb, float* __restrict__ pix2rgb,
                                float* __restrict__ pix2unitdepth, int32_t* __restrict__ winner) {
  const size_t p = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (p >= npix) return;
  const uint64_t key = zbuf[p];
  if (key == kEmpty) {
    if (pix2unitdepth) pix2unitdepth[p] = FLT_MAX;
    if (winner) winner[p] = -1;
    return;
  }
  const uint32_t i = 0xFFFFFFFEu - uint32_t(key & 0xffffffffu);
  if (pix2rgb) {
    pix2rgb[3 * p] = rgb[3 * size_t(i)];
    pix2rgb[3 * p + 1] = rgb[3 * size_t(i) + 1];
    pix2rgb[3 * p + 2] = rgb[3 * size_t(i) + 2];
  }
  if (pix2unitdepth) pix2unitdepth[p] = float(1.0 - (double(xyd[3 * size_t(i) + 2]) + 1.0) * 0.5);
  if (winner) winner[p] = int32_t(i);
}

__global__ void k_circle_zbuf(uint32_t n, const float* __restrict__ xyd, const float* __restrict__ rad, int w, int h,
                              int ts, uint64_t* __restrict__ zbuf) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float x = xyd[3 * i], y = xyd[3 * i + 1], r = rad[i];
  const int tile_w = (w + ts - 1) / ts, tile_h = (h + ts - 1) / ts;
  const float tsf = tile_inv(ts);
  // the circle's tile span, exactly as the tile lists compute it
  const int tx0 = tile_lo(fs(x, r), tsf, tile_w), ty0 = tile_lo(fs(y, r), tsf, tile_h);
  const int tx1 = tile_hi(fa(x, r), tsf, tile_w), ty1 = tile_hi(fa(y, r), tsf, tile_h);
  if (tx1 <= tx0 || ty1 <= ty0) return;
  const uint32_t hi = ~depth_bits(xyd[3 * i + 2]);
  const uint64_t key = (uint64_t(hi) << 32) | uint64_t(0xFFFFFFFEu - i);
  // candidate pixels: the span's pixels intersected with a 1-pixel-padded box
  int px0 = tx0 * ts, py0 = ty0 * ts, px1 = min(tx1 * ts, w), py1 = min(ty1 * ts, h);
  const float bx0 = floorf(x - r) - 1.f, by0 = floorf(y - r) - 1.f, bx1 = floorf(x + r) + 2.f,
              by1 = floorf(y + r) + 2.f;
  if (bx0 > float(px0)) px0 = bx0 < float(px1) ? int(bx0) : px1;
  if (by0 > float(py0)) py0 = by0 < float(py1) ? int(by0) : py1;
  if (bx1 < float(px1)) px1 = bx1 > float(px0) ? int(bx1) : px0;
  if (by1 < float(py1)) py1 = by1 > float(py0) ? int(by1) : py0;
  for (int iy = py0; iy < py1; ++iy) {
    const float dy = fs(y, float(iy) + 0.5f);
    for (int ix = px0; ix < px1; ++ix) {
      const float dx = fs(x, float(ix) + 0.5f);
      const float dist = sqrtf(fa(fm(dx, dx), fm(dy, dy)));
      if (dist > r) continue;
      atomicMin(reinterpret_cast<unsigned long long*>(zbuf + size_t(iy) * w + ix), (unsigned long long)key);
    }
  }
}

// colour_kind 0: float rgb[3] -> pix float[3]; 1: u32 rgba -> pix u32.
__global__ void k_circle_resolve(size_t npix, const uint64_t* __restrict__ zbuf, const void* __restrict__ colors,
                                 int color_kind, void* __restrict__ pix, int32_t* __restrict__ winner) {
  const size_t p = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (p >= npix) return;
  const uint64_t key = zbuf[p];
  if (key == kEmpty) {
    if (winner) winner[p] = -1;
    return;
  }
  const uint32_t i = 0xFFFFFFFEu - uint32_t(key & 0xffffffffu);
  if (pix) {
    if (color_kind == 0) {
      const float* c = static_cast<const float*>(colors);
      float* o = static_cast<float*>(pix);
      o[3 * p] = c[3 * size_t(i)];
      o[3 * p + 1] = c[3 * size_t(i) + 1];
      o[3 * p + 2] = c[3 * size_t(i) + 2];
    } else {
      static_cast<uint32_t*>(pix)[p] = static_cast<const uint32_t*>(colors)[i];
    }
  }
  if (winner) winner[p] = int32_t(i);
}

// ---------------------------------------------------------------------------
// Allocation-free variant of the point z-buffer.
//
// dsplat_point_rasterize_pix_zbuffer needs a W*H array of 64-bit keys from
// the caller.  Some callers cannot provide one: a render plug-in whose host
// application owns every device allocation and gives the library none, or a
// real-time loop that may not call cudaMalloc (it can block the whole device)
// and has no workspace to lend.  For them the keys live in this file-scope
// device array instead: 2^20 keys (8 MiB), enough for 1024x1024 or 1280x720.
// It is part of the module, so every GPU that loads libdsplat.so holds these
// 8 MiB until the process exits.
// ---------------------------------------------------------------------------
constexpr size_t kNoAllocMaxPixels = size_t(1) << 20;
static __device__ __align__(256) unsigned long long g_noalloc_zbuf[kNoAllocMaxPixels];

int report_error(int code, const char* msg);

namespace {
// Device address of g_noalloc_zbuf on the current device (host code only sees
// a host-side stand-in under that name).  Looked up on every call, with the
// caller's device current: the lookup is cheap, and a cached address would go
// stale if the caller reset the device (the module, and the array with it,
// is then loaded again at another address).
int noalloc_scratch(uint64_t** out) {
  void* p = nullptr;
  const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_zbuf);
  if (e != cudaSuccess || !p) {
    char msg[200];
    snprintf(msg, sizeof(msg), "cudaGetSymbolAddress(g_noalloc_zbuf) failed: %s", cudaGetErrorString(e));
    return report_error(DSPLAT_ERR_CUDA, msg);
  }
  *out = static_cast<uint64_t*>(p);
  return DSPLAT_OK;
}
}  // namespace
}  // namespace dsplat

// Same contract and results as dsplat_point_rasterize_pix_zbuffer, without the
// zbuf argument: the keys are kept in the library's own 2^20-entry device
// array.  Images larger than 2^20 pixels are rejected.  Every call looks the
// array's device address up (cudaGetSymbolAddress) on the current device; the
// first call on a device also loads the library's module there -- make that
// first call before any stream capture.  All calls share the one array (it is refilled at
// the start of every call), so calls whose GPU work overlaps -- on different
// streams or host threads -- race and must be serialised by the caller.
extern "C" int dsplat_point_rasterize_pix_zbuffer_noalloc(dsplat_stream stream, uint32_t num_pnt,
                                                          const float* pnt2pixxyndcz, const float* pnt2rgb,
                                                          float* pix2rgb, float* pix2unitdepth, int32_t* pix2winner,
                                                          uint32_t img_w, uint32_t img_h) {
  using namespace dsplat;
  const size_t npix = size_t(img_w) * img_h;
  if (npix == 0) return DSPLAT_OK;
  if (npix > kNoAllocMaxPixels) {
    char msg[160];
    snprintf(msg, sizeof(msg), "image of %zu pixels exceeds the allocation-free z-buffer limit of %zu pixels", npix,
             kNoAllocMaxPixels);
    return report_error(DSPLAT_ERR_INVALID_ARG, msg);
  }
  if ((num_pnt > 0 && !pnt2pixxyndcz) || (pix2rgb && !pnt2rgb)) return report_error(DSPLAT_ERR_INVALID_ARG, "null pointer");
  uint64_t* zbuf = nullptr;
  const int rc = noalloc_scratch(&zbuf);
  if (rc) return rc;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  k_fill_u64<<<unsigned((npix + 255) / 256), 256, 0, st>>>(zbuf, npix, ~0ull);
  count_launch();
  if (num_pnt > 0) {
    k_point_zbuf<<<(num_pnt + 255) / 256, 256, 0, st>>>(num_pnt, pnt2pixxyndcz, int(img_w), int(img_h), zbuf);
    count_launch();
  }
  k_point_resolve<<<unsigned((npix + 255) / 256), 256, 0, st>>>(npix, zbuf, pnt2pixxyndcz, pnt2rgb, pix2rgb,
                                                                pix2unitdepth, pix2winner);
  count_launch();
  if (cudaGetLastError() != cudaSuccess) return report_error(DSPLAT_ERR_CUDA, "allocation-free point z-buffer launch");
  return DSPLAT_OK;
}
