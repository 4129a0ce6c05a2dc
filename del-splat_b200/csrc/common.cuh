// common.cuh -- shared device helpers for the del-splat B200 kernels.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "dsplat.h"

#include <atomic>

#define DSPLAT_MAX_VIEWS 32

namespace dsplat {

// Host-side count of kernel launches issued by this library (dsplat_launch_count).
inline std::atomic<uint64_t> g_launches{0};
inline void count_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }

// ---------------------------------------------------------------------------
// Per-view constants, passed to kernels by value (<= 32 views, ~3 KB).
// ---------------------------------------------------------------------------
struct ViewDev {
  float mvp[16];   // column-major world -> NDC
  float campos[3];
  int32_t w, h;
  int32_t tile_w, tile_h;
  uint32_t item_base;  // first global (view, tile) item of this view
  uint32_t pix_base;   // first pixel of this view in the concatenated images
  uint32_t sb_base;    // first superblock of this view
  int32_t sb_log2;     // superblock side = 1 << sb_log2 tiles (0..3)
};

// superblock grid of a view
__host__ __device__ __forceinline__ int sb_cols(const ViewDev& d) {
  return (d.tile_w + (1 << d.sb_log2) - 1) >> d.sb_log2;
}
__host__ __device__ __forceinline__ int sb_rows(const ViewDev& d) {
  return (d.tile_h + (1 << d.sb_log2) - 1) >> d.sb_log2;
}

struct ViewBatch {
  int32_t num_views;
  int32_t ts;          // tile size in pixels (8, 16 or 32)
  uint32_t num_items;  // sum of tile counts
  uint32_t num_pix;    // sum of pixel counts
  uint32_t num_sb;     // sum of superblock counts
  uint32_t max_sb;     // largest per-view superblock count
  int32_t ppl;         // rasteriser pixels per lane (warp task = 32 * ppl pixels)
  uint32_t max_sb_side;  // largest per-view superblock column or row count (<= 255)
  ViewDev v[DSPLAT_MAX_VIEWS];
};

// Arguments of the fused rasteriser launches (host side).
struct FwdArgs {
  uint32_t n;
  const float4* rec;
  const uint2* list1;
  const uint32_t* off1;
  uint32_t nchunk;
  uint64_t capacity;
  const uint32_t* order;
  uint32_t* counter;
  float* out_rgb;
  float* out_T;
  uint32_t* out_last;
  const float* target;
  float* grad_pix;
  float* slab_loss;
  uint32_t* item_cost;
};

struct BwdArgs {
  uint32_t n;
  const float4* rec;
  const uint2* list1;
  const uint32_t* off1;
  uint32_t nchunk;
  uint64_t capacity;
  const uint32_t* order;
  uint32_t* counter;
  const float* grad_pix;
  const float* pix_T;
  const uint32_t* pix_last;
  float4* grad2d;
};



__device__ __forceinline__ int view_of_item(const ViewBatch& b, uint32_t item) {
  int v = 0;
#pragma unroll 1
  for (int k = 1; k < b.num_views; ++k)
    if (item >= b.v[k].item_base) v = k;
  return v;
}

// ---------------------------------------------------------------------------
// Non-contracted IEEE single-precision arithmetic.  The stages whose results
// are compared bit-for-bit with the CPU oracle use these (or are compiled
// with -fmad=false) so that no multiply-add is fused.
// ---------------------------------------------------------------------------
__device__ __forceinline__ float fm(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float fa(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float fs(float a, float b) { return __fsub_rn(a, b); }

// Deterministic exp(x): Cody-Waite reduction x = n*ln2 + r with ln2 split in
// a high part that has 9 trailing zero bits (so n*LN2_HI is exact for
// |n| < 512) and a low part, then the degree-7 Taylor polynomial of e^r on
// |r| <= ln2/2 (truncation error < 6e-9 relative) and an exact 2^n scaling.
// Only IEEE-exact operations are used, so the CPU oracle reproduces every
// bit.  Results below 2^-126 flush to zero.
__device__ __forceinline__ float dexp(float x) {
  if (x != x) return x;
  if (x < -87.0f) return 0.0f;
  if (x > 88.5f) return __int_as_float(0x7f800000);
  const float n = rintf(fm(x, 1.44269502162933349609375f));
  float r = fs(x, fm(n, 0.693145751953125f));
  r = fs(r, fm(n, 1.428606765330187045e-06f));
  float p = 1.984126984126984e-04f;  // 1/5040
  p = fa(fm(p, r), 1.388888888888889e-03f);  // 1/720
  p = fa(fm(p, r), 8.333333333333333e-03f);  // 1/120
  p = fa(fm(p, r), 4.166666666666667e-02f);  // 1/24
  p = fa(fm(p, r), 1.666666666666667e-01f);  // 1/6
  p = fa(fm(p, r), 0.5f);
  p = fa(fm(p, r), 1.0f);
  p = fa(fm(p, r), 1.0f);
  const int ni = (int)n;
  if (ni < -126) return 0.0f;
  return fm(p, __int_as_float((ni + 127) << 23));
}

// Fused multiply-add with a single rounding (IEEE fma; the CPU oracle's
// std::fma gives the same bits).
__device__ __forceinline__ float ff(float a, float b, float c) { return __fmaf_rn(a, b, c); }

// The rasterisers evaluate exp(-q/2) as 2^y with y = q * (-log2(e)/2); the
// factor is folded into the staged conic, so y comes out of the quadratic
// form directly.
constexpr float kNegHalfLog2e = -0.72134752044448170368f;
constexpr float kInvNegHalfLog2e = -1.38629436111989061883f;  // -2 ln 2

// Deterministic 2^y: y = n + f with n = nearest integer (the 1.5 * 2^23
// addition rounds y in the binade where the float spacing is 1; n is read
// back from the sum's bits), |f| <= 1/2, then a degree-5 polynomial
// 1 + f (c1 + f (c2 + ...)) fitted to 2^f on [-1/2, 1/2] by minimising the
// largest relative error (linear program on a dense grid, oracle/fit_exp2.py;
// 6.8e-8 before rounding, 2.2e-7 measured over every float f of the
// interval after float rounding and evaluation) in Horner form with fused
// multiply-adds, and the exact scaling by 2^n through the exponent field.  Every step is an exactly rounded IEEE operation, so the CPU oracle
// reproduces the result bit for bit.  Outside (-125, 123): 0 below, +inf
// above, NaN stays NaN.
constexpr float kExp2C1 = 0.6931465864181519f, kExp2C2 = 0.24022166430950165f, kExp2C3 = 0.055510472506284714f,
                kExp2C4 = 0.009674952365458012f, kExp2C5 = 0.0013202981790527701f;
__device__ __forceinline__ float exp2_det(float y) {
  if (!(fabsf(__fadd_rn(y, 1.f)) < 124.f)) {
    if (y != y) return y;
    return y < 0.f ? 0.f : __int_as_float(0x7f800000);
  }
  const float t = __fadd_rn(y, 12582912.f);
  const float f = __fsub_rn(y, __fsub_rn(t, 12582912.f));
  float p = kExp2C5;
  p = ff(p, f, kExp2C4);
  p = ff(p, f, kExp2C3);
  p = ff(p, f, kExp2C2);
  p = ff(p, f, kExp2C1);
  p = ff(p, f, 1.f);
  const uint32_t n = uint32_t(__float_as_int(t) - __float_as_int(12582912.f));
  return __int_as_float(int(uint32_t(__float_as_int(p)) + (n << 23)));
}

// Packed two-wide FP32 (sm_100 f32x2): each element is the exactly rounded
// IEEE result of the scalar operation, so packed and scalar sequences give
// the same bits.  f2 holds (lo, hi) = (first, second) element.
typedef unsigned long long f2;
__device__ __forceinline__ f2 f2_make(float lo, float hi) {
  f2 r;
  asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(lo), "f"(hi));
  return r;
}
__device__ __forceinline__ f2 f2_dup(float v) { return f2_make(v, v); }
__device__ __forceinline__ float f2_lo(f2 v) {
  float lo, hi;
  asm("mov.b64 {%0, %1}, %2;" : "=f"(lo), "=f"(hi) : "l"(v));
  return lo;
}
__device__ __forceinline__ float f2_hi(f2 v) {
  float lo, hi;
  asm("mov.b64 {%0, %1}, %2;" : "=f"(lo), "=f"(hi) : "l"(v));
  return hi;
}
__device__ __forceinline__ f2 add2(f2 a, f2 b) {
  f2 r;
  asm("add.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b));
  return r;
}
__device__ __forceinline__ f2 sub2(f2 a, f2 b) {
  f2 r;
  asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b));
  return r;
}
__device__ __forceinline__ f2 mul2(f2 a, f2 b) {
  f2 r;
  asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b));
  return r;
}
__device__ __forceinline__ f2 fma2(f2 a, f2 b, f2 c) {
  f2 r;
  asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(r) : "l"(a), "l"(b), "l"(c));
  return r;
}

// exp2_det2_inrange: exp2_det's fast path on both elements, packed; equal
// to exp2_det for elements in (-125, 123).  A caller that has bounded y to
// that range (see fwd_slab) uses it directly.
__device__ __forceinline__ f2 exp2_det2_inrange(f2 y) {
  const f2 magic = f2_dup(12582912.f);
  const f2 t = add2(y, magic);
  const f2 f = sub2(y, sub2(t, magic));
  f2 p = f2_dup(kExp2C5);
  p = fma2(p, f, f2_dup(kExp2C4));
  p = fma2(p, f, f2_dup(kExp2C3));
  p = fma2(p, f, f2_dup(kExp2C2));
  p = fma2(p, f, f2_dup(kExp2C1));
  p = fma2(p, f, f2_dup(1.f));
  // n << 23 = (bits(t) - bits(1.5 * 2^23)) << 23 = bits(t) << 23 modulo 2^32
  // (the low 9 bits of bits(1.5 * 2^23) are zero): one shift-add per element
  return f2_make(__uint_as_float(__float_as_uint(f2_lo(p)) + (__float_as_uint(f2_lo(t)) << 23)),
                 __uint_as_float(__float_as_uint(f2_hi(p)) + (__float_as_uint(f2_hi(t)) << 23)));
}
// exp2_det on both elements: the fast path runs packed, the (rare) case of
// an element outside (-125, 123) falls back to the scalar function; every
// element equals exp2_det of it.
__device__ __forceinline__ f2 exp2_det2(f2 y) {
  const float y0 = f2_lo(y), y1 = f2_hi(y);
  const f2 yp1 = add2(y, f2_dup(1.f));
  if (!(fabsf(f2_lo(yp1)) < 124.f) || !(fabsf(f2_hi(yp1)) < 124.f)) return f2_make(exp2_det(y0), exp2_det(y1));
  return exp2_det2_inrange(y);
}

// Hardware approximations (PTX ex2.approx / rcp.approx, flush-to-zero) for
// the backward, whose values need not reproduce the forward bit for bit.
__device__ __forceinline__ float ex2_approx(float y) {
  float r;
  asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(y));
  return r;
}
__device__ __forceinline__ float rcp_approx(float x) {
  float r;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
  return r;
}

// splat_gauss.cu:105 `alpha_sum > 0.999` is a double comparison; for a float
// alpha_sum it is exactly `alpha_sum >= 0.999f`.
constexpr float kAlphaBreak = 0.999f;

// tile_acceleration.h:43-46
__device__ __forceinline__ uint32_t depth_bits(float ndcz) {
  float zp1 = fa(ndcz, 1.f);
  if (zp1 <= 0.f) zp1 = 0.f;
  return __float_as_uint(zp1);
}

// tile_acceleration.h:22-31: [floor(min/ts), floor(max/ts)+1) clipped to the
// tile grid.  Out-of-range and NaN values clamp instead of overflowing.
// Tile sizes are powers of two (8, 16, 32), so a / ts is computed exactly as
// a * (1 / ts): the same correctly rounded value without a division
// (inv_ts = tile_inv(ts)).
__device__ __forceinline__ float tile_inv(int ts) { return ts == 8 ? 0.125f : ts == 16 ? 0.0625f : 0.03125f; }
__device__ __forceinline__ int tile_lo(float a, float inv_ts, int lim) {
  const float f = floorf(__fmul_rn(a, inv_ts));
  return (f >= 0.f) ? (f < float(lim) ? int(f) : lim) : 0;
}
__device__ __forceinline__ int tile_hi(float a, float inv_ts, int lim) {
  const float f = floorf(__fmul_rn(a, inv_ts));
  return (f >= 0.f) ? (f < float(lim) ? int(f) + 1 : lim) : 0;
}

// rect packing: x0 | y0 << 16 in .x, x1 | y1 << 16 in .y
__device__ __forceinline__ uint2 pack_rect(int x0, int y0, int x1, int y1) {
  return make_uint2(uint32_t(x0) | (uint32_t(y0) << 16),
                    uint32_t(x1) | (uint32_t(y1) << 16));
}

// ---------------------------------------------------------------------------
// Error flag (device) -- kernels record the first failure and return.
// ---------------------------------------------------------------------------
__device__ __forceinline__ void set_flag(uint32_t* flags, uint32_t bit) {
  atomicOr(flags, bit);
}
constexpr uint32_t kFlagPairOverflow = 1u;

}  // namespace dsplat

#define DSPLAT_CUDA_TRY(expr)                       \
  do {                                              \
    cudaError_t _e = (expr);                        \
    if (_e != cudaSuccess) return dsplat::map_err(_e); \
  } while (0)

namespace dsplat {
inline int map_err(cudaError_t e) {
  return e == cudaSuccess ? DSPLAT_OK : DSPLAT_ERR_CUDA;
}
}  // namespace dsplat
