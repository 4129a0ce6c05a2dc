// common.cuh -- shared device helpers for the del-splat B200 kernels.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "dsplat.h"
#include "exp_tables.cuh"

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



// The five parameter tensors of one fused Adam launch (k_adam_fused).
struct AdamSeg {
  float* p[5];
  const float* g[5];
  float* m[5];
  float* v[5];
  size_t end[5];  // cumulative element counts
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

// Fused multiply-add with a single rounding (IEEE fma; the CPU oracle's
// std::fma gives the same bits).
__device__ __forceinline__ float ff(float a, float b, float c) { return __fmaf_rn(a, b, c); }

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

// A packed product that keeps its own rounding when it feeds an add.  The
// assembler fuses a mul.rn.f32x2 whose result goes into an add.rn.f32x2 into
// one fused multiply-add (a single rounding) -- with or without -fmad=false,
// unlike the scalar mul.rn/add.rn pairs -- which changes the sum by an ulp
// now and then.  fma(a, b, -0) equals RN(a b) exactly (signed zeros
// included), and with the -0 held in a runtime value (nz: a kernel argument,
// (-0, -0)) there is no product left to fuse.
__device__ __forceinline__ f2 mul2_rn(f2 a, f2 b, f2 nz) { return fma2(a, b, nz); }

// ---------------------------------------------------------------------------
// expf_cr: e^x correctly rounded to single precision (the float nearest to
// the exact value), for every float x.  The blend evaluates exp(-q/2) with
// it, so its values are those of del-splat-cpu's f32 `exp` wherever that is
// correctly rounded too (glibc 2.39's expf is, except on about 1 input in
// 11,500 of [-110, 0], where it is one unit in the last place off).
//
// Fast path, |x| <= 87, single precision only:
//   k = nearest integer to x * 64/ln2 (the 1.5 * 2^23 addition rounds it);
//   r = x - k ln2/64 with ln2/64 = C1 + C2 + C3: k C1 and k C2 are exact
//     (11-bit constants, |k| < 2^13) and so are both subtractions, which
//     leaves rh exact and rl = -k C3 (|rl| < 2^-22) as a correction;
//   2^(j/64) (j = k mod 64) = TH (1 + R) from a 64-entry table (TH the
//     nearest float, R the float nearest to the remainder over TH);
//   y = TH (1 + R) e^r = TH (1 + rh + tail) with
//     tail = (rl + R)(1 + rh) + rh^2 (1/2 + rh/6 + rh^2/24) + O(2^-44),
//     evaluated as rh (rh p + (rl + R)) + (rl + R);
//   s = RN(TH + TH rh) by one fma, its rounding error TH rh + (TH - s)
//     (TH - s is exact: s and TH are within a factor 2) by a second fma,
//     ylo = TH tail + that error by a third: y = s + ylo.  If ylo +- 2^-37
//     round to the same float with s, the exact value rounds to it too
//     (rounding is monotonic and the error of s + ylo is below 2^-37 for y
//     in [0.99, 2)), so that float is the correctly rounded result; it is
//     scaled by 2^(k div 64) exactly.
// Otherwise (|x| > 87, NaN, or the rounding test failed -- about 4e-5 of
// the inputs), expf_cr_slow evaluates the same reduction in double precision
// (degree-6 polynomial, 2^(j/64) rounded to double) and rounds the double
// once to float, which also produces subnormal results, 0 and infinity.
// Both paths were compared with the correctly rounded value (float)e^x for
// all 2^32 float inputs and agree everywhere; every operation is an exactly
// rounded IEEE operation, so the result does not depend on the compiler.
// ---------------------------------------------------------------------------
constexpr float kExpMagic = 12582912.f;                            // 1.5 * 2^23
constexpr float kExpP3 = 0x1.555556p-3f, kExpP4 = 0x1.555556p-5f;  // 1/6, 1/24
constexpr float kExpTie = 0x1p-37f;
constexpr float kExpFastMax = 87.f;

static __device__ __noinline__ float expf_cr_slow(float x) {
  if (x != x) return x;
  if (x > 89.f) return __int_as_float(0x7f800000);
  if (x < -104.f) return 0.f;
  const double xd = double(x);
  const double t = __fma_rn(xd, kExpK64d, 0x1.8p52);
  const double kd = __dsub_rn(t, 0x1.8p52);
  double r = __fma_rn(kd, -kExpL1d, xd);
  r = __fma_rn(kd, -kExpL2d, r);
  const int k = __double2loint(t);  // the low word of t holds k
  double p = 1.0 / 720;
  p = __fma_rn(p, r, 1.0 / 120);
  p = __fma_rn(p, r, 1.0 / 24);
  p = __fma_rn(p, r, 1.0 / 6);
  p = __fma_rn(p, r, 0.5);
  p = __fma_rn(p, r, 1.0);
  const double tj = __ldg(&g_exp2_64d[k & 63]);
  double y = __fma_rn(tj, __dmul_rn(p, r), tj);
  y = __dmul_rn(y, __hiloint2double(((k >> 6) + 1023) << 20, 0));
  return __double2float_rn(y);
}

// The fast path's arithmetic, written once for one element (V = float) and
// for two (V = f2, packed): each packed operation rounds each element
// exactly as the scalar one, so both forms give the same bits.  Every
// product feeds an explicit fma, so no contraction can change a rounding.
__device__ __forceinline__ float vfma(float a, float b, float c) { return __fmaf_rn(a, b, c); }
__device__ __forceinline__ float vadd(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float vsub(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ f2 vfma(f2 a, f2 b, f2 c) { return fma2(a, b, c); }
__device__ __forceinline__ f2 vadd(f2 a, f2 b) { return add2(a, b); }
__device__ __forceinline__ f2 vsub(f2 a, f2 b) { return sub2(a, b); }
template <class V> __device__ __forceinline__ V vdup(float a);
template <> __device__ __forceinline__ float vdup<float>(float a) { return a; }
template <> __device__ __forceinline__ f2 vdup<f2>(float a) { return f2_dup(a); }

// tk = x 64/ln2 + 1.5 2^23: its low bits hold k (table index k & 63)
template <class V>
__device__ __forceinline__ V expf_cr_tk(V x) {
  return vfma(x, vdup<V>(kExpK64), vdup<V>(kExpMagic));
}
// ra, rb: s + ylo rounded with ylo moved by +-2^-37 (equal: the fast path
// holds), before the scaling by 2^(k div 64); th, rel = the table entry
template <class V>
__device__ __forceinline__ void expf_cr_round(V x, V tk, V th, V rel, V* ra, V* rb) {
  const V kf = vsub(tk, vdup<V>(kExpMagic));
  const V r1 = vfma(kf, vdup<V>(-kExpC1), x);
  const V rh = vfma(kf, vdup<V>(-kExpC2), r1);
  const V rlt = vfma(kf, vdup<V>(-kExpC3), rel);  // rl + R
  V p = vfma(rh, vdup<V>(kExpP4), vdup<V>(kExpP3));
  p = vfma(p, rh, vdup<V>(0.5f));
  const V tail = vfma(rh, vfma(rh, p, rlt), rlt);
  const V s = vfma(th, rh, th);
  const V ylo = vfma(th, tail, vfma(th, rh, vsub(th, s)));
  *ra = vadd(s, vadd(ylo, vdup<V>(kExpTie)));
  *rb = vadd(s, vsub(ylo, vdup<V>(kExpTie)));
}
// ra scaled by 2^(k div 64) (exact: no subnormal result for |x| <= 87)
__device__ __forceinline__ float expf_cr_scale(float ra, float tk) {
  return __uint_as_float(__float_as_uint(ra) + ((__float_as_uint(tk) << 17) & 0xff800000u));
}

// Scalar form, table read from global memory.
__device__ __forceinline__ float expf_cr(float x) {
  const float tk = expf_cr_tk(x);
  const float2 t = __ldg(&g_exp2_64[__float_as_uint(tk) & 63u]);
  float ra, rb;
  expf_cr_round(x, tk, t.x, t.y, &ra, &rb);
  return ra == rb && fabsf(x) <= kExpFastMax ? expf_cr_scale(ra, tk) : expf_cr_slow(x);
}

// Packed form for two elements, table in shared memory (tab: g_exp2_64 as
// two planes, tab[j] = hi and tab[64 + j] = rel, so that each element's
// value loads straight into its half of the packed operand).  RANGE: check
// |x| <= 87 per element (a caller that has bounded x for a whole batch
// passes false).  Each element equals expf_cr of it.
template <bool RANGE>
__device__ __forceinline__ f2 expf_cr2(f2 x, const float* tab) {
  const f2 tk = expf_cr_tk(x);
  const float k0 = f2_lo(tk), k1 = f2_hi(tk);
  const uint32_t j0 = __float_as_uint(k0) & 63u, j1 = __float_as_uint(k1) & 63u;
  f2 ra, rb;
  expf_cr_round(x, tk, f2_make(tab[j0], tab[j1]), f2_make(tab[64 + j0], tab[64 + j1]), &ra, &rb);
  float y0 = expf_cr_scale(f2_lo(ra), k0), y1 = expf_cr_scale(f2_hi(ra), k1);
  bool ok = ra == rb;  // both elements (64-bit compare; no zero or NaN in range)
  if (RANGE) ok = ok && fabsf(f2_lo(x)) <= kExpFastMax && fabsf(f2_hi(x)) <= kExpFastMax;
  if (!ok) {  // rare: settle each element on its own
    if (!(f2_lo(ra) == f2_lo(rb) && fabsf(f2_lo(x)) <= kExpFastMax)) y0 = expf_cr_slow(f2_lo(x));
    if (!(f2_hi(ra) == f2_hi(rb) && fabsf(f2_hi(x)) <= kExpFastMax)) y1 = expf_cr_slow(f2_hi(x));
  }
  return f2_make(y0, y1);
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

// Early exit of the front-to-back blend: del-splat-cpu stops once the f32
// alpha sum exceeds 0.999f (pnt2pixxyndcz.rs:93, `alpha_sum > 0.999` with an
// f32 left side).  The reference's CUDA kernel compares in double
// (splat_gauss.cu:105), which for a float sum is `>= 0.999f`; the two rules
// differ only when the sum equals 0.999f exactly.
constexpr float kAlphaStop = 0.999f;

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
