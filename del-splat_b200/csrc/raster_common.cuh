// raster_common.cuh -- what the tile rasterisers share (raster_fwd.cu,
// raster.cu): staged-entry layouts, list walkers, task geometry and the
// persistent-grid helpers.
//
// Forward (splat_gauss.cu:56-109 semantics): per pixel, walk the tile's list
// from the end (nearest: largest ndc_z) to the start; skip entries whose
// 3-sigma box does not contain the pixel centre (ix+.5, iy+.5);
// e = exp(-q/2) * opacity with q = d^T conic d; rgb += c*T*e; T *= 1-e;
// alpha_sum += T*e; stop once alpha_sum > 0.999f.
//
// B200 structure: the unit of work is a warp task.  With 8x8 tiles a task
// covers two horizontally adjacent tiles of one superblock (16x8 pixels, 4
// per lane); with 16x16 or 32x32 tiles a slab of one tile (32 lanes x 2..8
// pixels).  A lane's pixels share its column.  A warp stages 32 list entries
// at a time into its own shared-memory slots (one coalesced index load + one
// 48-byte record gather per lane; the next batch's index loads are issued
// before the current batch is walked), then every lane walks them with
// 128-bit broadcast reads, amortising each read over its pixels.  The fused path
// reads the entries straight out of the superblock list (1-8 tiles per
// side, see tiles.cu): a ballot over the 32 fetched entries keeps those whose
// tile span meets the task's tiles, compacted in order, so no per-tile list
// is ever materialised.  The forward evaluates a lane's pixels in pairs with
// packed f32x2 arithmetic; an entry whose exponent is bounded over its whole
// box at staging skips expf_cr's range check, and one whose box holds every
// row of the slab skips the per-slot row test (the same bits, fewer
// instructions; the backward measured slower with the row hoist).  A forward
// warp stops fetching as soon as all its pixels terminated (__any_sync), so
// no CTA-wide barrier exists anywhere.
// Warps pull tasks from a global counter (work stealing), longest first: one
// persistent launch covers views of different resolutions.
//
// The blend arithmetic is del-splat-cpu's (pnt2pixxyndcz.rs:86-93),
// operation for operation in single precision with no fused multiply-adds:
// q = A dx dx + B (dx dy + dy dx) + C dy dy, e = exp(-q/2) opacity with the
// correctly rounded expf_cr, e_out = T e, rgb += c e_out per channel,
// T *= 1 - e, alpha_sum += e_out, stop once alpha_sum > 0.999f.  The oracle
// performs the same sequence with exp evaluated in double and rounded once
// to float, so images, final transmittances and stop positions agree bit for
// bit; against del-splat-cpu itself (glibc expf) they differ only where
// glibc's expf is not correctly rounded.
//
// Backward (no reference counterpart): the same walk in reverse
// (back-to-front) from the saved stop position up to the list end; the
// transmittance in front of each entry is rebuilt from the saved final value,
// T_i = T_{i+1} / (1 - e_i), and the colour behind it is accumulated, so no
// per-pixel list is stored.  Each lane sums its pixels' contributions in
// registers as moments of t = G dL/dalpha (sum t, sum t dy, sum t dy^2 --
// dx is fixed per lane; w = dL/dq = -op/2 t is applied once per entry), the warp reduces the nine per-entry sums with a
// transposed butterfly (9 + 5 shuffles instead of 45), and nine lanes add
// the finished 2D gradient to the per-(view, point) record with one atomic
// instruction.
#pragma once
#include <type_traits>

#include "common.cuh"

namespace dsplat {

constexpr int kRasterWarps = 4;  // warps per CTA (independent tasks)
constexpr int kFwdGroup8 = 2;    // 8x8 tiles per forward task
constexpr int kBwdGroup8 = 2;    // 8x8 tiles per backward task (4 measured slower: registers, partial overlaps)
static_assert(kFwdGroup8 == kBwdGroup8, "the backward runs its tasks in the forward's order");

// The backward evaluates exp(-q/2) as 2^(k q) with k = -log2(e)/2 folded
// into the staged conic (hardware ex2.approx; see k_raster_bwd).
constexpr float kNegHalfLog2e = -0.72134752044448170368f;
constexpr float kInvNegHalfLog2e = -1.38629436111989061883f;  // -2 ln 2

struct Ent {  // one staged list entry (64 bytes), backward
  float4 a;   // px, py, k A, k 2B   (k = -log2(e)/2: exp(-q/2) = 2^(k q))
  float4 b;   // k C, opacity, r, g
  float4 c;   // b, box x0, box y0, box x1
  float4 d;   // box y1, point index (bits), list position (bits), -
  __device__ __forceinline__ void set_pos(uint32_t pos) { d.z = __uint_as_float(pos); }
};

// A staged entry for the forward, whose pixel slots are evaluated in pairs
// with packed two-wide FP32: every value a pair uses is stored twice, so a
// 64-bit shared load yields the packed operand (96 bytes).  The conic is
// kept as the reference reads it: (A, B, C) = (m0, m1, m2) with 2 m1 staged
// (exact), px and m0 once (they enter through the per-lane column term).
struct EntP {                // conic (A, B, C) staged times -1/2 (see make_entp)
  float4 a;  // py, py, -B, -B
  float4 b;  // -C/2, -C/2, opacity, opacity
  float4 c;  // r, r, g, g
  float4 d;  // b, b, px, -A/2
  float4 e;  // box x0, box x1, box y0, box y1
  float4 f;  // exponent in expf_cr's fast range (0/1 bits), list position (bits), -, -
  __device__ __forceinline__ void set_pos(uint32_t pos) { f.y = __uint_as_float(pos); }
};

__device__ __forceinline__ void make_entp(EntP* dst, float px, float py, float A, float B, float C, float op, float r,
                                          float g, float b, float x0, float y0, float x1, float y1) {
  // q = A dx^2 + 2B dx dy + C dy^2 of every pixel centre in the box is
  // bounded in magnitude by the same sum of absolute terms at the box's
  // farthest corner; below 170 (rounding adds far less than the margin to
  // 174) every exponent -q/2 of the entry lies in expf_cr's fast range and
  // the per-pixel range check is skipped.  NaN or infinite terms fail it.
  //
  // The conic is staged times -1/2 (exact), so that the walk forms the
  // exponent -q/2 directly: every product and sum of q scaled by -1/2 is the
  // scaled rounding of the same operation on the unscaled values, except
  // where an operand is subnormal -- and then |q| < 2^-100 and e^(-q/2)
  // rounds to 1 either way.
  const float B2 = fa(B, B);
  const float dxm = fmaxf(fabsf(x0 - px), fabsf(x1 - px)), dym = fmaxf(fabsf(y0 - py), fabsf(y1 - py));
  const float mag = fabsf(A) * dxm * dxm + fabsf(B2) * dxm * dym + fabsf(C) * dym * dym;
  const float hA = fm(A, -0.5f), hB2 = fm(B2, -0.5f), hC = fm(C, -0.5f);
  dst->a = make_float4(py, py, hB2, hB2);
  dst->b = make_float4(hC, hC, op, op);
  dst->c = make_float4(r, r, g, g);
  dst->d = make_float4(b, b, px, hA);
  dst->e = make_float4(x0, x1, y0, y1);
  dst->f = make_float4(__uint_as_float(mag < 170.f ? 1u : 0u), 0.f, 0.f, 0.f);
}

// The staged conic, scaled so that y = k q = kA dx^2 + (k2B dx + kC dy) dy.
__device__ __forceinline__ float4 scaled_conic_a(float px, float py, float A, float B) {
  return make_float4(px, py, fm(A, kNegHalfLog2e), fm(fa(B, B), kNegHalfLog2e));
}

template <int TS, int PPL_>
struct Geo {
  static constexpr int PPL = PPL_;                // pixels per lane
  static constexpr int ROW_STEP = 32 / TS;        // rows covered by the 32 lanes at once
  static constexpr int SLAB_ROWS = ROW_STEP * PPL;
  static constexpr int SLABS = TS / SLAB_ROWS;    // warp tasks per tile
  static_assert(SLABS * SLAB_ROWS == TS, "slab geometry");
};

// Fused-path task geometry: NT horizontally adjacent tiles of a superblock
// row per warp task (NT > 1 for 8x8 tiles, see k_raster_bwd), NT x the
// pixels per lane.
template <int TS, int PPL_, int NT>
struct TaskGeo {
  static constexpr int GX = NT * TS;   // task width in pixels
  static constexpr int PPL = NT * PPL_;
  static constexpr int ROW_STEP = 32 / GX;
  static constexpr int SLAB_ROWS = ROW_STEP * PPL;
  static constexpr int SLABS = TS / SLAB_ROWS;
  static_assert(SLABS * SLAB_ROWS == TS && GX <= 32, "task geometry");
};

__device__ __forceinline__ void stage_packed(Ent* dst, const float4* __restrict__ rec, uint32_t g) {
  const float4 r0 = __ldg(rec + 3 * size_t(g));
  const float4 r1 = __ldg(rec + 3 * size_t(g) + 1);
  const float4 r2 = __ldg(rec + 3 * size_t(g) + 2);
  dst->a = scaled_conic_a(r0.x, r0.y, r0.z, r0.w);
  dst->b = make_float4(fm(r1.x, kNegHalfLog2e), r1.y, r1.z, r1.w);
  dst->c = make_float4(r2.x, fs(r0.x, r2.y), fs(r0.y, r2.z), fa(r0.x, r2.y));
  dst->d = make_float4(fa(r0.y, r2.z), __uint_as_float(g), 0.f, 0.f);
}

struct AosSrc {
  const float *xyd, *conic, *aabb, *opacity, *rgb;
  __device__ __forceinline__ void stage(EntP* dst, uint32_t g) const {
    const size_t i = g;
    make_entp(dst, xyd[3 * i], xyd[3 * i + 1], conic[3 * i], conic[3 * i + 1], conic[3 * i + 2], opacity[i],
              rgb[3 * i], rgb[3 * i + 1], rgb[3 * i + 2], aabb[4 * i], aabb[4 * i + 1], aabb[4 * i + 2],
              aabb[4 * i + 3]);
  }
};

struct PackedSrc {
  const float4* rec;
  __device__ __forceinline__ void stage(Ent* dst, uint32_t g) const { stage_packed(dst, rec, g); }
  __device__ __forceinline__ void stage(EntP* dst, uint32_t g) const {
    const float4 r0 = __ldg(rec + 3 * size_t(g));
    const float4 r1 = __ldg(rec + 3 * size_t(g) + 1);
    const float4 r2 = __ldg(rec + 3 * size_t(g) + 2);
    make_entp(dst, r0.x, r0.y, r0.z, r0.w, r1.x, r1.y, r1.z, r1.w, r2.x, fs(r0.x, r2.y), fs(r0.y, r2.z),
              fa(r0.x, r2.y), fa(r0.y, r2.z));
  }
};

// Entry walkers: stage up to 32 entries of the list position range
// [pos0 - 32, pos0) (backwards) or [pos0, pos0 + 32) (forwards) into the
// warp's slots, in walk order, each with its list position (set_pos);
// return how many were staged.
// load() reads a lane's list word ahead of time (a prefetch while the
// previous batch is walked); stage() filters and gathers from it.
struct TileWalk {  // a per-tile list (tile2idx / idx2pnt)
  const uint32_t* idx2pnt;
  __device__ __forceinline__ uint2 load(uint32_t pos, bool valid) const {
    return make_uint2(valid ? idx2pnt[pos] : 0u, 0u);
  }
  template <class Src, class E>
  __device__ __forceinline__ int stage(const Src& src, E* sm, uint2 en, uint32_t pos, bool valid, int lane) const {
    if (valid) {
      src.stage(&sm[lane], en.x);
      sm[lane].set_pos(pos);
    }
    return __popc(__ballot_sync(0xffffffffu, valid));
  }
};

// A superblock list filtered to the tiles lx .. lx+nx-1 of one superblock row
// (a fused-path warp task): an entry is kept if its span meets any of them;
// ballot compaction keeps the list order.
struct SbWalkSpan {
  const uint2* list1;
  uint32_t lx, ly, nx;
  __device__ __forceinline__ uint2 load(uint32_t pos, bool valid) const {
    return valid ? list1[pos] : make_uint2(0u, 0u);
  }
  template <class Src, class E>
  __device__ __forceinline__ int stage(const Src& src, E* sm, uint2 en, uint32_t pos, bool valid, int lane) const {
    bool m = false;
    uint32_t g = 0;
    if (valid) {
      g = en.x;
      const uint32_t lr = en.y;
      m = lx < ((lr >> 8) & 15u) && lx + nx > (lr & 15u) && ly >= ((lr >> 4) & 15u) && ly < (lr >> 12);
    }
    const uint32_t bal = __ballot_sync(0xffffffffu, m);
    if (m) {
      const int slot = __popc(bal & ((1u << lane) - 1u));
      src.stage(&sm[slot], g);
      sm[slot].set_pos(pos);
    }
    return __popc(bal);
  }
};

// y = k q = (kA dx) dx + (k2B dx + kC dy) dy with the conic terms staged
// pre-scaled: kadxdx = (kA dx) dx and kb2dx = k2B dx are per entry and lane.
__device__ __forceinline__ float quad_y(float kC, float dy, float kb2dx, float kadxdx) {
  return ff(ff(kC, dy, kb2dx), dy, kadxdx);
}

// Copies expf_cr's 2^(j/64) table into the block's shared memory as two
// planes, hi at [j] and rel at [64 + j] (one barrier, at kernel start).
__device__ __forceinline__ void load_exp_table(float* tab) {
  for (int i = threadIdx.x; i < 64; i += blockDim.x) {
    const float2 t = g_exp2_64[i];
    tab[i] = t.x;
    tab[64 + i] = t.y;
  }
  __syncthreads();
}

// The superblock-list range of an item and the tile's place in it.
struct ItemGeo {
  int v, px0, py0;
  uint32_t s, e, lx, ly;
};

__device__ __forceinline__ ItemGeo item_geo(const ViewBatch& b, uint32_t item, const uint32_t* __restrict__ off1,
                                            uint32_t nchunk, uint64_t capacity) {
  ItemGeo g;
  g.v = view_of_item(b, item);
  const ViewDev& vd = b.v[g.v];
  const uint32_t t = item - vd.item_base;
  const uint32_t tx = t % uint32_t(vd.tile_w), ty = t / uint32_t(vd.tile_w);
  const int sl = vd.sb_log2;
  const uint32_t sb = vd.sb_base + (ty >> sl) * uint32_t(sb_cols(vd)) + (tx >> sl);
  g.s = uint32_t(min(uint64_t(off1[size_t(sb) * nchunk]), capacity));
  g.e = uint32_t(min(uint64_t(off1[size_t(sb + 1) * nchunk]), capacity));
  g.lx = tx & ((1u << sl) - 1u);
  g.ly = ty & ((1u << sl) - 1u);
  g.px0 = int(tx) * b.ts;
  g.py0 = int(ty) * b.ts;
  return g;
}

// ---------------------------------------------------------------------------
// host launch helpers
// ---------------------------------------------------------------------------
inline int num_sms() {
  static int sms = 0;
  if (!sms) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (sms <= 0) sms = 148;
  }
  return sms;
}

// Supported (tile size, pixels per lane) pairs; slabs per tile follow.
template <class K>
inline int persistent_grid(K kernel, uint32_t tasks) {
  int per_sm = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, 32 * kRasterWarps, 0);
  if (per_sm <= 0) per_sm = 4;
  int g = num_sms() * per_sm;
  const uint32_t ctas = (tasks + kRasterWarps - 1) / kRasterWarps;
  if (uint32_t(g) > ctas) g = int(ctas);
  return g < 1 ? 1 : g;
}

#define DSPLAT_RASTER_CONFIGS(X) X(8, 1) X(8, 2) X(16, 2) X(16, 4) X(16, 8) X(32, 4) X(32, 8)

}  // namespace dsplat
