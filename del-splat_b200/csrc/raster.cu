// raster.cu -- tile rasterisers.
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
#include <type_traits>

#include "common.cuh"

namespace dsplat {

constexpr int kRasterWarps = 4;  // warps per CTA (independent tasks)
constexpr int kFwdGroup8 = 2;    // 8x8 tiles per forward task
constexpr int kBwdGroup8 = 2;    // 8x8 tiles per backward task (4 measured slower: registers, partial overlaps)

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
struct EntP {
  float4 a;  // py, py, 2B, 2B
  float4 b;  // C, C, opacity, opacity
  float4 c;  // r, r, g, g
  float4 d;  // b, b, px, A
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
  const float B2 = fa(B, B);
  const float dxm = fmaxf(fabsf(x0 - px), fabsf(x1 - px)), dym = fmaxf(fabsf(y0 - py), fabsf(y1 - py));
  const float mag = fabsf(A) * dxm * dxm + fabsf(B2) * dxm * dym + fabsf(C) * dym * dym;
  dst->a = make_float4(py, py, B2, B2);
  dst->b = make_float4(C, C, op, op);
  dst->c = make_float4(r, r, g, g);
  dst->d = make_float4(b, b, px, A);
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

// ---------------------------------------------------------------------------
// Forward walk of one slab by one warp over the list range [s, e).  Slot k of
// every lane lies in the same row pair of the slab, so the per-slot skips
// (pixel done, row outside the entry's box) are uniform across the warp most
// of the time.
// ---------------------------------------------------------------------------
// CUDA_STOP: the stop test of the reference's CUDA kernel (alpha_sum >=
// 0.999f, its double comparison) instead of del-splat-cpu's (> 0.999f).
template <int TS, int PPL_, bool CUDA_STOP, class Walk, class Src>
__device__ __forceinline__ uint32_t fwd_slab(const Walk& walk, const Src& src, EntP* sm, const float2* tab, uint32_t s,
                                         uint32_t e,
                                         int px0, int py0, int w, int h, int xend, bool accumulate,
                                         float* __restrict__ out_rgb, size_t pix_base, float* __restrict__ out_T,
                                         uint32_t* __restrict__ out_last, const float* __restrict__ target,
                                         float* __restrict__ grad_pix, float* __restrict__ loss_slot) {
  using G = Geo<TS, PPL_>;
  constexpr int PPL = G::PPL;
  static_assert(PPL % 2 == 0, "pixel slots are evaluated in pairs");
  constexpr int NP = PPL / 2;
  const int lane = threadIdx.x & 31;
  const int ix = px0 + (lane % TS);
  const int iy0 = py0 + (lane / TS);
  const float fx = float(ix) + 0.5f;
  float T[PPL], as[PPL], c0[PPL], c1[PPL], c2[PPL], fy[PPL];
  uint32_t last[PPL];
  uint32_t live = 0;
#pragma unroll
  for (int k = 0; k < PPL; ++k) {
    const int iy = iy0 + k * G::ROW_STEP;
    fy[k] = float(iy) + 0.5f;
    T[k] = 1.f;
    as[k] = 0.f;
    c0[k] = c1[k] = c2[k] = 0.f;
    last[k] = s;
    if (ix < xend && iy < h) {
      live |= 1u << k;
      if (accumulate) {
        const size_t p = pix_base + size_t(iy) * w + ix;
        c0[k] = out_rgb[3 * p];
        c1[k] = out_rgb[3 * p + 1];
        c2[k] = out_rgb[3 * p + 2];
      }
    }
  }
  // slot pairs (2p, 2p+1) in packed registers during the walk
  f2 T2[NP], as2[NP], c02[NP], c12[NP], c22[NP], fy2[NP];
#pragma unroll
  for (int q = 0; q < NP; ++q) {
    T2[q] = f2_make(T[2 * q], T[2 * q + 1]);
    as2[q] = f2_make(as[2 * q], as[2 * q + 1]);
    c02[q] = f2_make(c0[2 * q], c0[2 * q + 1]);
    c12[q] = f2_make(c1[2 * q], c1[2 * q + 1]);
    c22[q] = f2_make(c2[2 * q], c2[2 * q + 1]);
    fy2[q] = f2_make(fy[2 * q], fy[2 * q + 1]);
  }
  // centres of the slab's first and last rows (the same for every lane)
  const float fy_first = float(py0) + 0.5f, fy_last = float(py0 + G::SLAB_ROWS - 1) + 0.5f;
  const uint32_t inside = live;
  uint32_t hi = e;
  uint2 en = hi > s ? walk.load(hi - 1u - uint32_t(lane), uint32_t(lane) < hi - s) : make_uint2(0u, 0u);
  while (hi > s) {
    const int cnt = int(min(32u, hi - s));
    const int k_staged = walk.stage(src, sm, en, hi - 1u - uint32_t(lane), lane < cnt, lane);
    {  // the next batch's list words arrive while this batch is blended
      const uint32_t hn = hi - uint32_t(cnt);
      if (hn > s) en = walk.load(hn - 1u - uint32_t(lane), uint32_t(lane) < hn - s);
    }
    __syncwarp();
    if (live) {
      for (int j = 0; j < k_staged; ++j) {
        const float4 ee = sm[j].e;
        if (!(ee.x <= fx && fx <= ee.y)) continue;
        const ulonglong2 qa = *reinterpret_cast<const ulonglong2*>(&sm[j].a);  // (py,py) (2B,2B)
        const ulonglong2 qb = *reinterpret_cast<const ulonglong2*>(&sm[j].b);  // (C,C) (op,op)
        const ulonglong2 qc = *reinterpret_cast<const ulonglong2*>(&sm[j].c);  // (r,r) (g,g)
        const float4 ed = sm[j].d;                                             // b, b, px, A
        const f2 qbl = f2_make(ed.x, ed.y);
        const float2 ef = *reinterpret_cast<const float2*>(&sm[j].f);
        // q = A dx dx + B (dx dy + dy dx) + C dy dy in the reference's
        // order (mat2_sym::mult_vec_from_both_sides); dx is fixed per lane,
        // so (A dx) dx is formed once per entry, and B (dx dy + dy dx) is
        // (2B)(dx dy) exactly
        const float dx = fs(fx, ed.z);
        const f2 adxdx2 = f2_dup(fm(fm(ed.w, dx), dx));
        const f2 dx2 = f2_dup(dx);
        const uint32_t pos = __float_as_uint(ef.y);
        // all instances compute the same bits: `inrange` skips expf_cr's
        // range check (proven by the entry's staged flag), `rows` the row
        // test of an entry whose box holds every row of the slab
        auto blend_slots = [&](auto inrange, auto rows) {
#pragma unroll
          for (int q = 0; q < NP; ++q) {
            // a slot is one row of the slab across the warp: the skips are
            // warp-uniform in practice
            const int k0 = 2 * q, k1 = 2 * q + 1;
            const bool a0 = ((live >> k0) & 1u) && (decltype(rows)::value || (ee.z <= fy[k0] && fy[k0] <= ee.w));
            const bool a1 = ((live >> k1) & 1u) && (decltype(rows)::value || (ee.z <= fy[k1] && fy[k1] <= ee.w));
            if (!(a0 || a1)) continue;
            const f2 dy2 = sub2(fy2[q], qa.x);
            const f2 qf = add2(add2(adxdx2, mul2(qa.y, mul2(dx2, dy2))), mul2(mul2(qb.x, dy2), dy2));
            const f2 g2 = expf_cr2<!decltype(inrange)::value>(mul2(qf, f2_dup(-0.5f)), tab);
            const f2 al = mul2(g2, qb.y);
            // an inactive slot of the pair takes alpha 0: its state is unchanged
            const f2 e2 = f2_make(a0 ? f2_lo(al) : 0.f, a1 ? f2_hi(al) : 0.f);
            const f2 eo2 = mul2(T2[q], e2);
            c02[q] = add2(c02[q], mul2(qc.x, eo2));
            c12[q] = add2(c12[q], mul2(qc.y, eo2));
            c22[q] = add2(c22[q], mul2(qbl, eo2));
            T2[q] = mul2(T2[q], sub2(f2_dup(1.f), e2));
            as2[q] = add2(as2[q], eo2);
            if (a0 && (CUDA_STOP ? f2_lo(as2[q]) >= kAlphaStop : f2_lo(as2[q]) > kAlphaStop)) {
              live &= ~(1u << k0);
              last[k0] = pos;
            }
            if (a1 && (CUDA_STOP ? f2_hi(as2[q]) >= kAlphaStop : f2_hi(as2[q]) > kAlphaStop)) {
              live &= ~(1u << k1);
              last[k1] = pos;
            }
          }
        };
        const bool all_rows = ee.z <= fy_first && fy_last <= ee.w;
        if (__float_as_uint(ef.x)) {
          if (all_rows)
            blend_slots(std::true_type{}, std::true_type{});
          else
            blend_slots(std::true_type{}, std::false_type{});
        } else {
          if (all_rows)
            blend_slots(std::false_type{}, std::true_type{});
          else
            blend_slots(std::false_type{}, std::false_type{});
        }
        if (!live) break;
      }
    }
    hi -= uint32_t(cnt);
    if (!__any_sync(0xffffffffu, live != 0u)) break;
    __syncwarp();
  }
#pragma unroll
  for (int q = 0; q < NP; ++q) {
    T[2 * q] = f2_lo(T2[q]);
    T[2 * q + 1] = f2_hi(T2[q]);
    c0[2 * q] = f2_lo(c02[q]);
    c0[2 * q + 1] = f2_hi(c02[q]);
    c1[2 * q] = f2_lo(c12[q]);
    c1[2 * q + 1] = f2_hi(c12[q]);
    c2[2 * q] = f2_lo(c22[q]);
    c2[2 * q + 1] = f2_hi(c22[q]);
  }
  float l = 0.f;
#pragma unroll
  for (int k = 0; k < PPL; ++k) {
    if (!((inside >> k) & 1u)) continue;
    const int iy = iy0 + k * G::ROW_STEP;
    const size_t p = pix_base + size_t(iy) * w + ix;
    out_rgb[3 * p] = c0[k];
    out_rgb[3 * p + 1] = c1[k];
    out_rgb[3 * p + 2] = c2[k];
    if (out_T) out_T[p] = T[k];
    if (out_last) out_last[p] = last[k];
    if (target) {
      const float d0 = c0[k] - target[3 * p], d1 = c1[k] - target[3 * p + 1], d2 = c2[k] - target[3 * p + 2];
      grad_pix[3 * p] = 2.f * d0;
      grad_pix[3 * p + 1] = 2.f * d1;
      grad_pix[3 * p + 2] = 2.f * d2;
      l += d0 * d0 + d1 * d1 + d2 * d2;
    }
  }
  if (target) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) l += __shfl_xor_sync(0xffffffffu, l, o);
    if (lane == 0) *loss_slot = l;
  }
  return e - hi;
}

// Copies expf_cr's 2^(j/64) table into the block's shared memory (one
// barrier, at kernel start).
__device__ __forceinline__ void load_exp_table(float2* tab) {
  for (int i = threadIdx.x; i < 64; i += blockDim.x) tab[i] = g_exp2_64[i];
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
// Fused-path forward: persistent, per-warp work stealing over slab tasks,
// walking each tile's entries out of its superblock list.
// slab_loss: one partial L2 loss per task (when target is given).
// ---------------------------------------------------------------------------
template <int TS, int PPL, int NT>
__global__ void __launch_bounds__(32 * kRasterWarps) k_raster_fwd(
    const ViewBatch b, uint32_t n, const float4* __restrict__ rec, const uint2* __restrict__ list1,
    const uint32_t* __restrict__ off1, uint32_t nchunk, uint64_t capacity, const uint32_t* __restrict__ order,
    uint32_t* __restrict__ work_counter, float* __restrict__ out_rgb, float* __restrict__ out_T,
    uint32_t* __restrict__ out_last, const float* __restrict__ target, float* __restrict__ grad_pix,
    float* __restrict__ slab_loss, uint32_t* __restrict__ item_cost) {
  using G = TaskGeo<TS, PPL, NT>;
  __shared__ EntP sm_all[kRasterWarps][32];
  __shared__ float2 tab[64];
  load_exp_table(tab);
  EntP* sm = sm_all[threadIdx.x >> 5];
  const int lane = threadIdx.x & 31;
  const uint32_t num_tasks = b.num_items * G::SLABS;
  for (;;) {
    uint32_t task = 0;
    if (lane == 0) task = atomicAdd(work_counter, 1u);
    task = __shfl_sync(0xffffffffu, task, 0);
    if (task >= num_tasks) return;
    const uint32_t item = order[task / G::SLABS], slab = task % G::SLABS;
    const ItemGeo ig = item_geo(b, item, off1, nchunk, capacity);
    const ViewDev& vd = b.v[ig.v];
    // tiles of this task (NT > 1: a run of a superblock row, see k_raster_bwd)
    uint32_t nx = 1;
    if (NT > 1) {
      nx = min(uint32_t(NT), 1u << vd.sb_log2);
      if (ig.lx % nx) {  // carried by the run's leftmost tile
        if (target && slab_loss && lane == 0) slab_loss[size_t(item) * G::SLABS + slab] = 0.f;
        continue;
      }
    }
    PackedSrc src{rec + 3 * size_t(ig.v) * n};
    SbWalkSpan walk{list1, ig.lx, ig.ly, nx};
    const int xend = min(vd.w, ig.px0 + int(nx) * TS);
    const uint32_t walked = fwd_slab<G::GX, G::PPL, false>(
        walk, src, sm, tab, ig.s, ig.e, ig.px0, ig.py0 + int(slab) * G::SLAB_ROWS, vd.w, vd.h, xend, false, out_rgb,
        vd.pix_base, out_T, out_last, target, grad_pix, slab_loss ? slab_loss + size_t(item) * G::SLABS + slab : nullptr);
    // scheduling hint for the backward and the next forward: list positions walked
    if (lane == 0 && walked) atomicMax(&item_cost[item], walked);
    __syncwarp();
  }
}

// Drop-in forward (splat_gauss.rs:46-94): AoS inputs and per-tile lists,
// accumulates into pix2rgb.
template <int TS, int PPL, bool CUDA_STOP>
__global__ void __launch_bounds__(32 * kRasterWarps) k_raster_fwd_aos(
    int w, int h, int tile_w, uint32_t num_tasks, float* __restrict__ pix2rgb, AosSrc src,
    const uint32_t* __restrict__ tile2idx, const uint32_t* __restrict__ idx2pnt, float* __restrict__ out_T,
    uint32_t* __restrict__ out_last) {
  using G = Geo<TS, PPL>;
  __shared__ EntP sm_all[kRasterWarps][32];
  __shared__ float2 tab[64];
  load_exp_table(tab);
  EntP* sm = sm_all[threadIdx.x >> 5];
  const uint32_t task = blockIdx.x * kRasterWarps + (threadIdx.x >> 5);
  if (task >= num_tasks) return;
  const uint32_t tile = task / G::SLABS, slab = task % G::SLABS;
  const int px0 = int(tile % uint32_t(tile_w)) * TS;
  const int py0 = int(tile / uint32_t(tile_w)) * TS + int(slab) * G::SLAB_ROWS;
  TileWalk walk{idx2pnt};
  fwd_slab<TS, PPL, CUDA_STOP>(walk, src, sm, tab, tile2idx[tile], tile2idx[tile + 1], px0, py0, w, h, w, true, pix2rgb, 0, out_T,
                    out_last, nullptr, nullptr, nullptr);
}

// ---------------------------------------------------------------------------
// Fused-path backward.  grad2d[(v*N+g)*3 + k] float4:
//   (d px, d py, d A, d B) (d C, d opacity, d r, d g) (d b, 0, 0, 0)
// exp and 1/(1-alpha) use the hardware approximations: gradients need not
// reproduce the forward bit for bit (the discrete structure -- boxes, stop
// positions -- comes from the forward).
// ---------------------------------------------------------------------------
// NT > 1 (8x8 tiles): one task covers NT horizontally adjacent tiles of one
// superblock row (fewer where the superblock is narrower), NT x as wide with
// NT x the pixels per lane, so that the per-entry warp reduction serves NT x
// the pixels.  The run's leftmost tile leads the task; the other tiles' tasks
// are empty.  The walk keeps entries whose span meets any of the tiles and
// every pixel still tests the entry's box, which contains the pixel only if
// the entry is in that pixel's own tile list, so each pixel sees exactly its
// tile's entries (and its stop position is a position in the shared
// superblock list).  The forward groups tiles the same way.
template <int TS, int PPL_, int NT>
__global__ void __launch_bounds__(32 * kRasterWarps) k_raster_bwd(
    const ViewBatch b, uint32_t n, const float4* __restrict__ rec, const uint2* __restrict__ list1,
    const uint32_t* __restrict__ off1, uint32_t nchunk, uint64_t capacity, const uint32_t* __restrict__ order,
    uint32_t* __restrict__ work_counter, const float* __restrict__ grad_pix, const float* __restrict__ pix_T,
    const uint32_t* __restrict__ pix_last, float4* __restrict__ grad2d) {
  using G = TaskGeo<TS, PPL_, NT>;
  constexpr int PPL = G::PPL;
  __shared__ Ent sm_all[kRasterWarps][32];
  Ent* sm = sm_all[threadIdx.x >> 5];
  const int lane = threadIdx.x & 31;
  const uint32_t num_tasks = b.num_items * G::SLABS;
  for (;;) {
    uint32_t task = 0;
    if (lane == 0) task = atomicAdd(work_counter, 1u);
    task = __shfl_sync(0xffffffffu, task, 0);
    if (task >= num_tasks) return;
    const uint32_t item = order[task / G::SLABS], slab = task % G::SLABS;
    const ItemGeo ig = item_geo(b, item, off1, nchunk, capacity);
    const ViewDev& vd = b.v[ig.v];
    // tiles of this task: 1, or 2 when the superblock holds the right neighbour
    uint32_t nx = 1;
    if (NT > 1) {
      nx = min(uint32_t(NT), 1u << vd.sb_log2);
      if (ig.lx % nx) continue;  // the group's leftmost tile carries it
    }
    const int col = lane % G::GX;
    const int ix = ig.px0 + col;
    const int iy0 = ig.py0 + int(slab) * G::SLAB_ROWS + (lane / G::GX);
    const bool col_in = col < int(nx) * TS;
    const float fx = float(ix) + 0.5f;
    const uint32_t s = ig.s, e = ig.e;
    // per pixel: T in front of the current entry, S = d . (colour behind it),
    // d = dL/dpixel
    float Tc[PPL], S[PPL], d0[PPL], d1[PPL], d2[PPL];
    uint32_t last[PPL];
    uint32_t lo_min = e;
#pragma unroll
    for (int k = 0; k < PPL; ++k) {
      const int iy = iy0 + k * G::ROW_STEP;
      Tc[k] = 1.f;
      S[k] = 0.f;
      d0[k] = d1[k] = d2[k] = 0.f;
      last[k] = e;  // outside pixels process nothing
      if (col_in && ix < vd.w && iy < vd.h) {
        const size_t p = size_t(vd.pix_base) + size_t(iy) * vd.w + ix;
        Tc[k] = pix_T[p];
        last[k] = pix_last[p];
        d0[k] = grad_pix[3 * p];
        d1[k] = grad_pix[3 * p + 1];
        d2[k] = grad_pix[3 * p + 2];
        lo_min = min(lo_min, last[k]);
      }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) lo_min = min(lo_min, __shfl_xor_sync(0xffffffffu, lo_min, o));
    PackedSrc src{rec + 3 * size_t(ig.v) * n};
    SbWalkSpan walk{list1, ig.lx, ig.ly, nx};
    float* gv = reinterpret_cast<float*>(grad2d + 3 * size_t(ig.v) * n);
    const uint32_t lo0 = max(s, lo_min);
    uint2 en = lo0 < e ? walk.load(lo0 + uint32_t(lane), uint32_t(lane) < e - lo0) : make_uint2(0u, 0u);
    for (uint32_t lo = lo0; lo < e; lo += 32) {
      const int cnt = int(min(32u, e - lo));
      const int k_staged = walk.stage(src, sm, en, lo + uint32_t(lane), lane < cnt, lane);
      // the next batch's list words arrive while this batch is processed
      if (lo + 32u < e) en = walk.load(lo + 32u + uint32_t(lane), uint32_t(lane) < e - (lo + 32u));
      __syncwarp();
      for (int j = 0; j < k_staged; ++j) {
        const float4 ea = sm[j].a, eb = sm[j].b, ec = sm[j].c, ed = sm[j].d;
        const uint32_t pos = __float_as_uint(ed.z);
        // v[]: this lane's sums over its pixels of (t dx, t dy, t dx^2,
        // t dx dy, t dy^2, t, dL/dr, dL/dg) with t = G dL/dalpha (its sum
        // is dL/dop; w = dL/dq = -op/2 t); gb = dL/db
        float v[8], gb = 0.f;
#pragma unroll
        for (int i = 0; i < 8; ++i) v[i] = 0.f;
        bool any = false;
        const float dx = fx - ea.x;
        if (ec.y <= fx && fx <= ec.w) {
          const float kadxdx = ea.z * dx * dx, kb2dx = ea.w * dx;
          // moments of t = G dL/dalpha (v[5] = sum t, tdy = sum t dy, tdyy =
          // sum t dy^2); w = dL/dq = -op/2 t, the factor is applied once per
          // entry after the warp reduction
          float tdy = 0.f, tdyy = 0.f;
#pragma unroll
          for (int k = 0; k < PPL; ++k) {
            const float fy = float(iy0 + k * G::ROW_STEP) + 0.5f;
            if (pos < last[k] || !(ec.z <= fy && fy <= ed.x)) continue;
            any = true;
            const float dy = fy - ea.y;
            const float Gv = ex2_approx(quad_y(eb.x, dy, kb2dx, kadxdx));
            const float al = Gv * eb.y;
            const float iom = rcp_approx(1.f - al);
            Tc[k] *= iom;
            const float wgt = al * Tc[k];
            const float drgb = d0[k] * eb.z + d1[k] * eb.w + d2[k] * ec.x;
            const float dLde = Tc[k] * drgb - iom * S[k];
            S[k] += wgt * drgb;
            v[6] += wgt * d0[k];
            v[7] += wgt * d1[k];
            gb += wgt * d2[k];
            const float t = Gv * dLde;
            v[5] += t;
            const float tdy_p = t * dy;
            tdy += tdy_p;
            tdyy += tdy_p * dy;
          }
          v[0] = v[5] * dx;
          v[1] = tdy;
          v[2] = v[0] * dx;
          v[3] = tdy * dx;
          v[4] = tdyy;
        }
        if (__any_sync(0xffffffffu, any)) {
          // transposed butterfly: after the offset-16/8/4 steps lane L holds a
          // partial sum of v[L >> 2]; offsets 2 and 1 finish it
#pragma unroll
          for (int i = 0; i < 4; ++i) {
            const bool up = lane & 16;
            const float send = up ? v[i] : v[i + 4], keep = up ? v[i + 4] : v[i];
            v[i] = keep + __shfl_xor_sync(0xffffffffu, send, 16);
          }
#pragma unroll
          for (int i = 0; i < 2; ++i) {
            const bool up = lane & 8;
            const float send = up ? v[i] : v[i + 2], keep = up ? v[i + 2] : v[i];
            v[i] = keep + __shfl_xor_sync(0xffffffffu, send, 8);
          }
          {
            const bool up = lane & 4;
            const float send = up ? v[0] : v[1], keep = up ? v[1] : v[0];
            v[0] = keep + __shfl_xor_sync(0xffffffffu, send, 4);
          }
          v[0] += __shfl_xor_sync(0xffffffffu, v[0], 2);
          v[0] += __shfl_xor_sync(0xffffffffu, v[0], 1);
#pragma unroll
          for (int o = 16; o > 0; o >>= 1) gb += __shfl_xor_sync(0xffffffffu, gb, o);
          const float m0 = __shfl_sync(0xffffffffu, v[0], 0), m1 = __shfl_sync(0xffffffffu, v[0], 4);
          // with the w moments m_i = -op/2 (t moments): d px = -2 (A m0 +
          // B m1), d py = -2 (B m0 + C m1), d A = m2, d B = 2 m3, d C = m4
          // (raw conic recovered from the staged one)
          const float A = ea.z * kInvNegHalfLog2e, B = ea.w * (0.5f * kInvNegHalfLog2e),
                      C = eb.x * kInvNegHalfLog2e;
          const int k = lane >> 2;
          float out = v[0];
          if (k == 0) out = -2.f * (A * m0 + B * m1);
          if (k == 1) out = -2.f * (B * m0 + C * m1);
          if (k == 3) out = 2.f * v[0];
          if (k < 5) out *= -0.5f * eb.y;  // the moments of t become moments of w = dL/dq
          float* dst = gv + 12 * size_t(__float_as_uint(ed.y));
          if ((lane & 3) == 0) atomicAdd(dst + k, out);
          if (lane == 1) atomicAdd(dst + 8, gb);
        }
      }
      __syncwarp();
    }
  }
}

// ---------------------------------------------------------------------------
// Circle tile painter (splat_circle.cu:93-132): ascending walk, the last
// covering entry wins; covered iff sqrt(dx^2+dy^2) <= rad.
// ---------------------------------------------------------------------------
template <int TS>
__global__ void __launch_bounds__(TS* TS) k_circle_splat_tiles(int w, int h, int tile_w, float* __restrict__ pix2rgb,
                                                              const float* __restrict__ xyd,
                                                              const float* __restrict__ rad,
                                                              const float* __restrict__ rgb,
                                                              const uint32_t* __restrict__ tile2idx,
                                                              const uint32_t* __restrict__ idx2pnt) {
  constexpr int NT = TS * TS;
  __shared__ float s_x[NT], s_y[NT], s_r[NT];
  __shared__ uint32_t s_g[NT];
  const int tid = threadIdx.x;
  const uint32_t tile = blockIdx.y * uint32_t(tile_w) + blockIdx.x;
  const int ix = int(blockIdx.x) * TS + (tid % TS), iy = int(blockIdx.y) * TS + (tid / TS);
  const bool inside = ix < w && iy < h;
  const float fx = float(ix) + 0.5f, fy = float(iy) + 0.5f;
  const uint32_t s = tile2idx[tile], e = tile2idx[tile + 1];
  int64_t win = -1;
  for (uint32_t lo = s; lo < e; lo += NT) {
    const int cnt = int(min(uint32_t(NT), e - lo));
    if (tid < cnt) {
      const uint32_t g = idx2pnt[lo + uint32_t(tid)];
      s_x[tid] = xyd[3 * size_t(g)];
      s_y[tid] = xyd[3 * size_t(g) + 1];
      s_r[tid] = rad[g];
      s_g[tid] = g;
    }
    __syncthreads();
    for (int j = 0; j < cnt; ++j) {
      const float dx = fs(s_x[j], fx), dy = fs(s_y[j], fy);
      const float dist = sqrtf(fa(fm(dx, dx), fm(dy, dy)));
      if (!(dist > s_r[j])) win = s_g[j];
    }
    __syncthreads();
  }
  if (inside && win >= 0) {
    const size_t pix = size_t(iy) * w + ix;
    pix2rgb[3 * pix] = rgb[3 * size_t(win)];
    pix2rgb[3 * pix + 1] = rgb[3 * size_t(win) + 1];
    pix2rgb[3 * pix + 2] = rgb[3 * size_t(win) + 2];
  }
}

// ---------------------------------------------------------------------------
// host launch helpers
// ---------------------------------------------------------------------------
static int num_sms() {
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
bool raster_config_ok(int ts, int ppl) {
  return (ts == 8 && (ppl == 1 || ppl == 2)) || (ts == 16 && (ppl == 2 || ppl == 4 || ppl == 8)) ||
         (ts == 32 && (ppl == 4 || ppl == 8));
}
int raster_default_ppl(int ts) { return ts == 8 ? 2 : 4; }
uint32_t raster_slabs_per_tile(int ts, int ppl) { return uint32_t(ts * ts / (32 * ppl)); }

template <class K>
static int persistent_grid(K kernel, uint32_t tasks) {
  int per_sm = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, 32 * kRasterWarps, 0);
  if (per_sm <= 0) per_sm = 4;
  int g = num_sms() * per_sm;
  const uint32_t ctas = (tasks + kRasterWarps - 1) / kRasterWarps;
  if (uint32_t(g) > ctas) g = int(ctas);
  return g < 1 ? 1 : g;
}

template <int TS, int PPL>
static void launch_fwd(cudaStream_t st, const ViewBatch& b, const FwdArgs& a) {
  constexpr int NT = TS == 8 ? kFwdGroup8 : 1;
  const uint32_t tasks = b.num_items * TaskGeo<TS, PPL, NT>::SLABS;
  k_raster_fwd<TS, PPL, NT><<<persistent_grid(k_raster_fwd<TS, PPL, NT>, tasks), 32 * kRasterWarps, 0, st>>>(
      b, a.n, a.rec, a.list1, a.off1, a.nchunk, a.capacity, a.order, a.counter, a.out_rgb, a.out_T, a.out_last,
      a.target, a.grad_pix, a.slab_loss, a.item_cost);
  count_launch();
}

// tiles per backward task (see k_raster_bwd): 2 for 8x8 tiles
int raster_bwd_group(int ts) { return ts == 8 ? kBwdGroup8 : 1; }
int raster_fwd_group(int ts) { return ts == 8 ? kFwdGroup8 : 1; }

template <int TS, int PPL>
static void launch_bwd(cudaStream_t st, const ViewBatch& b, const BwdArgs& a) {
  constexpr int NT = TS == 8 ? kBwdGroup8 : 1;
  const uint32_t tasks = b.num_items * TaskGeo<TS, PPL, NT>::SLABS;
  k_raster_bwd<TS, PPL, NT><<<persistent_grid(k_raster_bwd<TS, PPL, NT>, tasks), 32 * kRasterWarps, 0, st>>>(
      b, a.n, a.rec, a.list1, a.off1, a.nchunk, a.capacity, a.order, a.counter, a.grad_pix, a.pix_T, a.pix_last,
      a.grad2d);
  count_launch();
}

#define DSPLAT_RASTER_CONFIGS(X) X(8, 1) X(8, 2) X(16, 2) X(16, 4) X(16, 8) X(32, 4) X(32, 8)

cudaError_t raster_fwd(cudaStream_t st, const ViewBatch& b, const FwdArgs& a) {
#define X(T, P)                        \
  if (b.ts == T && b.ppl == P) {       \
    launch_fwd<T, P>(st, b, a);        \
    return cudaGetLastError();         \
  }
  DSPLAT_RASTER_CONFIGS(X)
#undef X
  return cudaErrorInvalidValue;
}

cudaError_t raster_bwd(cudaStream_t st, const ViewBatch& b, const BwdArgs& a) {
#define X(T, P)                        \
  if (b.ts == T && b.ppl == P) {       \
    launch_bwd<T, P>(st, b, a);        \
    return cudaGetLastError();         \
  }
  DSPLAT_RASTER_CONFIGS(X)
#undef X
  return cudaErrorInvalidValue;
}

template <int TS, int PPL, bool CUDA_STOP>
static void launch_aos(cudaStream_t st, int w, int h, float* pix2rgb, const AosSrc& src, const uint32_t* tile2idx,
                       const uint32_t* idx2pnt, float* out_T, uint32_t* out_last) {
  const int tw = (w + TS - 1) / TS, th = (h + TS - 1) / TS;
  const uint32_t tasks = uint32_t(tw) * uint32_t(th) * Geo<TS, PPL>::SLABS;
  const unsigned grid = (tasks + kRasterWarps - 1) / kRasterWarps;
  k_raster_fwd_aos<TS, PPL, CUDA_STOP><<<grid, 32 * kRasterWarps, 0, st>>>(w, h, tw, tasks, pix2rgb, src, tile2idx,
                                                                           idx2pnt, out_T, out_last);
  count_launch();
}

template <bool CUDA_STOP>
static cudaError_t launch_aos_ts(cudaStream_t st, int ts, int w, int h, float* pix2rgb, const AosSrc& src,
                                 const uint32_t* tile2idx, const uint32_t* idx2pnt, float* out_T,
                                 uint32_t* out_last) {
  switch (ts) {
    case 8:
      launch_aos<8, 2, CUDA_STOP>(st, w, h, pix2rgb, src, tile2idx, idx2pnt, out_T, out_last);
      break;
    case 16:
      launch_aos<16, 4, CUDA_STOP>(st, w, h, pix2rgb, src, tile2idx, idx2pnt, out_T, out_last);
      break;
    case 32:
      launch_aos<32, 4, CUDA_STOP>(st, w, h, pix2rgb, src, tile2idx, idx2pnt, out_T, out_last);
      break;
    default:
      return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

cudaError_t raster_fwd_aos(cudaStream_t st, int ts, int w, int h, float* pix2rgb, const float* xyd, const float* conic,
                           const float* aabb, const float* opacity, const float* rgb, const uint32_t* tile2idx,
                           const uint32_t* idx2pnt, float* out_T, uint32_t* out_last, bool cuda_stop) {
  if (w <= 0 || h <= 0) return cudaSuccess;
  const AosSrc src{xyd, conic, aabb, opacity, rgb};
  return cuda_stop ? launch_aos_ts<true>(st, ts, w, h, pix2rgb, src, tile2idx, idx2pnt, out_T, out_last)
                   : launch_aos_ts<false>(st, ts, w, h, pix2rgb, src, tile2idx, idx2pnt, out_T, out_last);
}

// expf_cr elementwise (exposed so that it can be checked against a
// correctly rounded reference on every float).
__global__ void k_expf_cr(size_t n, const float* __restrict__ x, float* __restrict__ y) {
  const size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i < n) y[i] = expf_cr(x[i]);
}

cudaError_t expf_cr_launch(cudaStream_t st, size_t n, const float* x, float* y) {
  if (n == 0) return cudaSuccess;
  k_expf_cr<<<unsigned((n + 255) / 256), 256, 0, st>>>(n, x, y);
  count_launch();
  return cudaGetLastError();
}

cudaError_t circle_splat_tiles(cudaStream_t st, int ts, int w, int h, float* pix2rgb, const float* xyd,
                               const float* rad, const float* rgb, const uint32_t* tile2idx, const uint32_t* idx2pnt) {
  const int tw = (w + ts - 1) / ts, th = (h + ts - 1) / ts;
  if (tw == 0 || th == 0) return cudaSuccess;
  switch (ts) {
    case 8:
      k_circle_splat_tiles<8><<<dim3(tw, th), 64, 0, st>>>(w, h, tw, pix2rgb, xyd, rad, rgb, tile2idx, idx2pnt);
      break;
    case 16:
      k_circle_splat_tiles<16><<<dim3(tw, th), 256, 0, st>>>(w, h, tw, pix2rgb, xyd, rad, rgb, tile2idx, idx2pnt);
      break;
    case 32:
      k_circle_splat_tiles<32><<<dim3(tw, th), 1024, 0, st>>>(w, h, tw, pix2rgb, xyd, rad, rgb, tile2idx, idx2pnt);
      break;
    default:
      return cudaErrorInvalidValue;
  }
  count_launch();
  return cudaGetLastError();
}

}  // namespace dsplat
