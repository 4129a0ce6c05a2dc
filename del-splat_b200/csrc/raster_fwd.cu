// raster_fwd.cu -- the forward rasterisers (see raster_common.cuh).
//
// The blend must perform del-splat-cpu's operations one IEEE rounding at a
// time.  The file is built with -fmad=false (no scalar multiply-add is
// contracted), and every packed product whose result feeds an add is formed
// with mul2_rn (an fma with a runtime -0 addend, kernel argument nz), because
// the assembler contracts packed mul/add pairs regardless of that flag.  The
// fused multiply-adds the exponential wants are written out (fma2) and stay
// fused.
#include "raster_common.cuh"

namespace dsplat {

// ---------------------------------------------------------------------------
// Forward walk of one slab by one warp over the list range [s, e).  Slot k of
// every lane lies in the same row pair of the slab, so the per-slot skips
// (pixel done, row outside the entry's box) are uniform across the warp most
// of the time.
// ---------------------------------------------------------------------------
// CUDA_STOP: the stop test of the reference's CUDA kernel (alpha_sum >=
// 0.999f, its double comparison) instead of del-splat-cpu's (> 0.999f).
// SPLIT (a 16x8 task of two 8x8 tiles, 4 slots per lane): lane L covers
// column L % 8 of both tiles at rows L / 8 and L / 8 + 4, slot pair 0 in the
// left tile and pair 1 in the right one, so that an entry whose box meets
// one tile keeps every lane of the warp busy on one pair and skips the
// other pair warp-wide.  Otherwise lane L covers column L % TS, slot k at
// row L / TS + k (32 / TS).
template <int TS, int PPL_, bool CUDA_STOP, bool SPLIT, class Walk, class Src>
__device__ __forceinline__ uint32_t fwd_slab(const Walk& walk, const Src& src, EntP* sm, float4* park,
                                         uint32_t* park_pos, const float* tab, float nz,
                                         uint32_t s, uint32_t e, int px0, int py0, int w, int h, int xend, bool accumulate,
                                         float* __restrict__ out_rgb, size_t pix_base, float* __restrict__ out_T,
                                         uint32_t* __restrict__ out_last, const float* __restrict__ target,
                                         float* __restrict__ grad_pix, float* __restrict__ loss_slot) {
  using G = Geo<TS, PPL_>;
  constexpr int PPL = G::PPL;
  static_assert(PPL % 2 == 0, "pixel slots are evaluated in pairs");
  constexpr int NP = PPL / 2;
  static_assert(!SPLIT || (TS == 16 && PPL == 4), "split lanes: two 8-wide tiles, two slot pairs");
  constexpr int COLS = SPLIT ? TS / 2 : TS;
  constexpr int RSTEP = SPLIT ? 4 : G::ROW_STEP;
  const int lane = threadIdx.x & 31;
  const int col = lane % COLS, row0 = lane / COLS;
  auto slot_x = [&](int k) { return px0 + col + (SPLIT ? (k / 2) * COLS : 0); };
  auto slot_y = [&](int k) { return py0 + row0 + (SPLIT ? k % 2 : k) * RSTEP; };
  float fxp[NP];  // column centre of each slot pair
#pragma unroll
  for (int q = 0; q < NP; ++q) fxp[q] = float(slot_x(2 * q)) + 0.5f;
  float T[PPL], as[PPL], c0[PPL], c1[PPL], c2[PPL], fy[PPL];
  uint32_t live = 0;
#pragma unroll
  for (int k = 0; k < PPL; ++k) {
    const int ix = slot_x(k), iy = slot_y(k);
    fy[k] = float(iy) + 0.5f;
    T[k] = 1.f;
    as[k] = 0.f;
    c0[k] = c1[k] = c2[k] = 0.f;
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
  const f2 nz2 = f2_dup(nz);  // (-0, -0), a runtime value (see mul2_rn)
  // a slot that stops parks its final values in the warp's shared area
  // (park[k][lane] = T, r, g, b; park_pos[k][lane] = its stop position); its
  // registers are no longer read, and the outputs are written after the walk
  const uint32_t inside = live;
  // centres of the slab's first and last rows (the same for every lane)
  const float fy_first = float(py0) + 0.5f, fy_last = float(py0 + G::SLAB_ROWS - 1) + 0.5f;
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
        // column tests: the slot pairs' columns (one column unless SPLIT)
        const bool cin0 = ee.x <= fxp[0] && fxp[0] <= ee.y;
        const bool cin1 = SPLIT ? (ee.x <= fxp[NP - 1] && fxp[NP - 1] <= ee.y) : cin0;
        if (!(cin0 || cin1)) continue;
        const ulonglong2 qa = *reinterpret_cast<const ulonglong2*>(&sm[j].a);  // (py,py) (2B,2B)
        const ulonglong2 qb = *reinterpret_cast<const ulonglong2*>(&sm[j].b);  // (C,C) (op,op)
        const ulonglong2 qc = *reinterpret_cast<const ulonglong2*>(&sm[j].c);  // (r,r) (g,g)
        const float4 ed = sm[j].d;                                             // b, b, px, A
        const f2 qbl = f2_make(ed.x, ed.y);
        const float2 ef = *reinterpret_cast<const float2*>(&sm[j].f);
        // -q/2 with q = A dx dx + B (dx dy + dy dx) + C dy dy in the
        // reference's order (mat2_sym::mult_vec_from_both_sides), from the
        // conic staged times -1/2; dx is fixed per slot pair, so (A dx) dx
        // is formed once per entry and column, and B (dx dy + dy dx) is
        // (2B)(dx dy) exactly
        auto col_terms = [&](float fxq, f2* adxdx2, f2* dx2) {
          const float dx = fs(fxq, ed.z);
          *adxdx2 = f2_dup(__fmaf_rn(fm(ed.w, dx), dx, nz));
          *dx2 = f2_dup(dx);
        };
        f2 adxdx2_1 = 0, dx2_1 = 0;  // the lane's column (all pairs) unless SPLIT
        if (!SPLIT) col_terms(fxp[0], &adxdx2_1, &dx2_1);
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
            if (SPLIT && !(q == 0 ? cin0 : cin1)) continue;
            // a0/a1: the slot's row lies in the box.  A stopped slot's
            // registers are no longer read (its outputs are written), so only
            // the row test masks the update
            const bool a0 = decltype(rows)::value || (ee.z <= fy[k0] && fy[k0] <= ee.w);
            const bool a1 = decltype(rows)::value || (ee.z <= fy[k1] && fy[k1] <= ee.w);
            if (!((((live >> k0) & 1u) && a0) || (((live >> k1) & 1u) && a1))) continue;
            f2 adxdx2 = adxdx2_1, dx2 = dx2_1;
            if (SPLIT) col_terms(fxp[q], &adxdx2, &dx2);
            const f2 dy2 = sub2(fy2[q], qa.x);
            const f2 qf = add2(add2(adxdx2, mul2_rn(qa.y, mul2(dx2, dy2), nz2)),
                               mul2_rn(mul2(qb.x, dy2), dy2, nz2));
            const f2 g2 = expf_cr2<!decltype(inrange)::value>(qf, tab);
            const f2 al = mul2_rn(g2, qb.y, nz2);
            // a live slot whose row is outside the box takes alpha 0: its
            // state is unchanged
            const f2 e2 = decltype(rows)::value ? al : f2_make(a0 ? f2_lo(al) : 0.f, a1 ? f2_hi(al) : 0.f);
            const f2 eo2 = mul2_rn(T2[q], e2, nz2);
            c02[q] = add2(c02[q], mul2_rn(qc.x, eo2, nz2));
            c12[q] = add2(c12[q], mul2_rn(qc.y, eo2, nz2));
            c22[q] = add2(c22[q], mul2_rn(qbl, eo2, nz2));
            T2[q] = mul2(T2[q], sub2(f2_dup(1.f), e2));
            as2[q] = add2(as2[q], eo2);
            // a stopped slot's alpha sum is parked at -inf (it stays -inf
            // or NaN, which no test passes), and a live slot keeps a sum at
            // or below the threshold until it stops, so one test of the
            // pair's larger sum finds every slot that stops at this entry
            const float amax = fmaxf(f2_lo(as2[q]), f2_hi(as2[q]));
            if (CUDA_STOP ? amax >= kAlphaStop : amax > kAlphaStop) {  // rare
              float s0 = f2_lo(as2[q]), s1 = f2_hi(as2[q]);
              if (CUDA_STOP ? s0 >= kAlphaStop : s0 > kAlphaStop) {
                live &= ~(1u << k0);
                park[k0 * 32 + lane] = make_float4(f2_lo(T2[q]), f2_lo(c02[q]), f2_lo(c12[q]), f2_lo(c22[q]));
                park_pos[k0 * 32 + lane] = pos;
                s0 = -INFINITY;
              }
              if (CUDA_STOP ? s1 >= kAlphaStop : s1 > kAlphaStop) {
                live &= ~(1u << k1);
                park[k1 * 32 + lane] = make_float4(f2_hi(T2[q]), f2_hi(c02[q]), f2_hi(c12[q]), f2_hi(c22[q]));
                park_pos[k1 * 32 + lane] = pos;
                s1 = -INFINITY;
              }
              as2[q] = f2_make(s0, s1);
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
  // slots still walking at the end walked the whole list (stop position s)
#pragma unroll
  for (int q = 0; q < NP; ++q) {
    if ((live >> (2 * q)) & 1u) {
      park[2 * q * 32 + lane] = make_float4(f2_lo(T2[q]), f2_lo(c02[q]), f2_lo(c12[q]), f2_lo(c22[q]));
      park_pos[2 * q * 32 + lane] = s;
    }
    if ((live >> (2 * q + 1)) & 1u) {
      park[(2 * q + 1) * 32 + lane] = make_float4(f2_hi(T2[q]), f2_hi(c02[q]), f2_hi(c12[q]), f2_hi(c22[q]));
      park_pos[(2 * q + 1) * 32 + lane] = s;
    }
  }
  float l = 0.f;
#pragma unroll
  for (int k = 0; k < PPL; ++k) {
    if (!((inside >> k) & 1u)) continue;
    const float4 o = park[k * 32 + lane];
    const size_t p = pix_base + size_t(slot_y(k)) * w + slot_x(k);
    out_rgb[3 * p] = o.y;
    out_rgb[3 * p + 1] = o.z;
    out_rgb[3 * p + 2] = o.w;
    if (out_T) out_T[p] = o.x;
    if (out_last) out_last[p] = park_pos[k * 32 + lane];
    if (target) {
      const float d0 = o.y - target[3 * p], d1 = o.z - target[3 * p + 1], d2 = o.w - target[3 * p + 2];
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
    float* __restrict__ slab_loss, uint32_t* __restrict__ item_cost, float nz) {
  using G = TaskGeo<TS, PPL, NT>;
  __shared__ EntP sm_all[kRasterWarps][32];
  __shared__ float4 park_all[kRasterWarps][G::PPL * 32];
  __shared__ uint32_t park_pos_all[kRasterWarps][G::PPL * 32];
  __shared__ float tab[128];
  load_exp_table(tab);
  EntP* sm = sm_all[threadIdx.x >> 5];
  float4* park = park_all[threadIdx.x >> 5];
  uint32_t* park_pos = park_pos_all[threadIdx.x >> 5];
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
    const uint32_t walked = fwd_slab<G::GX, G::PPL, false, NT == 2 && G::PPL == 4>(
        walk, src, sm, park, park_pos, tab, nz, ig.s, ig.e, ig.px0, ig.py0 + int(slab) * G::SLAB_ROWS, vd.w, vd.h, xend, false, out_rgb,
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
    uint32_t* __restrict__ out_last, float nz) {
  using G = Geo<TS, PPL>;
  __shared__ EntP sm_all[kRasterWarps][32];
  __shared__ float4 park_all[kRasterWarps][PPL * 32];
  __shared__ uint32_t park_pos_all[kRasterWarps][PPL * 32];
  __shared__ float tab[128];
  load_exp_table(tab);
  EntP* sm = sm_all[threadIdx.x >> 5];
  float4* park = park_all[threadIdx.x >> 5];
  uint32_t* park_pos = park_pos_all[threadIdx.x >> 5];
  const uint32_t task = blockIdx.x * kRasterWarps + (threadIdx.x >> 5);
  if (task >= num_tasks) return;
  const uint32_t tile = task / G::SLABS, slab = task % G::SLABS;
  const int px0 = int(tile % uint32_t(tile_w)) * TS;
  const int py0 = int(tile / uint32_t(tile_w)) * TS + int(slab) * G::SLAB_ROWS;
  TileWalk walk{idx2pnt};
  fwd_slab<TS, PPL, CUDA_STOP, false>(walk, src, sm, park, park_pos, tab, nz, tile2idx[tile], tile2idx[tile + 1], px0, py0, w, h, w, true, pix2rgb, 0, out_T,
                    out_last, nullptr, nullptr, nullptr);
}

template <int TS, int PPL>
static void launch_fwd(cudaStream_t st, const ViewBatch& b, const FwdArgs& a) {
  constexpr int NT = TS == 8 ? kFwdGroup8 : 1;
  const uint32_t tasks = b.num_items * TaskGeo<TS, PPL, NT>::SLABS;
  k_raster_fwd<TS, PPL, NT><<<persistent_grid(k_raster_fwd<TS, PPL, NT>, tasks), 32 * kRasterWarps, 0, st>>>(
      b, a.n, a.rec, a.list1, a.off1, a.nchunk, a.capacity, a.order, a.counter, a.out_rgb, a.out_T, a.out_last,
      a.target, a.grad_pix, a.slab_loss, a.item_cost, -0.f);
  count_launch();
}

int raster_fwd_group(int ts) { return ts == 8 ? kFwdGroup8 : 1; }

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

template <int TS, int PPL, bool CUDA_STOP>
static void launch_aos(cudaStream_t st, int w, int h, float* pix2rgb, const AosSrc& src, const uint32_t* tile2idx,
                       const uint32_t* idx2pnt, float* out_T, uint32_t* out_last) {
  const int tw = (w + TS - 1) / TS, th = (h + TS - 1) / TS;
  const uint32_t tasks = uint32_t(tw) * uint32_t(th) * Geo<TS, PPL>::SLABS;
  const unsigned grid = (tasks + kRasterWarps - 1) / kRasterWarps;
  k_raster_fwd_aos<TS, PPL, CUDA_STOP><<<grid, 32 * kRasterWarps, 0, st>>>(w, h, tw, tasks, pix2rgb, src, tile2idx,
                                                                           idx2pnt, out_T, out_last, -0.f);
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

}  // namespace dsplat
