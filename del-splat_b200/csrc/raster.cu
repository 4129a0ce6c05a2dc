// raster.cu -- the backward rasteriser, the circle tile painter and the
// raster configuration queries (see raster_common.cuh; the forward lives in
// raster_fwd.cu).
#include "raster_common.cuh"

namespace dsplat {

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
            // alpha < 1 is a precondition (opacity < 1); the floor only
            // keeps gradients finite if an input breaks it
            const float iom = rcp_approx(fmaxf(1.f - al, 1e-7f));
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

bool raster_config_ok(int ts, int ppl) {
  return (ts == 8 && (ppl == 1 || ppl == 2)) || (ts == 16 && (ppl == 2 || ppl == 4 || ppl == 8)) ||
         (ts == 32 && (ppl == 4 || ppl == 8));
}
int raster_default_ppl(int ts) { return ts == 8 ? 2 : 4; }
uint32_t raster_slabs_per_tile(int ts, int ppl) { return uint32_t(ts * ts / (32 * ppl)); }

template <int TS, int PPL>
static void launch_bwd(cudaStream_t st, const ViewBatch& b, const BwdArgs& a) {
  constexpr int NT = TS == 8 ? kBwdGroup8 : 1;
  const uint32_t tasks = b.num_items * TaskGeo<TS, PPL, NT>::SLABS;
  k_raster_bwd<TS, PPL, NT><<<persistent_grid(k_raster_bwd<TS, PPL, NT>, tasks), 32 * kRasterWarps, 0, st>>>(
      b, a.n, a.rec, a.list1, a.off1, a.nchunk, a.capacity, a.order, a.counter, a.grad_pix, a.pix_T, a.pix_last,
      a.grad2d);
  count_launch();
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
