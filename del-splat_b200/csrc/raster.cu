// raster.cu -- tile rasterisers.
//
// Forward (splat_gauss.cu:56-109 semantics): per pixel, walk the tile's list
// from the end (nearest: largest ndc_z) to the start; skip entries whose
// 3-sigma box does not contain the pixel centre (ix+.5, iy+.5);
// e = exp(-q/2) * opacity with q = d^T conic d; rgb += c*T*e; T *= 1-e;
// alpha_sum += T*e; stop once alpha_sum > 0.999.
//
// B200 structure: one CTA per (view, tile) work item, TS*TS threads = one
// pixel each.  Entries are staged cooperatively into shared memory in batches
// of TS*TS (one coalesced index load + one 48-byte record gather per thread),
// every pixel then walks the batch from shared memory.  A CTA stops loading
// as soon as __syncthreads_count says every pixel has terminated.  The
// fused-path kernels are persistent: CTAs pull items from a global counter
// (work stealing), so views of different resolutions share one launch.
//
// The blend arithmetic uses non-contracted IEEE operations and dexp() so that
// the oracle reproduces it exactly, including every early-exit decision.
//
// Backward (no reference counterpart): the same walk in reverse
// (back-to-front) from the saved stop position up to the list end; the
// transmittance in front of each entry is rebuilt from the saved final value,
// T_i = T_{i+1} / (1 - e_i), and the colour behind it is accumulated, so no
// per-pixel list is stored.  Per-entry gradients are summed across the warp
// with shuffles and added to the per-(view, point) 2D gradient with one
// vectorised float4 atomic per component group.
#include "common.cuh"

namespace dsplat {

struct SmemEnt {
  float* px;
  float* py;
  float* a;
  float* b;
  float* c;
  float* op;
  float* r;
  float* g;
  float* bl;
  float* x0;
  float* y0;
  float* x1;
  float* y1;
  uint32_t* gid;
};

template <int NT>
__device__ __forceinline__ SmemEnt carve(float* s) {
  SmemEnt e;
  e.px = s;
  e.py = s + NT;
  e.a = s + 2 * NT;
  e.b = s + 3 * NT;
  e.c = s + 4 * NT;
  e.op = s + 5 * NT;
  e.r = s + 6 * NT;
  e.g = s + 7 * NT;
  e.bl = s + 8 * NT;
  e.x0 = s + 9 * NT;
  e.y0 = s + 10 * NT;
  e.x1 = s + 11 * NT;
  e.y1 = s + 12 * NT;
  e.gid = reinterpret_cast<uint32_t*>(s + 13 * NT);
  return e;
}
constexpr int kSmemFloatsPerEnt = 14;

__device__ __forceinline__ void stage_packed(const SmemEnt& S, int j, const float4* __restrict__ rec, uint32_t g) {
  const float4 r0 = __ldg(rec + 3 * size_t(g));
  const float4 r1 = __ldg(rec + 3 * size_t(g) + 1);
  const float4 r2 = __ldg(rec + 3 * size_t(g) + 2);
  S.px[j] = r0.x;
  S.py[j] = r0.y;
  S.a[j] = r0.z;
  S.b[j] = r0.w;
  S.c[j] = r1.x;
  S.op[j] = r1.y;
  S.r[j] = r1.z;
  S.g[j] = r1.w;
  S.bl[j] = r2.x;
  S.x0[j] = fs(r0.x, r2.y);
  S.y0[j] = fs(r0.y, r2.z);
  S.x1[j] = fa(r0.x, r2.y);
  S.y1[j] = fa(r0.y, r2.z);
  S.gid[j] = g;
}

__device__ __forceinline__ void stage_aos(const SmemEnt& S, int j, const float* __restrict__ xyd,
                                          const float* __restrict__ conic, const float* __restrict__ aabb,
                                          const float* __restrict__ opacity, const float* __restrict__ rgb,
                                          uint32_t g) {
  S.px[j] = xyd[3 * size_t(g)];
  S.py[j] = xyd[3 * size_t(g) + 1];
  S.a[j] = conic[3 * size_t(g)];
  S.b[j] = conic[3 * size_t(g) + 1];
  S.c[j] = conic[3 * size_t(g) + 2];
  S.op[j] = opacity[g];
  S.r[j] = rgb[3 * size_t(g)];
  S.g[j] = rgb[3 * size_t(g) + 1];
  S.bl[j] = rgb[3 * size_t(g) + 2];
  S.x0[j] = aabb[4 * size_t(g)];
  S.y0[j] = aabb[4 * size_t(g) + 1];
  S.x1[j] = aabb[4 * size_t(g) + 2];
  S.y1[j] = aabb[4 * size_t(g) + 3];
  S.gid[j] = g;
}

struct PixState {
  float T, asum, c0, c1, c2;
  uint32_t last;
  bool done;
};

// Walks staged entries j = 0..cnt-1 (entry j sits at list position hi-1-j).
__device__ __forceinline__ void blend_batch(const SmemEnt& S, int cnt, uint32_t hi, float fx, float fy,
                                            PixState& st) {
  if (st.done) return;
  for (int j = 0; j < cnt; ++j) {
    if (!(S.x0[j] <= fx && fx <= S.x1[j] && S.y0[j] <= fy && fy <= S.y1[j])) continue;
    const float dx = fs(fx, S.px[j]);
    const float dy = fs(fy, S.py[j]);
    const float q = fa(fa(fm(fm(S.a[j], dx), dx), fm(S.b[j], fa(fm(dx, dy), fm(dy, dx)))), fm(fm(S.c[j], dy), dy));
    const float e = fm(dexp(fm(-0.5f, q)), S.op[j]);
    const float eo = fm(st.T, e);
    st.c0 = fa(st.c0, fm(S.r[j], eo));
    st.c1 = fa(st.c1, fm(S.g[j], eo));
    st.c2 = fa(st.c2, fm(S.bl[j], eo));
    st.T = fm(st.T, fs(1.f, e));
    st.asum = fa(st.asum, eo);
    if (st.asum >= kAlphaBreak) {
      st.done = true;
      st.last = hi - 1u - uint32_t(j);
      return;
    }
  }
}

// ---------------------------------------------------------------------------
// Fused-path forward: persistent, work-stealing over (view, tile) items.
// outputs (per pixel of the concatenated images): rgb[3], T, last list pos.
// If `target` is given, also writes the L2-loss pixel gradient 2(C - target)
// and per-item partial losses.
// ---------------------------------------------------------------------------
template <int TS>
__global__ void __launch_bounds__(TS* TS) k_raster_fwd(const ViewBatch b, uint32_t n, const float4* __restrict__ rec,
                                                      const uint32_t* __restrict__ item_start,
                                                      const uint32_t* __restrict__ idx2pnt,
                                                      uint32_t* __restrict__ work_counter, float* __restrict__ out_rgb,
                                                      float* __restrict__ out_T, uint32_t* __restrict__ out_last,
                                                      const float* __restrict__ target, float* __restrict__ grad_pix,
                                                      float* __restrict__ item_loss) {
  constexpr int NT = TS * TS;
  extern __shared__ float smem[];
  const SmemEnt S = carve<NT>(smem);
  __shared__ uint32_t s_item;
  __shared__ float s_loss[NT / 32];
  const int tid = threadIdx.x;
  for (;;) {
    if (tid == 0) s_item = atomicAdd(work_counter, 1u);
    __syncthreads();
    const uint32_t item = s_item;
    __syncthreads();
    if (item >= b.num_items) return;
    const int v = view_of_item(b, item);
    const ViewDev& vd = b.v[v];
    const uint32_t t = item - vd.item_base;
    const int ix = int(t % uint32_t(vd.tile_w)) * TS + (tid % TS);
    const int iy = int(t / uint32_t(vd.tile_w)) * TS + (tid / TS);
    const bool inside = ix < vd.w && iy < vd.h;
    const float fx = float(ix) + 0.5f, fy = float(iy) + 0.5f;
    const uint32_t s = item_start[item], e = item_start[item + 1];
    PixState st{1.f, 0.f, 0.f, 0.f, 0.f, s, !inside};
    const float4* recv = rec + 3 * size_t(v) * n;
    for (uint32_t hi = e; hi > s;) {
      const int cnt = int(min(uint32_t(NT), hi - s));
      if (tid < cnt) {
        const uint32_t g = idx2pnt[hi - 1u - uint32_t(tid)];
        stage_packed(S, tid, recv, g);
      }
      __syncthreads();
      blend_batch(S, cnt, hi, fx, fy, st);
      hi -= uint32_t(cnt);
      if (__syncthreads_count(!st.done) == 0) break;
    }
    float l = 0.f;
    if (inside) {
      const size_t pix = size_t(vd.pix_base) + size_t(iy) * vd.w + ix;
      out_rgb[3 * pix] = st.c0;
      out_rgb[3 * pix + 1] = st.c1;
      out_rgb[3 * pix + 2] = st.c2;
      out_T[pix] = st.T;
      out_last[pix] = st.last;
      if (target) {
        const float d0 = st.c0 - target[3 * pix], d1 = st.c1 - target[3 * pix + 1],
                    d2 = st.c2 - target[3 * pix + 2];
        grad_pix[3 * pix] = 2.f * d0;
        grad_pix[3 * pix + 1] = 2.f * d1;
        grad_pix[3 * pix + 2] = 2.f * d2;
        l = d0 * d0 + d1 * d1 + d2 * d2;
      }
    }
    if (target) {
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) l += __shfl_xor_sync(0xffffffffu, l, o);
      if ((tid & 31) == 0) s_loss[tid >> 5] = l;
      __syncthreads();
      if (tid == 0) {
        float acc = 0.f;
        for (int w = 0; w < NT / 32; ++w) acc += s_loss[w];
        item_loss[item] = acc;
      }
    }
    __syncthreads();
  }
}

// ---------------------------------------------------------------------------
// Drop-in forward (splat_gauss.rs:46-94): AoS inputs, one CTA per tile, adds
// into pix2rgb like the reference.  Optional T / stop-position outputs.
// ---------------------------------------------------------------------------
template <int TS>
__global__ void __launch_bounds__(TS* TS) k_raster_fwd_aos(int w, int h, int tile_w, float* __restrict__ pix2rgb,
                                                          const float* __restrict__ xyd, const float* __restrict__ conic,
                                                          const float* __restrict__ aabb,
                                                          const float* __restrict__ opacity,
                                                          const float* __restrict__ rgb,
                                                          const uint32_t* __restrict__ tile2idx,
                                                          const uint32_t* __restrict__ idx2pnt,
                                                          float* __restrict__ out_T, uint32_t* __restrict__ out_last) {
  constexpr int NT = TS * TS;
  extern __shared__ float smem[];
  const SmemEnt S = carve<NT>(smem);
  const int tid = threadIdx.x;
  const uint32_t tile = blockIdx.y * uint32_t(tile_w) + blockIdx.x;
  const int ix = int(blockIdx.x) * TS + (tid % TS), iy = int(blockIdx.y) * TS + (tid / TS);
  const bool inside = ix < w && iy < h;
  const float fx = float(ix) + 0.5f, fy = float(iy) + 0.5f;
  const uint32_t s = tile2idx[tile], e = tile2idx[tile + 1];
  PixState st{1.f, 0.f, 0.f, 0.f, 0.f, s, !inside};
  if (inside) {
    const size_t pix = size_t(iy) * w + ix;
    st.c0 = pix2rgb[3 * pix];
    st.c1 = pix2rgb[3 * pix + 1];
    st.c2 = pix2rgb[3 * pix + 2];
  }
  for (uint32_t hi = e; hi > s;) {
    const int cnt = int(min(uint32_t(NT), hi - s));
    if (tid < cnt) stage_aos(S, tid, xyd, conic, aabb, opacity, rgb, idx2pnt[hi - 1u - uint32_t(tid)]);
    __syncthreads();
    blend_batch(S, cnt, hi, fx, fy, st);
    hi -= uint32_t(cnt);
    if (__syncthreads_count(!st.done) == 0) break;
  }
  if (inside) {
    const size_t pix = size_t(iy) * w + ix;
    pix2rgb[3 * pix] = st.c0;
    pix2rgb[3 * pix + 1] = st.c1;
    pix2rgb[3 * pix + 2] = st.c2;
    if (out_T) out_T[pix] = st.T;
    if (out_last) out_last[pix] = st.last;
  }
}

// ---------------------------------------------------------------------------
// Fused-path backward.  grad2d[(v*N+g)*3 + k] float4:
//   (d px, d py, d A, d B) (d C, d opacity, d r, d g) (d b, 0, 0, 0)
// ---------------------------------------------------------------------------
template <int TS>
__global__ void __launch_bounds__(TS* TS) k_raster_bwd(const ViewBatch b, uint32_t n, const float4* __restrict__ rec,
                                                      const uint32_t* __restrict__ item_start,
                                                      const uint32_t* __restrict__ idx2pnt,
                                                      uint32_t* __restrict__ work_counter,
                                                      const float* __restrict__ grad_pix,
                                                      const float* __restrict__ pix_T,
                                                      const uint32_t* __restrict__ pix_last,
                                                      float4* __restrict__ grad2d) {
  constexpr int NT = TS * TS;
  extern __shared__ float smem[];
  const SmemEnt S = carve<NT>(smem);
  __shared__ uint32_t s_item;
  __shared__ uint32_t s_min_last;
  const int tid = threadIdx.x;
  const int lane = tid & 31;
  for (;;) {
    if (tid == 0) {
      s_item = atomicAdd(work_counter, 1u);
      s_min_last = 0xffffffffu;
    }
    __syncthreads();
    const uint32_t item = s_item;
    if (item >= b.num_items) return;
    const int v = view_of_item(b, item);
    const ViewDev& vd = b.v[v];
    const uint32_t t = item - vd.item_base;
    const int ix = int(t % uint32_t(vd.tile_w)) * TS + (tid % TS);
    const int iy = int(t / uint32_t(vd.tile_w)) * TS + (tid / TS);
    const bool inside = ix < vd.w && iy < vd.h;
    const float fx = float(ix) + 0.5f, fy = float(iy) + 0.5f;
    const uint32_t s = item_start[item], e = item_start[item + 1];
    float Tcur = 1.f, dC0 = 0.f, dC1 = 0.f, dC2 = 0.f;
    uint32_t last = e;
    if (inside) {
      const size_t pix = size_t(vd.pix_base) + size_t(iy) * vd.w + ix;
      Tcur = pix_T[pix];
      last = pix_last[pix];
      dC0 = grad_pix[3 * pix];
      dC1 = grad_pix[3 * pix + 1];
      dC2 = grad_pix[3 * pix + 2];
      atomicMin(&s_min_last, last);
    }
    __syncthreads();
    const uint32_t lo0 = max(s, s_min_last);
    float acc0 = 0.f, acc1 = 0.f, acc2 = 0.f;
    const float4* recv = rec + 3 * size_t(v) * n;
    float4* gv = grad2d + 3 * size_t(v) * n;
    for (uint32_t lo = lo0; lo < e; lo += NT) {
      const int cnt = int(min(uint32_t(NT), e - lo));
      if (tid < cnt) stage_packed(S, tid, recv, idx2pnt[lo + uint32_t(tid)]);
      __syncthreads();
      for (int j = 0; j < cnt; ++j) {
        const uint32_t pos = lo + uint32_t(j);
        bool act = inside && pos >= last && S.x0[j] <= fx && fx <= S.x1[j] && S.y0[j] <= fy && fy <= S.y1[j];
        float gpx = 0.f, gpy = 0.f, gA = 0.f, gB = 0.f, gC = 0.f, gop = 0.f, gr = 0.f, gg = 0.f, gb = 0.f;
        if (act) {
          const float A = S.a[j], B = S.b[j], C = S.c[j], op = S.op[j];
          const float dx = fs(fx, S.px[j]);
          const float dy = fs(fy, S.py[j]);
          const float q = fa(fa(fm(fm(A, dx), dx), fm(B, fa(fm(dx, dy), fm(dy, dx)))), fm(fm(C, dy), dy));
          const float G = dexp(fm(-0.5f, q));
          const float ee = fm(G, op);
          const float om = 1.f - ee;
          Tcur = Tcur / om;
          const float wgt = ee * Tcur;
          const float cr = S.r[j], cg = S.g[j], cb = S.bl[j];
          const float iom = 1.f / om;
          const float dLde = dC0 * (cr * Tcur - acc0 * iom) + dC1 * (cg * Tcur - acc1 * iom) +
                             dC2 * (cb * Tcur - acc2 * iom);
          acc0 += cr * wgt;
          acc1 += cg * wgt;
          acc2 += cb * wgt;
          gr = wgt * dC0;
          gg = wgt * dC1;
          gb = wgt * dC2;
          gop = G * dLde;
          const float dLdq = dLde * op * G * -0.5f;
          gA = dLdq * dx * dx;
          gB = dLdq * 2.f * dx * dy;
          gC = dLdq * dy * dy;
          gpx = -dLdq * (2.f * A * dx + 2.f * B * dy);
          gpy = -dLdq * (2.f * B * dx + 2.f * C * dy);
        }
        if (__any_sync(0xffffffffu, act)) {
#pragma unroll
          for (int o = 16; o > 0; o >>= 1) {
            gpx += __shfl_xor_sync(0xffffffffu, gpx, o);
            gpy += __shfl_xor_sync(0xffffffffu, gpy, o);
            gA += __shfl_xor_sync(0xffffffffu, gA, o);
            gB += __shfl_xor_sync(0xffffffffu, gB, o);
            gC += __shfl_xor_sync(0xffffffffu, gC, o);
            gop += __shfl_xor_sync(0xffffffffu, gop, o);
            gr += __shfl_xor_sync(0xffffffffu, gr, o);
            gg += __shfl_xor_sync(0xffffffffu, gg, o);
            gb += __shfl_xor_sync(0xffffffffu, gb, o);
          }
          if (lane == 0) {
            float4* dst = gv + 3 * size_t(S.gid[j]);
            atomicAdd(dst, make_float4(gpx, gpy, gA, gB));
            atomicAdd(dst + 1, make_float4(gC, gop, gr, gg));
            atomicAdd(reinterpret_cast<float*>(dst + 2), gb);
          }
        }
      }
      __syncthreads();
    }
    __syncthreads();
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
template <int TS>
static cudaError_t launch_fwd_t(cudaStream_t st, int grid, const ViewBatch& b, uint32_t n, const float4* rec,
                                const uint32_t* item_start, const uint32_t* idx2pnt, uint32_t* counter, float* out_rgb,
                                float* out_T, uint32_t* out_last, const float* target, float* grad_pix,
                                float* item_loss) {
  constexpr int NT = TS * TS;
  const size_t sm = size_t(kSmemFloatsPerEnt) * NT * sizeof(float);
  static bool attr_set = false;
  if (!attr_set) {
    cudaError_t e = cudaFuncSetAttribute(k_raster_fwd<TS>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(sm));
    if (e != cudaSuccess) return e;
    attr_set = true;
  }
  k_raster_fwd<TS><<<grid, NT, sm, st>>>(b, n, rec, item_start, idx2pnt, counter, out_rgb, out_T, out_last, target,
                                         grad_pix, item_loss); count_launch();
  return cudaGetLastError();
}

template <int TS>
static cudaError_t launch_bwd_t(cudaStream_t st, int grid, const ViewBatch& b, uint32_t n, const float4* rec,
                                const uint32_t* item_start, const uint32_t* idx2pnt, uint32_t* counter,
                                const float* grad_pix, const float* pix_T, const uint32_t* pix_last, float4* grad2d) {
  constexpr int NT = TS * TS;
  const size_t sm = size_t(kSmemFloatsPerEnt) * NT * sizeof(float);
  static bool attr_set = false;
  if (!attr_set) {
    cudaError_t e = cudaFuncSetAttribute(k_raster_bwd<TS>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(sm));
    if (e != cudaSuccess) return e;
    attr_set = true;
  }
  k_raster_bwd<TS><<<grid, NT, sm, st>>>(b, n, rec, item_start, idx2pnt, counter, grad_pix, pix_T, pix_last, grad2d); count_launch();
  return cudaGetLastError();
}

static int persistent_grid(int ts, uint32_t items) {
  static int sms = 0;
  if (!sms) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (sms <= 0) sms = 148;
  }
  const int per_sm = ts == 8 ? 16 : (ts == 16 ? 4 : 1);
  int g = sms * per_sm;
  if (uint32_t(g) > items) g = int(items);
  return g < 1 ? 1 : g;
}

cudaError_t raster_fwd(cudaStream_t st, const ViewBatch& b, uint32_t n, const float4* rec, const uint32_t* item_start,
                       const uint32_t* idx2pnt, uint32_t* counter, float* out_rgb, float* out_T, uint32_t* out_last,
                       const float* target, float* grad_pix, float* item_loss) {
  const int grid = persistent_grid(b.ts, b.num_items);
  switch (b.ts) {
    case 8:
      return launch_fwd_t<8>(st, grid, b, n, rec, item_start, idx2pnt, counter, out_rgb, out_T, out_last, target,
                             grad_pix, item_loss);
    case 16:
      return launch_fwd_t<16>(st, grid, b, n, rec, item_start, idx2pnt, counter, out_rgb, out_T, out_last, target,
                              grad_pix, item_loss);
    case 32:
      return launch_fwd_t<32>(st, grid, b, n, rec, item_start, idx2pnt, counter, out_rgb, out_T, out_last, target,
                              grad_pix, item_loss);
  }
  return cudaErrorInvalidValue;
}

cudaError_t raster_bwd(cudaStream_t st, const ViewBatch& b, uint32_t n, const float4* rec, const uint32_t* item_start,
                       const uint32_t* idx2pnt, uint32_t* counter, const float* grad_pix, const float* pix_T,
                       const uint32_t* pix_last, float4* grad2d) {
  const int grid = persistent_grid(b.ts, b.num_items);
  switch (b.ts) {
    case 8:
      return launch_bwd_t<8>(st, grid, b, n, rec, item_start, idx2pnt, counter, grad_pix, pix_T, pix_last, grad2d);
    case 16:
      return launch_bwd_t<16>(st, grid, b, n, rec, item_start, idx2pnt, counter, grad_pix, pix_T, pix_last, grad2d);
    case 32:
      return launch_bwd_t<32>(st, grid, b, n, rec, item_start, idx2pnt, counter, grad_pix, pix_T, pix_last, grad2d);
  }
  return cudaErrorInvalidValue;
}

template <int TS>
static cudaError_t launch_aos_t(cudaStream_t st, int w, int h, float* pix2rgb, const float* xyd, const float* conic,
                                const float* aabb, const float* opacity, const float* rgb, const uint32_t* tile2idx,
                                const uint32_t* idx2pnt, float* out_T, uint32_t* out_last) {
  constexpr int NT = TS * TS;
  const int tw = (w + TS - 1) / TS, th = (h + TS - 1) / TS;
  if (tw == 0 || th == 0) return cudaSuccess;
  const size_t sm = size_t(kSmemFloatsPerEnt) * NT * sizeof(float);
  static bool attr_set = false;
  if (!attr_set) {
    cudaError_t e = cudaFuncSetAttribute(k_raster_fwd_aos<TS>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(sm));
    if (e != cudaSuccess) return e;
    attr_set = true;
  }
  k_raster_fwd_aos<TS><<<dim3(tw, th), NT, sm, st>>>(w, h, tw, pix2rgb, xyd, conic, aabb, opacity, rgb, tile2idx,
                                                     idx2pnt, out_T, out_last); count_launch();
  return cudaGetLastError();
}

cudaError_t raster_fwd_aos(cudaStream_t st, int ts, int w, int h, float* pix2rgb, const float* xyd, const float* conic,
                           const float* aabb, const float* opacity, const float* rgb, const uint32_t* tile2idx,
                           const uint32_t* idx2pnt, float* out_T, uint32_t* out_last) {
  switch (ts) {
    case 8:
      return launch_aos_t<8>(st, w, h, pix2rgb, xyd, conic, aabb, opacity, rgb, tile2idx, idx2pnt, out_T, out_last);
    case 16:
      return launch_aos_t<16>(st, w, h, pix2rgb, xyd, conic, aabb, opacity, rgb, tile2idx, idx2pnt, out_T, out_last);
    case 32:
      return launch_aos_t<32>(st, w, h, pix2rgb, xyd, conic, aabb, opacity, rgb, tile2idx, idx2pnt, out_T, out_last);
  }
  return cudaErrorInvalidValue;
}

cudaError_t circle_splat_tiles(cudaStream_t st, int ts, int w, int h, float* pix2rgb, const float* xyd,
                               const float* rad, const float* rgb, const uint32_t* tile2idx, const uint32_t* idx2pnt) {
  const int tw = (w + ts - 1) / ts, th = (h + ts - 1) / ts;
  if (tw == 0 || th == 0) return cudaSuccess;
  switch (ts) {
    case 8:
      k_circle_splat_tiles<8><<<dim3(tw, th), 64, 0, st>>>(w, h, tw, pix2rgb, xyd, rad, rgb, tile2idx, idx2pnt); count_launch();
      break;
    case 16:
      k_circle_splat_tiles<16><<<dim3(tw, th), 256, 0, st>>>(w, h, tw, pix2rgb, xyd, rad, rgb, tile2idx, idx2pnt); count_launch();
      break;
    case 32:
      k_circle_splat_tiles<32><<<dim3(tw, th), 1024, 0, st>>>(w, h, tw, pix2rgb, xyd, rad, rgb, tile2idx, idx2pnt); count_launch();
      break;
    default:
      return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

}  // namespace dsplat
