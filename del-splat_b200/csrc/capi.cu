// capi.cu -- the extern "C" entry points declared in include/dsplat.h.
//
// Host orchestration only: argument checks, workspace carving and the launch
// sequence of each entry point.  No device memory is allocated here; every
// buffer comes from the caller.
#include <algorithm>
#include <cstdio>
#include <cstring>
#include <string>

#include "common.cuh"

namespace dsplat {
// kernels and launchers defined in the other translation units
__global__ void k_gauss_project_ref(uint32_t, const float*, const float*, const float*, const float*, int, int, float*,
                                    float*, float*);
__global__ void k_circle_project_ref(uint32_t, const float*, const float*, int, int, float, float*, float*);
__global__ void k_prep_tiles(uint32_t, const float*, const float*, const float*, int, int, int, uint2*, uint32_t*,
                             uint32_t*);
__global__ void k_fused_project(uint32_t, uint32_t, int, const float*, const float*, const float*, const float*,
                                const float*, const ViewBatch, float4*, uint2*, uint32_t*, uint32_t*);
__global__ void k_project_bwd_geom(uint32_t, const float*, const float*, const float*, const ViewBatch,
                                   float4*, float*, float*, float*, float*);
__global__ void k_project_bwd_colour(uint32_t, int, const float*, const float*, const ViewBatch, float4*,
                                     float*, float*, unsigned long long*, unsigned long long);
__global__ void k_prepare_grad2d(const unsigned long long*, unsigned long long, float4*, size_t);
__global__ void k_adam(size_t, float*, const float*, float*, float*, float, float, float, float, float, float);
int raster_fwd_group(int ts);
__global__ void k_pad_keys(uint32_t*, uint32_t, uint32_t, uint32_t);
__global__ void k_sb_count(const uint32_t*, const uint2*, uint32_t, uint32_t, const ViewBatch, uint32_t*,
                           unsigned long long*);
__global__ void k_sb_scatter(const uint32_t*, const uint2*, uint32_t, uint32_t, const ViewBatch, const uint32_t*,
                             uint64_t, uint2*, uint32_t*);
__global__ void k_sb_scatter_staged(const uint32_t*, const uint2*, uint32_t, uint32_t, const ViewBatch, const uint32_t*,
                                    uint64_t, uint2*, uint32_t*, uint32_t);
size_t sb_scatter_staged_smem(uint32_t max_sb, uint32_t max_side, uint32_t qcap);
__global__ void k_tile_count(const uint2*, const uint32_t*, uint32_t, uint64_t, const ViewBatch, uint32_t*);
__global__ void k_tile_scatter(const uint2*, const uint32_t*, uint32_t, uint64_t, const ViewBatch, const uint32_t*,
                               uint32_t*, uint32_t*, uint32_t*);
__global__ void k_clamp_ranges(uint32_t*, uint32_t, uint64_t, uint32_t*);
__global__ void k_check_capacity(const unsigned long long*, uint64_t, uint32_t*);
__global__ void k_make_keys64(const uint32_t*, const uint32_t*, const float*, const unsigned long long*, uint64_t,
                              uint64_t*);
__global__ void k_fill_u64(uint64_t*, size_t, uint64_t);
__global__ void k_point_zbuf(uint32_t, const float*, int, int, uint64_t*);
__global__ void k_point_resolve(size_t, const uint64_t*, const float*, const float*, float*, float*, int32_t*);
__global__ void k_circle_zbuf(uint32_t, const float*, const float*, int, int, int, uint64_t*);
__global__ void k_circle_resolve(size_t, const uint64_t*, const void*, int, void*, int32_t*);

size_t scan_tmp_words(size_t n);
size_t radix_hist_words(size_t n);
cudaError_t exclusive_scan(cudaStream_t, const uint32_t*, uint32_t*, size_t, uint32_t*);
cudaError_t radix_sort(cudaStream_t, uint32_t*, uint32_t*, uint32_t*, uint32_t*, size_t, const uint32_t*, int, uint32_t,
                       uint32_t*, uint32_t*, bool*, const uint2*, uint32_t, uint2*, bool, uint32_t);
cudaError_t raster_fwd(cudaStream_t, const ViewBatch&, const FwdArgs&);
cudaError_t raster_bwd(cudaStream_t, const ViewBatch&, const BwdArgs&);
bool raster_config_ok(int ts, int ppl);
int raster_default_ppl(int ts);
uint32_t raster_slabs_per_tile(int ts, int ppl);
__global__ void k_order_hist(const ViewBatch, const uint32_t*, uint32_t, const uint32_t*, int, uint32_t*);
__global__ void k_order_scatter(const ViewBatch, const uint32_t*, uint32_t, const uint32_t*, int, uint32_t*,
                                uint32_t*);
cudaError_t raster_fwd_aos(cudaStream_t, int, int, int, float*, const float*, const float*, const float*, const float*,
                           const float*, const uint32_t*, const uint32_t*, float*, uint32_t*, bool);
cudaError_t expf_cr_launch(cudaStream_t, size_t, const float*, float*);
cudaError_t circle_splat_tiles(cudaStream_t, int, int, int, float*, const float*, const float*, const float*,
                               const uint32_t*, const uint32_t*);

__global__ void k_adam_fused(AdamSeg, double, double, double, double, const int32_t*);
__global__ void k_adam_step_inc(int32_t*);

__global__ void k_one_minus(const float* __restrict__ T, float* __restrict__ out, size_t n) {
  const size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i < n) out[i] = 1.f - T[i];
}

namespace {

thread_local std::string g_last_error;

// Optional CUDA events recorded at stage boundaries of the batched calls
// (profiling hook, dsplat_set_stage_events).
thread_local cudaEvent_t g_stage_ev[16];
thread_local int g_stage_n = 0;
inline void stage_mark(cudaStream_t st, int k) {
  if (k < g_stage_n && g_stage_ev[k]) cudaEventRecord(g_stage_ev[k], st);
}

int fail(int code, const char* msg) {
  g_last_error = msg;
  return code;
}

int cuda_fail(cudaError_t e, const char* where) {
  char buf[256];
  snprintf(buf, sizeof(buf), "%s: %s", where, cudaGetErrorString(e));
  g_last_error = buf;
  return DSPLAT_ERR_CUDA;
}

#define TRY_CUDA(expr, where)                    \
  do {                                           \
    cudaError_t _e = (expr);                     \
    if (_e != cudaSuccess) return cuda_fail(_e, where); \
  } while (0)

inline unsigned blocks_for(size_t n, unsigned t) { return unsigned((n + t - 1) / t); }
inline bool ts_ok(uint32_t ts) { return ts == 8 || ts == 16 || ts == 32; }
inline size_t align_up(size_t x, size_t a) { return (x + a - 1) / a * a; }
inline uint32_t ceil_div(uint32_t a, uint32_t b) { return (a + b - 1) / b; }
inline int bits_for(uint32_t n_items) {
  int b = 0;
  while ((1ull << b) < uint64_t(n_items)) ++b;
  return b;
}
constexpr uint32_t kSortTile = 4096;

// Simple bump allocator over the caller's workspace.
struct Carver {
  char* base;
  size_t off = 0;
  explicit Carver(void* p) : base(static_cast<char*>(p)) {}
  template <class T>
  T* take(size_t count, size_t* off_out = nullptr) {
    off = align_up(off, 256);
    if (off_out) *off_out = off;
    T* p = base ? reinterpret_cast<T*>(base + off) : nullptr;
    off += count * sizeof(T);
    return p;
  }
};

// ---------------------------------------------------------------------------
// Tile lists from rank order (shared by the drop-in and batched paths):
// stage 1 superblock multisplit, stage 2 per-tile multisplit; see tiles.cu.
// ---------------------------------------------------------------------------
constexpr uint32_t kChunk = 4096;  // ranks per stage-1 chunk (= kSortTile)

struct ListsWs {
  uint32_t *cnt1, *off1, *tcnt;
  uint2* list1;
};

size_t lists_scan_words(const ViewBatch& b, uint32_t npad) {
  const size_t a = size_t(b.num_sb) * (npad / kChunk) + 1, c = size_t(b.num_items) + 1;
  return a > c ? a : c;
}

void carve_lists(Carver& c, const ViewBatch& b, uint32_t npad, size_t cap, ListsWs* L, size_t* off_list1,
                 size_t* off_off1) {
  const size_t m = size_t(b.num_sb) * (npad / kChunk) + 1;
  L->cnt1 = c.take<uint32_t>(m);
  L->off1 = c.take<uint32_t>(m, off_off1);
  L->list1 = c.take<uint2>(cap, off_list1);
  L->tcnt = c.take<uint32_t>(size_t(b.num_items) + 1);
}

// Stage 1: superblock lists of (point, local tile span) in rank order.
// flags[6..7] <- tile pairs P (u64), flags[8..9] <- superblock entries
// (capacity needed, u64); flags[0] |= overflow when they exceed capacity.
int build_sb_lists(cudaStream_t st, const ViewBatch& b, uint32_t n, uint32_t npad, const uint32_t* order,
                   const uint2* srect, const ListsWs& L, uint32_t* scan_tmp, uint64_t capacity, uint32_t* flags) {
  const uint32_t nchunk = npad / kChunk;
  const size_t m = size_t(b.num_sb) * nchunk;
  const unsigned grid1 = unsigned(b.num_views) * nchunk;
  const size_t smem1 = size_t(b.max_sb) * sizeof(uint32_t);
  const size_t smem3 = 8 * smem1 + 8 * 2 * size_t(b.max_sb_side) * sizeof(uint32_t);
  if (smem3 > 48 * 1024) {
    if (smem3 > 200 * 1024) return fail(DSPLAT_ERR_UNSUPPORTED, "too many superblocks in one view");
    TRY_CUDA(cudaFuncSetAttribute(k_sb_scatter, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem3)), "attr");
  }
  unsigned long long* totals = reinterpret_cast<unsigned long long*>(flags + 6);
  k_sb_count<<<grid1, 256, smem1, st>>>(order, srect, n, npad, b, L.cnt1, totals);
  count_launch();
  TRY_CUDA(cudaMemsetAsync(L.cnt1 + m, 0, sizeof(uint32_t), st), "memset");
  TRY_CUDA(exclusive_scan(st, L.cnt1, L.off1, m + 1, scan_tmp), "scan");
  k_check_capacity<<<1, 32, 0, st>>>(totals + 1, capacity, flags);
  count_launch();
  // staged scatter (coalesced list stores) when its shared memory fits
  constexpr uint32_t kStageEntries = 3072;
  const size_t smem_staged = sb_scatter_staged_smem(b.max_sb, b.max_sb_side, kStageEntries);
  if (smem_staged <= 100 * 1024) {
    if (smem_staged > 48 * 1024)
      TRY_CUDA(cudaFuncSetAttribute(k_sb_scatter_staged, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    int(smem_staged)),
               "attr");
    k_sb_scatter_staged<<<grid1, 256, smem_staged, st>>>(order, srect, n, npad, b, L.off1, capacity, L.list1, flags,
                                                         kStageEntries);
  } else {
    k_sb_scatter<<<grid1, 256, smem3, st>>>(order, srect, n, npad, b, L.off1, capacity, L.list1, flags);
  }
  count_launch();
  TRY_CUDA(cudaGetLastError(), "superblock lists");
  return DSPLAT_OK;
}

// Stage 2 (reference-format output only): per-tile lists tile2idx/idx2pnt.
int build_tile_lists(cudaStream_t st, const ViewBatch& b, uint32_t npad, const ListsWs& L, uint32_t* scan_tmp,
                     uint32_t* item_start, uint32_t* idx2pnt, uint32_t* out_tile, uint64_t capacity,
                     uint32_t* flags) {
  const uint32_t nchunk = npad / kChunk;
  TRY_CUDA(cudaMemsetAsync(L.tcnt + b.num_items, 0, sizeof(uint32_t), st), "memset");
  k_tile_count<<<b.num_sb, 256, 0, st>>>(L.list1, L.off1, nchunk, capacity, b, L.tcnt);
  count_launch();
  TRY_CUDA(exclusive_scan(st, L.tcnt, item_start, size_t(b.num_items) + 1, scan_tmp), "scan");
  k_tile_scatter<<<b.num_sb, 256, 0, st>>>(L.list1, L.off1, nchunk, capacity, b, item_start, idx2pnt, out_tile,
                                           flags);
  count_launch();
  k_clamp_ranges<<<64, 256, 0, st>>>(item_start, b.num_items, capacity, flags);
  count_launch();
  TRY_CUDA(cudaGetLastError(), "tile lists");
  return DSPLAT_OK;
}

cudaError_t order_tasks(cudaStream_t st, const ViewBatch& b, const uint32_t* off1, uint32_t nchunk,
                        const uint32_t* cost, int nt, uint32_t* sched, uint32_t* order) {
  cudaError_t e = cudaMemsetAsync(sched, 0, 80 * sizeof(uint32_t), st);
  if (e != cudaSuccess) return e;
  k_order_hist<<<296, 256, 0, st>>>(b, off1, nchunk, cost, nt, sched);
  count_launch();
  k_order_scatter<<<296, 256, 0, st>>>(b, off1, nchunk, cost, nt, sched, order);
  count_launch();
  return cudaGetLastError();
}

// Superblock side per view.  A tile walks its whole superblock list when its
// pixels never saturate (silhouettes, sparse regions), so the list length,
// ~ visible points x superblock area / view area, bounds the slowest raster
// task; stage 1 instead pays per superblock a point spans.  Rule: the
// largest side (8 tiles at most) that still splits the view into at least
// kSbMinPerView superblocks -- a fixed fraction of the view -- within the
// per-view limits of the stage-1 kernels (255 per side, kSbMaxPerView).
constexpr uint32_t kSbMinPerView = 200;
constexpr uint32_t kSbMaxPerView = 4096;

int choose_sb_log2(int tile_w, int tile_h) {
  int s = 3;
  while (s > 0) {
    const uint32_t cw = uint32_t((tile_w + (1 << s) - 1) >> s), ch = uint32_t((tile_h + (1 << s) - 1) >> s);
    if (cw * ch >= kSbMinPerView) break;
    const uint32_t nw = uint32_t((tile_w + (1 << (s - 1)) - 1) >> (s - 1));
    const uint32_t nh = uint32_t((tile_h + (1 << (s - 1)) - 1) >> (s - 1));
    if (nw > 255 || nh > 255 || nw * nh > kSbMaxPerView) break;
    --s;
  }
  return s;
}

void fill_sb_layout(ViewBatch* b) {
  uint32_t sb = 0, mx = 0, side = 1;
  for (int v = 0; v < b->num_views; ++v) {
    ViewDev& d = b->v[v];
    d.sb_base = sb;
    d.sb_log2 = choose_sb_log2(d.tile_w, d.tile_h);
    const uint32_t c = uint32_t(sb_cols(d)) * uint32_t(sb_rows(d));
    sb += c;
    mx = c > mx ? c : mx;
    side = std::max(side, uint32_t(std::max(sb_cols(d), sb_rows(d))));
  }
  b->num_sb = sb;
  b->max_sb = mx;
  b->max_sb_side = side;
}

// ---------------------------------------------------------------------------
// Single-view tile list builder shared by the Gaussian and circle entries.
// ---------------------------------------------------------------------------
struct TileWs {
  uint32_t* flags;  // [0] flags, [1] total pairs
  uint2* rect;
  uint2* srect;  // tile spans in depth order (written by the sort's last pass)
  uint32_t *cnt, *dka, *dva, *dkb, *dvb, *hist, *scan_tmp, *out_tile;
  ListsWs lists;
  size_t bytes;
};

ViewBatch single_view_batch(int w, int h, int ts, uint32_t tile_w, uint32_t tile_h) {
  ViewBatch b;
  memset(&b, 0, sizeof(b));
  b.num_views = 1;
  b.ts = ts;
  b.ppl = raster_default_ppl(ts);
  b.num_items = tile_w * tile_h;
  b.num_pix = uint32_t(w) * uint32_t(h);
  b.v[0].w = w;
  b.v[0].h = h;
  b.v[0].tile_w = int(tile_w);
  b.v[0].tile_h = int(tile_h);
  fill_sb_layout(&b);
  return b;
}

TileWs carve_tiles(void* ws, uint32_t n, uint32_t tile_w, uint32_t tile_h, uint64_t pairs) {
  const uint32_t npad = ceil_div(n > 0 ? n : 1, kSortTile) * kSortTile;
  const size_t cap = pairs > 0 ? pairs : 1;
  const ViewBatch b = single_view_batch(int(tile_w) * 8, int(tile_h) * 8, 8, tile_w, tile_h);
  Carver c(ws);
  TileWs t;
  t.flags = c.take<uint32_t>(16);
  t.rect = c.take<uint2>(n + 1);
  t.srect = c.take<uint2>(npad);
  t.cnt = c.take<uint32_t>(size_t(n) + 1);
  t.dka = c.take<uint32_t>(npad);
  t.dva = c.take<uint32_t>(npad);
  t.dkb = c.take<uint32_t>(npad);
  t.dvb = c.take<uint32_t>(npad);
  const size_t hw = radix_hist_words(npad);
  t.hist = c.take<uint32_t>(hw);
  size_t sw = lists_scan_words(b, npad);
  if (hw > sw) sw = hw;
  if (size_t(n) + 1 > sw) sw = size_t(n) + 1;
  t.scan_tmp = c.take<uint32_t>(scan_tmp_words(sw));
  size_t d0, d1;
  carve_lists(c, b, npad, cap, &t.lists, &d0, &d1);
  t.out_tile = c.take<uint32_t>(cap);
  t.bytes = c.off;
  return t;
}

// counts only: prep + sum
int tiles_count(cudaStream_t st, uint32_t n, const float* xyd, const float* aabb, const float* rad, uint32_t tile_w,
                uint32_t tile_h, uint32_t ts, void* ws, size_t ws_bytes, uint64_t* num_pairs) {
  if (!num_pairs) return fail(DSPLAT_ERR_INVALID_ARG, "num_pairs is null");
  if (!ts_ok(ts)) return fail(DSPLAT_ERR_UNSUPPORTED, "tile_size must be 8, 16 or 32");
  TileWs t = carve_tiles(nullptr, n, tile_w, tile_h, 0);
  if (!ws || ws_bytes < t.bytes) return fail(DSPLAT_ERR_WORKSPACE, "workspace too small");
  t = carve_tiles(ws, n, tile_w, tile_h, 0);
  *num_pairs = 0;
  if (n == 0 || tile_w == 0 || tile_h == 0) return DSPLAT_OK;
  k_prep_tiles<<<blocks_for(n, 256), 256, 0, st>>>(n, xyd, aabb, rad, int(ts), int(tile_w), int(tile_h), t.rect,
                                                  t.dka, t.cnt);
  count_launch();
  TRY_CUDA(cudaMemsetAsync(t.cnt + n, 0, sizeof(uint32_t), st), "memset");
  TRY_CUDA(exclusive_scan(st, t.cnt, t.dkb, size_t(n) + 1, t.scan_tmp), "scan");
  uint32_t total = 0;
  TRY_CUDA(cudaMemcpyAsync(&total, t.dkb + n, sizeof(uint32_t), cudaMemcpyDeviceToHost, st), "memcpy");
  TRY_CUDA(cudaStreamSynchronize(st), "sync");
  *num_pairs = total;
  return DSPLAT_OK;
}

int tiles_fill(cudaStream_t st, uint32_t n, const float* xyd, const float* aabb, const float* rad, int img_w,
               int img_h, uint32_t tile_w, uint32_t tile_h, uint32_t ts, uint32_t* tile2idx, uint32_t* idx2pnt,
               uint64_t capacity, uint64_t* keys64, void* ws, size_t ws_bytes) {
  if (!ts_ok(ts)) return fail(DSPLAT_ERR_UNSUPPORTED, "tile_size must be 8, 16 or 32");
  if ((tile_w + 7) / 8 > 255 || (tile_h + 7) / 8 > 255)
    return fail(DSPLAT_ERR_UNSUPPORTED, "image too large for the tile size (at most 255x255 superblocks)");
  if (!tile2idx || (!idx2pnt && capacity > 0)) return fail(DSPLAT_ERR_INVALID_ARG, "null output");
  if (n > 0 && !xyd) return fail(DSPLAT_ERR_INVALID_ARG, "null input");
  TileWs t = carve_tiles(nullptr, n, tile_w, tile_h, capacity);
  if (!ws || ws_bytes < t.bytes) return fail(DSPLAT_ERR_WORKSPACE, "workspace too small");
  t = carve_tiles(ws, n, tile_w, tile_h, capacity);
  const uint32_t T = tile_w * tile_h;
  TRY_CUDA(cudaMemsetAsync(t.flags, 0, 16 * sizeof(uint32_t), st), "memset");
  if (n == 0 || T == 0 || capacity == 0) {
    TRY_CUDA(cudaMemsetAsync(tile2idx, 0, (size_t(T) + 1) * sizeof(uint32_t), st), "memset");
    return DSPLAT_OK;
  }
  const uint32_t npad = ceil_div(n, kSortTile) * kSortTile;
  ViewBatch b = single_view_batch(img_w, img_h, int(ts), tile_w, tile_h);
  if (npad > n) {
    k_pad_keys<<<blocks_for(npad - n, 256), 256, 0, st>>>(t.dka, n, npad, 1);
    count_launch();
  }
  k_prep_tiles<<<blocks_for(n, 256), 256, 0, st>>>(n, xyd, aabb, rad, int(ts), int(tile_w), int(tile_h), t.rect,
                                                  t.dka, t.cnt);
  count_launch();
  bool in_b = false;
  TRY_CUDA(radix_sort(st, t.dka, t.dva, t.dkb, t.dvb, npad, nullptr, 32, 1, t.hist, t.scan_tmp, &in_b, t.rect, n,
                      t.srect, true, n),
           "depth sort");
  const uint32_t* order = in_b ? t.dvb : t.dva;
  int rc = build_sb_lists(st, b, n, npad, order, t.srect, t.lists, t.scan_tmp, capacity, t.flags);
  if (rc) return rc;
  rc = build_tile_lists(st, b, npad, t.lists, t.scan_tmp, tile2idx, idx2pnt, keys64 ? t.out_tile : nullptr, capacity,
                        t.flags);
  if (rc) return rc;
  if (keys64) {
    k_make_keys64<<<1184, 256, 0, st>>>(t.out_tile, idx2pnt, xyd,
                                        reinterpret_cast<const unsigned long long*>(t.flags + 6), capacity, keys64);
    count_launch();
  }
  TRY_CUDA(cudaGetLastError(), "launch");
  return DSPLAT_OK;
}

// ---------------------------------------------------------------------------
// Batched Gaussian state
// ---------------------------------------------------------------------------
struct BatchWs {
  dsplat_batch_layout L;
  uint32_t* flags;
  float4* rec;
  uint2* rect;
  uint2* srect;  // tile spans in depth order per view (written by the sort's last pass)
  uint32_t *cnt, *dka, *dva, *dkb, *dvb, *hist, *scan_tmp;
  ListsWs lists;
  float* pix_T;
  uint32_t* pix_stop;
  float* grad_pix;
  float* slab_loss;
  float4* grad2d;
  unsigned long long* grad2d_tag;  // == grad2d_tag_value(): grad2d is all zero
  uint32_t *sched, *task_order, *item_cost;
};

int make_batch(int64_t n64, int32_t nv, const dsplat_view* views, int32_t ts, int32_t ppl, ViewBatch* b) {
  if (nv < 1 || nv > DSPLAT_MAX_VIEWS) return fail(DSPLAT_ERR_INVALID_ARG, "num_views must be in [1, 32]");
  if (!views) return fail(DSPLAT_ERR_INVALID_ARG, "views is null");
  if (!ts_ok(uint32_t(ts))) return fail(DSPLAT_ERR_UNSUPPORTED, "tile_size must be 8, 16 or 32");
  if (ppl == 0) ppl = raster_default_ppl(ts);
  if (!raster_config_ok(ts, ppl))
    return fail(DSPLAT_ERR_UNSUPPORTED, "pixels_per_lane must be 2 (8x8 tiles), 2/4/8 (16x16) or 4/8 (32x32)");
  if (n64 < 0 || n64 > int64_t(0x7fffffff)) return fail(DSPLAT_ERR_INVALID_ARG, "num_pnt out of range");
  memset(b, 0, sizeof(*b));
  b->num_views = nv;
  b->ts = ts;
  b->ppl = ppl;
  uint64_t items = 0, pix = 0;
  for (int v = 0; v < nv; ++v) {
    const dsplat_view& s = views[v];
    if (s.width <= 0 || s.height <= 0 || s.width > 16384 || s.height > 16384)
      return fail(DSPLAT_ERR_INVALID_ARG, "bad view size (1..16384 pixels per side)");
    ViewDev& d = b->v[v];
    memcpy(d.mvp, s.mvp, sizeof(d.mvp));
    memcpy(d.campos, s.campos, sizeof(d.campos));
    d.w = s.width;
    d.h = s.height;
    d.tile_w = (s.width + ts - 1) / ts;
    d.tile_h = (s.height + ts - 1) / ts;
    if ((d.tile_w + 7) / 8 > 255 || (d.tile_h + 7) / 8 > 255)
      return fail(DSPLAT_ERR_UNSUPPORTED, "view too large for the tile size (at most 255x255 superblocks)");
    d.item_base = uint32_t(items);
    d.pix_base = uint32_t(pix);
    items += uint64_t(d.tile_w) * d.tile_h;
    pix += uint64_t(s.width) * s.height;
  }
  if (items >= 0xffffffffull || pix * 3 >= 0xffffffffull) return fail(DSPLAT_ERR_INVALID_ARG, "batch too large");
  b->num_items = uint32_t(items);
  b->num_pix = uint32_t(pix);
  fill_sb_layout(b);
  return DSPLAT_OK;
}

// Value of the workspace's grad2d tag meaning "grad2d is all zero for this
// layout": a fixed pattern mixed with the layout, so that a fresh workspace
// or one carved for another batch is cleared before use.
unsigned long long grad2d_tag_value(const dsplat_batch_layout& L, uint32_t n, int32_t views) {
  unsigned long long h = 0x6a09e667f3bcc909ull;
  const unsigned long long parts[4] = {L.total_bytes, L.off_grad2d, n, uint64_t(uint32_t(views))};
  for (unsigned long long x : parts) {
    h ^= x + 0x9e3779b97f4a7c15ull + (h << 6) + (h >> 2);
    h *= 0xbf58476d1ce4e5b9ull;
  }
  return h | 1ull;
}

BatchWs carve_batch(void* ws, uint32_t n, const ViewBatch& b, uint64_t capacity) {
  const uint32_t V = uint32_t(b.num_views);
  const uint32_t npad = ceil_div(n > 0 ? n : 1, kSortTile) * kSortTile;
  const size_t cap = capacity > 0 ? capacity : 1;
  const size_t VN = size_t(V) * n, Vp = size_t(V) * npad;
  Carver c(ws);
  BatchWs w;
  dsplat_batch_layout& L = w.L;
  memset(&L, 0, sizeof(L));
  L.num_items = b.num_items;
  L.num_pix = b.num_pix;
  L.npad = npad;
  L.slabs_per_tile = raster_slabs_per_tile(b.ts, b.ppl);
  w.flags = c.take<uint32_t>(16, &L.off_flags);
  w.rec = c.take<float4>(3 * VN + 3, &L.off_rec);
  w.rect = c.take<uint2>(VN + 1, &L.off_rect);
  w.srect = c.take<uint2>(Vp);
  w.cnt = c.take<uint32_t>(VN + 1, &L.off_cnt);
  w.dka = c.take<uint32_t>(Vp);
  w.dva = c.take<uint32_t>(Vp, &L.off_order);  // 4 passes of 8 bits end back in (dka, dva)
  w.dkb = c.take<uint32_t>(Vp);
  w.dvb = c.take<uint32_t>(Vp);
  const size_t hw = radix_hist_words(Vp);
  w.hist = c.take<uint32_t>(hw);
  size_t sw = lists_scan_words(b, npad);
  if (hw > sw) sw = hw;
  w.scan_tmp = c.take<uint32_t>(scan_tmp_words(sw));
  carve_lists(c, b, npad, cap, &w.lists, &L.off_sb_list, &L.off_sb_start);
  L.sb_chunks = npad / kChunk;
  L.num_sb = b.num_sb;
  for (int v = 0; v < b.num_views; ++v) L.sb_log2[v] = b.v[v].sb_log2;
  w.pix_T = c.take<float>(b.num_pix, &L.off_pix_T);
  w.pix_stop = c.take<uint32_t>(b.num_pix, &L.off_pix_stop);
  w.grad_pix = c.take<float>(size_t(b.num_pix) * 3, &L.off_grad_pix);
  w.slab_loss = c.take<float>(size_t(b.num_items) * L.slabs_per_tile, &L.off_slab_loss);
  w.grad2d = c.take<float4>(3 * VN + 3, &L.off_grad2d);
  w.grad2d_tag = c.take<unsigned long long>(1);
  w.sched = c.take<uint32_t>(80);
  w.task_order = c.take<uint32_t>(size_t(b.num_items) + 1);
  w.item_cost = c.take<uint32_t>(size_t(b.num_items) + 1);
  L.total_bytes = align_up(c.off, 256);
  return w;
}

int check_params(const dsplat_gauss_params* p) {
  if (!p) return fail(DSPLAT_ERR_INVALID_ARG, "params is null");
  if (p->sh_degree < -1 || p->sh_degree > 3) return fail(DSPLAT_ERR_INVALID_ARG, "sh_degree must be -1..3");
  if (p->num_pnt > 0 && (!p->means || !p->log_scales || !p->quats || !p->opacity || !p->colors))
    return fail(DSPLAT_ERR_INVALID_ARG, "null parameter pointer");
  return DSPLAT_OK;
}

}  // namespace

// Records the message returned by dsplat_last_error() for entry points that
// live in other translation units.
int report_error(int code, const char* msg) { return fail(code, msg); }

}  // namespace dsplat

using namespace dsplat;

extern "C" {

const char* dsplat_version(void) { return "dsplat-b200 0.1.0 (sm_100a)"; }
const char* dsplat_last_error(void) { return g_last_error.c_str(); }

int dsplat_gauss_pnt2splat3_to_pnt2splat2(dsplat_stream stream, uint32_t num_pnt, const float* pnt2xyz,
                                          const float* pnt2scale, const float* pnt2quat, float* pnt2pixxydepth,
                                          float* pnt2pixconvinv, float* pnt2pixaabb,
                                          const float* transform_world2ndc, uint32_t img_w, uint32_t img_h) {
  if (num_pnt == 0) return DSPLAT_OK;
  if (!pnt2xyz || !pnt2scale || !pnt2quat || !pnt2pixxydepth || !pnt2pixconvinv || !pnt2pixaabb ||
      !transform_world2ndc)
    return fail(DSPLAT_ERR_INVALID_ARG, "null pointer");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  k_gauss_project_ref<<<blocks_for(num_pnt, 256), 256, 0, st>>>(num_pnt, pnt2xyz, pnt2quat, pnt2scale,
                                                                transform_world2ndc, int(img_w), int(img_h),
                                                                pnt2pixxydepth, pnt2pixconvinv, pnt2pixaabb); count_launch();
  TRY_CUDA(cudaGetLastError(), "k_gauss_project_ref");
  return DSPLAT_OK;
}

size_t dsplat_tile2idx_workspace_size(uint32_t num_pnt, uint32_t tile_w, uint32_t tile_h, uint64_t num_pairs) {
  return carve_tiles(nullptr, num_pnt, tile_w, tile_h, num_pairs).bytes;
}

int dsplat_gauss_tile2idx_count(dsplat_stream stream, uint32_t num_pnt, const float* pnt2pixaabb, uint32_t img_w,
                                uint32_t img_h, uint32_t tile_size, void* workspace, size_t workspace_bytes,
                                uint64_t* num_pairs) {
  if (!ts_ok(tile_size)) return fail(DSPLAT_ERR_UNSUPPORTED, "tile_size must be 8, 16 or 32");
  if (num_pnt > 0 && !pnt2pixaabb) return fail(DSPLAT_ERR_INVALID_ARG, "null pnt2pixaabb");
  const uint32_t tw = ceil_div(img_w, tile_size), th = ceil_div(img_h, tile_size);
  // xyd is not needed for counting; pass the aabb pointer as a dummy centre array
  return tiles_count(static_cast<cudaStream_t>(stream), num_pnt, pnt2pixaabb, pnt2pixaabb, nullptr, tw, th,
                     tile_size, workspace, workspace_bytes, num_pairs);
}

int dsplat_gauss_tile2idx_idx2pnt(dsplat_stream stream, uint32_t num_pnt, const float* pnt2pixxydepth,
                                  const float* pnt2pixaabb, uint32_t img_w, uint32_t img_h, uint32_t tile_size,
                                  uint32_t* tile2idx, uint32_t* idx2pnt, uint64_t capacity, uint64_t* idx2tiledepth,
                                  void* workspace, size_t workspace_bytes) {
  if (!ts_ok(tile_size)) return fail(DSPLAT_ERR_UNSUPPORTED, "tile_size must be 8, 16 or 32");
  if (num_pnt > 0 && (!pnt2pixaabb || !pnt2pixxydepth)) return fail(DSPLAT_ERR_INVALID_ARG, "null input");
  const uint32_t tw = ceil_div(img_w, tile_size), th = ceil_div(img_h, tile_size);
  return tiles_fill(static_cast<cudaStream_t>(stream), num_pnt, pnt2pixxydepth, pnt2pixaabb, nullptr, int(img_w),
                    int(img_h), tw, th, tile_size, tile2idx, idx2pnt, capacity, idx2tiledepth, workspace,
                    workspace_bytes);
}

int dsplat_gauss_rasterize_pnt2splat2_stop(dsplat_stream stream, uint32_t img_w, uint32_t img_h, float* pix2rgb,
                                           const float* pnt2pixxydepth, const float* pnt2pixconvinv,
                                           const float* pnt2pixaabb, const float* pnt2opacity, const float* pnt2rgb,
                                           uint32_t tile_size, const uint32_t* tile2idx, const uint32_t* idx2pnt,
                                           float* pix2transmit, uint32_t* pix2stop, int32_t stop_rule) {
  if (!ts_ok(tile_size)) return fail(DSPLAT_ERR_UNSUPPORTED, "tile_size must be 8, 16 or 32");
  if (stop_rule != DSPLAT_STOP_CPU && stop_rule != DSPLAT_STOP_CUDA)
    return fail(DSPLAT_ERR_INVALID_ARG, "stop_rule must be DSPLAT_STOP_CPU or DSPLAT_STOP_CUDA");
  if (img_w == 0 || img_h == 0) return DSPLAT_OK;
  if (!pix2rgb || !tile2idx) return fail(DSPLAT_ERR_INVALID_ARG, "null pointer");
  TRY_CUDA(raster_fwd_aos(static_cast<cudaStream_t>(stream), int(tile_size), int(img_w), int(img_h), pix2rgb,
                          pnt2pixxydepth, pnt2pixconvinv, pnt2pixaabb, pnt2opacity, pnt2rgb, tile2idx, idx2pnt,
                          pix2transmit, pix2stop, stop_rule == DSPLAT_STOP_CUDA),
           "raster_fwd_aos");
  return DSPLAT_OK;
}

int dsplat_gauss_rasterize_pnt2splat2(dsplat_stream stream, uint32_t img_w, uint32_t img_h, float* pix2rgb,
                                      const float* pnt2pixxydepth, const float* pnt2pixconvinv,
                                      const float* pnt2pixaabb, const float* pnt2opacity, const float* pnt2rgb,
                                      uint32_t tile_size, const uint32_t* tile2idx, const uint32_t* idx2pnt,
                                      float* pix2transmit, uint32_t* pix2stop) {
  return dsplat_gauss_rasterize_pnt2splat2_stop(stream, img_w, img_h, pix2rgb, pnt2pixxydepth, pnt2pixconvinv,
                                                pnt2pixaabb, pnt2opacity, pnt2rgb, tile_size, tile2idx, idx2pnt,
                                                pix2transmit, pix2stop, DSPLAT_STOP_CPU);
}

int dsplat_expf_cr(dsplat_stream stream, uint64_t n, const float* x, float* y) {
  if (n == 0) return DSPLAT_OK;
  if (!x || !y) return fail(DSPLAT_ERR_INVALID_ARG, "null pointer");
  TRY_CUDA(expf_cr_launch(static_cast<cudaStream_t>(stream), size_t(n), x, y), "k_expf_cr");
  return DSPLAT_OK;
}

int dsplat_circle_pnt2splat3_to_pnt2splat2(dsplat_stream stream, uint32_t num_pnt, const float* pnt2xyz,
                                           float* pnt2pixxydepth, float* pnt2pixrad,
                                           const float* transform_world2ndc, uint32_t img_w, uint32_t img_h,
                                           float radius) {
  if (num_pnt == 0) return DSPLAT_OK;
  if (!pnt2xyz || !pnt2pixxydepth || !pnt2pixrad || !transform_world2ndc)
    return fail(DSPLAT_ERR_INVALID_ARG, "null pointer");
  k_circle_project_ref<<<blocks_for(num_pnt, 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(
      num_pnt, pnt2xyz, transform_world2ndc, int(img_w), int(img_h), radius, pnt2pixxydepth, pnt2pixrad); count_launch();
  TRY_CUDA(cudaGetLastError(), "k_circle_project_ref");
  return DSPLAT_OK;
}

int dsplat_circle_tile2idx_count(dsplat_stream stream, uint32_t num_pnt, const float* pnt2pixxydepth,
                                 const float* pnt2pixrad, uint32_t tile_w, uint32_t tile_h, uint32_t tile_size,
                                 void* workspace, size_t workspace_bytes, uint64_t* num_pairs) {
  if (num_pnt > 0 && (!pnt2pixxydepth || !pnt2pixrad)) return fail(DSPLAT_ERR_INVALID_ARG, "null input");
  return tiles_count(static_cast<cudaStream_t>(stream), num_pnt, pnt2pixxydepth, nullptr, pnt2pixrad, tile_w, tile_h,
                     tile_size, workspace, workspace_bytes, num_pairs);
}

int dsplat_circle_tile2idx_idx2pnt(dsplat_stream stream, uint32_t num_pnt, const float* pnt2pixxydepth,
                                   const float* pnt2pixrad, uint32_t tile_w, uint32_t tile_h, uint32_t tile_size,
                                   uint32_t* tile2idx, uint32_t* idx2pnt, uint64_t capacity,
                                   uint64_t* idx2tiledepth, void* workspace, size_t workspace_bytes) {
  if (num_pnt > 0 && (!pnt2pixxydepth || !pnt2pixrad)) return fail(DSPLAT_ERR_INVALID_ARG, "null input");
  return tiles_fill(static_cast<cudaStream_t>(stream), num_pnt, pnt2pixxydepth, nullptr, pnt2pixrad,
                    int(tile_w * tile_size), int(tile_h * tile_size), tile_w, tile_h, tile_size, tile2idx, idx2pnt,
                    capacity, idx2tiledepth, workspace, workspace_bytes);
}

int dsplat_circle_splat(dsplat_stream stream, uint32_t img_w, uint32_t img_h, float* pix2rgb,
                        const float* pnt2pixxydepth, const float* pnt2pixrad, const float* pnt2rgb,
                        uint32_t tile_size, const uint32_t* tile2idx, const uint32_t* idx2pnt) {
  if (!ts_ok(tile_size)) return fail(DSPLAT_ERR_UNSUPPORTED, "tile_size must be 8, 16 or 32");
  if (img_w == 0 || img_h == 0) return DSPLAT_OK;
  if (!pix2rgb || !tile2idx) return fail(DSPLAT_ERR_INVALID_ARG, "null pointer");
  TRY_CUDA(circle_splat_tiles(static_cast<cudaStream_t>(stream), int(tile_size), int(img_w), int(img_h), pix2rgb,
                              pnt2pixxydepth, pnt2pixrad, pnt2rgb, tile2idx, idx2pnt),
           "circle_splat_tiles");
  return DSPLAT_OK;
}

int dsplat_circle_splat_zbuffer(dsplat_stream stream, uint32_t num_pnt, const float* pnt2pixxydepth,
                                const float* pnt2pixrad, const void* colors, int32_t color_kind, void* pix,
                                int32_t* pix2winner, uint32_t img_w, uint32_t img_h, uint32_t tile_size,
                                uint64_t* zbuf) {
  if (!ts_ok(tile_size)) return fail(DSPLAT_ERR_UNSUPPORTED, "tile_size must be 8, 16 or 32");
  if (color_kind != 0 && color_kind != 1) return fail(DSPLAT_ERR_INVALID_ARG, "color_kind must be 0 or 1");
  const size_t npix = size_t(img_w) * img_h;
  if (npix == 0) return DSPLAT_OK;
  if (!zbuf || (num_pnt > 0 && (!pnt2pixxydepth || !pnt2pixrad)) || (pix && !colors))
    return fail(DSPLAT_ERR_INVALID_ARG, "null pointer");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  k_fill_u64<<<blocks_for(npix, 256), 256, 0, st>>>(zbuf, npix, ~0ull); count_launch();
  if (num_pnt > 0) {
    k_circle_zbuf<<<blocks_for(num_pnt, 128), 128, 0, st>>>(num_pnt, pnt2pixxydepth, pnt2pixrad, int(img_w),
                                                           int(img_h), int(tile_size), zbuf);
    count_launch();
  }
  k_circle_resolve<<<blocks_for(npix, 256), 256, 0, st>>>(npix, zbuf, colors, color_kind, pix, pix2winner); count_launch();
  TRY_CUDA(cudaGetLastError(), "circle zbuffer");
  return DSPLAT_OK;
}

int dsplat_point_rasterize_pix_zbuffer(dsplat_stream stream, uint32_t num_pnt, const float* pnt2pixxyndcz,
                                       const float* pnt2rgb, float* pix2rgb, float* pix2unitdepth,
                                       int32_t* pix2winner, uint32_t img_w, uint32_t img_h, uint64_t* zbuf) {
  const size_t npix = size_t(img_w) * img_h;
  if (npix == 0) return DSPLAT_OK;
  if (!zbuf || (num_pnt > 0 && !pnt2pixxyndcz) || (pix2rgb && !pnt2rgb))
    return fail(DSPLAT_ERR_INVALID_ARG, "null pointer");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  k_fill_u64<<<blocks_for(npix, 256), 256, 0, st>>>(zbuf, npix, ~0ull); count_launch();
  if (num_pnt > 0) {
    k_point_zbuf<<<blocks_for(num_pnt, 256), 256, 0, st>>>(num_pnt, pnt2pixxyndcz, int(img_w), int(img_h), zbuf);
    count_launch();
  }
  k_point_resolve<<<blocks_for(npix, 256), 256, 0, st>>>(npix, zbuf, pnt2pixxyndcz, pnt2rgb, pix2rgb, pix2unitdepth,
                                                         pix2winner); count_launch();
  TRY_CUDA(cudaGetLastError(), "point zbuffer");
  return DSPLAT_OK;
}

int dsplat_point_rasterize_pix(dsplat_stream stream, uint32_t num_pnt, const float* pnt2pixxyndcz,
                               const float* pnt2rgb, float* pix2rgb, uint32_t img_w, uint32_t img_h, uint64_t* zbuf) {
  return dsplat_point_rasterize_pix_zbuffer(stream, num_pnt, pnt2pixxyndcz, pnt2rgb, pix2rgb, nullptr, nullptr,
                                            img_w, img_h, zbuf);
}

int dsplat_gauss_batch_layout(int64_t num_pnt, int32_t num_views, const dsplat_view* views, int32_t tile_size,
                              int32_t pixels_per_lane, uint64_t pair_capacity, dsplat_batch_layout* out) {
  if (!out) return fail(DSPLAT_ERR_INVALID_ARG, "out is null");
  ViewBatch b;
  int rc = make_batch(num_pnt, num_views, views, tile_size, pixels_per_lane, &b);
  if (rc) return rc;
  *out = carve_batch(nullptr, uint32_t(num_pnt), b, pair_capacity).L;
  return DSPLAT_OK;
}

int dsplat_gauss_batch_forward(dsplat_stream stream, const dsplat_gauss_params* params, int32_t num_views,
                               const dsplat_view* views, int32_t tile_size, int32_t pixels_per_lane,
                               uint64_t pair_capacity, void* workspace, size_t workspace_bytes, float* out_rgb,
                               float* out_alpha, const float* target) {
  int rc = check_params(params);
  if (rc) return rc;
  ViewBatch b;
  rc = make_batch(params->num_pnt, num_views, views, tile_size, pixels_per_lane, &b);
  if (rc) return rc;
  if (pair_capacity > 0xfffff000ull) return fail(DSPLAT_ERR_INVALID_ARG, "pair_capacity must fit in u32");
  const uint32_t n = uint32_t(params->num_pnt);
  BatchWs w = carve_batch(nullptr, n, b, pair_capacity);
  if (!workspace || workspace_bytes < w.L.total_bytes) return fail(DSPLAT_ERR_WORKSPACE, "workspace too small");
  if (!out_rgb) return fail(DSPLAT_ERR_INVALID_ARG, "out_rgb is null");
  w = carve_batch(workspace, n, b, pair_capacity);
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const uint32_t V = uint32_t(num_views), npad = w.L.npad;
  const size_t Vp = size_t(V) * npad;
  stage_mark(st, 0);
  TRY_CUDA(cudaMemsetAsync(w.flags, 0, 16 * sizeof(uint32_t), st), "memset");
  if (n == 0 || pair_capacity == 0) {
    TRY_CUDA(cudaMemsetAsync(w.lists.off1, 0, (size_t(b.num_sb) * (npad / kChunk) + 1) * 4, st), "memset");
  } else {
    if (npad > n) {
      k_pad_keys<<<blocks_for(size_t(npad - n) * V, 256), 256, 0, st>>>(w.dka, n, npad, V);
      count_launch();
    }
    k_fused_project<<<blocks_for(n, 128), 128, 0, st>>>(n, npad, params->sh_degree, params->means,
                                                        params->log_scales, params->quats, params->opacity,
                                                        params->colors, b, w.rec, w.rect, w.dka, nullptr);
    count_launch();
    stage_mark(st, 1);
    bool in_b = false;
    TRY_CUDA(radix_sort(st, w.dka, w.dva, w.dkb, w.dvb, Vp, nullptr, 32, V, w.hist, w.scan_tmp, &in_b, w.rect, n,
                        w.srect, true, n),
             "depth sort");
    stage_mark(st, 2);
    const uint32_t* order = in_b ? w.dvb : w.dva;
    int rc2 = build_sb_lists(st, b, n, npad, order, w.srect, w.lists, w.scan_tmp, pair_capacity, w.flags);
    if (rc2) return rc2;
    stage_mark(st, 3);
  }
  // longest-first raster task order (costs measured by the previous forward)
  TRY_CUDA(order_tasks(st, b, w.lists.off1, npad / kChunk, w.item_cost, raster_fwd_group(b.ts), w.sched,
                       w.task_order),
           "task order");
  TRY_CUDA(cudaMemsetAsync(w.item_cost, 0, size_t(b.num_items) * sizeof(uint32_t), st), "memset");
  stage_mark(st, 4);
  const FwdArgs fa{n,           w.rec,   w.lists.list1, w.lists.off1, npad / kChunk, pair_capacity, w.task_order,
                   w.flags + 2, out_rgb, w.pix_T,       w.pix_stop,   target,        w.grad_pix,    w.slab_loss,
                   w.item_cost};
  TRY_CUDA(raster_fwd(st, b, fa),
           "raster_fwd");
  stage_mark(st, 5);
  if (out_alpha) {
    k_one_minus<<<blocks_for(b.num_pix, 256), 256, 0, st>>>(w.pix_T, out_alpha, b.num_pix);
    count_launch();
  }
  TRY_CUDA(cudaGetLastError(), "forward");
  return DSPLAT_OK;
}

int dsplat_gauss_batch_backward(dsplat_stream stream, const dsplat_gauss_params* params, int32_t num_views,
                                const dsplat_view* views, int32_t tile_size, int32_t pixels_per_lane,
                                uint64_t pair_capacity, void* workspace, size_t workspace_bytes, const float* grad_rgb,
                                const dsplat_gauss_grads* grads) {
  int rc = check_params(params);
  if (rc) return rc;
  if (!grads || (params->num_pnt > 0 && (!grads->means || !grads->log_scales || !grads->quats || !grads->opacity ||
                                         !grads->colors)))
    return fail(DSPLAT_ERR_INVALID_ARG, "null gradient pointer");
  ViewBatch b;
  rc = make_batch(params->num_pnt, num_views, views, tile_size, pixels_per_lane, &b);
  if (rc) return rc;
  const uint32_t n = uint32_t(params->num_pnt);
  BatchWs w = carve_batch(nullptr, n, b, pair_capacity);
  if (!workspace || workspace_bytes < w.L.total_bytes) return fail(DSPLAT_ERR_WORKSPACE, "workspace too small");
  w = carve_batch(workspace, n, b, pair_capacity);
  if (n == 0) return DSPLAT_OK;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const size_t VN = size_t(num_views) * n;
  stage_mark(st, 6);
  // grad2d must start at zero; the projection backward zeroes what it
  // consumes, so only a buffer not known to be clean is cleared here
  const unsigned long long tag = grad2d_tag_value(w.L, n, num_views);
  k_prepare_grad2d<<<blocks_for(3 * VN, 256) < 4096 ? blocks_for(3 * VN, 256) : 4096, 256, 0, st>>>(
      w.grad2d_tag, tag, w.grad2d, 3 * VN);
  count_launch();
  TRY_CUDA(cudaMemsetAsync(w.flags + 3, 0, sizeof(uint32_t), st), "memset");
  // the forward's longest-first task order: it ranks the tasks by the walks
  // of the forward before it, the same measure as this forward's (equal once
  // the scene stops changing), and every order gives the same results
  stage_mark(st, 7);
  const BwdArgs ba{n,           w.rec,    w.lists.list1,  w.lists.off1, w.L.npad / kChunk, pair_capacity,
                   w.task_order, w.flags + 3, grad_rgb ? grad_rgb : w.grad_pix, w.pix_T, w.pix_stop, w.grad2d};
  TRY_CUDA(raster_bwd(st, b, ba),
           "raster_bwd");
  stage_mark(st, 8);
  k_project_bwd_geom<<<blocks_for(n, 128), 128, 0, st>>>(n, params->means, params->log_scales, params->quats, b,
                                                         w.grad2d, grads->means, grads->log_scales, grads->quats,
                                                         grads->opacity);
  count_launch();
  k_project_bwd_colour<<<blocks_for(n, 128), 128, 0, st>>>(n, params->sh_degree, params->means, params->colors, b,
                                                           w.grad2d, grads->means, grads->colors, w.grad2d_tag,
                                                           tag);
  count_launch();
  stage_mark(st, 9);
  TRY_CUDA(cudaGetLastError(), "backward");
  return DSPLAT_OK;
}

int dsplat_gauss_batch_status(dsplat_stream stream, const void* workspace, uint32_t* flags, uint64_t* capacity_needed,
                              uint64_t* tile_pairs) {
  if (!workspace) return fail(DSPLAT_ERR_INVALID_ARG, "workspace is null");
  uint32_t h[10] = {};
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  TRY_CUDA(cudaMemcpyAsync(h, workspace, sizeof(h), cudaMemcpyDeviceToHost, st), "memcpy");
  TRY_CUDA(cudaStreamSynchronize(st), "sync");
  uint64_t pairs, entries;
  memcpy(&pairs, h + 6, 8);
  memcpy(&entries, h + 8, 8);
  if (flags) *flags = h[0];
  if (capacity_needed) *capacity_needed = entries;
  if (tile_pairs) *tile_pairs = pairs;
  return (h[0] & kFlagPairOverflow) ? DSPLAT_ERR_CAPACITY : DSPLAT_OK;
}

int dsplat_gauss_adam_step(dsplat_stream stream, int64_t num_pnt, int32_t sh_degree,
                           const dsplat_gauss_tensors* params, const dsplat_gauss_grads* grads,
                           const dsplat_gauss_tensors* exp_avg, const dsplat_gauss_tensors* exp_avg_sq, double lr,
                           double beta1, double beta2, double eps, int32_t* step) {
  if (num_pnt <= 0) return DSPLAT_OK;
  if (!params || !grads || !exp_avg || !exp_avg_sq || !step) return fail(DSPLAT_ERR_INVALID_ARG, "null argument");
  if (sh_degree < -1 || sh_degree > 3) return fail(DSPLAT_ERR_INVALID_ARG, "sh_degree must be -1..3");
  const size_t n = size_t(num_pnt);
  const size_t K = sh_degree < 0 ? 1 : size_t(sh_degree + 1) * size_t(sh_degree + 1);
  const size_t counts[5] = {3 * n, 3 * n, 4 * n, n, 3 * K * n};
  float* const ps[5] = {params->means, params->log_scales, params->quats, params->opacity, params->colors};
  const float* const gs[5] = {grads->means, grads->log_scales, grads->quats, grads->opacity, grads->colors};
  float* const ms[5] = {exp_avg->means, exp_avg->log_scales, exp_avg->quats, exp_avg->opacity, exp_avg->colors};
  float* const vs[5] = {exp_avg_sq->means, exp_avg_sq->log_scales, exp_avg_sq->quats, exp_avg_sq->opacity,
                        exp_avg_sq->colors};
  AdamSeg seg;
  size_t acc = 0;
  for (int k = 0; k < 5; ++k) {
    if (!ps[k] || !gs[k] || !ms[k] || !vs[k]) return fail(DSPLAT_ERR_INVALID_ARG, "null tensor");
    seg.p[k] = ps[k];
    seg.g[k] = gs[k];
    seg.m[k] = ms[k];
    seg.v[k] = vs[k];
    acc += counts[k];
    seg.end[k] = acc;
  }
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  k_adam_fused<<<unsigned(std::min<size_t>(blocks_for(acc, 256), 148 * 16)), 256, 0, st>>>(seg, lr, beta1, beta2,
                                                                                         eps, step);
  count_launch();
  k_adam_step_inc<<<1, 32, 0, st>>>(step);
  count_launch();
  TRY_CUDA(cudaGetLastError(), "adam");
  return DSPLAT_OK;
}

int dsplat_adam_step(dsplat_stream stream, int64_t n, float* param, const float* grad, float* exp_avg,
                     float* exp_avg_sq, float lr, float beta1, float beta2, float eps, int32_t step) {
  if (n <= 0) return DSPLAT_OK;
  if (!param || !grad || !exp_avg || !exp_avg_sq || step < 1) return fail(DSPLAT_ERR_INVALID_ARG, "bad argument");
  const float bc1 = 1.f - powf(beta1, float(step)), bc2 = 1.f - powf(beta2, float(step));
  k_adam<<<blocks_for(size_t(n), 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(
      size_t(n), param, grad, exp_avg, exp_avg_sq, lr, beta1, beta2, eps, bc1, bc2); count_launch();
  TRY_CUDA(cudaGetLastError(), "adam");
  return DSPLAT_OK;
}

}  // extern "C"

extern "C" uint64_t dsplat_launch_count(void) { return dsplat::g_launches.load(); }

extern "C" int dsplat_set_stage_events(void* const* events, int32_t count) {
  if (count < 0 || count > 16 || (count > 0 && !events)) return fail(DSPLAT_ERR_INVALID_ARG, "bad event list");
  for (int k = 0; k < count; ++k) g_stage_ev[k] = static_cast<cudaEvent_t>(events[k]);
  g_stage_n = count;
  return DSPLAT_OK;
}
