/*
 * dsplat.h -- C ABI of the B200 splatting library (libdsplat.so).
 *
 * Plain C: device pointers, sizes and a cudaStream_t (passed as void*).
 * Every call is asynchronous on the given stream unless it says otherwise,
 * returns a status code and never aborts.  The library allocates no device
 * memory: outputs and workspaces belong to the caller (size them with the
 * *_workspace_size queries).  Thread-safe as long as two calls do not share a
 * workspace at the same time.
 *
 * Each entry point cites the del-splat (nobuyuki83/del-splat) interface it
 * replaces.  Array conventions follow the reference:
 *   pnt2xyz [N,3], pnt2quat [N,4] (x,y,z,w), pnt2scale [N,3] (std-dev),
 *   transform_world2ndc [16] column-major (larger ndc_z = nearer),
 *   pnt2pixxydepth [N,3] (pixel x, pixel y, ndc z), pnt2pixconvinv [N,3]
 *   (conic a,b,c), pnt2pixaabb [N,4] (xmin,ymin,xmax,ymax),
 *   tile2idx [T+1] u32, idx2pnt [P] u32, pix2rgb [H,W,3] f32.
 */
#ifndef DSPLAT_H
#define DSPLAT_H
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define DSPLAT_OK 0
#define DSPLAT_ERR_INVALID_ARG 1  /* null pointer, bad size or shape     */
#define DSPLAT_ERR_CAPACITY 2     /* pair buffer too small (see *_status) */
#define DSPLAT_ERR_CUDA 3         /* a CUDA runtime call failed           */
#define DSPLAT_ERR_WORKSPACE 4    /* workspace smaller than required      */
#define DSPLAT_ERR_UNSUPPORTED 5  /* e.g. tile size other than 8/16/32    */

typedef void* dsplat_stream; /* cudaStream_t */

/* Library version string and the message of the last failed call on this
 * host thread. */
const char* dsplat_version(void);
const char* dsplat_last_error(void);
/* Number of kernel launches this library has issued in the process. */
uint64_t dsplat_launch_count(void);

/* ===================== del-splat-cudarc :: splat_gauss ================== */

/* del-splat-cudarc/src/splat_gauss.rs:6-44 pnt2splat3_to_pnt2splat2
 * (kernel splat_gauss.cu:10-53). */
int dsplat_gauss_pnt2splat3_to_pnt2splat2(dsplat_stream stream, uint32_t num_pnt, const float* pnt2xyz,
                                          const float* pnt2scale, const float* pnt2quat, float* pnt2pixxydepth,
                                          float* pnt2pixconvinv, float* pnt2pixaabb,
                                          const float* transform_world2ndc, uint32_t img_w, uint32_t img_h);

/* Workspace for the tile2idx / idx2pnt builders below (Gaussian and circle). */
size_t dsplat_tile2idx_workspace_size(uint32_t num_pnt, uint32_t tile_w, uint32_t tile_h, uint64_t num_pairs);

/* del-splat-cudarc/src/splat_gauss.rs:96-195 tile2idx_idx2pnt, split in two
 * because the reference allocates its outputs: (1) count -- synchronises the
 * stream and returns the pair total P on the host, like the reference's D2H
 * read at splat_gauss.rs:147; (2) fill caller buffers tile2idx[T+1] and
 * idx2pnt[capacity] (capacity >= P).  idx2tiledepth (nullable) receives the
 * sorted 64-bit keys (tile << 32 | bits(max(ndc_z+1, 0))).  Unlike the
 * reference, the given tile_size is used throughout (the reference
 * hard-codes 16 in its count/fill launches, splat_gauss.rs:127,176). */
int dsplat_gauss_tile2idx_count(dsplat_stream stream, uint32_t num_pnt, const float* pnt2pixaabb, uint32_t img_w,
                                uint32_t img_h, uint32_t tile_size, void* workspace, size_t workspace_bytes,
                                uint64_t* num_pairs);
int dsplat_gauss_tile2idx_idx2pnt(dsplat_stream stream, uint32_t num_pnt, const float* pnt2pixxydepth,
                                  const float* pnt2pixaabb, uint32_t img_w, uint32_t img_h, uint32_t tile_size,
                                  uint32_t* tile2idx, uint32_t* idx2pnt, uint64_t capacity, uint64_t* idx2tiledepth,
                                  void* workspace, size_t workspace_bytes);

/* del-splat-cudarc/src/splat_gauss.rs:46-94 rasterize_pnt2splat2 (kernel
 * splat_gauss.cu:56-109): accumulates into pix2rgb like the reference.
 * pix2transmit [H,W] and pix2stop [H,W] (nullable) receive the final
 * transmittance and the list position where each pixel's walk stopped.
 * The blend performs del-splat-cpu's f32 operations (pnt2pixxyndcz.rs:86-93)
 * with a correctly rounded exp and its stop test alpha_sum > 0.999f. */
int dsplat_gauss_rasterize_pnt2splat2(dsplat_stream stream, uint32_t img_w, uint32_t img_h, float* pix2rgb,
                                      const float* pnt2pixxydepth, const float* pnt2pixconvinv,
                                      const float* pnt2pixaabb, const float* pnt2opacity, const float* pnt2rgb,
                                      uint32_t tile_size, const uint32_t* tile2idx, const uint32_t* idx2pnt,
                                      float* pix2transmit, uint32_t* pix2stop);

/* The same with a choice of stop test: DSPLAT_STOP_CPU is del-splat-cpu's
 * (pnt2pixxyndcz.rs:93, f32 alpha_sum > 0.999f), DSPLAT_STOP_CUDA the
 * reference CUDA kernel's (splat_gauss.cu:105, `alpha_sum > 0.999` in double,
 * i.e. alpha_sum >= 0.999f).  The two reference paths disagree exactly when
 * a pixel's sum lands on 0.999f. */
#define DSPLAT_STOP_CPU 0
#define DSPLAT_STOP_CUDA 1
int dsplat_gauss_rasterize_pnt2splat2_stop(dsplat_stream stream, uint32_t img_w, uint32_t img_h, float* pix2rgb,
                                           const float* pnt2pixxydepth, const float* pnt2pixconvinv,
                                           const float* pnt2pixaabb, const float* pnt2opacity, const float* pnt2rgb,
                                           uint32_t tile_size, const uint32_t* tile2idx, const uint32_t* idx2pnt,
                                           float* pix2transmit, uint32_t* pix2stop, int32_t stop_rule);

/* No reference counterpart: the blend's exponential, y[i] = e^x[i]
 * correctly rounded to float (the exp that del-splat-cpu's f32 `exp` call
 * approximates to within one unit in the last place), elementwise. */
int dsplat_expf_cr(dsplat_stream stream, uint64_t n, const float* x, float* y);

/* ===================== del-splat-cudarc :: splat_circle ================= */

/* del-splat-cudarc/src/splat_circle.rs:96-132 pnt2splat3_to_pnt2splat2
 * (kernel splat_circle.cu:7-41). */
int dsplat_circle_pnt2splat3_to_pnt2splat2(dsplat_stream stream, uint32_t num_pnt, const float* pnt2xyz,
                                           float* pnt2pixxydepth, float* pnt2pixrad,
                                           const float* transform_world2ndc, uint32_t img_w, uint32_t img_h,
                                           float radius);

/* del-splat-cudarc/src/splat_circle.rs:3-94 tile2idx_idx2pnt(tile_shape, ..):
 * same two-step contract as the Gaussian version; box = centre +- radius. */
int dsplat_circle_tile2idx_count(dsplat_stream stream, uint32_t num_pnt, const float* pnt2pixxydepth,
                                 const float* pnt2pixrad, uint32_t tile_w, uint32_t tile_h, uint32_t tile_size,
                                 void* workspace, size_t workspace_bytes, uint64_t* num_pairs);
int dsplat_circle_tile2idx_idx2pnt(dsplat_stream stream, uint32_t num_pnt, const float* pnt2pixxydepth,
                                   const float* pnt2pixrad, uint32_t tile_w, uint32_t tile_h, uint32_t tile_size,
                                   uint32_t* tile2idx, uint32_t* idx2pnt, uint64_t capacity,
                                   uint64_t* idx2tiledepth, void* workspace, size_t workspace_bytes);

/* del-splat-cudarc/src/splat_circle.rs:134-177 splat (kernel
 * splat_circle.cu:93-132): painter over the tile lists; writes covered pixels. */
int dsplat_circle_splat(dsplat_stream stream, uint32_t img_w, uint32_t img_h, float* pix2rgb,
                        const float* pnt2pixxydepth, const float* pnt2pixrad, const float* pnt2rgb,
                        uint32_t tile_size, const uint32_t* tile2idx, const uint32_t* idx2pnt);

/* Circle splat through a packed 64-bit depth|index z-buffer (no tile lists);
 * same winners as dsplat_circle_splat over tile lists of tile_size.
 * colors: color_kind 0 -> float rgb [N,3] into pix float [H,W,3];
 *         color_kind 1 -> u32 rgba [N] into pix u32 [H,W].
 * zbuf: caller workspace of img_w*img_h u64.  pix2winner [H,W] nullable. */
int dsplat_circle_splat_zbuffer(dsplat_stream stream, uint32_t num_pnt, const float* pnt2pixxydepth,
                                const float* pnt2pixrad, const void* colors, int32_t color_kind, void* pix,
                                int32_t* pix2winner, uint32_t img_w, uint32_t img_h, uint32_t tile_size,
                                uint64_t* zbuf);

/* ===================== del-splat-dlpack :: splat_point ================== */

/* del-splat-dlpack/src/splat_point.rs:47-106 point_splat_rasterize_pix_zbuffer
 * (kernel splat_point.cu:49-74): nearest point per pixel; pix2unitdepth gets
 * 1-(ndc_z+1)/2 of the winner or FLT_MAX; pix2rgb untouched where empty.
 * zbuf: caller workspace of img_w*img_h u64.  pix2winner nullable. */
int dsplat_point_rasterize_pix_zbuffer(dsplat_stream stream, uint32_t num_pnt, const float* pnt2pixxyndcz,
                                       const float* pnt2rgb, float* pix2rgb, float* pix2unitdepth,
                                       int32_t* pix2winner, uint32_t img_w, uint32_t img_h, uint64_t* zbuf);

/* No counterpart in the reference.  dsplat_point_rasterize_pix_zbuffer for
 * callers that cannot hand the library device memory (e.g. a plug-in whose
 * host application owns every GPU allocation, or a loop that must not call
 * cudaMalloc): no zbuf argument and nothing is allocated; the 64-bit keys live
 * in a fixed 2^20-entry (8 MiB) array inside the library, so img_w*img_h must
 * be <= 1048576 (larger images return DSPLAT_ERR_INVALID_ARG).  Each call
 * looks the array's address up on the current device; the first call on a
 * device also loads the library there, so make it before any stream capture.
 * Calls share the array: calls whose GPU work overlaps race. */
int dsplat_point_rasterize_pix_zbuffer_noalloc(dsplat_stream stream, uint32_t num_pnt, const float* pnt2pixxyndcz,
                                               const float* pnt2rgb, float* pix2rgb, float* pix2unitdepth,
                                               int32_t* pix2winner, uint32_t img_w, uint32_t img_h);

/* del-splat-dlpack/src/splat_point.rs:12-43 point_splat_rasterize_pix (the
 * reference has only a CPU branch, its GPU arm is todo!()). */
int dsplat_point_rasterize_pix(dsplat_stream stream, uint32_t num_pnt, const float* pnt2pixxyndcz,
                               const float* pnt2rgb, float* pix2rgb, uint32_t img_w, uint32_t img_h, uint64_t* zbuf);

/* ============ differentiable, batched Gaussian splatting (new) =========== */
/* No reference counterpart: the reference is forward-only and one view at a
 * time.  Parameters: means [N,3], log_scales [N,3], quats [N,4] (x,y,z,w,
 * normalised inside), opacity [N] (used as is), colors [N,3] RGB when
 * sh_degree < 0, else SH coefficients [N,(sh_degree+1)^2,3]. */
typedef struct {
  float mvp[16];    /* column-major world->NDC */
  float campos[3];  /* camera centre, for the SH view direction */
  int32_t width, height;
} dsplat_view;

typedef struct {
  int64_t num_pnt;
  int32_t sh_degree; /* -1 (RGB) or 0..3 */
  const float* means;
  const float* log_scales;
  const float* quats;
  const float* opacity;
  const float* colors;
} dsplat_gauss_params;

typedef struct { /* gradients, accumulated (+=) */
  float* means;
  float* log_scales;
  float* quats;
  float* opacity;
  float* colors;
} dsplat_gauss_grads;

/* Byte offsets of the batch state inside the workspace (for inspection).
 * Tile lists of the batched path live in superblock form: superblock s
 * (square blocks of 2^sb_log2[v] tiles per side, chosen per view from its
 * tile grid; view v's superblocks start at the sum of the earlier views'
 * counts, row-major inside the view) owns the entries
 * sb_list[sb_start[s * sb_chunks] .. sb_start[(s + 1) * sb_chunks]), each a
 * (point index, span) pair where span packs the tiles it covers inside the
 * superblock as x0 | y0 << 4 | x1 << 8 | y1 << 12; filtering a superblock list
 * by tile gives that tile's list in the reference's order. */
typedef struct {
  size_t total_bytes;
  uint32_t num_items; /* sum over views of tiles */
  uint32_t num_pix;   /* sum over views of pixels */
  uint32_t npad;      /* per-view padded point count of the depth sort */
  uint32_t slabs_per_tile; /* raster warp tasks per tile (4 for 32x32 tiles, else 1) */
  uint32_t num_sb;    /* superblocks over all views */
  uint32_t sb_chunks; /* entries of sb_start per superblock */
  size_t off_flags;      /* u32[16]: [0] flags, [6..7] tile pairs (u64), [8..9] superblock entries (u64) */
  size_t off_rec;        /* float4[V*N*3] per-view 2D records (written where the tile span is not empty) */
  size_t off_rect;       /* uint2[V*N] tile spans */
  size_t off_cnt;        /* u32[V*N] reserved (tiles per point; not written by the batched forward) */
  size_t off_order;      /* u32[V*npad] points in depth order per view */
  size_t off_sb_start;   /* u32[num_sb*sb_chunks+1] superblock list offsets */
  size_t off_sb_list;    /* uint2[capacity] superblock lists */
  size_t off_pix_T;      /* f32[num_pix] final transmittance */
  size_t off_pix_stop;   /* u32[num_pix] sb_list position where the walk stopped */
  size_t off_grad_pix;   /* f32[num_pix*3] dL/dpixel (loss gradient) */
  size_t off_slab_loss;  /* f32[num_items*slabs_per_tile] partial L2 losses */
  size_t off_grad2d;     /* float4[V*N*3] per-view 2D gradients (zero again after each backward) */
  int32_t sb_log2[32];   /* per view: superblock side = 1 << sb_log2 tiles (0..3) */
} dsplat_batch_layout;

/* tile_size: 8, 16 or 32.  pixels_per_lane: rasteriser work split, one warp
 * task covers 32 * pixels_per_lane pixels of a tile: 2 for 8x8 tiles, 2/4/8
 * for 16x16, 4/8 for 32x32; 0 picks the default (2, 4, 4).  Both are
 * throughput knobs only: results do not depend on pixels_per_lane. */
int dsplat_gauss_batch_layout(int64_t num_pnt, int32_t num_views, const dsplat_view* views, int32_t tile_size,
                              int32_t pixels_per_lane, uint64_t capacity, dsplat_batch_layout* out);

/* Forward over all views: projection (+SH), depth sort, superblock lists and
 * rasterisation in one launch sequence, no host sync (CUDA-graph
 * capturable).  capacity: superblock-list entries (see _status).  out_rgb: concatenated [H_v,W_v,3] images; out_alpha
 * (nullable): 1 - T per pixel.  target (nullable, same layout as out_rgb):
 * also computes the L2 loss sum (per-item partials in the workspace) and
 * its pixel gradient for dsplat_gauss_batch_backward. */
int dsplat_gauss_batch_forward(dsplat_stream stream, const dsplat_gauss_params* params, int32_t num_views,
                               const dsplat_view* views, int32_t tile_size, int32_t pixels_per_lane,
                               uint64_t capacity, void* workspace,
                               size_t workspace_bytes, float* out_rgb, float* out_alpha, const float* target);

/* Backward of the last forward on this workspace.  grad_rgb (nullable):
 * dL/d out_rgb; null uses the L2-loss gradient stored by the forward. */
int dsplat_gauss_batch_backward(dsplat_stream stream, const dsplat_gauss_params* params, int32_t num_views,
                                const dsplat_view* views, int32_t tile_size, int32_t pixels_per_lane,
                                uint64_t capacity, void* workspace,
                                size_t workspace_bytes, const float* grad_rgb, const dsplat_gauss_grads* grads);

/* Synchronises the stream and reports, for the last forward, the flags (bit 0:
 * capacity overflow -- outputs undefined), the capacity it needed (superblock
 * entries) and its number of (tile, point) pairs. */
int dsplat_gauss_batch_status(dsplat_stream stream, const void* workspace, uint32_t* flags, uint64_t* capacity_needed,
                              uint64_t* tile_pairs);

/* Profiling hook: CUDA events (cudaEvent_t) recorded on the launch stream at
 * the stage boundaries of the batched calls on this host thread:
 * forward 0 start, 1 projected, 2 depth-sorted, 3 pairs emitted, 4 tile lists
 * ready, 5 rasterised; backward 6 start, 7 gradients cleared, 8 backward
 * raster done, 9 projection backward done.  count 0 disables. */
int dsplat_set_stage_events(void* const* events, int32_t count);

/* Mutable parameter tensors (same shapes as dsplat_gauss_params). */
typedef struct {
  float* means;
  float* log_scales;
  float* quats;
  float* opacity;
  float* colors;
} dsplat_gauss_tensors;

/* No reference counterpart (the reference does not train).  One fused Adam
 * update of all five parameter tensors, the form torch.optim.Adam computes
 * (no weight decay): step is a device int32 holding the number of updates
 * done so far; the call uses step + 1 for the bias corrections and stores it,
 * so a captured graph replays with the right count.  Opacity is kept in
 * [0, 0.999] after the update (the blend needs alpha < 1). */
int dsplat_gauss_adam_step(dsplat_stream stream, int64_t num_pnt, int32_t sh_degree,
                           const dsplat_gauss_tensors* params, const dsplat_gauss_grads* grads,
                           const dsplat_gauss_tensors* exp_avg, const dsplat_gauss_tensors* exp_avg_sq, double lr,
                           double beta1, double beta2, double eps, int32_t* step);

/* Adam (bias-corrected) on one parameter tensor, in place. */
int dsplat_adam_step(dsplat_stream stream, int64_t n, float* param, const float* grad, float* exp_avg,
                     float* exp_avg_sq, float lr, float beta1, float beta2, float eps, int32_t step);

#ifdef __cplusplus
}
#endif
#endif /* DSPLAT_H */
