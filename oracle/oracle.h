/*
 * oracle.h -- CPU restatement of nobuyuki83/del-splat's splatting path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker for the CUDA
 * implementation in del-splat_b200/.  Only tests/, __graft_entry__.smoke()
 * and bench.py's CPU-baseline / reference arms may load it.  Nothing in the
 * product path calls it.
 *
 * Parity status: the tile-pair key format, the tile span, the point
 * z-buffer and the blend (splat_gauss.cu:56-109, with the C library's expf
 * and its double stop test) are pinned against the reference's own CUDA
 * sources compiled on the CPU (oracle/ref/, output oracle/_ref/).  The
 * del-geo helpers those sources call (matrix products, the projected
 * covariance, its safe inverse, the quadratic form) live in an absent crate
 * and are restated here; that part is "parity unpinned" (no golden vector
 * exists upstream).
 *
 * Conventions (all arrays row-major, f32 unless stated):
 *   mvp[16]            column-major 4x4 world->NDC, larger ndc_z = nearer
 *   pnt2pixxydepth     [N,3] pixel x, pixel y, ndc z
 *   pnt2pixconvinv     [N,3] conic (a, b, c) of the 2x2 inverse covariance
 *   pnt2pixaabb        [N,4] xmin, ymin, xmax, ymax in pixels
 *   tile2idx           [T+1] u32, idx2pnt [P] u32, keys [P] u64
 *   image              [H,W,3], pixel (ix,iy) centre at (ix+0.5, iy+0.5)
 */
#ifndef DSPLAT_ORACLE_H
#define DSPLAT_ORACLE_H
#include <stdint.h>
#ifdef __cplusplus
extern "C" {
#endif

/* ---- reference forward path, FP32 ---------------------------------- */
void orc_gauss_project(int64_t n, const float* xyz, const float* quat,
                       const float* scale, const float* mvp, int w, int h,
                       float* xyd, float* conic, float* aabb);
void orc_circle_project(int64_t n, const float* xyz, const float* mvp, int w,
                        int h, float radius, float* xyd, float* rad);
void orc_circle_aabb(int64_t n, const float* xyd, const float* rad,
                     float* aabb);
uint64_t orc_tile2pnt_count(int64_t n, const float* aabb, int tile_w,
                            int tile_h, int ts, uint32_t* tile2idx);
void orc_tile2pnt_fill(int64_t n, const float* aabb, const float* xyd,
                       int tile_w, int tile_h, int ts, const uint32_t* tile2idx,
                       uint32_t* idx2pnt, uint64_t* keys);
/* Blend (pnt2pixxyndcz.rs:86-93 arithmetic).  mode bit 1: the C library's
 * expf instead of the correctly rounded exp; mode bit 2: the CUDA kernel's
 * double stop test (alpha_sum >= 0.999f) instead of del-splat-cpu's
 * alpha_sum > 0.999f.  The plain entry points use mode 0. */
void orc_gauss_rasterize_tiled(int w, int h, int ts, const uint32_t* tile2idx,
                               const uint32_t* idx2pnt, const float* xyd,
                               const float* conic, const float* aabb,
                               const float* opacity, const float* rgb,
                               float* pix_rgb, float* pix_T,
                               int32_t* pix_last, int nthreads);
void orc_gauss_rasterize_tiled_mode(int w, int h, int ts,
                                    const uint32_t* tile2idx,
                                    const uint32_t* idx2pnt, const float* xyd,
                                    const float* conic, const float* aabb,
                                    const float* opacity, const float* rgb,
                                    float* pix_rgb, float* pix_T,
                                    int32_t* pix_last, int nthreads, int mode);
void orc_gauss_render_naive(int64_t n, const float* xyd, const float* conic,
                            const float* aabb, const float* opacity,
                            const float* rgb, int w, int h, float* pix_rgb);
void orc_gauss_render_naive_mode(int64_t n, const float* xyd,
                                 const float* conic, const float* aabb,
                                 const float* opacity, const float* rgb, int w,
                                 int h, float* pix_rgb, int mode);
/* exp(x) correctly rounded to float, elementwise */
void orc_expf_cr(int64_t n, const float* x, float* out);
void orc_circle_splat_tiled(int w, int h, int ts, const uint32_t* tile2idx,
                            const uint32_t* idx2pnt, const float* xyd,
                            const float* rad, int32_t* winner);
void orc_point_render_sort_depth(int64_t n, const float* xyd, int w, int h,
                                 int32_t* winner);

/* ---- differentiable path (no upstream counterpart), FP32 mirror ------ */
void orc_fused_project(int64_t n, const float* means, const float* log_scales,
                       const float* quats, const float* colors, int sh_deg,
                       const float* mvp, const float* campos, int w, int h,
                       float* xyd, float* conic, float* aabb, float* rgb);
void orc_sh_eval(int64_t n, const float* means, const float* colors,
                 int sh_deg, const float* campos, float* rgb);

/* ---- FP64 gradient oracle --------------------------------------------
 * The discrete structure (tile lists, per-pixel stop position, per-Gaussian
 * AABB used for the inclusion test) is frozen from a forward run; the loss
 * is then a smooth function of the parameters, which is what the analytic
 * backward differentiates.  loss = sum_pix sum_ch (C - target)^2.        */
typedef struct {
  int64_t n;
  int sh_deg;                 /* -1: colors are RGB [N,3]; 0..3: SH [N,K,3] */
  const float* means;         /* [N,3] */
  const float* log_scales;    /* [N,3] */
  const float* quats;         /* [N,4] (x,y,z,w), normalised inside */
  const float* opacity;       /* [N]   */
  const float* colors;        /* [N,3] or [N,K,3] */
  const float* mvp;           /* [16]  */
  const float* campos;        /* [3]   */
  int w, h, ts;
  const uint32_t* tile2idx;   /* [T+1] */
  const uint32_t* idx2pnt;    /* [P]   */
  const int32_t* pix_last;    /* [H*W] absolute list position where the walk stopped */
  const float* aabb;          /* [N,4] frozen inclusion boxes */
  const float* target;        /* [H,W,3] */
} orc64_scene;

double orc64_loss(const orc64_scene* s, const uint8_t* tile_mask,
                  double* pix_rgb);
/* grads: means[N,3], log_scales[N,3], quats[N,4], opacity[N], colors[N,K*3] */
double orc64_backward(const orc64_scene* s, double* g_means,
                      double* g_log_scales, double* g_quats, double* g_opacity,
                      double* g_colors);
/* central difference of the loss w.r.t. one scalar parameter.
 * kind: 0 means, 1 log_scales, 2 quats, 3 opacity, 4 colors */
double orc64_fd(const orc64_scene* s, int kind, int64_t gauss, int comp,
                double h);

/* ---- FP32 CPU pipeline used as the timed CPU baseline --------------- */
/* One view, fwd + bwd, FP32, OpenMP over tiles.  Returns pairs. */
uint64_t orc_cpu_fwd_bwd(const orc64_scene* s, int nthreads, float* pix_rgb,
                         float* g_means, float* g_log_scales, float* g_quats,
                         float* g_opacity, float* g_colors);

#ifdef __cplusplus
}
#endif
#endif
