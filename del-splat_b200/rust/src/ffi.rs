//! Raw declarations of the C ABI in include/dsplat.h (libdsplat.so).
//! Device pointers are passed as raw pointers, streams as `*mut c_void`
//! (a `CUstream`).  tests/test_capi.py checks these against the header.
#![allow(non_camel_case_types)]
use std::ffi::{c_char, c_void};

pub type dsplat_stream = *mut c_void;

pub const DSPLAT_OK: i32 = 0;
pub const DSPLAT_ERR_INVALID_ARG: i32 = 1;
pub const DSPLAT_ERR_CAPACITY: i32 = 2;
pub const DSPLAT_ERR_CUDA: i32 = 3;
pub const DSPLAT_ERR_WORKSPACE: i32 = 4;
pub const DSPLAT_ERR_UNSUPPORTED: i32 = 5;
pub const DSPLAT_STOP_CPU: i32 = 0;
pub const DSPLAT_STOP_CUDA: i32 = 1;

extern "C" {
    pub fn dsplat_version() -> *const c_char;
    pub fn dsplat_last_error() -> *const c_char;
    pub fn dsplat_launch_count() -> u64;

    pub fn dsplat_gauss_pnt2splat3_to_pnt2splat2(
        stream: dsplat_stream, num_pnt: u32, pnt2xyz: *const f32, pnt2scale: *const f32, pnt2quat: *const f32,
        pnt2pixxydepth: *mut f32, pnt2pixconvinv: *mut f32, pnt2pixaabb: *mut f32,
        transform_world2ndc: *const f32, img_w: u32, img_h: u32,
    ) -> i32;
    pub fn dsplat_tile2idx_workspace_size(num_pnt: u32, tile_w: u32, tile_h: u32, num_pairs: u64) -> usize;
    pub fn dsplat_gauss_tile2idx_count(
        stream: dsplat_stream, num_pnt: u32, pnt2pixaabb: *const f32, img_w: u32, img_h: u32, tile_size: u32,
        workspace: *mut c_void, workspace_bytes: usize, num_pairs: *mut u64,
    ) -> i32;
    pub fn dsplat_gauss_tile2idx_idx2pnt(
        stream: dsplat_stream, num_pnt: u32, pnt2pixxydepth: *const f32, pnt2pixaabb: *const f32, img_w: u32,
        img_h: u32, tile_size: u32, tile2idx: *mut u32, idx2pnt: *mut u32, capacity: u64, idx2tiledepth: *mut u64,
        workspace: *mut c_void, workspace_bytes: usize,
    ) -> i32;
    pub fn dsplat_gauss_rasterize_pnt2splat2(
        stream: dsplat_stream, img_w: u32, img_h: u32, pix2rgb: *mut f32, pnt2pixxydepth: *const f32,
        pnt2pixconvinv: *const f32, pnt2pixaabb: *const f32, pnt2opacity: *const f32, pnt2rgb: *const f32,
        tile_size: u32, tile2idx: *const u32, idx2pnt: *const u32, pix2transmit: *mut f32, pix2stop: *mut u32,
    ) -> i32;
    pub fn dsplat_gauss_rasterize_pnt2splat2_stop(
        stream: dsplat_stream, img_w: u32, img_h: u32, pix2rgb: *mut f32, pnt2pixxydepth: *const f32,
        pnt2pixconvinv: *const f32, pnt2pixaabb: *const f32, pnt2opacity: *const f32, pnt2rgb: *const f32,
        tile_size: u32, tile2idx: *const u32, idx2pnt: *const u32, pix2transmit: *mut f32, pix2stop: *mut u32,
        stop_rule: i32,
    ) -> i32;
    pub fn dsplat_expf_cr(stream: dsplat_stream, n: u64, x: *const f32, y: *mut f32) -> i32;

    pub fn dsplat_circle_pnt2splat3_to_pnt2splat2(
        stream: dsplat_stream, num_pnt: u32, pnt2xyz: *const f32, pnt2pixxydepth: *mut f32, pnt2pixrad: *mut f32,
        transform_world2ndc: *const f32, img_w: u32, img_h: u32, radius: f32,
    ) -> i32;
    pub fn dsplat_circle_tile2idx_count(
        stream: dsplat_stream, num_pnt: u32, pnt2pixxydepth: *const f32, pnt2pixrad: *const f32, tile_w: u32,
        tile_h: u32, tile_size: u32, workspace: *mut c_void, workspace_bytes: usize, num_pairs: *mut u64,
    ) -> i32;
    pub fn dsplat_circle_tile2idx_idx2pnt(
        stream: dsplat_stream, num_pnt: u32, pnt2pixxydepth: *const f32, pnt2pixrad: *const f32, tile_w: u32,
        tile_h: u32, tile_size: u32, tile2idx: *mut u32, idx2pnt: *mut u32, capacity: u64, idx2tiledepth: *mut u64,
        workspace: *mut c_void, workspace_bytes: usize,
    ) -> i32;
    pub fn dsplat_circle_splat(
        stream: dsplat_stream, img_w: u32, img_h: u32, pix2rgb: *mut f32, pnt2pixxydepth: *const f32,
        pnt2pixrad: *const f32, pnt2rgb: *const f32, tile_size: u32, tile2idx: *const u32, idx2pnt: *const u32,
    ) -> i32;
    pub fn dsplat_circle_splat_zbuffer(
        stream: dsplat_stream, num_pnt: u32, pnt2pixxydepth: *const f32, pnt2pixrad: *const f32,
        colors: *const c_void, color_kind: i32, pix: *mut c_void, pix2winner: *mut i32, img_w: u32, img_h: u32,
        tile_size: u32, zbuf: *mut u64,
    ) -> i32;

    pub fn dsplat_point_rasterize_pix_zbuffer(
        stream: dsplat_stream, num_pnt: u32, pnt2pixxyndcz: *const f32, pnt2rgb: *const f32, pix2rgb: *mut f32,
        pix2unitdepth: *mut f32, pix2winner: *mut i32, img_w: u32, img_h: u32, zbuf: *mut u64,
    ) -> i32;
    pub fn dsplat_point_rasterize_pix_zbuffer_noalloc(
        stream: dsplat_stream, num_pnt: u32, pnt2pixxyndcz: *const f32, pnt2rgb: *const f32, pix2rgb: *mut f32,
        pix2unitdepth: *mut f32, pix2winner: *mut i32, img_w: u32, img_h: u32,
    ) -> i32;
    pub fn dsplat_point_rasterize_pix(
        stream: dsplat_stream, num_pnt: u32, pnt2pixxyndcz: *const f32, pnt2rgb: *const f32, pix2rgb: *mut f32,
        img_w: u32, img_h: u32, zbuf: *mut u64,
    ) -> i32;
}
