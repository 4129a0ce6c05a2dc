//! del-splat-cudarc/src/splat_gauss.rs, over libdsplat.so.
use crate::{check, ffi};
use del_cudarc_sys::{cu::CUstream, CuVec};

fn st(stream: CUstream) -> ffi::dsplat_stream {
    stream as ffi::dsplat_stream
}

/// splat_gauss.rs:6-44: projection of 3D Gaussians to pixel-space
/// (centre + ndc z, conic, 3-sigma box).
pub fn pnt2splat3_to_pnt2splat2(
    stream: CUstream,
    pnt2xyz: &CuVec<f32>,
    pnt2scale: &CuVec<f32>,
    pnt2quat: &CuVec<f32>,
    pnt2pixxydepth: &CuVec<f32>,
    pnt2pixconvinv: &CuVec<f32>,
    pnt2pixaabb: &CuVec<f32>,
    transform_world2ndc: &CuVec<f32>,
    img_shape: (u32, u32),
) -> anyhow::Result<()> {
    let num_pnt = (pnt2xyz.n / 3) as u32;
    let rc = unsafe {
        ffi::dsplat_gauss_pnt2splat3_to_pnt2splat2(
            st(stream),
            num_pnt,
            pnt2xyz.dptr as *const f32,
            pnt2scale.dptr as *const f32,
            pnt2quat.dptr as *const f32,
            pnt2pixxydepth.dptr as *mut f32,
            pnt2pixconvinv.dptr as *mut f32,
            pnt2pixaabb.dptr as *mut f32,
            transform_world2ndc.dptr as *const f32,
            img_shape.0,
            img_shape.1,
        )
    };
    check(rc, "pnt2splat3_to_pnt2splat2")
}

/// splat_gauss.rs:46-94: front-to-back blend over the tile lists, added into
/// pix2rgb_dev.
#[allow(clippy::too_many_arguments)]
pub fn rasterize_pnt2splat2(
    stream: CUstream,
    img_shape: (u32, u32),
    pix2rgb_dev: &CuVec<f32>,
    pnt2pixxydepth_dev: &CuVec<f32>,
    pnt2pixconvinv_dev: &CuVec<f32>,
    pnt2pixaabb_dev: &CuVec<f32>,
    pnt2opacity_dev: &CuVec<f32>,
    pnt2rgb: &CuVec<f32>,
    tile_size: u32,
    tile2idx_dev: &CuVec<u32>,
    idx2pnt_dev: &CuVec<u32>,
) -> anyhow::Result<()> {
    let rc = unsafe {
        ffi::dsplat_gauss_rasterize_pnt2splat2(
            st(stream),
            img_shape.0,
            img_shape.1,
            pix2rgb_dev.dptr as *mut f32,
            pnt2pixxydepth_dev.dptr as *const f32,
            pnt2pixconvinv_dev.dptr as *const f32,
            pnt2pixaabb_dev.dptr as *const f32,
            pnt2opacity_dev.dptr as *const f32,
            pnt2rgb.dptr as *const f32,
            tile_size,
            tile2idx_dev.dptr as *const u32,
            idx2pnt_dev.dptr as *const u32,
            std::ptr::null_mut(),
            std::ptr::null_mut(),
        )
    };
    check(rc, "rasterize_pnt2splat2")
}

/// splat_gauss.rs:96-195: (tile2idx [T+1], idx2pnt [P]) for the image's
/// tile grid, each tile's list in (depth, point) order.  The given tile size
/// is used throughout (the reference hard-codes 16 in its launches).
pub fn tile2idx_idx2pnt(
    stream: CUstream,
    img_shape: (u32, u32),
    tile_size: u32,
    pnt2pixxydepth: &CuVec<f32>,
    pnt2pixaabb: &CuVec<f32>,
) -> anyhow::Result<(CuVec<u32>, CuVec<u32>)> {
    let num_pnt = (pnt2pixxydepth.n / 3) as u32;
    let tile_w = img_shape.0.div_ceil(tile_size);
    let tile_h = img_shape.1.div_ceil(tile_size);
    let ws_bytes = unsafe { ffi::dsplat_tile2idx_workspace_size(num_pnt, tile_w, tile_h, 0) };
    let ws = CuVec::<u8>::alloc_zeros(ws_bytes.max(1), stream).unwrap();
    let mut num_pairs = 0u64;
    let rc = unsafe {
        ffi::dsplat_gauss_tile2idx_count(
            st(stream),
            num_pnt,
            pnt2pixaabb.dptr as *const f32,
            img_shape.0,
            img_shape.1,
            tile_size,
            ws.dptr as *mut std::ffi::c_void,
            ws_bytes,
            &mut num_pairs,
        )
    };
    check(rc, "tile2idx_count")?;
    let ws_bytes = unsafe { ffi::dsplat_tile2idx_workspace_size(num_pnt, tile_w, tile_h, num_pairs) };
    let ws = CuVec::<u8>::alloc_zeros(ws_bytes.max(1), stream).unwrap();
    let tile2idx = CuVec::<u32>::alloc_zeros((tile_w * tile_h) as usize + 1, stream).unwrap();
    let idx2pnt = CuVec::<u32>::alloc_zeros((num_pairs as usize).max(1), stream).unwrap();
    let rc = unsafe {
        ffi::dsplat_gauss_tile2idx_idx2pnt(
            st(stream),
            num_pnt,
            pnt2pixxydepth.dptr as *const f32,
            pnt2pixaabb.dptr as *const f32,
            img_shape.0,
            img_shape.1,
            tile_size,
            tile2idx.dptr as *mut u32,
            idx2pnt.dptr as *mut u32,
            num_pairs,
            std::ptr::null_mut(),
            ws.dptr as *mut std::ffi::c_void,
            ws_bytes,
        )
    };
    check(rc, "tile2idx_idx2pnt")?;
    Ok((tile2idx, idx2pnt))
}
