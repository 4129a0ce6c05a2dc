//! del-splat-cudarc/src/splat_circle.rs, over libdsplat.so.
use crate::{check, ffi};
use del_cudarc_sys::{cu, cu::CUstream, CuVec};

fn st(stream: CUstream) -> ffi::dsplat_stream {
    stream as ffi::dsplat_stream
}

/// splat_circle.rs:3-94: tile lists of circles (box = centre +- radius) on a
/// tile grid of tile_shape, 16-pixel tiles as in the reference.
pub fn tile2idx_idx2pnt(
    stream: CUstream,
    tile_shape: (u32, u32),
    pnt2pixxydepth: &CuVec<f32>,
    pnt2pixrad: &CuVec<f32>,
) -> anyhow::Result<(CuVec<u32>, CuVec<u32>)> {
    const TILE_SIZE: u32 = 16;
    let num_pnt = (pnt2pixxydepth.n / 3) as u32;
    let ws_bytes = unsafe { ffi::dsplat_tile2idx_workspace_size(num_pnt, tile_shape.0, tile_shape.1, 0) };
    let ws = CuVec::<u8>::alloc_zeros(ws_bytes.max(1), stream).unwrap();
    let mut num_pairs = 0u64;
    let rc = unsafe {
        ffi::dsplat_circle_tile2idx_count(
            st(stream),
            num_pnt,
            pnt2pixxydepth.dptr as *const f32,
            pnt2pixrad.dptr as *const f32,
            tile_shape.0,
            tile_shape.1,
            TILE_SIZE,
            ws.dptr as *mut std::ffi::c_void,
            ws_bytes,
            &mut num_pairs,
        )
    };
    check(rc, "circle tile2idx_count")?;
    let ws_bytes = unsafe { ffi::dsplat_tile2idx_workspace_size(num_pnt, tile_shape.0, tile_shape.1, num_pairs) };
    let ws = CuVec::<u8>::alloc_zeros(ws_bytes.max(1), stream).unwrap();
    let tile2idx = CuVec::<u32>::alloc_zeros((tile_shape.0 * tile_shape.1) as usize + 1, stream).unwrap();
    let idx2pnt = CuVec::<u32>::alloc_zeros((num_pairs as usize).max(1), stream).unwrap();
    let rc = unsafe {
        ffi::dsplat_circle_tile2idx_idx2pnt(
            st(stream),
            num_pnt,
            pnt2pixxydepth.dptr as *const f32,
            pnt2pixrad.dptr as *const f32,
            tile_shape.0,
            tile_shape.1,
            TILE_SIZE,
            tile2idx.dptr as *mut u32,
            idx2pnt.dptr as *mut u32,
            num_pairs,
            std::ptr::null_mut(),
            ws.dptr as *mut std::ffi::c_void,
            ws_bytes,
        )
    };
    check(rc, "circle tile2idx_idx2pnt")?;
    Ok((tile2idx, idx2pnt))
}

/// splat_circle.rs:96-132: circle centre (pixel x, y, ndc z) and pixel
/// radius of a world-space sphere of the given radius.
pub fn pnt2splat3_to_pnt2splat2(
    stream: cu::CUstream,
    pnt2xyz: &CuVec<f32>,
    pnt2pixxydepth: &CuVec<f32>,
    pnt2pixrad: &CuVec<f32>,
    transform_world2ndc: &CuVec<f32>,
    img_shape: (u32, u32),
    radius: f32,
) -> anyhow::Result<()> {
    let num_pnt = (pnt2xyz.n / 3) as u32;
    let rc = unsafe {
        ffi::dsplat_circle_pnt2splat3_to_pnt2splat2(
            st(stream),
            num_pnt,
            pnt2xyz.dptr as *const f32,
            pnt2pixxydepth.dptr as *mut f32,
            pnt2pixrad.dptr as *mut f32,
            transform_world2ndc.dptr as *const f32,
            img_shape.0,
            img_shape.1,
            radius,
        )
    };
    check(rc, "circle pnt2splat3_to_pnt2splat2")
}

/// splat_circle.rs:134-177: painter over the tile lists (the nearest
/// covering circle's colour per pixel).
#[allow(clippy::too_many_arguments)]
pub fn splat(
    stream: CUstream,
    img_shape: (u32, u32),
    pix2rgb_dev: &CuVec<f32>,
    pnt2pixxydepth_dev: &CuVec<f32>,
    pnt2pixrad_dev: &CuVec<f32>,
    pnt2rgb: &CuVec<f32>,
    tile_size: u32,
    tile2idx_dev: &CuVec<u32>,
    idx2pnt_dev: &CuVec<u32>,
) -> anyhow::Result<()> {
    let rc = unsafe {
        ffi::dsplat_circle_splat(
            st(stream),
            img_shape.0,
            img_shape.1,
            pix2rgb_dev.dptr as *mut f32,
            pnt2pixxydepth_dev.dptr as *const f32,
            pnt2pixrad_dev.dptr as *const f32,
            pnt2rgb.dptr as *const f32,
            tile_size,
            tile2idx_dev.dptr as *const u32,
            idx2pnt_dev.dptr as *const u32,
        )
    };
    check(rc, "circle splat")
}
