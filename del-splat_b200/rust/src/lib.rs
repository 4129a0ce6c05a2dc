//! del-splat-cudarc's launch wrappers (`splat_gauss`, `splat_circle`) over
//! the C ABI of libdsplat.so (`include/dsplat.h`, bound in [`ffi`]).
//!
//! The functions keep the reference's signatures (del-splat-cudarc/src/
//! splat_gauss.rs, splat_circle.rs): `CUstream` first, `&CuVec<_>` buffers,
//! `anyhow::Result`.  Buffers that the reference allocates inside
//! `tile2idx_idx2pnt` are allocated here with `CuVec::alloc_zeros` as well,
//! after one count call that synchronises the stream, as the reference's
//! read of the pair total does.
pub mod ffi;
#[cfg(feature = "cuda")]
pub mod splat_circle;
#[cfg(feature = "cuda")]
pub mod splat_gauss;

/// Turns a dsplat status code into an `anyhow::Error` carrying
/// `dsplat_last_error()`.
pub fn check(code: i32, what: &str) -> anyhow::Result<()> {
    if code == ffi::DSPLAT_OK {
        return Ok(());
    }
    let msg = unsafe { std::ffi::CStr::from_ptr(ffi::dsplat_last_error()) };
    Err(anyhow::anyhow!("{}: dsplat error {} ({})", what, code, msg.to_string_lossy()))
}
