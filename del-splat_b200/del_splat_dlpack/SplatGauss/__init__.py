"""Gaussian splatting entry points (new in this package; the reference exposes
its Gaussian path only through the Rust del-splat-cudarc crate)."""
