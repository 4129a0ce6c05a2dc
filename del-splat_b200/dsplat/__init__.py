"""dsplat -- host side of the B200 splatting library (libdsplat.so).

Modules:
  _native  ctypes binding of the C ABI (include/dsplat.h)
  cudarc   mirror of del-splat-cudarc's launch wrappers over torch tensors
  gauss    batched, differentiable Gaussian rendering (GaussBatch, render)
  scenes   cameras and seeded synthetic scenes
  ply      PLY readers (del-splat-cpu/src/io_ply.rs)
"""
from . import scenes  # noqa: F401

__all__ = ["scenes"]
