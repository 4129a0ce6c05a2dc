"""Functions of the reference's PyO3 extension module (del-splat-dlpack/src),
same names and arguments, backed by libdsplat.so.

Arguments arrive as DLPack capsules (or tensors) exported on ``stream_ptr``.
Outputs are preallocated by the caller and written in place.  Device
dispatch: CUDA -> libdsplat.so; CPU tensors raise NotImplementedError (this
package has no CPU path; the reference ran del-splat-cpu there).  Shape and
dtype checks raise ValueError/TypeError where the reference panicked.
"""
from __future__ import annotations

import ctypes

import torch

from dsplat import _native as N
from dsplat import ply as _ply


def _t(x) -> torch.Tensor:
    return x if isinstance(x, torch.Tensor) else torch.from_dlpack(x)


def _check(t: torch.Tensor, name: str, shape, device):
    if t.dtype != torch.float32:
        raise TypeError(f"{name}: expected float32, got {t.dtype}")
    if t.device != device:
        raise ValueError(f"{name}: on {t.device}, expected {device}")
    if len(shape) != t.dim() or any(s != -1 and s != d for s, d in zip(shape, t.shape)):
        raise ValueError(f"{name}: expected shape {tuple(shape)}, got {tuple(t.shape)}")
    if not t.is_contiguous():
        raise ValueError(f"{name}: expected a contiguous tensor")


def _cuda_only(device: torch.device, fn: str):
    if device.type != "cuda":
        raise NotImplementedError(f"{fn}: del-splat-b200 implements the CUDA branch only (device {device})")


def points_load_ply(path: str):
    """del-splat-dlpack/src/points.rs:11-20 -> (pnt2xyz capsule [N,3], pnt2rgb capsule [N,3]) on the CPU."""
    xyz, rgb = _ply.read_xyzrgb(path)
    return torch.from_numpy(xyz).__dlpack__(), torch.from_numpy(rgb).__dlpack__()


def circle_splat_from_project_spheres(pnt2xyz, radius, transform_world2ndc, img_shape, pnt2pixxyndcz, pnt2pixrad,
                                      stream_ptr=0):
    """del-splat-dlpack/src/splat_circle.rs:11-75 (its GPU arm looked up a nonexistent
    `splat_sphere` fatbin; here it runs the circle projection kernel)."""
    pnt2xyz, transform_world2ndc = _t(pnt2xyz), _t(transform_world2ndc)
    pnt2pixxyndcz, pnt2pixrad = _t(pnt2pixxyndcz), _t(pnt2pixrad)
    dev = pnt2xyz.device
    n = pnt2xyz.shape[0]
    _check(pnt2xyz, "pnt2xyz", (n, 3), dev)
    _check(transform_world2ndc, "transform_world2ndc", (16,), dev)
    _check(pnt2pixxyndcz, "pnt2pixxyndcz", (n, 3), dev)
    _check(pnt2pixrad, "pnt2pixrad", (n,), dev)
    _cuda_only(dev, "circle_splat_from_project_spheres")
    N.check(N.lib().dsplat_circle_pnt2splat3_to_pnt2splat2(
        int(stream_ptr), n, pnt2xyz.data_ptr(), pnt2pixxyndcz.data_ptr(), pnt2pixrad.data_ptr(),
        transform_world2ndc.data_ptr(), int(img_shape[0]), int(img_shape[1]), float(radius)),
        "circle_splat_from_project_spheres")


def point_splat_rasterize_pix(pnt2pixxyndcz, pnt2rgb, pix2rgb, stream_ptr=0):
    """del-splat-dlpack/src/splat_point.rs:12-43 (the reference's GPU arm was todo!())."""
    pnt2pixxyndcz, pnt2rgb, pix2rgb = _t(pnt2pixxyndcz), _t(pnt2rgb), _t(pix2rgb)
    dev = pnt2pixxyndcz.device
    n = pnt2pixxyndcz.shape[0]
    _check(pnt2pixxyndcz, "pnt2pixxyndcz", (n, 3), dev)
    _check(pnt2rgb, "pnt2rgb", (n, 3), dev)
    _check(pix2rgb, "pix2rgb", (-1, -1, 3), dev)
    _cuda_only(dev, "point_splat_rasterize_pix")
    h, w = pix2rgb.shape[0], pix2rgb.shape[1]
    zbuf = torch.empty(max(1, w * h), dtype=torch.int64, device=dev)
    N.check(N.lib().dsplat_point_rasterize_pix(int(stream_ptr), n, pnt2pixxyndcz.data_ptr(), pnt2rgb.data_ptr(),
                                               pix2rgb.data_ptr(), w, h, zbuf.data_ptr()),
            "point_splat_rasterize_pix")


def point_splat_rasterize_pix_zbuffer(pnt2pixxyndcz, pnt2rgb, pix2rgb, pix2unitdepth, stream_ptr=0):
    """del-splat-dlpack/src/splat_point.rs:47-106: nearest point per pixel; pix2unitdepth gets
    1-(ndc_z+1)/2 of the winner or FLT_MAX."""
    pnt2pixxyndcz, pnt2rgb = _t(pnt2pixxyndcz), _t(pnt2rgb)
    pix2rgb, pix2unitdepth = _t(pix2rgb), _t(pix2unitdepth)
    dev = pnt2pixxyndcz.device
    n = pnt2pixxyndcz.shape[0]
    h, w = pix2rgb.shape[0], pix2rgb.shape[1]
    _check(pnt2pixxyndcz, "pnt2pixxyndcz", (n, 3), dev)
    _check(pnt2rgb, "pnt2rgb", (n, 3), dev)
    _check(pix2rgb, "pix2rgb", (h, w, 3), dev)
    _check(pix2unitdepth, "pix2unitdepth", (h, w), dev)
    _cuda_only(dev, "point_splat_rasterize_pix_zbuffer")
    zbuf = torch.empty(max(1, w * h), dtype=torch.int64, device=dev)
    N.check(N.lib().dsplat_point_rasterize_pix_zbuffer(
        int(stream_ptr), n, pnt2pixxyndcz.data_ptr(), pnt2rgb.data_ptr(), pix2rgb.data_ptr(),
        pix2unitdepth.data_ptr(), None, w, h, zbuf.data_ptr()), "point_splat_rasterize_pix_zbuffer")
