"""Gaussian splatting with torch tensors.

* ``project`` / ``tile2idx_idx2pnt`` / ``rasterize``: the reference's
  Gaussian path (del-splat-cudarc/src/splat_gauss.rs) as torch functions.
* ``render``: differentiable, batched over cameras (torch.autograd).
"""
from typing import List, Sequence

import torch

from dsplat import cudarc
from dsplat.gauss import GaussBatch, render as _render
from dsplat.scenes import Camera


def project(pnt2xyz, pnt2scale, pnt2quat, transform_world2ndc, img_shape):
    """splat_gauss.rs:6-44 -> (pnt2pixxydepth [N,3], pnt2pixconvinv [N,3], pnt2pixaabb [N,4]).
    transform_world2ndc: 16 floats, column-major."""
    n = pnt2xyz.shape[0]
    dev = pnt2xyz.device
    xyd = torch.empty((n, 3), dtype=torch.float32, device=dev)
    conic = torch.empty((n, 3), dtype=torch.float32, device=dev)
    aabb = torch.empty((n, 4), dtype=torch.float32, device=dev)
    cudarc.splat_gauss_pnt2splat3_to_pnt2splat2(None, pnt2xyz.contiguous(), pnt2scale.contiguous(),
                                                pnt2quat.contiguous(), xyd, conic, aabb,
                                                transform_world2ndc.contiguous().reshape(16), img_shape)
    return xyd, conic, aabb


def tile2idx_idx2pnt(img_shape, tile_size, pnt2pixxydepth, pnt2pixaabb):
    """splat_gauss.rs:96-195 -> (tile2idx [T+1], idx2pnt [P]) int32."""
    return cudarc.splat_gauss_tile2idx_idx2pnt(None, img_shape, tile_size, pnt2pixxydepth, pnt2pixaabb)


def rasterize(img_shape, pnt2pixxydepth, pnt2pixconvinv, pnt2pixaabb, pnt2opacity, pnt2rgb, tile_size, tile2idx,
              idx2pnt):
    """splat_gauss.rs:46-94 -> pix2rgb [H,W,3] (black background)."""
    w, h = img_shape
    pix2rgb = torch.zeros((h, w, 3), dtype=torch.float32, device=pnt2pixxydepth.device)
    cudarc.splat_gauss_rasterize_pnt2splat2(None, img_shape, pix2rgb, pnt2pixxydepth, pnt2pixconvinv, pnt2pixaabb,
                                            pnt2opacity, pnt2rgb, tile_size, tile2idx, idx2pnt)
    return pix2rgb


def make_batch(num_pnt: int, cameras: Sequence[Camera], tile_size: int = 16, sh_degree: int = 3,
               pair_capacity: int = 1 << 20) -> GaussBatch:
    return GaussBatch(num_pnt, cameras, tile_size, sh_degree, pair_capacity)


def render(means, log_scales, quats, opacity, colors, batch: GaussBatch) -> List[torch.Tensor]:
    """Differentiable render of every camera of ``batch`` (list of [H,W,3])."""
    return _render(means, log_scales, quats, opacity, colors, batch)
