import torch

from .. import util_torch


def from_project_spheres(
        pnt2xyz: torch.Tensor,
        radius: float,
        transform_world2ndc: torch.Tensor,
        img_shape):
    """del_splat_dlpack/SplatCircle/torch.py:6-40: (pnt2pixxyndcz [N,3], pnt2pixrad [N]).
    transform_world2ndc is a row-major 4x4 tensor, transposed to column-major here."""
    device = pnt2xyz.device
    num_pnt = pnt2xyz.shape[0]
    assert transform_world2ndc.device == device
    assert transform_world2ndc.shape == (4, 4)
    assert transform_world2ndc.dtype == torch.float32
    pnt2pixxyndcz = torch.empty((num_pnt, 3), device=device, dtype=torch.float32)
    pnt2pixrad = torch.empty((num_pnt,), device=device, dtype=torch.float32)
    transform_world2ndc = transform_world2ndc.transpose(0, 1).flatten()
    stream_ptr = 0
    if device.type == "cuda":
        torch.cuda.set_device(device)
        stream_ptr = torch.cuda.current_stream(device).cuda_stream
    from .. import SplatCircle

    SplatCircle.from_project_spheres(
        util_torch.to_dlpack_safe(pnt2xyz, stream_ptr),
        radius,
        util_torch.to_dlpack_safe(transform_world2ndc, stream_ptr),
        img_shape,
        util_torch.to_dlpack_safe(pnt2pixxyndcz, stream_ptr),
        util_torch.to_dlpack_safe(pnt2pixrad, stream_ptr),
        stream_ptr)
    return pnt2pixxyndcz, pnt2pixrad


def splat_zbuffer(pnt2pixxyndcz: torch.Tensor, pnt2pixrad: torch.Tensor, colors: torch.Tensor, img_shape,
                  tile_size: int = 16):
    """Circle splat with the packed depth|index z-buffer (no tile lists).  colors float [N,3]
    -> [H,W,3] float image; int32 RGBA [N] -> [H,W] int32 image.  Uncovered pixels are 0."""
    from dsplat import cudarc
    return cudarc.circle_splat_zbuffer(None, img_shape, pnt2pixxyndcz.contiguous(), pnt2pixrad.contiguous(),
                                       colors.contiguous(), tile_size)
