"""Python mirror of del-splat-cudarc's launch wrappers, over torch CUDA tensors.

Same function names, argument order and meaning as the reference's Rust L2
API (``CuVec`` -> contiguous CUDA tensor, ``CUstream`` -> stream handle as an
int, or None for torch's current stream):

* splat_gauss.rs:6-44    ``splat_gauss_pnt2splat3_to_pnt2splat2``
* splat_gauss.rs:96-195  ``splat_gauss_tile2idx_idx2pnt`` (allocates and
  returns (tile2idx, idx2pnt) like the reference; synchronises once to read
  the pair count, as the reference does at splat_gauss.rs:147)
* splat_gauss.rs:46-94   ``splat_gauss_rasterize_pnt2splat2`` (adds into pix2rgb)
* splat_circle.rs:96-132 ``splat_circle_pnt2splat3_to_pnt2splat2``
* splat_circle.rs:3-94   ``splat_circle_tile2idx_idx2pnt``
* splat_circle.rs:134-177 ``splat_circle_splat``

Errors raise ``RuntimeError`` (the reference returns anyhow::Result and
panics inside on launch failures).
"""
from __future__ import annotations

import ctypes
from typing import Optional, Tuple

import torch

from . import _native as N


def _st(stream: Optional[int], dev: torch.device) -> int:
    return int(stream) if stream is not None else torch.cuda.current_stream(dev).cuda_stream


def _chk(t: torch.Tensor, name: str, numel: Optional[int] = None, dtype=torch.float32) -> int:
    if not isinstance(t, torch.Tensor) or not t.is_cuda:
        raise RuntimeError(f"{name}: expected a CUDA tensor (del-splat-b200 has no CPU path)")
    if t.dtype != dtype:
        raise TypeError(f"{name}: expected {dtype}, got {t.dtype}")
    if not t.is_contiguous():
        raise ValueError(f"{name}: expected a contiguous tensor")
    if numel is not None and t.numel() != numel:
        raise ValueError(f"{name}: expected {numel} elements, got {t.numel()}")
    return t.data_ptr()


def tile_shape(img_shape: Tuple[int, int], tile_size: int) -> Tuple[int, int]:
    return ((img_shape[0] + tile_size - 1) // tile_size, (img_shape[1] + tile_size - 1) // tile_size)


def splat_gauss_pnt2splat3_to_pnt2splat2(stream, pnt2xyz, pnt2scale, pnt2quat, pnt2pixxydepth, pnt2pixconvinv,
                                         pnt2pixaabb, transform_world2ndc, img_shape) -> None:
    n = pnt2xyz.numel() // 3
    args = [_chk(pnt2xyz, "pnt2xyz", 3 * n), _chk(pnt2scale, "pnt2scale", 3 * n), _chk(pnt2quat, "pnt2quat", 4 * n),
            _chk(pnt2pixxydepth, "pnt2pixxydepth", 3 * n), _chk(pnt2pixconvinv, "pnt2pixconvinv", 3 * n),
            _chk(pnt2pixaabb, "pnt2pixaabb", 4 * n), _chk(transform_world2ndc, "transform_world2ndc", 16)]
    N.check(N.lib().dsplat_gauss_pnt2splat3_to_pnt2splat2(
        _st(stream, pnt2xyz.device), n, args[0], args[1], args[2], args[3], args[4], args[5], args[6],
        int(img_shape[0]), int(img_shape[1])), "pnt2splat3_to_pnt2splat2")


def _tile_lists(stream, count_fn, fill_fn, n, dev, pre_args, tw, th, ts, with_keys):
    L = N.lib()
    st = _st(stream, dev)
    ws_bytes = L.dsplat_tile2idx_workspace_size(n, tw, th, 0)
    ws = torch.empty(max(1, ws_bytes), dtype=torch.uint8, device=dev)
    num = N.c_u64(0)
    N.check(count_fn(st, n, *pre_args["count"], tw, th, ts, ws.data_ptr(), ws.numel(), ctypes.byref(num)),
            "tile2idx_count")
    P = int(num.value)
    ws_bytes = L.dsplat_tile2idx_workspace_size(n, tw, th, P)
    if ws_bytes > ws.numel():
        ws = torch.empty(ws_bytes, dtype=torch.uint8, device=dev)
    tile2idx = torch.empty(tw * th + 1, dtype=torch.int32, device=dev)
    idx2pnt = torch.empty(max(P, 1), dtype=torch.int32, device=dev)
    keys = torch.empty(max(P, 1), dtype=torch.int64, device=dev) if with_keys else None
    N.check(fill_fn(st, n, *pre_args["fill"], tw, th, ts, tile2idx.data_ptr(), idx2pnt.data_ptr(), P,
                    keys.data_ptr() if keys is not None else None, ws.data_ptr(), ws.numel()), "tile2idx_idx2pnt")
    idx2pnt = idx2pnt[:P]
    if keys is not None:
        return tile2idx, idx2pnt, keys[:P]
    return tile2idx, idx2pnt


def splat_gauss_tile2idx_idx2pnt(stream, img_shape, tile_size, pnt2pixxydepth, pnt2pixaabb, with_keys=False):
    """Returns (tile2idx [T+1], idx2pnt [P]) as int32 tensors (u32 bit patterns);
    with_keys=True also returns the sorted u64 keys (tile << 32 | depth bits)."""
    n = pnt2pixxydepth.numel() // 3
    xyd = _chk(pnt2pixxydepth, "pnt2pixxydepth", 3 * n)
    aabb = _chk(pnt2pixaabb, "pnt2pixaabb", 4 * n)
    tw, th = tile_shape(img_shape, tile_size)
    L = N.lib()

    def count_fn(st, n_, aabb_, tw_, th_, ts_, ws, wsb, num):
        return L.dsplat_gauss_tile2idx_count(st, n_, aabb_, int(img_shape[0]), int(img_shape[1]), ts_, ws, wsb, num)

    def fill_fn(st, n_, xyd_, aabb_, tw_, th_, ts_, t2i, i2p, cap, keys, ws, wsb):
        return L.dsplat_gauss_tile2idx_idx2pnt(st, n_, xyd_, aabb_, int(img_shape[0]), int(img_shape[1]), ts_, t2i,
                                               i2p, cap, keys, ws, wsb)

    return _tile_lists(stream, count_fn, fill_fn, n, pnt2pixxydepth.device,
                       {"count": [aabb], "fill": [xyd, aabb]}, tw, th, int(tile_size), with_keys)


def splat_gauss_rasterize_pnt2splat2(stream, img_shape, pix2rgb, pnt2pixxydepth, pnt2pixconvinv, pnt2pixaabb,
                                     pnt2opacity, pnt2rgb, tile_size, tile2idx, idx2pnt, pix2transmit=None,
                                     pix2stop=None, stop_rule: int = N.STOP_CPU) -> None:
    """Adds the tiled front-to-back blend into pix2rgb.  stop_rule: N.STOP_CPU
    (del-splat-cpu, alpha_sum > 0.999f, the default) or N.STOP_CUDA (the
    reference CUDA kernel's double comparison)."""
    n = pnt2pixxydepth.numel() // 3
    w, h = int(img_shape[0]), int(img_shape[1])
    tw, th = tile_shape(img_shape, tile_size)
    if tile2idx.numel() != tw * th + 1:
        raise ValueError(f"tile2idx: expected {tw * th + 1} entries, got {tile2idx.numel()}")
    N.check(N.lib().dsplat_gauss_rasterize_pnt2splat2_stop(
        _st(stream, pix2rgb.device), w, h, _chk(pix2rgb, "pix2rgb", w * h * 3),
        _chk(pnt2pixxydepth, "pnt2pixxydepth", 3 * n), _chk(pnt2pixconvinv, "pnt2pixconvinv", 3 * n),
        _chk(pnt2pixaabb, "pnt2pixaabb", 4 * n), _chk(pnt2opacity, "pnt2opacity", n), _chk(pnt2rgb, "pnt2rgb", 3 * n),
        int(tile_size), _chk(tile2idx, "tile2idx", dtype=tile2idx.dtype), _chk(idx2pnt, "idx2pnt", dtype=idx2pnt.dtype),
        _chk(pix2transmit, "pix2transmit", w * h) if pix2transmit is not None else None,
        _chk(pix2stop, "pix2stop", w * h, dtype=pix2stop.dtype) if pix2stop is not None else None, int(stop_rule)),
        "rasterize_pnt2splat2")


def expf_cr(x: torch.Tensor, stream=None) -> torch.Tensor:
    """The blend's exponential: e^x correctly rounded to float32, elementwise."""
    y = torch.empty_like(x)
    N.check(N.lib().dsplat_expf_cr(_st(stream, x.device), x.numel(), _chk(x, "x"), y.data_ptr()), "expf_cr")
    return y


def splat_circle_pnt2splat3_to_pnt2splat2(stream, pnt2xyz, pnt2pixxydepth, pnt2pixrad, transform_world2ndc,
                                          img_shape, radius: float) -> None:
    n = pnt2xyz.numel() // 3
    N.check(N.lib().dsplat_circle_pnt2splat3_to_pnt2splat2(
        _st(stream, pnt2xyz.device), n, _chk(pnt2xyz, "pnt2xyz", 3 * n), _chk(pnt2pixxydepth, "pnt2pixxydepth", 3 * n),
        _chk(pnt2pixrad, "pnt2pixrad", n), _chk(transform_world2ndc, "transform_world2ndc", 16),
        int(img_shape[0]), int(img_shape[1]), float(radius)), "circle pnt2splat3_to_pnt2splat2")


def splat_circle_tile2idx_idx2pnt(stream, tile_shape_, pnt2pixxydepth, pnt2pixrad, tile_size=16, with_keys=False):
    """splat_circle.rs:3-94 (tile size 16 as the reference hard-codes it)."""
    n = pnt2pixxydepth.numel() // 3
    xyd = _chk(pnt2pixxydepth, "pnt2pixxydepth", 3 * n)
    rad = _chk(pnt2pixrad, "pnt2pixrad", n)
    tw, th = int(tile_shape_[0]), int(tile_shape_[1])
    L = N.lib()
    return _tile_lists(stream, L.dsplat_circle_tile2idx_count, L.dsplat_circle_tile2idx_idx2pnt, n,
                       pnt2pixxydepth.device, {"count": [xyd, rad], "fill": [xyd, rad]}, tw, th, int(tile_size),
                       with_keys)


def splat_circle_splat(stream, img_shape, pix2rgb, pnt2pixxydepth, pnt2pixrad, pnt2rgb, tile_size, tile2idx,
                       idx2pnt) -> None:
    n = pnt2pixxydepth.numel() // 3
    w, h = int(img_shape[0]), int(img_shape[1])
    N.check(N.lib().dsplat_circle_splat(
        _st(stream, pix2rgb.device), w, h, _chk(pix2rgb, "pix2rgb", w * h * 3),
        _chk(pnt2pixxydepth, "pnt2pixxydepth", 3 * n), _chk(pnt2pixrad, "pnt2pixrad", n),
        _chk(pnt2rgb, "pnt2rgb", 3 * n), int(tile_size), _chk(tile2idx, "tile2idx", dtype=tile2idx.dtype),
        _chk(idx2pnt, "idx2pnt", dtype=idx2pnt.dtype)), "circle splat")


def circle_splat_zbuffer(stream, img_shape, pnt2pixxydepth, pnt2pixrad, colors, tile_size=16, want_winner=False):
    """Circle splat through the packed 64-bit z-buffer.  colors: float [N,3] -> image [H,W,3] float, or
    int32/uint32-bit [N] RGBA -> image [H,W] int32 (u32 bit patterns)."""
    n = pnt2pixxydepth.numel() // 3
    w, h = int(img_shape[0]), int(img_shape[1])
    dev = pnt2pixxydepth.device
    if colors.dtype == torch.float32:
        kind = 0
        pix = torch.zeros((h, w, 3), dtype=torch.float32, device=dev)
        cptr = _chk(colors, "colors", 3 * n)
    else:
        kind = 1
        pix = torch.zeros((h, w), dtype=torch.int32, device=dev)
        cptr = _chk(colors, "colors", n, dtype=colors.dtype)
    zbuf = torch.empty(w * h, dtype=torch.int64, device=dev)
    win = torch.empty((h, w), dtype=torch.int32, device=dev) if want_winner else None
    N.check(N.lib().dsplat_circle_splat_zbuffer(
        _st(stream, dev), n, _chk(pnt2pixxydepth, "pnt2pixxydepth", 3 * n), _chk(pnt2pixrad, "pnt2pixrad", n), cptr,
        kind, pix.data_ptr(), win.data_ptr() if win is not None else None, w, h, int(tile_size), zbuf.data_ptr()),
        "circle zbuffer")
    return (pix, win) if want_winner else pix
