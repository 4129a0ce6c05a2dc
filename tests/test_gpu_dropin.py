"""Parity of the reference-facing entry points (del-splat-cudarc / dlpack API)
against the CPU oracle and the reference-generated fixtures.
Bar: bit-exact for projections, tile lists, keys, permutations, stop
positions and z-buffer winners; images max-abs <= 1e-4 (observed: exact)."""
import os

import numpy as np
import pytest
import torch

from dsplat import cudarc, scenes
from gpu_util import F, T, U32

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(__file__), "golden")
IMG_TOL = 1e-4


def _project(orc, dev, sc, w, h):
    cam = sc.cameras[0]
    n = sc.n
    xyd, conic, aabb = (torch.empty((n, k), device=dev) for k in (3, 3, 4))
    cudarc.splat_gauss_pnt2splat3_to_pnt2splat2(None, T(sc.means, dev), T(sc.scales, dev), T(sc.quats, dev), xyd,
                                                conic, aabb, T(cam.mvp, dev), (w, h))
    return xyd, conic, aabb


@pytest.mark.parametrize("size", [(256, 256), (250, 130), (1, 1)])
def test_gauss_projection_bitexact(orc, dev, size):
    sc = scenes.config0(n=16384, size=size)
    xyd, conic, aabb = _project(orc, dev, sc, *size)
    o = orc.gauss_project(sc.means, sc.quats, sc.scales, sc.cameras[0].mvp, *size)
    for g, c in zip((xyd, conic, aabb), o):
        assert np.array_equal(F(g).view(np.uint32), c.view(np.uint32))


def test_circle_projection_bitexact(orc, dev):
    pts = scenes.config1(n=50000, size=(320, 200))
    n = pts.xyz.shape[0]
    xyd = torch.empty((n, 3), device=dev)
    rad = torch.empty((n,), device=dev)
    cudarc.splat_circle_pnt2splat3_to_pnt2splat2(None, T(pts.xyz, dev), xyd, rad, T(pts.camera.mvp, dev),
                                                 (320, 200), 0.01)
    oxyd, orad = orc.circle_project(pts.xyz, pts.camera.mvp, 320, 200, 0.01)
    assert np.array_equal(F(xyd).view(np.uint32), oxyd.view(np.uint32))
    assert np.array_equal(F(rad).view(np.uint32), orad.view(np.uint32))


@pytest.mark.parametrize("ts,size", [(16, (256, 256)), (8, (256, 256)), (32, (256, 256)), (16, (250, 130))])
def test_gauss_tile_lists_bitexact(orc, dev, ts, size):
    sc = scenes.config0(n=16384, size=size)
    xyd, conic, aabb = _project(orc, dev, sc, *size)
    t2i, i2p, keys = cudarc.splat_gauss_tile2idx_idx2pnt(None, size, ts, xyd, aabb, with_keys=True)
    o_t, o_i, o_k = orc.tile2pnt(F(xyd), F(aabb), size[0], size[1], ts)
    assert np.array_equal(U32(t2i), o_t)
    assert np.array_equal(U32(i2p), o_i)
    assert np.array_equal(F(keys).view(np.uint64), o_k)


@pytest.mark.parametrize("name", ["tiles_gauss_small.npz", "tiles_circle_small.npz"])
def test_tile_lists_match_reference_fixtures(dev, name):
    d = np.load(os.path.join(GOLD, name))
    w, h, ts = (int(x) for x in d["shape"])
    t2i, i2p, keys = cudarc.splat_gauss_tile2idx_idx2pnt(None, (w, h), ts, T(d["xyd"], dev), T(d["aabb"], dev),
                                                         with_keys=True)
    assert np.array_equal(U32(t2i), d["tile2idx"])
    assert np.array_equal(U32(i2p), d["idx2pnt"])
    assert np.array_equal(F(keys).view(np.uint64), d["keys"])
    if "rad" in d:
        tw, th = (w + ts - 1) // ts, (h + ts - 1) // ts
        c2i, c_i2p, c_keys = cudarc.splat_circle_tile2idx_idx2pnt(None, (tw, th), T(d["xyd"], dev),
                                                                  T(d["rad"], dev), ts, with_keys=True)
        assert np.array_equal(U32(c2i), d["tile2idx"])
        assert np.array_equal(U32(c_i2p), d["idx2pnt"])
        assert np.array_equal(F(c_keys).view(np.uint64), d["keys"])


def test_tile_lists_edge_cases(orc, dev):
    # empty input
    e = torch.empty((0, 3), device=dev)
    t2i, i2p = cudarc.splat_gauss_tile2idx_idx2pnt(None, (64, 32), 16, e, torch.empty((0, 4), device=dev))
    assert U32(t2i).tolist() == [0] * 9 and i2p.numel() == 0
    # everything off screen, huge boxes, exact depth ties, NaN-free degenerate zero-size boxes
    rng = np.random.default_rng(5)
    n = 4000
    xyd = np.stack([rng.uniform(-300, 400, n), rng.uniform(-300, 300, n), rng.uniform(-1.5, 1.5, n)], 1)
    xyd = xyd.astype(np.float32)
    xyd[::7, 2] = xyd[0, 2]                      # depth ties -> index order
    half = rng.uniform(0, 200, (n, 2)).astype(np.float32)
    half[::11] = 0.0                             # zero-size boxes
    aabb = np.concatenate([xyd[:, :2] - half, xyd[:, :2] + half], 1).astype(np.float32)
    for ts in (8, 16, 32):
        t2i, i2p, keys = cudarc.splat_gauss_tile2idx_idx2pnt(None, (200, 120), ts, T(xyd, dev), T(aabb, dev),
                                                             with_keys=True)
        o_t, o_i, o_k = orc.tile2pnt(xyd, aabb, 200, 120, ts)
        assert np.array_equal(U32(t2i), o_t) and np.array_equal(U32(i2p), o_i)
        assert np.array_equal(F(keys).view(np.uint64), o_k)


@pytest.mark.parametrize("ts", [8, 16, 32])
def test_gauss_raster_matches_oracle(orc, dev, ts):
    size = (256, 256)
    sc = scenes.config0(n=16384, size=size)
    xyd, conic, aabb = _project(orc, dev, sc, *size)
    t2i, i2p = cudarc.splat_gauss_tile2idx_idx2pnt(None, size, ts, xyd, aabb)
    img = torch.zeros((256, 256, 3), device=dev)
    Tm = torch.empty((256, 256), device=dev)
    stop = torch.empty((256, 256), dtype=torch.int32, device=dev)
    cudarc.splat_gauss_rasterize_pnt2splat2(None, size, img, xyd, conic, aabb, T(sc.opacity, dev),
                                            T(sc.colors, dev), ts, t2i, i2p, Tm, stop)
    o_img, o_T, o_last = orc.gauss_rasterize_tiled(256, 256, ts, U32(t2i), U32(i2p), F(xyd), F(conic), F(aabb),
                                                   sc.opacity, sc.colors)
    assert np.abs(F(img) - o_img).max() <= IMG_TOL
    assert np.array_equal(F(img), o_img)          # same IEEE ops, same order
    assert np.array_equal(F(Tm), o_T)
    assert np.array_equal(F(stop), o_last)


def test_gauss_raster_accumulates_like_reference(orc, dev):
    size = (64, 48)
    sc = scenes.config0(n=2000, size=size)
    xyd, conic, aabb = _project(orc, dev, sc, *size)
    t2i, i2p = cudarc.splat_gauss_tile2idx_idx2pnt(None, size, 16, xyd, aabb)
    base = torch.full((48, 64, 3), 0.25, device=dev)
    cudarc.splat_gauss_rasterize_pnt2splat2(None, size, base, xyd, conic, aabb, T(sc.opacity, dev),
                                            T(sc.colors, dev), 16, t2i, i2p)
    o_img, _, _ = orc.gauss_rasterize_tiled(64, 48, 16, U32(t2i), U32(i2p), F(xyd), F(conic), F(aabb),
                                            sc.opacity, sc.colors)
    assert np.abs(F(base) - (o_img + 0.25)).max() <= IMG_TOL


def test_circle_splat_tiles_and_zbuffer_bitexact(orc, dev):
    w, h = 300, 200
    pts = scenes.config1(n=60000, size=(w, h))
    n = pts.xyz.shape[0]
    xyd = torch.empty((n, 3), device=dev)
    rad = torch.empty((n,), device=dev)
    cudarc.splat_circle_pnt2splat3_to_pnt2splat2(None, T(pts.xyz, dev), xyd, rad, T(pts.camera.mvp, dev), (w, h),
                                                 0.01)
    rgb = torch.rand((n, 3), device=dev)
    tw, th = (w + 15) // 16, (h + 15) // 16
    t2i, i2p = cudarc.splat_circle_tile2idx_idx2pnt(None, (tw, th), xyd, rad)
    img = torch.zeros((h, w, 3), device=dev)
    cudarc.splat_circle_splat(None, (w, h), img, xyd, rad, rgb, 16, t2i, i2p)
    win = orc.circle_splat_tiled(w, h, 16, U32(t2i), U32(i2p), F(xyd), F(rad))
    exp = np.where((win >= 0)[..., None], F(rgb)[np.maximum(win, 0)], 0.0).astype(np.float32)
    assert np.array_equal(F(img), exp)
    zimg, zwin = cudarc.circle_splat_zbuffer(None, (w, h), xyd, rad, rgb, 16, want_winner=True)
    assert np.array_equal(F(zwin), win)
    assert np.array_equal(F(zimg), exp)


def test_point_zbuffer_matches_painter_and_reference(orc, dev):
    d = np.load(os.path.join(GOLD, "point_zbuffer_small.npz"))
    w, h = (int(x) for x in d["shape"])
    from del_splat_dlpack import del_splat_dlpack as L3
    pix = torch.zeros((h, w, 3), device=dev)
    depth = torch.empty((h, w), device=dev)
    L3.point_splat_rasterize_pix_zbuffer(T(d["xyd"], dev), T(d["rgb"], dev), pix, depth,
                                         torch.cuda.current_stream().cuda_stream)
    assert np.array_equal(F(depth), d["depth"])          # reference splat_point.cu output
    hit = d["depth"] < np.finfo(np.float32).max
    assert np.array_equal(F(pix)[hit], d["rgb_out"][hit])
    win = orc.point_render_sort_depth(d["xyd"], w, h)
    assert np.array_equal(win >= 0, hit)


def _config1_zbuffer(orc, dev, n, size):
    """Config 1's circle z-buffer (u32 RGBA, pixel radius 1..4) on the GPU and
    the oracle's tiled painter (splat_circle.cu:93-132 order: the nearest
    covering point wins, ties to the larger index)."""
    w, h = size
    pts = scenes.config1(n=n, size=size)
    m = pts.xyz.shape[0]
    xyd = torch.empty((m, 3), device=dev)
    rad0 = torch.empty((m,), device=dev)
    cudarc.splat_circle_pnt2splat3_to_pnt2splat2(None, T(pts.xyz, dev), xyd, rad0, T(pts.camera.mvp, dev), size,
                                                 0.0)
    rad = T(pts.radius_px, dev)
    rgba = T(pts.rgba.view(np.int32), dev)
    pix, win = cudarc.circle_splat_zbuffer(None, size, xyd, rad, rgba, 16, want_winner=True)
    oxyd, _ = orc.circle_project(pts.xyz, pts.camera.mvp, w, h, 0.0)
    assert np.array_equal(F(xyd).view(np.uint32), oxyd.view(np.uint32))
    aabb = orc.circle_aabb(oxyd, pts.radius_px)
    t2i, i2p, _ = orc.tile2pnt(oxyd, aabb, w, h, 16, with_keys=False)
    o_win = orc.circle_splat_tiled(w, h, 16, t2i, i2p, oxyd, pts.radius_px)
    expect = np.where(o_win >= 0, pts.rgba[np.maximum(o_win, 0)], 0).astype(np.uint32)
    return F(pix).view(np.uint32), F(win), expect, o_win


def test_circle_zbuffer_u32_rgba_small(orc, dev):
    pix, win, expect, o_win = _config1_zbuffer(orc, dev, 40000, (160, 120))
    assert (o_win >= 0).sum() > 1000
    assert np.array_equal(win, o_win)
    assert np.array_equal(pix, expect)


def test_circle_zbuffer_config1_full_size(orc, dev):
    """Config 1 itself: 1,048,576 points, 1024x1024, radius 1..4 px, u32 RGBA;
    winners and pixels bit-exact."""
    pix, win, expect, o_win = _config1_zbuffer(orc, dev, 1 << 20, (1024, 1024))
    assert (o_win >= 0).mean() > 0.5
    assert np.array_equal(win, o_win)
    assert np.array_equal(pix, expect)
