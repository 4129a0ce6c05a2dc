"""The reference-facing entry points either side of the path, on the GPU:
del-splat-dlpack's circle projection and point rasteriser (module functions
and their torch wrappers), a render of the reference's own 3DGS capture
(a subset of asset/bulba.ply, tests/golden/bulba_subset.ply) and of views
read from a COLMAP model, each against the CPU oracle."""
import os

import numpy as np
import pytest
import torch

from dsplat import colmap, scenes
from dsplat.gauss import GaussBatch
from dsplat.render_ply import load_scene
from gpu_util import F, T, params_of
from test_host import _colmap_files

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(__file__), "golden")


def _check_batch_against_oracle(orc, sc, batch):
    for v, cam in enumerate(sc.cameras):
        xyd, conic, aabb, rgb = orc.fused_project(sc.means, sc.log_scales, sc.quats, sc.colors, sc.sh_degree,
                                                  cam.mvp, cam.campos, cam.width, cam.height)
        t2i, i2p, _ = orc.tile2pnt(xyd, aabb, cam.width, cam.height, 16, with_keys=False)
        o_img, o_T, _ = orc.gauss_rasterize_tiled(cam.width, cam.height, 16, t2i, i2p, xyd, conic, aabb,
                                                  sc.opacity, rgb, nthreads=8)
        assert len(i2p) > 0
        assert np.array_equal(F(batch.images()[v]), o_img)
        assert np.array_equal(F(batch.per_pixel("T")[v]), o_T)


def test_bulba_capture_eight_orbit_views(orc, dev):
    """io_ply.rs:128-227 conversions, then 8 orbit views at 640x480 in one
    batched forward: bit-exact against the oracle on every view."""
    cams = scenes.sphere_cameras(np.random.default_rng(7), 8, 3.0, [(640, 480)])
    sc = load_scene(os.path.join(GOLD, "bulba_subset.ply"), cams)
    batch = GaussBatch(sc.n, cams, 8, 3, pair_capacity=1 << 20, device=dev)
    batch.ensure_capacity(params_of(sc, dev))
    batch.forward(params_of(sc, dev))
    torch.cuda.synchronize()
    _check_batch_against_oracle(orc, sc, batch)


def test_colmap_views_render(orc, dev, tmp_path):
    """PINHOLE views of a COLMAP binary model (two cameras of different size)
    rendered in one batch."""
    d = _colmap_files(tmp_path)
    views = colmap.views_from_model(colmap.read_cameras(d / "cameras.bin"), colmap.read_images(d / "images.bin"),
                                    near=0.5, far=50.0)
    sc = scenes.config0(seed=31, n=8000, size=(64, 64))
    sc.cameras = views
    batch = GaussBatch(sc.n, views, 16, -1, pair_capacity=1 << 20, device=dev)
    batch.ensure_capacity(params_of(sc, dev))
    batch.forward(params_of(sc, dev))
    torch.cuda.synchronize()
    _check_batch_against_oracle(orc, sc, batch)


def test_circle_splat_from_project_spheres_and_torch_wrapper(orc, dev):
    """del-splat-dlpack/src/splat_circle.rs:11-75 (module function and
    SplatCircle.torch.from_project_spheres) against the oracle's projection."""
    from del_splat_dlpack import del_splat_dlpack
    from del_splat_dlpack.SplatCircle import torch as sct
    pts = scenes.config1(n=40000, size=(320, 240))
    n = pts.xyz.shape[0]
    mvp_col = pts.camera.mvp
    o_xyd, o_rad = orc.circle_project(pts.xyz, mvp_col, 320, 240, 0.015)
    xyd = torch.empty((n, 3), device=dev)
    rad = torch.empty((n,), device=dev)
    st = torch.cuda.current_stream().cuda_stream
    del_splat_dlpack.circle_splat_from_project_spheres(T(pts.xyz, dev), 0.015, T(mvp_col, dev), (320, 240), xyd, rad,
                                                       st)
    torch.cuda.synchronize()
    assert np.array_equal(F(xyd).view(np.uint32), o_xyd.view(np.uint32))
    assert np.array_equal(F(rad).view(np.uint32), o_rad.view(np.uint32))
    m_row = T(mvp_col.reshape(4, 4).T.copy(), dev)  # the torch wrapper takes the row-major 4x4
    xyd2, rad2 = sct.from_project_spheres(T(pts.xyz, dev), 0.015, m_row, (320, 240))
    torch.cuda.synchronize()
    assert torch.equal(xyd2, xyd) and torch.equal(rad2, rad)


def test_point_rasterize_pix_torch_wrapper(orc, dev):
    """SplatPoint.torch.rasterize_pix (the reference's GPU arm was todo!()):
    nearest point per pixel, as the oracle's render_pix_sort_depth painter
    (pnt2pixxyndcz.rs:1-40) picks it when no two points tie in depth."""
    from del_splat_dlpack.SplatPoint import torch as spt
    rng = np.random.default_rng(41)
    n, w, h = 30000, 120, 90
    xyd = np.stack([rng.uniform(0, w, n), rng.uniform(0, h, n), rng.uniform(-0.999, 0.999, n)], 1).astype(np.float32)
    rgb = rng.uniform(0, 1, (n, 3)).astype(np.float32)
    img = F(spt.rasterize_pix(T(xyd, dev), T(rgb, dev), (w, h)))
    win = orc.point_render_sort_depth(xyd, w, h)
    expect = np.where((win >= 0)[..., None], rgb[np.maximum(win, 0)], 0.0).astype(np.float32)
    assert (win >= 0).mean() > 0.9
    assert np.array_equal(img, expect)
