"""The CPU oracle against the reference's own code (oracle/_ref: the
reference's tile_acceleration.h and splat_point.cu compiled as host C++) and
against the committed fixtures that code produced."""
import os

import numpy as np
import pytest

from dsplat import scenes

GOLD = os.path.join(os.path.dirname(__file__), "golden")


def _cfg0_projected(orc, n=16384, size=(256, 256), seed=0):
    sc = scenes.config0(seed=seed, n=n, size=size)
    cam = sc.cameras[0]
    xyd, conic, aabb = orc.gauss_project(sc.means, sc.quats, sc.scales, cam.mvp, cam.width, cam.height)
    return sc, xyd, conic, aabb


@pytest.mark.parametrize("ts", [8, 16, 32])
def test_tile_lists_match_reference_code(orc, ts):
    if not orc.ref_available():
        pytest.skip("oracle/_ref not built (needs the del-splat sources)")
    _, xyd, _, aabb = _cfg0_projected(orc)
    t_o, i_o, k_o = orc.tile2pnt(xyd, aabb, 256, 256, ts)
    t_r, i_r, k_r = orc.ref_tile2pnt(xyd, aabb, 256, 256, ts)
    assert np.array_equal(t_o, t_r)
    assert np.array_equal(i_o, i_r)
    assert np.array_equal(k_o, k_r)


def test_circle_tile_lists_match_reference_code(orc):
    if not orc.ref_available():
        pytest.skip("oracle/_ref not built")
    pts = scenes.config1(n=20000, size=(200, 120))
    cam = pts.camera
    xyd, rad = orc.circle_project(pts.xyz, cam.mvp, cam.width, cam.height, 0.01)
    aabb = orc.circle_aabb(xyd, rad)
    t_o, i_o, k_o = orc.tile2pnt(xyd, aabb, 200, 120, 16)
    t_r, i_r, k_r = orc.ref_tile2pnt(xyd, aabb, 200, 120, 16)
    assert np.array_equal(t_o, t_r) and np.array_equal(i_o, i_r) and np.array_equal(k_o, k_r)


def test_point_painter_matches_reference_zbuffer(orc):
    """render_pix_sort_depth (restated) vs splat_point.cu run serially: same
    winner per pixel whenever no two points tie in unit depth."""
    if not orc.ref_available():
        pytest.skip("oracle/_ref not built")
    rng = np.random.default_rng(7)
    n, w, h = 20000, 64, 48
    xyd = np.stack([rng.uniform(-0.9, w + 3, n), rng.uniform(-0.9, h + 3, n), rng.uniform(-0.999, 0.999, n)],
                   1).astype(np.float32)
    rgb = rng.uniform(0, 1, (n, 3)).astype(np.float32)
    depth_r, img_r = orc.ref_point_zbuffer(xyd, rgb, w, h)
    win = orc.point_render_sort_depth(xyd, w, h)
    hit = win >= 0
    assert np.array_equal(hit, depth_r < np.finfo(np.float32).max)
    ud = orc.point_unitdepth(xyd[:, 2])
    assert np.array_equal(ud[win[hit]], depth_r[hit])
    assert np.array_equal(rgb[win[hit]], img_r[hit])


def test_naive_renderer_equals_tiled(orc):
    """pnt2pixxyndcz.rs:42 (global sort, untiled) and splat_gauss.cu:56 (tiled)
    give the same image when every ndc_z is inside (-1, 1)."""
    sc, xyd, conic, aabb = _cfg0_projected(orc, n=3000, size=(96, 64))
    assert np.all(np.abs(xyd[:, 2]) < 1)
    t2i, i2p, _ = orc.tile2pnt(xyd, aabb, 96, 64, 16)
    img_t, _, _ = orc.gauss_rasterize_tiled(96, 64, 16, t2i, i2p, xyd, conic, aabb, sc.opacity, sc.colors)
    img_n = orc.gauss_render_naive(xyd, conic, aabb, sc.opacity, sc.colors, 96, 64)
    assert np.array_equal(img_t, img_n)


@pytest.mark.parametrize("name", ["tiles_gauss_small.npz", "tiles_circle_small.npz"])
def test_oracle_matches_reference_fixtures(orc, name):
    d = np.load(os.path.join(GOLD, name))
    w, h, ts = (int(x) for x in d["shape"])
    t2i, i2p, keys = orc.tile2pnt(d["xyd"], d["aabb"], w, h, ts)
    assert np.array_equal(t2i, d["tile2idx"])
    assert np.array_equal(i2p, d["idx2pnt"])
    assert np.array_equal(keys, d["keys"])


def test_oracle_matches_reference_zbuffer_fixture(orc):
    d = np.load(os.path.join(GOLD, "point_zbuffer_small.npz"))
    w, h = (int(x) for x in d["shape"])
    win = orc.point_render_sort_depth(d["xyd"], w, h)
    hit = win >= 0
    assert np.array_equal(hit, d["depth"] < np.finfo(np.float32).max)
    assert np.array_equal(orc.point_unitdepth(d["xyd"][win[hit], 2]), d["depth"][hit])
