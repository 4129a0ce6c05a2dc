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


# ---------------------------------------------------------------- the blend and the projection kernels
# oracle/_ref also holds splat_gauss.cu and splat_circle.cu compiled for the
# host (C library expf, the kernel's double stop test, no contraction), their
# del-geo calls resolved to the oracle's restatement.

@pytest.mark.parametrize("ts,size", [(16, (256, 256)), (8, (120, 72)), (32, (250, 130))])
def test_blend_matches_reference_kernel(orc, ts, size):
    if not orc.ref_available():
        pytest.skip("oracle/_ref not built")
    sc, xyd, conic, aabb = _cfg0_projected(orc, n=16384 if size == (256, 256) else 6000, size=size)
    t2i, i2p, _ = orc.tile2pnt(xyd, aabb, *size, ts, with_keys=False)
    ref = orc.ref_gauss_rasterize(*size, ts, t2i, i2p, xyd, conic, aabb, sc.opacity, sc.colors)
    img, _, _ = orc.gauss_rasterize_tiled(*size, ts, t2i, i2p, xyd, conic, aabb, sc.opacity, sc.colors,
                                          nthreads=8, mode=orc.BLEND_LIBM_EXP | orc.BLEND_CUDA_STOP)
    assert np.array_equal(img.view(np.uint32), ref.view(np.uint32))


@pytest.mark.parametrize("size", [(256, 256), (250, 130)])
def test_projection_composition_matches_reference_kernel(orc, size):
    """splat_gauss.cu:10-53 run on the host (del-geo restated) == the oracle's projection."""
    if not orc.ref_available():
        pytest.skip("oracle/_ref not built")
    sc = scenes.config0(n=16384, size=size)
    cam = sc.cameras[0]
    o = orc.gauss_project(sc.means, sc.quats, sc.scales, cam.mvp, *size)
    r = orc.ref_gauss_project(sc.means, sc.quats, sc.scales, cam.mvp, *size)
    for a, b in zip(o, r):
        assert np.array_equal(a.view(np.uint32), b.view(np.uint32))


def test_circle_kernels_match_reference(orc):
    """splat_circle.cu:7-41 (projection) and :93-132 (painter) run on the host
    == the oracle's circle projection and tiled painter."""
    if not orc.ref_available():
        pytest.skip("oracle/_ref not built")
    pts = scenes.config1(n=30000, size=(200, 120))
    cam = pts.camera
    xyd, rad = orc.circle_project(pts.xyz, cam.mvp, 200, 120, 0.01)
    rx, rr = orc.ref_circle_project(pts.xyz, cam.mvp, 200, 120, 0.01)
    assert np.array_equal(xyd.view(np.uint32), rx.view(np.uint32))
    assert np.array_equal(rad.view(np.uint32), rr.view(np.uint32))
    aabb = orc.circle_aabb(xyd, rad)
    t2i, i2p, _ = orc.tile2pnt(xyd, aabb, 200, 120, 16, with_keys=False)
    rgb = np.random.default_rng(3).uniform(0, 1, (xyd.shape[0], 3)).astype(np.float32)
    win = orc.circle_splat_tiled(200, 120, 16, t2i, i2p, xyd, rad)
    img = np.zeros((120, 200, 3), np.float32)
    img[win >= 0] = rgb[win[win >= 0]]
    ref = orc.ref_circle_rasterize(200, 120, 16, t2i, i2p, xyd, rad, rgb)
    assert (win >= 0).sum() > 1000
    assert np.array_equal(img, ref)


def test_untiled_and_tiled_blend_agree(orc):
    """del-splat-cpu's untiled render_gauss_sort_depth (pnt2pixxyndcz.rs:42-100)
    and the tiled walk visit every pixel's Gaussians in the same order, so with
    the same arithmetic they agree bit for bit."""
    sc, xyd, conic, aabb = _cfg0_projected(orc, n=4000, size=(96, 64))
    t2i, i2p, _ = orc.tile2pnt(xyd, aabb, 96, 64, 16, with_keys=False)
    for mode in (0, orc.BLEND_LIBM_EXP):
        naive = orc.gauss_render_naive(xyd, conic, aabb, sc.opacity, sc.colors, 96, 64, mode=mode)
        tiled, _, _ = orc.gauss_rasterize_tiled(96, 64, 16, t2i, i2p, xyd, conic, aabb, sc.opacity, sc.colors,
                                                mode=mode)
        assert np.array_equal(naive, tiled)


def test_correctly_rounded_exp_stays_within_1e4_of_libm_blend(orc):
    """The product's arithmetic (correctly rounded exp) against del-splat-cpu's
    literal f32 arithmetic (the C library's expf): the two exps differ on about
    1 input in 11,500, so images agree to float rounding and the stop
    positions coincide at config 0."""
    sc, xyd, conic, aabb = _cfg0_projected(orc)
    t2i, i2p, _ = orc.tile2pnt(xyd, aabb, 256, 256, 16, with_keys=False)
    a, Ta, la = orc.gauss_rasterize_tiled(256, 256, 16, t2i, i2p, xyd, conic, aabb, sc.opacity, sc.colors,
                                          nthreads=8, mode=0)
    b, Tb, lb = orc.gauss_rasterize_tiled(256, 256, 16, t2i, i2p, xyd, conic, aabb, sc.opacity, sc.colors,
                                          nthreads=8, mode=orc.BLEND_LIBM_EXP)
    assert np.abs(a - b).max() <= 1e-4
    assert np.abs(Ta - Tb).max() <= 1e-4
    assert np.array_equal(la, lb)


def test_expf_cr_is_correctly_rounded(orc):
    rng = np.random.default_rng(11)
    x = np.concatenate([rng.uniform(-110, 90, 1 << 20), rng.standard_normal(1 << 16) * 1e-3,
                        [0.0, -0.0, -87.0, 87.0, -103.9, -104.5, 88.7, 89.5]]).astype(np.float32)
    got = orc.expf_cr(x)
    with np.errstate(over="ignore"):
        want = np.exp(x.astype(np.float64)).astype(np.float32)
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32))
    s = orc.expf_cr(np.array([np.nan, -np.inf, np.inf], np.float32))
    assert np.isnan(s[0]) and s[1] == 0.0 and s[2] == np.inf
