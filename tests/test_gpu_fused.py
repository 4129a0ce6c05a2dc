"""Batched, fused forward (projection + SH, depth sort, pair emission, tile
sort, ranges, persistent raster) against the CPU oracle, and batched vs the
plain per-view path.  Bar: records, tile lists and stop positions bit-exact;
images max-abs <= 1e-4 (observed exact); batched == per-view."""
import numpy as np
import pytest
import torch

from dsplat import scenes
from dsplat.gauss import GaussBatch
from gpu_util import F, U32, params_of

pytestmark = pytest.mark.gpu
IMG_TOL = 1e-4


def _scene(sh_deg, n=20000, seed=3):
    rng = np.random.default_rng(seed)
    base = scenes.config0(seed=seed, n=n, size=(64, 64))
    if sh_deg >= 0:
        base.colors = scenes._sh_colors(rng, n, sh_deg)
    base.sh_degree = sh_deg
    cams = [scenes.Camera.look_at_origin((0.3, 0.2, -3.0), 256, 256),
            scenes.Camera.look_at_origin((2.0, 1.0, 2.0), 200, 120),
            scenes.Camera.look_at_origin((-2.5, -0.5, 1.0), 64, 48)]
    base.cameras = cams
    return base


def _check_view(orc, batch, sc, v, ts):
    cam = sc.cameras[v]
    w, h = cam.width, cam.height
    xyd, conic, aabb, rgb = orc.fused_project(sc.means, sc.log_scales, sc.quats, sc.colors.reshape(sc.n, -1),
                                              sc.sh_degree, cam.mvp, cam.campos, w, h)
    o_t, o_i, _ = orc.tile2pnt(xyd, aabb, w, h, ts)
    # records are written for the points that have tiles in this view
    vis = np.zeros(sc.n, bool)
    vis[np.unique(o_i)] = True
    assert vis.any()
    rec = F(batch.records()[v])[vis]
    vxyd, vconic, vrgb, vaabb = xyd[vis], conic[vis], rgb[vis], aabb[vis]
    assert np.array_equal(rec[:, 0:2].view(np.uint32), vxyd[:, :2].view(np.uint32))
    assert np.array_equal(rec[:, 2:4].view(np.uint32), vconic[:, :2].view(np.uint32))
    assert np.array_equal(rec[:, 4].view(np.uint32), vconic[:, 2].view(np.uint32))
    assert np.array_equal(rec[:, 11].view(np.uint32), vxyd[:, 2].view(np.uint32))
    assert np.array_equal(rec[:, [6, 7, 8]].view(np.uint32), vrgb.view(np.uint32))
    gpu_aabb = np.stack([rec[:, 0] - rec[:, 9], rec[:, 1] - rec[:, 10], rec[:, 0] + rec[:, 9],
                         rec[:, 1] + rec[:, 10]], 1).astype(np.float32)
    assert np.array_equal(gpu_aabb.view(np.uint32), vaabb.view(np.uint32))
    t2i, i2p, stop = batch.tile_lists(v)
    assert np.array_equal(t2i, o_t)
    assert np.array_equal(i2p, o_i)
    o_img, o_T, o_last = orc.gauss_rasterize_tiled(w, h, ts, o_t, o_i, xyd, conic, aabb, sc.opacity, rgb)
    img = F(batch.images()[v])
    assert np.abs(img - o_img).max() <= IMG_TOL
    assert np.array_equal(img, o_img)
    assert np.array_equal(F(batch.per_pixel("T")[v]), o_T)
    assert np.array_equal(stop, o_last)


@pytest.mark.parametrize("sh_deg,ts,ppl", [(-1, 16, 0), (0, 16, 2), (1, 8, 2), (3, 8, 1), (3, 16, 4), (3, 16, 8), (3, 32, 4),
                                            (2, 32, 8)])
def test_batched_forward_matches_oracle(orc, dev, sh_deg, ts, ppl):
    sc = _scene(sh_deg)
    batch = GaussBatch(sc.n, sc.cameras, ts, sh_deg, pair_capacity=1000, device=dev, pixels_per_lane=ppl)
    p = params_of(sc, dev)
    pairs = batch.ensure_capacity(p)
    assert pairs > 0 and batch.status()[0] == 0
    torch.cuda.synchronize()
    for v in range(len(sc.cameras)):
        _check_view(orc, batch, sc, v, ts)


def test_plain_per_view_equals_batched(dev):
    sc = _scene(3)
    p = params_of(sc, dev)
    batch = GaussBatch(sc.n, sc.cameras, 16, 3, pair_capacity=1000, device=dev)
    batch.ensure_capacity(p)
    imgs = [F(x) for x in batch.images()]
    for v, cam in enumerate(sc.cameras):
        one = GaussBatch(sc.n, [cam], 16, 3, pair_capacity=1000, device=dev)
        one.ensure_capacity(p)
        assert np.array_equal(F(one.images()[0]), imgs[v])


def test_capacity_overflow_is_reported_not_fatal(dev):
    sc = _scene(-1)
    p = params_of(sc, dev)
    batch = GaussBatch(sc.n, sc.cameras, 16, -1, pair_capacity=777, device=dev)
    batch.forward(p)
    flags, needed, pairs = batch.status()
    assert flags & 1 and needed > 777 and pairs >= needed
    batch.ensure_capacity(p)
    assert batch.status()[0] == 0


def test_empty_scene(dev):
    cams = [scenes.Camera.look_at_origin((0, 0, -3), 40, 30)]
    z = lambda *s: torch.zeros(s, device=dev)  # noqa: E731
    p = dict(means=z(0, 3), log_scales=z(0, 3), quats=z(0, 4), opacity=z(0), colors=z(0, 3))
    batch = GaussBatch(0, cams, 16, -1, pair_capacity=16, device=dev)
    img = batch.forward(p)
    assert float(img.abs().max()) == 0.0


def test_graph_captured_step_matches_eager(dev):
    """The whole batched fwd+bwd step captured into a CUDA graph gives the same
    images and gradients as the eager calls."""
    from dsplat.gauss import CapturedStep
    sc = _scene(3, n=8000)
    p = params_of(sc, dev)
    batch = GaussBatch(sc.n, sc.cameras, 16, 3, pair_capacity=1000, device=dev, pixels_per_lane=2)
    batch.ensure_capacity(p)
    npix = int(batch.layout.num_pix)
    target = torch.rand(npix * 3, device=dev)
    grads = {k: torch.zeros_like(v) for k, v in p.items()}
    batch.forward(p, target=target)
    batch.backward(p, grads)
    torch.cuda.synchronize()
    img_eager = batch.out_rgb.clone()
    g_eager = {k: v.clone() for k, v in grads.items()}
    step = CapturedStep(batch, p, grads, target)
    step.replay()
    torch.cuda.synchronize()
    assert torch.equal(batch.out_rgb, img_eager)
    for k in g_eager:  # float atomics may add in another order: compare at the group's scale
        scale = g_eager[k].abs().max()
        assert (grads[k] - g_eager[k]).abs().max() <= 1e-4 * scale, k


def test_autotuner_picks_a_supported_config(dev):
    from dsplat import autotune
    sc = _scene(0, n=4000)
    p = params_of(sc, dev)
    npix = sum(c.width * c.height for c in sc.cameras)
    rep = {}
    ts, ppl = autotune.tune(p, sc.cameras, 0, torch.rand(npix * 3, device=dev), use_cache=False, report=rep)
    assert (ts, ppl) in autotune.CANDIDATES and len(rep["timings_ms"]) == len(autotune.CANDIDATES)


def test_repeated_backward_accumulates_exactly_twice(dev):
    """The projection backward zeroes the per-view 2D gradients it consumes;
    a second backward of the same forward must see them rebuilt from zero:
    gradients after two backward calls are twice those after one (the same
    atomics order is not guaranteed, so the comparison is to 1e-5 relative)."""
    sc = _scene(3, n=8000, seed=9)
    p = params_of(sc, dev)
    batch = GaussBatch(sc.n, sc.cameras, 8, 3, pair_capacity=1 << 18, device=dev, pixels_per_lane=2)
    batch.ensure_capacity(p)
    tgt = torch.rand(int(batch.layout.num_pix) * 3, device=dev)
    batch.forward(p, target=tgt)
    g1 = {k: torch.zeros_like(v) for k, v in p.items()}
    batch.backward(p, g1)
    g2 = {k: torch.zeros_like(v) for k, v in p.items()}
    batch.backward(p, g2)
    batch.backward(p, g2)
    torch.cuda.synchronize(dev)
    for k in p:
        a, b = F(g1[k]).astype(np.float64) * 2, F(g2[k]).astype(np.float64)
        scale = max(np.abs(a).max(), 1e-30)
        assert np.abs(a - b).max() <= 1e-5 * scale, k
        assert np.abs(a).max() > 0, k


def test_large_splats_take_the_direct_scatter_path(orc, dev):
    """Splats whose boxes span dozens of superblocks give sub-passes with more
    list entries than the superblock scatter stages in shared memory; those
    write their entries directly.  Lists, images and stops stay bit-exact."""
    rng = np.random.default_rng(17)
    sc = scenes.config0(seed=17, n=3000, size=(64, 64))
    sc.log_scales = rng.uniform(-1.6, -1.0, (sc.n, 3)).astype(np.float32)  # boxes of ~100-300 px
    sc.cameras = [scenes.Camera.look_at_origin((0.2, -0.1, -3.0), 512, 512),
                  scenes.Camera.look_at_origin((1.5, 2.0, 1.5), 384, 256)]
    p = params_of(sc, dev)
    batch = GaussBatch(sc.n, sc.cameras, 8, sc.sh_degree, pair_capacity=1 << 20, device=dev, pixels_per_lane=2)
    batch.ensure_capacity(p)
    _, needed, _ = batch.status()
    # 3000 points = 6 sub-passes of 512 ranks per view: on average each holds
    # more list entries than the 3072 the scatter stages
    assert needed > len(sc.cameras) * 6 * 3072
    for v in range(len(sc.cameras)):
        _check_view(orc, batch, sc, v, 8)


def test_thousands_of_superblocks_take_the_unstaged_scatter(orc, dev):
    """A 3072x3072 view at 8x8 tiles has 48x48 = 2304 superblocks: the staged
    superblock scatter would need more than its 100 KB shared-memory budget,
    so the lists are built by the unstaged kernel.  Lists, images and stops
    stay bit-exact."""
    sc = scenes.config0(seed=23, n=4000, size=(64, 64))
    sc.cameras = [scenes.Camera.look_at_origin((0.1, 0.3, -3.0), 3072, 3072)]
    p = params_of(sc, dev)
    batch = GaussBatch(sc.n, sc.cameras, 8, sc.sh_degree, pair_capacity=1 << 20, device=dev, pixels_per_lane=2)
    assert int(batch.layout.sb_log2[0]) == 3 and int(batch.layout.num_sb) == 48 * 48
    batch.ensure_capacity(p)
    assert batch.status()[0] == 0
    _check_view(orc, batch, sc, 0, 8)


def test_headline_batch_matches_plain_and_oracle(orc, dev):
    """The benchmarked batch (config 3: 1,048,576 Gaussians, SH 3, 16 views of
    mixed resolution) in one batched forward, against the plain per-view path
    on every view (max-abs <= 1e-4; observed bit-exact) and against the oracle
    on the first view and the first 1920x1080 view."""
    sc = scenes.config3(n=1 << 20, views=16)
    p = params_of(sc, dev)
    batch = GaussBatch(sc.n, sc.cameras, 8, 3, pair_capacity=1 << 26, device=dev)
    batch.ensure_capacity(p)
    batch.forward(p)
    imgs = [F(x) for x in batch.images()]
    worst = 0.0
    for v, cam in enumerate(sc.cameras):
        one = GaussBatch(sc.n, [cam], 8, 3, pair_capacity=1 << 24, device=dev)
        one.ensure_capacity(p)
        one.forward(p)
        worst = max(worst, float(np.abs(F(one.images()[0]) - imgs[v]).max()))
        del one
    print(f"headline batch vs plain per-view: max|img| {worst:.3g}")
    assert worst <= IMG_TOL
    big = next(v for v, c in enumerate(sc.cameras) if c.width == 1920)
    for v in sorted({0, big}):
        cam = sc.cameras[v]
        xyd, conic, aabb, rgb = orc.fused_project(sc.means, sc.log_scales, sc.quats, sc.colors, 3, cam.mvp,
                                                  cam.campos, cam.width, cam.height)
        t2i, i2p, _ = orc.tile2pnt(xyd, aabb, cam.width, cam.height, 16, with_keys=False)
        o_img, _, _ = orc.gauss_rasterize_tiled(cam.width, cam.height, 16, t2i, i2p, xyd, conic, aabb, sc.opacity,
                                                rgb, nthreads=16)
        assert np.array_equal(imgs[v], o_img)


def test_training_batch_matches_plain(dev):
    """The training workload's batch (config 4: 4,194,304 Gaussians, SH 3,
    8 views at 1920x1080) in one batched forward, against the plain per-view
    path on every view (max-abs <= 1e-4; observed bit-exact)."""
    sc = scenes.config4()
    p = params_of(sc, dev)
    batch = GaussBatch(sc.n, sc.cameras, 8, 3, pair_capacity=1 << 26, device=dev)
    pairs = batch.ensure_capacity(p)
    assert pairs > 3_000_000_000  # about 3.9 G tile pairs, near the 32-bit range
    batch.forward(p)
    imgs = [F(x) for x in batch.images()]
    worst = 0.0
    for v, cam in enumerate(sc.cameras):
        one = GaussBatch(sc.n, [cam], 8, 3, pair_capacity=1 << 25, device=dev)
        one.ensure_capacity(p)
        one.forward(p)
        worst = max(worst, float(np.abs(F(one.images()[0]) - imgs[v]).max()))
        del one
    torch.cuda.empty_cache()
    print(f"config-4 batch vs plain per-view: max|img| {worst:.3g}")
    assert worst <= IMG_TOL
