"""Backward rasteriser + projection backward against the FP64 gradient oracle.

The discrete structure (tile lists, per-pixel stop positions, 3-sigma boxes)
is taken from the GPU forward and frozen; the oracle's loss is then a smooth
function of the parameters.  Checks:
  * FP64 analytic backward vs FP64 central differences (h = 1e-4): the oracle
    is right (relative error <= 1e-4 -- the O(h^2) truncation of the central
    difference -- with a floor of 1e-3 x group max);
  * GPU (FP32) vs FP64 central differences on 64 random parameters:
    |g_gpu - g_fd| <= 1e-3 * max(|g_fd|, 1e-2 * group max);
  * GPU vs FP64 analytic on every parameter, same tolerance.
"""
import numpy as np
import pytest
import torch

from dsplat import scenes
from dsplat.gauss import GaussBatch
from gpu_util import F, U32, params_of

pytestmark = pytest.mark.gpu
GROUPS = ["means", "log_scales", "quats", "opacity", "colors"]


def _run(orc, dev, sc, target, ts=16):
    cam = sc.cameras[0]
    p = params_of(sc, dev)
    batch = GaussBatch(sc.n, [cam], ts, sc.sh_degree, pair_capacity=1000, device=dev)
    batch.ensure_capacity(p)
    tgt = torch.from_numpy(target.reshape(-1)).to(dev)
    batch.forward(p, target=tgt)
    grads = {k: torch.zeros_like(v) for k, v in p.items()}
    batch.backward(p, grads)
    torch.cuda.synchronize()
    rec = F(batch.records()[0])
    aabb = np.stack([rec[:, 0] - rec[:, 9], rec[:, 1] - rec[:, 10], rec[:, 0] + rec[:, 9],
                     rec[:, 1] + rec[:, 10]], 1).astype(np.float32)
    t2i, i2p, last = batch.tile_lists(0)
    S = orc.Scene(sc.means, sc.log_scales, sc.quats, sc.opacity, sc.colors.reshape(sc.n, -1), sc.sh_degree,
                  cam.mvp, cam.campos, cam.width, cam.height, ts, t2i, i2p, last.astype(np.int32), aabb, target)
    return batch, {k: F(v).reshape(sc.n, -1).astype(np.float64) for k, v in grads.items()}, S


def _close(a, b, scale, rel, floor):
    return np.abs(a - b) <= rel * np.maximum(np.abs(b), floor * scale)


@pytest.mark.parametrize("sh_deg", [-1, 3])
def test_gradients_small(orc, dev, sh_deg):
    rng = np.random.default_rng(21)
    sc = scenes.config0(seed=21, n=3000, size=(96, 72))
    if sh_deg >= 0:
        sc.colors = scenes._sh_colors(rng, sc.n, sh_deg)
        sc.sh_degree = sh_deg
    target = rng.uniform(0, 1, (72, 96, 3)).astype(np.float32)
    batch, g_gpu, S = _run(orc, dev, sc, target)
    L64, img64 = S.loss(with_image=True)
    assert np.abs(img64 - F(batch.images()[0])).max() < 1e-4
    L, g64 = S.backward()
    for k in GROUPS:
        ref = g64[k].reshape(sc.n, -1)
        scale = np.abs(ref).max()
        ok = _close(g_gpu[k], ref, scale, 1e-3, 1e-2)
        assert ok.mean() > 0.999, (k, ok.mean(), np.abs(g_gpu[k] - ref).max(), scale)
    # FD on 64 random parameters of visible Gaussians
    vis = np.unique(batch.tile_lists(0)[1])
    picks = []
    for _ in range(64):
        k = GROUPS[rng.integers(0, len(GROUPS))]
        g = int(rng.choice(vis))
        c = int(rng.integers(0, g64[k].reshape(sc.n, -1).shape[1]))
        picks.append((k, g, c))
    bad = []
    for k, g, c in picks:
        fd = S.fd(k, g, c, 1e-4)
        an = g64[k].reshape(sc.n, -1)[g, c]
        gp = g_gpu[k][g, c]
        scale = np.abs(g64[k]).max()
        if not _close(np.array(an), np.array(fd), scale, 1e-4, 1e-3):
            bad.append(("analytic", k, g, c, an, fd))
        if not _close(np.array(gp), np.array(fd), scale, 1e-3, 1e-2):
            bad.append(("gpu", k, g, c, gp, fd))
    assert not bad, bad[:8]


def test_gradients_config2_scale(orc, dev):
    """262,144 Gaussians, SH 3, 1280x720, L2 loss against a U[0,1] target:
    GPU gradients vs FP64 central differences on 64 random parameters of
    visible Gaussians, and vs the FP64 analytic backward on every parameter."""
    sc, target = scenes.config2()
    batch, g_gpu, S = _run(orc, dev, sc, target, ts=16)
    L, g64 = S.backward()
    for k in GROUPS:
        ref = g64[k].reshape(sc.n, -1)
        scale = np.abs(ref).max()
        ok = _close(g_gpu[k], ref, scale, 1e-3, 1e-2)
        assert ok.mean() > 0.999, (k, ok.mean(), np.abs(g_gpu[k] - ref).max(), scale)
    rng = np.random.default_rng(22)
    vis = np.unique(batch.tile_lists(0)[1])
    bad = []
    for _ in range(64):
        k = GROUPS[rng.integers(0, len(GROUPS))]
        g = int(rng.choice(vis))
        c = int(rng.integers(0, g64[k].reshape(sc.n, -1).shape[1]))
        fd = S.fd(k, g, c, 1e-4)
        gp = g_gpu[k][g, c]
        scale = np.abs(g64[k]).max()
        if not _close(np.array(gp), np.array(fd), scale, 1e-3, 1e-2):
            bad.append((k, g, c, gp, fd))
    assert not bad, bad[:8]
