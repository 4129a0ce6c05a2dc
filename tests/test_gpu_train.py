"""The training-side API: the torch.autograd entry point of del-splat-dlpack,
the fused Adam against torch.optim.Adam, the graph-captured training step,
capacity growth on overflow and the 64-bit tile-pair total."""
import numpy as np
import pytest
import torch

from dsplat import scenes
from dsplat.gauss import Adam, CapturedStep, GaussBatch
from gpu_util import F, params_of

pytestmark = pytest.mark.gpu


def _scene(n=6000, seed=21):
    sc = scenes.config0(seed=seed, n=n, size=(64, 64))
    sc.colors = scenes._sh_colors(np.random.default_rng(seed), n, 3)
    sc.sh_degree = 3
    sc.cameras = [scenes.Camera.look_at_origin((0.4, 0.3, -3.0), 160, 120),
                  scenes.Camera.look_at_origin((2.0, 1.0, 2.0), 96, 64)]
    return sc


def _rel(a, b):
    return float((a - b).abs().max() / b.abs().max().clamp_min(1e-30))


def test_render_autograd_matches_batch_backward(dev):
    """del_splat_dlpack.SplatGauss.torch.render + loss.backward() == the
    batch's own forward/backward with the same dL/dimage."""
    from del_splat_dlpack.SplatGauss import torch as sg
    sc = _scene()
    p = params_of(sc, dev)
    leaves = {k: v.clone().requires_grad_(True) for k, v in p.items()}
    batch = sg.make_batch(sc.n, sc.cameras, 16, 3, pair_capacity=1 << 18)
    imgs = sg.render(leaves["means"], leaves["log_scales"], leaves["quats"], leaves["opacity"], leaves["colors"],
                     batch)
    w = [torch.rand_like(im) for im in imgs]
    loss = sum((im * wi).sum() for im, wi in zip(imgs, w))
    loss.backward()
    ref = GaussBatch(sc.n, sc.cameras, 16, 3, pair_capacity=1 << 18, device=dev)
    ref.ensure_capacity(p)
    ref.forward(p)
    for a, b in zip(ref.images(), imgs):
        assert torch.equal(a, b.detach())
    grads = {k: torch.zeros_like(v) for k, v in p.items()}
    ref.backward(p, grads, torch.cat([x.reshape(-1) for x in w]))
    for k in p:
        assert _rel(leaves[k].grad, grads[k]) <= 1e-5, k


def test_render_grows_the_lists_on_overflow(dev):
    """A batch created with a tiny list capacity still renders the full image:
    the autograd forward reads the overflow flag and grows the lists."""
    from dsplat.gauss import render
    sc = _scene()
    p = params_of(sc, dev)
    small = GaussBatch(sc.n, sc.cameras, 16, 3, pair_capacity=64, device=dev)
    imgs = render(p["means"], p["log_scales"], p["quats"], p["opacity"], p["colors"], small)
    assert small.capacity > 64
    ref = GaussBatch(sc.n, sc.cameras, 16, 3, pair_capacity=1 << 18, device=dev)
    ref.ensure_capacity(p)
    ref.forward(p)
    for a, b in zip(ref.images(), imgs):
        assert torch.equal(a, b)


def test_render_backward_after_a_later_forward_raises(dev):
    """The forward state (stop positions, final transmittance, tile lists)
    lives in the batch's workspace: a backward of a render that a later
    forward on the same batch has overwritten raises instead of returning
    the later forward's gradients; the latest render's backward still works."""
    from dsplat.gauss import render
    sc = _scene()
    p = params_of(sc, dev)
    leaves = {k: v.clone().requires_grad_(True) for k, v in p.items()}
    batch = GaussBatch(sc.n, sc.cameras, 16, 3, pair_capacity=1 << 18, device=dev)
    args = (leaves["means"], leaves["log_scales"], leaves["quats"], leaves["opacity"], leaves["colors"], batch)
    first = sum(im.sum() for im in render(*args))
    second = sum(im.sum() for im in render(*args))
    with pytest.raises(RuntimeError, match="another forward"):
        first.backward()
    second.backward()
    assert all(torch.isfinite(v.grad).all() for v in leaves.values())


def test_fused_adam_matches_torch_optim(dev):
    torch.manual_seed(0)
    n, K = 5000, 16
    shapes = dict(means=(n, 3), log_scales=(n, 3), quats=(n, 4), opacity=(n,), colors=(n, 3 * K))
    ours = {k: torch.randn(s, device=dev) for k, s in shapes.items()}
    ours["opacity"] = torch.rand(n, device=dev) * 0.8 + 0.1
    theirs = {k: v.clone().requires_grad_(True) for k, v in ours.items()}
    opt = torch.optim.Adam(list(theirs.values()), lr=1e-3, betas=(0.9, 0.999), eps=1e-8)
    adam = Adam(ours, 3, lr=1e-3, betas=(0.9, 0.999), eps=1e-8)
    for _ in range(5):
        grads = {k: torch.randn_like(v) for k, v in ours.items()}
        for k in theirs:
            theirs[k].grad = grads[k].clone()
        opt.step()
        adam.step(grads)
    assert int(adam.step_count.item()) == 5
    for k in ours:
        assert _rel(ours[k], theirs[k].detach()) <= 1e-6, k
        assert _rel(adam.exp_avg_sq[k], opt.state[theirs[k]]["exp_avg_sq"]) <= 1e-6, k


def test_fused_adam_keeps_opacity_below_one(dev):
    p = {k: torch.zeros(s, device=dev) for k, s in dict(means=(10, 3), log_scales=(10, 3), quats=(10, 4),
                                                            opacity=(10,), colors=(10, 3)).items()}
    p["opacity"].fill_(0.9985)
    adam = Adam(p, -1, lr=0.1)
    g = {k: torch.zeros_like(v) for k, v in p.items()}
    g["opacity"].fill_(-1.0)  # pushes opacity up
    g["colors"].fill_(1.0)
    adam.step(g)
    assert float(p["opacity"].max()) <= 0.999 + 1e-7
    assert float(p["colors"].max()) < 0.0


def test_adam_inside_a_graph_matches_eager(dev):
    """The fused Adam captured in a CUDA graph and replayed three times ==
    three eager calls, bit for bit (same gradients; the step count advances on
    the device)."""
    torch.manual_seed(3)
    n = 4000
    base = dict(means=torch.randn(n, 3, device=dev), log_scales=torch.randn(n, 3, device=dev),
                quats=torch.randn(n, 4, device=dev), opacity=torch.rand(n, device=dev) * 0.8 + 0.1,
                colors=torch.randn(n, 48, device=dev))
    grads = {k: torch.randn_like(v) for k, v in base.items()}
    eager = {k: v.clone() for k, v in base.items()}
    a_eager = Adam(eager, 3, lr=1e-3)
    for _ in range(3):
        a_eager.step(grads)
    graphed = {k: v.clone() for k, v in base.items()}
    a_graph = Adam(graphed, 3, lr=1e-3)
    side = torch.cuda.Stream()
    side.wait_stream(torch.cuda.current_stream())
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g, stream=side):
        a_graph.step(grads)
    for _ in range(3):
        g.replay()
    torch.cuda.synchronize()
    assert int(a_graph.step_count.item()) == 3
    for k in base:
        assert torch.equal(graphed[k], eager[k]), k
        assert torch.equal(a_graph.exp_avg_sq[k], a_eager.exp_avg_sq[k]), k


def test_captured_train_step_trains(dev):
    """forward + backward + fused Adam in one captured graph: replays keep the
    lists within capacity, keep every parameter finite and lower the loss."""
    sc = _scene()
    tgt = torch.cat([torch.from_numpy(t.reshape(-1)) for t in scenes.targets_for(sc)]).to(dev)
    p = params_of(sc, dev)
    g = {k: torch.zeros_like(v) for k, v in p.items()}
    batch = GaussBatch(sc.n, sc.cameras, 16, 3, pair_capacity=1 << 18, device=dev, check_overflow=False)
    batch.ensure_capacity(p)
    adam = Adam(p, 3, lr=1e-2)
    step = CapturedStep(batch, p, g, tgt, warmup=1, optimizer=adam)
    losses = []
    for _ in range(20):
        step.replay()
        losses.append(float(batch.slab_loss().sum()))
    torch.cuda.synchronize()
    assert batch.status()[0] == 0
    assert int(adam.step_count.item()) == 21
    assert all(bool(torch.isfinite(v).all()) for v in p.values())
    assert float(p["opacity"].max()) <= 0.999 + 1e-7
    assert losses[-1] < losses[0]


def test_pair_total_beyond_32_bits(dev):
    """17,000 Gaussians whose 3-sigma boxes each cover a whole 4096x4096 view
    at 8x8 tiles: 17,000 x 512 x 512 = 4,456,448,000 tile pairs (> 2^32).
    With a small list capacity the forward reports the overflow and the exact
    64-bit pair total."""
    n = 17000
    rng = np.random.default_rng(9)
    cam = scenes.Camera.look_at_origin((0.0, 0.0, -3.0), 4096, 4096)
    sc = scenes.GaussScene(means=rng.uniform(-0.05, 0.05, (n, 3)).astype(np.float32),
                           log_scales=np.full((n, 3), np.log(3.0), np.float32),
                           quats=np.tile(np.array([0, 0, 0, 1], np.float32), (n, 1)),
                           opacity=np.full(n, 0.5, np.float32),
                           colors=rng.uniform(0, 1, (n, 3)).astype(np.float32), sh_degree=-1, cameras=[cam],
                           tile_size=8)
    batch = GaussBatch(n, [cam], 8, -1, pair_capacity=4096, device=dev, check_overflow=False)
    batch.forward(params_of(sc, dev))
    flags, needed, pairs = batch.status()
    assert flags & 1
    assert pairs == n * 512 * 512
    assert needed > 4096
