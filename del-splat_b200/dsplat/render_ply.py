"""Render a 3D Gaussian Splatting PLY file from orbit cameras.

    python -m dsplat.render_ply scene.ply [--views 8] [--width 1280] [--height 720]
                                [--tile 8] [--out DIR]

Reads the standard 3DGS layout (dsplat.ply.read_3d_gauss_splat: position,
f_dc + 45 f_rest SH coefficients, logit opacity, log scale, quaternion),
centres and scales the scene into the unit cube, places `--views` cameras
on a radius-3 sphere looking at it (seeded), renders all views in one
batched forward, writes one PNG per view, and times the CUDA-graph captured
forward + backward (L2 loss against a random target) of the batch.  The
del-splat-cpu examples do the same with a single camera
(examples/cpu_splat_gauss_ply.rs).
"""
from __future__ import annotations

import argparse
import json
import os

import numpy as np
import torch

from . import ply, scenes
from .gauss import CapturedStep, GaussBatch
from .image import save_png


def load_scene(path: str, cameras) -> scenes.GaussScene:
    d = ply.read_3d_gauss_splat(path)
    ctr = d["xyz"].mean(0)
    ext = float(np.percentile(np.abs(d["xyz"] - ctr), 95, axis=0).max()) or 1.0
    means = ((d["xyz"] - ctr) / ext * 0.8).astype(np.float32)
    log_scales = (d["log_scale"] + np.float32(np.log(0.8 / ext))).astype(np.float32)
    return scenes.GaussScene(means, log_scales, d["quat"], d["opacity"], d["sh_coeffs"], 3, cameras, 8)


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("ply")
    ap.add_argument("--views", type=int, default=8)
    ap.add_argument("--width", type=int, default=1280)
    ap.add_argument("--height", type=int, default=720)
    ap.add_argument("--tile", type=int, default=8)
    ap.add_argument("--seed", type=int, default=7)
    ap.add_argument("--out", default="renders")
    ap.add_argument("--steps", type=int, default=50)
    a = ap.parse_args(argv)
    cams = scenes.sphere_cameras(np.random.default_rng(a.seed), a.views, 3.0, [(a.width, a.height)])
    sc = load_scene(a.ply, cams)
    dev = torch.device("cuda")
    p = {k: torch.from_numpy(np.ascontiguousarray(v)).to(dev) for k, v in dict(
        means=sc.means, log_scales=sc.log_scales, quats=sc.quats, opacity=sc.opacity,
        colors=sc.colors.reshape(sc.n, -1)).items()}
    b = GaussBatch(sc.n, cams, a.tile, 3, pair_capacity=1 << 20, device=dev)
    b.ensure_capacity(p)
    tgt = torch.rand(int(b.layout.num_pix) * 3, device=dev)
    b.forward(p, target=tgt)
    os.makedirs(a.out, exist_ok=True)
    for v, img in enumerate(b.images()):
        save_png(os.path.join(a.out, f"view{v:02d}.png"), img)
    grads = {k: torch.zeros_like(x) for k, x in p.items()}
    step = CapturedStep(b, p, grads, tgt)
    for _ in range(5):
        step.replay()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(a.steps):
        step.replay()
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / a.steps
    flags, _, pairs = b.status()
    print(json.dumps({"gaussians": sc.n, "views": a.views, "resolution": f"{a.width}x{a.height}",
                      "fwd_bwd_ms_per_step": ms, "views_per_s": a.views / (ms / 1e3), "tile_pairs": int(pairs),
                      "capacity_overflow": bool(flags & 1), "images": a.out}))


if __name__ == "__main__":
    main()
