"""Autotuner for the batched Gaussian path: picks the tile size (8, 16, 32)
and the rasteriser's pixels per lane by timing real forward + backward steps
of the caller's workload, and caches the choice per (GPU, point-count bucket,
SH degree, set of resolutions).  Results never depend on the choice; only
throughput does.
"""
from __future__ import annotations

import json
import math
import os
from typing import Dict, Iterable, Optional, Sequence, Tuple

import torch

from .gauss import GaussBatch
from .scenes import Camera

CANDIDATES: Tuple[Tuple[int, int], ...] = ((8, 1), (8, 2), (16, 2), (16, 4), (32, 4))
_memo: Dict[str, Tuple[int, int]] = {}


def _key(n: int, cameras: Sequence[Camera], sh_degree: int, device: torch.device) -> str:
    res = sorted({(c.width, c.height) for c in cameras})
    bucket = int(math.log2(max(n, 1)))
    return json.dumps([torch.cuda.get_device_name(device), bucket, sh_degree, res, len(cameras)])


def _cache_path() -> str:
    return os.environ.get("DSPLAT_AUTOTUNE_CACHE", os.path.join(os.path.expanduser("~"), ".cache",
                                                                  "dsplat_autotune.json"))


def _load() -> dict:
    try:
        with open(_cache_path()) as f:
            return json.load(f)
    except (OSError, ValueError):
        return {}


def _store(key: str, val) -> None:
    d = _load()
    d[key] = val
    try:
        os.makedirs(os.path.dirname(_cache_path()), exist_ok=True)
        with open(_cache_path(), "w") as f:
            json.dump(d, f)
    except OSError:
        pass


def time_config(params: Dict[str, torch.Tensor], cameras: Sequence[Camera], sh_degree: int, tile_size: int,
                ppl: int, target: torch.Tensor, steps: int = 3, device: Optional[torch.device] = None) -> float:
    """Milliseconds per fwd+bwd step of one (tile size, pixels per lane) configuration."""
    dev = device or params["means"].device
    n = params["means"].shape[0]
    batch = GaussBatch(n, cameras, tile_size, sh_degree, pair_capacity=1 << 20, device=dev, pixels_per_lane=ppl)
    batch.ensure_capacity(params)
    grads = {k: torch.zeros_like(v) for k, v in params.items()}

    def step():
        batch.forward(params, target=target)
        batch.backward(params, grads)

    step()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize(dev)
    e0.record()
    for _ in range(steps):
        step()
    e1.record()
    torch.cuda.synchronize(dev)
    ms = e0.elapsed_time(e1) / steps
    del batch, grads
    torch.cuda.empty_cache()
    return ms


def tune(params: Dict[str, torch.Tensor], cameras: Sequence[Camera], sh_degree: int, target: torch.Tensor,
         candidates: Iterable[Tuple[int, int]] = CANDIDATES, use_cache: bool = True,
         report: Optional[dict] = None) -> Tuple[int, int]:
    """Best (tile_size, pixels_per_lane) for this workload (timed, cached)."""
    dev = params["means"].device
    key = _key(params["means"].shape[0], cameras, sh_degree, dev)
    if use_cache:
        if key in _memo:
            return _memo[key]
        hit = _load().get(key)
        if hit:
            _memo[key] = (int(hit[0]), int(hit[1]))
            return _memo[key]
    timings = {}
    for ts, ppl in candidates:
        timings[f"{ts}/{ppl}"] = time_config(params, cameras, sh_degree, ts, ppl, target)
    best = min(timings, key=timings.get)
    choice = tuple(int(x) for x in best.split("/"))
    _memo[key] = choice
    _store(key, list(choice))
    if report is not None:
        report.update({"timings_ms": timings, "choice": best})
    return choice
