"""Torch-facing wrappers of the batched Gaussian pipeline (C ABI in dsplat.h).

``GaussBatch`` owns one workspace for a fixed list of cameras and drives
``dsplat_gauss_batch_forward`` / ``_backward``.  ``render`` is the
differentiable entry point (a ``torch.autograd.Function``).  Torch is used
for device memory and the current stream only; every stage runs in
libdsplat.so.
"""
from __future__ import annotations

import ctypes
from typing import Dict, List, Optional, Sequence

import numpy as np
import torch

from . import _native as N
from .scenes import Camera

PARAM_NAMES = ("means", "log_scales", "quats", "opacity", "colors")


def _stream_ptr(device: torch.device) -> int:
    return torch.cuda.current_stream(device).cuda_stream


def _require_cuda(t: torch.Tensor, name: str) -> None:
    if not t.is_cuda:
        raise RuntimeError(f"{name}: del-splat-b200 runs on CUDA devices only (got {t.device})")
    if t.dtype != torch.float32:
        raise TypeError(f"{name}: expected float32, got {t.dtype}")
    if not t.is_contiguous():
        raise ValueError(f"{name}: expected a contiguous tensor")


def make_views(cameras: Sequence[Camera]):
    arr = (N.View * len(cameras))()
    for i, c in enumerate(cameras):
        arr[i].mvp[:] = [float(x) for x in np.asarray(c.mvp, np.float32).reshape(16)]
        arr[i].campos[:] = [float(x) for x in np.asarray(c.campos, np.float32).reshape(3)]
        arr[i].width = int(c.width)
        arr[i].height = int(c.height)
    return arr


def params_struct(p: Dict[str, torch.Tensor], sh_degree: int) -> N.GaussParams:
    for k in PARAM_NAMES:
        _require_cuda(p[k], k)
    n = p["means"].shape[0]
    return N.GaussParams(n, sh_degree, p["means"].data_ptr(), p["log_scales"].data_ptr(), p["quats"].data_ptr(),
                         p["opacity"].data_ptr(), p["colors"].data_ptr())


class GaussBatch:
    """Workspace + launches for rendering N Gaussians into a fixed set of views.

    The forward state (tile lists, stop positions, transmittance) lives in the
    workspace until the next forward; ``backward`` uses the latest forward.
    """

    def __init__(self, num_pnt: int, cameras: Sequence[Camera], tile_size: int = 16, sh_degree: int = 3,
                 pair_capacity: int = 1 << 20, device: Optional[torch.device] = None, pixels_per_lane: int = 0,
                 check_overflow: bool = True):
        self.device = torch.device(device or "cuda")
        # render() reads the overflow flag after each forward (one host sync);
        # False keeps the forward free of host syncs (graph capture) and
        # leaves the check to the caller (status())
        self.check_overflow = bool(check_overflow)
        self.generation = 0  # forwards issued on this batch (the autograd render checks it)
        self.n = int(num_pnt)
        self.cameras = list(cameras)
        self.tile_size = int(tile_size)
        self.ppl = int(pixels_per_lane)
        self.sh_degree = int(sh_degree)
        self.views = make_views(self.cameras)
        self.num_views = len(self.cameras)
        self.pix_offsets = np.cumsum([0] + [c.width * c.height for c in self.cameras]).tolist()
        self._alloc(int(pair_capacity))

    # ----------------------------------------------------------- workspace
    def _alloc(self, capacity: int) -> None:
        self.capacity = max(1, capacity)
        L = N.BatchLayout()
        N.check(N.lib().dsplat_gauss_batch_layout(self.n, self.num_views, self.views, self.tile_size, self.ppl,
                                                  self.capacity, ctypes.byref(L)), "batch_layout")
        self.layout = L
        self.ws = torch.empty(int(L.total_bytes), dtype=torch.uint8, device=self.device)
        self.out_rgb = torch.empty(int(L.num_pix) * 3, dtype=torch.float32, device=self.device)

    def ensure_capacity(self, params: Dict[str, torch.Tensor], slack: float = 1.05) -> int:
        """Run one forward, read the capacity it needed and grow the lists; returns the tile pairs."""
        self.forward(params)
        flags, needed, pairs = self.status()
        if needed > self.capacity:
            self._alloc(int(needed * slack) + 1024)
            self.forward(params)
            flags, needed, pairs = self.status()
            if flags:
                raise RuntimeError("list capacity still exceeded after resize")
        return pairs

    def status(self):
        """(flags, capacity needed, tile pairs) of the last forward (synchronises)."""
        f = N.c_u32(0)
        need = N.c_u64(0)
        p = N.c_u64(0)
        N.lib().dsplat_gauss_batch_status(_stream_ptr(self.device), self.ws.data_ptr(), ctypes.byref(f),
                                          ctypes.byref(need), ctypes.byref(p))
        return int(f.value), int(need.value), int(p.value)

    # ----------------------------------------------------------- launches
    def forward(self, params: Dict[str, torch.Tensor], target: Optional[torch.Tensor] = None,
                out_alpha: Optional[torch.Tensor] = None, out_rgb: Optional[torch.Tensor] = None) -> torch.Tensor:
        ps = params_struct(params, self.sh_degree)
        out = self.out_rgb if out_rgb is None else out_rgb
        if target is not None:
            _require_cuda(target, "target")
        N.check(N.lib().dsplat_gauss_batch_forward(
            _stream_ptr(self.device), ctypes.byref(ps), self.num_views, self.views, self.tile_size, self.ppl,
            self.capacity, self.ws.data_ptr(), self.ws.numel(), out.data_ptr(),
            out_alpha.data_ptr() if out_alpha is not None else None,
            target.data_ptr() if target is not None else None), "batch_forward")
        self.generation += 1
        return out

    def backward(self, params: Dict[str, torch.Tensor], grads: Dict[str, torch.Tensor],
                 grad_rgb: Optional[torch.Tensor] = None) -> None:
        ps = params_struct(params, self.sh_degree)
        for k in PARAM_NAMES:
            _require_cuda(grads[k], "grad " + k)
        gs = N.GaussGrads(grads["means"].data_ptr(), grads["log_scales"].data_ptr(), grads["quats"].data_ptr(),
                          grads["opacity"].data_ptr(), grads["colors"].data_ptr())
        if grad_rgb is not None:
            _require_cuda(grad_rgb, "grad_rgb")
        N.check(N.lib().dsplat_gauss_batch_backward(
            _stream_ptr(self.device), ctypes.byref(ps), self.num_views, self.views, self.tile_size, self.ppl,
            self.capacity, self.ws.data_ptr(), self.ws.numel(), grad_rgb.data_ptr() if grad_rgb is not None else None,
            ctypes.byref(gs)), "batch_backward")

    # ----------------------------------------------------------- views of the workspace
    def _ws(self, off: int, count: int, dtype: torch.dtype) -> torch.Tensor:
        itemsize = torch.empty((), dtype=dtype).element_size()
        return self.ws[off: off + count * itemsize].view(dtype)

    def images(self, flat: Optional[torch.Tensor] = None) -> List[torch.Tensor]:
        flat = self.out_rgb if flat is None else flat
        out = []
        for v, c in enumerate(self.cameras):
            a, b = self.pix_offsets[v], self.pix_offsets[v + 1]
            out.append(flat[3 * a: 3 * b].view(c.height, c.width, 3))
        return out

    def per_pixel(self, name: str) -> List[torch.Tensor]:
        L = self.layout
        off = {"T": L.off_pix_T, "stop": L.off_pix_stop}[name]
        dt = torch.float32 if name == "T" else torch.int32
        flat = self._ws(off, int(L.num_pix), dt)
        return [flat[self.pix_offsets[v]: self.pix_offsets[v + 1]].view(c.height, c.width)
                for v, c in enumerate(self.cameras)]

    def tile_lists(self, view: int):
        """Per-tile lists of one view in the reference's format, rebuilt on the host
        from the superblock lists: (tile2idx [T+1] u32, idx2pnt [P] u32,
        stop [H,W] i64 = each pixel's stop position as an idx2pnt position)."""
        L = self.layout
        ts = self.tile_size

        def grid(v):
            tw_, th_ = (self.cameras[v].width + ts - 1) // ts, (self.cameras[v].height + ts - 1) // ts
            side_ = 1 << int(L.sb_log2[v])
            return tw_, th_, side_, (tw_ + side_ - 1) // side_, (th_ + side_ - 1) // side_

        sb_base = sum(grid(v)[3] * grid(v)[4] for v in range(view))
        c = self.cameras[view]
        tw, th, side, sbw, _ = grid(view)
        ch = int(L.sb_chunks)
        starts = self._ws(L.off_sb_start, int(L.num_sb) * ch + 1, torch.int32).cpu().numpy().view(np.uint32)
        ent = self._ws(L.off_sb_list, 2 * self.capacity, torch.int32).cpu().numpy().view(np.uint32).reshape(-1, 2)
        stop_sb = self.per_pixel("stop")[view].cpu().numpy().view(np.uint32).astype(np.int64)
        tile2idx = np.zeros(tw * th + 1, np.uint32)
        lists, positions = [], []
        for t in range(tw * th):
            tx, ty = t % tw, t // tw
            sb = sb_base + (ty // side) * sbw + (tx // side)
            s, e = int(starts[sb * ch]), int(starts[(sb + 1) * ch])
            lr = ent[s:e, 1]
            lx, ly = tx % side, ty % side
            m = (lx >= (lr & 15)) & (lx < ((lr >> 8) & 15)) & (ly >= ((lr >> 4) & 15)) & (ly < (lr >> 12))
            lists.append(ent[s:e, 0][m])
            positions.append(s + np.nonzero(m)[0])
            tile2idx[t + 1] = tile2idx[t] + int(m.sum())
        idx2pnt = np.concatenate(lists).astype(np.uint32) if lists else np.zeros(0, np.uint32)
        stop = np.zeros((c.height, c.width), np.int64)
        for t in range(tw * th):
            tx, ty = t % tw, t // tw
            ys, xs = slice(ty * ts, min(ty * ts + ts, c.height)), slice(tx * ts, min(tx * ts + ts, c.width))
            stop[ys, xs] = tile2idx[t] + np.searchsorted(positions[t], stop_sb[ys, xs])
        return tile2idx, idx2pnt, stop

    def slab_loss(self) -> torch.Tensor:
        """Partial L2 losses of the last forward with a target (sum = loss)."""
        L = self.layout
        return self._ws(L.off_slab_loss, int(L.num_items) * int(L.slabs_per_tile), torch.float32)

    def grad2d(self) -> torch.Tensor:
        return self._ws(self.layout.off_grad2d, self.num_views * self.n * 12, torch.float32).view(
            self.num_views, self.n, 12)

    def records(self) -> torch.Tensor:
        """[V, N, 12] per-view 2D records of the last forward; rows of points
        whose tile span in that view is empty are not written."""
        return self._ws(self.layout.off_rec, self.num_views * self.n * 12, torch.float32).view(
            self.num_views, self.n, 12)


class _RenderFn(torch.autograd.Function):
    @staticmethod
    def forward(ctx, means, log_scales, quats, opacity, colors, batch: GaussBatch):
        params = dict(means=means.detach(), log_scales=log_scales.detach(), quats=quats.detach(),
                      opacity=opacity.detach(), colors=colors.detach())
        out = torch.empty(int(batch.layout.num_pix) * 3, dtype=torch.float32, device=means.device)
        batch.forward(params, out_rgb=out)
        if batch.check_overflow:
            flags, needed, _ = batch.status()
            if flags:  # the lists outgrew the capacity: grow once and render again
                batch._alloc(int(needed * 1.05) + 1024)
                batch.forward(params, out_rgb=out)
                flags, needed, _ = batch.status()
                if flags:
                    raise RuntimeError(f"tile-list capacity exceeded ({needed} entries needed, "
                                       f"{batch.capacity} available)")
        ctx.batch = batch
        ctx.generation = batch.generation
        ctx.save_for_backward(means, log_scales, quats, opacity, colors)
        return out

    @staticmethod
    def backward(ctx, grad_rgb):
        if ctx.batch.generation != ctx.generation:
            # the batch's workspace (stop positions, final transmittance, tile
            # lists) now holds a later forward's state
            raise RuntimeError("render(): the batch ran another forward before this render's backward; "
                               "call backward first or render with a separate GaussBatch")
        means, log_scales, quats, opacity, colors = ctx.saved_tensors
        params = dict(means=means.detach(), log_scales=log_scales.detach(), quats=quats.detach(),
                      opacity=opacity.detach(), colors=colors.detach())
        grads = {k: torch.zeros_like(v) for k, v in params.items()}
        ctx.batch.backward(params, grads, grad_rgb.contiguous())
        return grads["means"], grads["log_scales"], grads["quats"], grads["opacity"], grads["colors"], None


def render(means, log_scales, quats, opacity, colors, batch: GaussBatch) -> List[torch.Tensor]:
    """Differentiable render of all views of ``batch``; returns [H,W,3] images.

    The backward of the returned images runs the hand-written backward
    rasteriser and projection backward.  Call backward before the next render
    on the same batch (the forward state lives in its workspace); a backward
    after a later forward on the batch raises RuntimeError.
    """
    flat = _RenderFn.apply(means, log_scales, quats, opacity, colors, batch)
    return batch.images(flat)


def adam_step(param: torch.Tensor, grad: torch.Tensor, exp_avg: torch.Tensor, exp_avg_sq: torch.Tensor,
              lr: float, beta1: float, beta2: float, eps: float, step: int) -> None:
    N.check(N.lib().dsplat_adam_step(_stream_ptr(param.device), param.numel(), param.data_ptr(), grad.data_ptr(),
                                     exp_avg.data_ptr(), exp_avg_sq.data_ptr(), lr, beta1, beta2, eps, step),
            "adam_step")


def _tensors(d: Dict[str, torch.Tensor]) -> N.GaussTensors:
    for k in PARAM_NAMES:
        _require_cuda(d[k], k)
    return N.GaussTensors(*(d[k].data_ptr() for k in PARAM_NAMES))


class Adam:
    """Fused Adam over the five parameter tensors of a scene: one
    ``dsplat_gauss_adam_step`` launch per step, the same update as
    ``torch.optim.Adam`` (no weight decay).  The step count lives on the
    device, so the update can sit inside a captured CUDA graph.  Opacity is
    kept in [0, 0.999] after every update (the blend needs alpha < 1)."""

    def __init__(self, params: Dict[str, torch.Tensor], sh_degree: int, lr: float = 1e-3, betas=(0.9, 0.999),
                 eps: float = 1e-8):
        self.params, self.sh_degree = params, int(sh_degree)
        self.lr, self.betas, self.eps = float(lr), (float(betas[0]), float(betas[1])), float(eps)
        self.exp_avg = {k: torch.zeros_like(v) for k, v in params.items()}
        self.exp_avg_sq = {k: torch.zeros_like(v) for k, v in params.items()}
        self.step_count = torch.zeros(1, dtype=torch.int32, device=params["means"].device)

    def step(self, grads: Dict[str, torch.Tensor]) -> None:
        p = self.params
        g = N.GaussGrads(*(grads[k].data_ptr() for k in PARAM_NAMES))
        N.check(N.lib().dsplat_gauss_adam_step(
            _stream_ptr(p["means"].device), p["means"].shape[0], self.sh_degree, ctypes.byref(_tensors(p)),
            ctypes.byref(g), ctypes.byref(_tensors(self.exp_avg)), ctypes.byref(_tensors(self.exp_avg_sq)),
            self.lr, self.betas[0], self.betas[1], self.eps, self.step_count.data_ptr()), "gauss_adam_step")


class CapturedStep:
    """A whole batched training step (zero grads, forward with L2 loss,
    backward, and the optimizer's update when one is given) captured into one
    CUDA graph.  The batch's forward has no host synchronisation (fixed list
    capacity, overflow reported by a device flag), so the step replays with
    zero host work per kernel."""

    def __init__(self, batch: GaussBatch, params: Dict[str, torch.Tensor], grads: Dict[str, torch.Tensor],
                 target: torch.Tensor, warmup: int = 2, optimizer: Optional[Adam] = None,
                 out_rgb: Optional[torch.Tensor] = None):
        self.batch, self.params, self.grads, self.target = batch, params, grads, target
        self.optimizer = optimizer
        self.out_rgb = out_rgb  # None: the batch's own image buffer
        side = torch.cuda.Stream(batch.device)
        side.wait_stream(torch.cuda.current_stream(batch.device))
        with torch.cuda.stream(side):
            for _ in range(warmup):
                self._step()
        torch.cuda.current_stream(batch.device).wait_stream(side)
        torch.cuda.synchronize(batch.device)
        self.graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(self.graph):
            self._step()
        torch.cuda.synchronize(batch.device)

    def _step(self):
        for g in self.grads.values():
            g.zero_()
        self.batch.forward(self.params, target=self.target, out_rgb=self.out_rgb)
        self.batch.backward(self.params, self.grads)
        if self.optimizer is not None:
            self.optimizer.step(self.grads)

    def replay(self):
        self.graph.replay()
