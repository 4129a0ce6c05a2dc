"""Helpers shared by the GPU parity tests."""
import numpy as np
import torch


def T(a, dev, dtype=None):
    t = torch.from_numpy(np.ascontiguousarray(a))
    if dtype is not None:
        t = t.to(dtype)
    return t.to(dev)


def U32(t):
    return t.detach().cpu().numpy().view(np.uint32)


def F(t):
    return t.detach().cpu().numpy()


def params_of(scene, dev):
    return dict(means=T(scene.means, dev), log_scales=T(scene.log_scales, dev), quats=T(scene.quats, dev),
                opacity=T(scene.opacity, dev), colors=T(scene.colors.reshape(scene.n, -1), dev))
