"""The allocation-free point z-buffer entry point against the allocating one.

dsplat_point_rasterize_pix_zbuffer_noalloc exists for callers that cannot lend
the library device memory (a plug-in whose host application owns every GPU
allocation, or a loop that must not call cudaMalloc): it keeps its 64-bit
depth|index keys in a fixed 2^20-entry array inside libdsplat.so instead of a
caller workspace.  This file is collected last on purpose, so a run that stops
at the first failure has already run every other test; it also passes when
run alone in a fresh process.

Checked through the C ABI: two calls in a row (a larger image, then a smaller
one, so stale keys from the first call would show) give exactly the
allocating entry point's pixels, unit depths and winners (the same integer
keys decide both: tolerance 0), and an image above the limit is rejected.
"""
import ctypes

import numpy as np
import pytest
import torch

from dsplat import _native as N

pytestmark = pytest.mark.gpu
MAX_PIXELS = 1 << 20


def _points(seed, n, w, h):
    rng = np.random.default_rng(seed)
    xyd = np.stack([rng.uniform(-2, w + 2, n), rng.uniform(-2, h + 2, n), rng.uniform(-1.05, 1.05, n)], 1)
    xyd = xyd.astype(np.float32)
    xyd[::97, 2] = xyd[0, 2]  # depth ties: the larger index must win in both
    rgb = rng.uniform(0, 1, (n, 3)).astype(np.float32)
    return xyd, rgb


def _run(fn_name, dev, xyd, rgb, w, h):
    L = N.lib()
    st = torch.cuda.current_stream(dev).cuda_stream
    x = torch.from_numpy(xyd).to(dev)
    c = torch.from_numpy(rgb).to(dev)
    pix = torch.full((h, w, 3), -7.0, device=dev)
    depth = torch.empty((h, w), device=dev)
    win = torch.empty((h, w), dtype=torch.int32, device=dev)
    n = xyd.shape[0]
    if fn_name == "alloc":
        zbuf = torch.empty(w * h, dtype=torch.int64, device=dev)
        rc = L.dsplat_point_rasterize_pix_zbuffer(st, n, x.data_ptr(), c.data_ptr(), pix.data_ptr(), depth.data_ptr(),
                                                  win.data_ptr(), w, h, zbuf.data_ptr())
    else:
        rc = L.dsplat_point_rasterize_pix_zbuffer_noalloc(st, n, x.data_ptr(), c.data_ptr(), pix.data_ptr(),
                                                          depth.data_ptr(), win.data_ptr(), w, h)
    assert rc == 0, L.dsplat_last_error()
    torch.cuda.synchronize(dev)
    return pix.cpu().numpy(), depth.cpu().numpy(), win.cpu().numpy()


def test_noalloc_point_zbuffer_matches_allocating_entry_point(dev):
    for seed, (w, h), n in ((1, (1024, 1000), 400000), (2, (320, 200), 30000)):
        xyd, rgb = _points(seed, n, w, h)
        ref = _run("alloc", dev, xyd, rgb, w, h)
        got = _run("noalloc", dev, xyd, rgb, w, h)
        for a, b in zip(ref, got):
            assert np.array_equal(a, b)
        assert (got[2] >= 0).any() and (got[2] < 0).any()


def test_noalloc_point_zbuffer_rejects_images_over_the_limit(dev):
    L = N.lib()
    x = torch.zeros((4, 3), device=dev)
    rc = L.dsplat_point_rasterize_pix_zbuffer_noalloc(torch.cuda.current_stream(dev).cuda_stream, 4, x.data_ptr(),
                                                      x.data_ptr(), None, None, None, 1025, 1024)
    assert rc == 1
    assert b"exceeds" in L.dsplat_last_error()
    assert 1025 * 1024 > MAX_PIXELS
