"""The C-ABI library loads without a GPU and exports every entry point that
include/*.h declares; argument validation works without touching a GPU."""
import ctypes
import os
import re

import pytest

from dsplat import _native as N

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    names = set()
    for f in os.listdir(os.path.join(ROOT, "include")):
        if f.endswith(".h"):
            src = open(os.path.join(ROOT, "include", f)).read()
            names |= set(re.findall(r"^\s*(?:int|size_t|uint64_t|const char\*)\s+(dsplat_\w+)\s*\(", src, re.M))
    return names


def test_library_loads_and_exports_all_symbols():
    L = N.lib()
    names = _declared()
    assert len(names) >= 19
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing
    assert set(N.SIGNATURES) >= names, sorted(names - set(N.SIGNATURES))


def test_version_and_argument_checks_need_no_gpu():
    L = N.lib()
    assert b"sm_100a" in L.dsplat_version()
    # unsupported tile size is rejected before any CUDA call
    rc = L.dsplat_gauss_rasterize_pnt2splat2(None, 4, 4, None, None, None, None, None, None, 12, None, None,
                                             None, None)
    assert rc == 5 and b"tile_size" in L.dsplat_last_error()
    lay = N.BatchLayout()
    views = (N.View * 1)()
    views[0].width, views[0].height = 100, 50
    assert L.dsplat_gauss_batch_layout(1000, 1, views, 16, 0, 5000, ctypes.byref(lay)) == 0
    assert lay.num_items == 7 * 4 and lay.num_pix == 5000 and lay.total_bytes > 0
    assert L.dsplat_gauss_batch_layout(1000, 0, views, 16, 0, 5000, ctypes.byref(lay)) == 1
    assert L.dsplat_gauss_batch_layout(1000, 1, views, 24, 0, 5000, ctypes.byref(lay)) == 5
    assert L.dsplat_gauss_batch_layout(1000, 1, views, 16, 3, 5000, ctypes.byref(lay)) == 5
    assert L.dsplat_tile2idx_workspace_size(1000, 7, 4, 100) > L.dsplat_tile2idx_workspace_size(1000, 7, 4, 0)


def test_layout_grows_with_capacity_and_views():
    L = N.lib()
    v = (N.View * 2)()
    for i in range(2):
        v[i].width, v[i].height = 640, 480
    a, b = N.BatchLayout(), N.BatchLayout()
    L.dsplat_gauss_batch_layout(10000, 1, v, 16, 0, 1 << 16, ctypes.byref(a))
    L.dsplat_gauss_batch_layout(10000, 2, v, 16, 0, 1 << 20, ctypes.byref(b))
    assert b.total_bytes > a.total_bytes and b.num_items == 2 * a.num_items
