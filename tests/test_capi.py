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


def _sb_rule(tile_w, tile_h, min_per_view=200, max_per_view=4096):
    """The superblock side rule: the largest side (8 tiles at most) that still
    splits the view into >= min_per_view superblocks, within 255 superblocks
    per side and max_per_view per view."""
    s = 3
    while s > 0:
        cw, ch = -(-tile_w // (1 << s)), -(-tile_h // (1 << s))
        if cw * ch >= min_per_view:
            break
        nw, nh = -(-tile_w // (1 << (s - 1))), -(-tile_h // (1 << (s - 1)))
        if nw > 255 or nh > 255 or nw * nh > max_per_view:
            break
        s -= 1
    return s


@pytest.mark.parametrize("ts", [8, 16, 32])
def test_superblock_side_per_view_follows_the_rule(ts):
    L = N.lib()
    sizes = [(320, 240), (640, 480), (1280, 720), (1920, 1080), (64, 64), (16000, 8), (4096, 4096), (1, 1)]
    v = (N.View * len(sizes))()
    for i, (w, h) in enumerate(sizes):
        v[i].width, v[i].height = w, h
    lay = N.BatchLayout()
    assert L.dsplat_gauss_batch_layout(5000, len(sizes), v, ts, 0, 1 << 16, ctypes.byref(lay)) == 0
    total_sb = 0
    for i, (w, h) in enumerate(sizes):
        tw, th = -(-w // ts), -(-h // ts)
        s = _sb_rule(tw, th)
        assert lay.sb_log2[i] == s, (w, h, ts, lay.sb_log2[i], s)
        total_sb += -(-tw // (1 << s)) * -(-th // (1 << s))
    assert lay.num_sb == total_sb
    # the bench's views at 8x8 tiles: 1, 2, 3, 3 (64-pixel superblocks at 720p/1080p)
    if ts == 8:
        assert list(lay.sb_log2[:4]) == [1, 2, 3, 3]
        # more than 255 superblocks of 8 tiles in a row is rejected
        v[5].width = 16384
        assert L.dsplat_gauss_batch_layout(5000, len(sizes), v, ts, 0, 1 << 16, ctypes.byref(lay)) == 5
        assert b"superblocks" in L.dsplat_last_error()


def test_plain_c_client_builds_and_runs(tmp_path):
    """The header and library are usable from C alone (the boundary a Rust or
    C host binds): compile tests/c_abi_smoke.c with gcc, link libdsplat.so."""
    import shutil
    import subprocess
    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        pytest.skip("no C compiler")
    exe = tmp_path / "c_abi_smoke"
    libdir = os.path.dirname(N.LIB_PATH)
    r = subprocess.run([cc, "-std=c99", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"),
                        os.path.join(ROOT, "tests", "c_abi_smoke.c"), "-L", libdir, "-ldsplat",
                        "-Wl,-rpath," + libdir, "-o", str(exe)], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    run = subprocess.run([str(exe)], capture_output=True, text=True, timeout=120)
    assert run.returncode == 0, run.stdout + run.stderr
    assert "sm_100a" in run.stdout and "rejected" in run.stdout


def _c_decls():
    """name -> number of parameters, for every entry point in include/*.h."""
    out = {}
    for f in os.listdir(os.path.join(ROOT, "include")):
        if not f.endswith(".h"):
            continue
        src = re.sub(r"/\*.*?\*/", "", open(os.path.join(ROOT, "include", f)).read(), flags=re.S)
        for m in re.finditer(r"(?:int|size_t|uint64_t|const char\*)\s+(dsplat_\w+)\s*\(([^)]*)\)\s*;", src):
            args = m.group(2).strip()
            out[m.group(1)] = 0 if args in ("", "void") else args.count(",") + 1
    return out


def test_rust_shim_declarations_match_the_header():
    """del-splat_b200/rust (the del-splat-cudarc replacement, built where cargo
    exists) declares the C ABI by hand; every extern "C" function it declares
    must exist in include/dsplat.h with the same number of parameters, and it
    must cover the drop-in entry points its wrappers call."""
    src = open(os.path.join(ROOT, "del-splat_b200", "rust", "src", "ffi.rs")).read()
    rust = {}
    for m in re.finditer(r"pub fn (dsplat_\w+)\s*\(([^)]*)\)", src, re.S):
        args = [a for a in m.group(2).split(",") if a.strip()]
        rust[m.group(1)] = len(args)
    header = _c_decls()
    assert len(rust) >= 17
    for name, n in rust.items():
        assert name in header, name
        assert header[name] == n, (name, n, header[name])
    wrappers = (open(os.path.join(ROOT, "del-splat_b200", "rust", "src", "splat_gauss.rs")).read() +
                open(os.path.join(ROOT, "del-splat_b200", "rust", "src", "splat_circle.rs")).read())
    called = set(re.findall(r"ffi::(dsplat_\w+)\(", wrappers))
    assert called <= set(rust)
    for fn in ("pnt2splat3_to_pnt2splat2", "rasterize_pnt2splat2", "tile2idx_idx2pnt", "splat"):
        assert re.search(r"pub fn " + fn + r"\(", wrappers), fn
