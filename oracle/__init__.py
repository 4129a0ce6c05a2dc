"""CPU oracle for del-splat's splatting path -- TEST INFRASTRUCTURE ONLY.

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU arms may
import this package.  It wraps two shared libraries with ctypes:

* ``oracle/_build/liboracle.so`` -- the C++ restatement (oracle/oracle.cpp) of
  del-splat-cpu and the reference CUDA kernels, plus an FP64 gradient oracle.
* ``oracle/_ref/libdsplat_ref.so`` -- the reference's own
  ``tile_acceleration.h``, ``splat_point.cu``, ``splat_gauss.cu`` and
  ``splat_circle.cu`` compiled as host C++ (oracle/ref/), used to pin the
  restatement.  Present only when it was built from a del-splat checkout;
  ``ref_available()`` says whether it is.

Parity status: tile spans, key bits, the point z-buffer, the blend (with the
C library's expf and the kernel's double stop test) and the way the
reference's kernels compose the del-geo helpers are pinned against the
reference's own code; the del-geo helpers themselves (absent crate) are a
restatement whose parity with upstream is unpinned.

Blend modes (``mode`` arguments): 0 is the product's arithmetic -- del-splat-
cpu's f32 operations with a correctly rounded exp and the f32 stop test
``alpha_sum > 0.999f``; ``BLEND_LIBM_EXP`` uses the C library's expf (what
del-splat-cpu's ``f32::exp`` calls), ``BLEND_CUDA_STOP`` the CUDA kernel's
double stop test (``alpha_sum >= 0.999f``).
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from typing import Optional

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = os.path.join(_HERE, "_build", "liboracle.so")
_REF = os.path.join(_HERE, "_ref", "libdsplat_ref.so")

_lib: Optional[ctypes.CDLL] = None
_ref: Optional[ctypes.CDLL] = None

_f32p = ctypes.POINTER(ctypes.c_float)
_f64p = ctypes.POINTER(ctypes.c_double)
_u32p = ctypes.POINTER(ctypes.c_uint32)
_i32p = ctypes.POINTER(ctypes.c_int32)
_u64p = ctypes.POINTER(ctypes.c_uint64)
_u8p = ctypes.POINTER(ctypes.c_uint8)
_i64 = ctypes.c_int64
_int = ctypes.c_int


BLEND_LIBM_EXP = 1
BLEND_CUDA_STOP = 2


def build(reference_root: Optional[str] = None) -> None:
    """Compile the oracle, and the pin when ``reference_root`` (or the
    DSPLAT_REFERENCE_ROOT environment variable) names a del-splat checkout."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    ref = reference_root or os.environ.get("DSPLAT_REFERENCE_ROOT")
    if ref and os.path.isdir(os.path.join(ref, "del-splat-cuda-kernels")):
        subprocess.run(["make", "-s", "-C", os.path.join(_HERE, "ref"), f"REF={ref}"], check=True)


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB):
            build()
        _lib = ctypes.CDLL(_LIB)
        _declare(_lib)
    return _lib


def ref_available() -> bool:
    return os.path.exists(_REF)


def ref() -> ctypes.CDLL:
    global _ref
    if _ref is None:
        _ref = ctypes.CDLL(_REF)
        _ref.ref_tiles_count.restype = ctypes.c_uint64
        _ref.ref_tiles_count.argtypes = [_i64, _f32p, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32, _u32p]
        _ref.ref_tiles_fill.restype = None
        _ref.ref_tiles_fill.argtypes = [_i64, _f32p, _f32p, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32, _u32p, _u64p]
        _ref.ref_point_zbuffer.restype = None
        _ref.ref_point_zbuffer.argtypes = [ctypes.c_uint32, _f32p, _f32p, _f32p, _f32p, _int, _int]
        u32 = ctypes.c_uint32
        _ref.ref_gauss_project.restype = None
        _ref.ref_gauss_project.argtypes = [u32, _f32p, _f32p, _f32p, _f32p, u32, u32, _f32p, _f32p, _f32p]
        _ref.ref_gauss_rasterize.restype = None
        _ref.ref_gauss_rasterize.argtypes = [u32, u32, _f32p, _f32p, _f32p, _f32p, _f32p, _f32p, u32, _u32p, _u32p]
        _ref.ref_circle_project.restype = None
        _ref.ref_circle_project.argtypes = [u32, _f32p, _f32p, u32, u32, ctypes.c_float, _f32p, _f32p]
        _ref.ref_circle_rasterize.restype = None
        _ref.ref_circle_rasterize.argtypes = [u32, u32, _f32p, u32, _u32p, _u32p, _f32p, _f32p, _f32p]
    return _ref


class Scene64(ctypes.Structure):
    _fields_ = [
        ("n", _i64), ("sh_deg", _int),
        ("means", _f32p), ("log_scales", _f32p), ("quats", _f32p), ("opacity", _f32p),
        ("colors", _f32p), ("mvp", _f32p), ("campos", _f32p),
        ("w", _int), ("h", _int), ("ts", _int),
        ("tile2idx", _u32p), ("idx2pnt", _u32p), ("pix_last", _i32p), ("aabb", _f32p),
        ("target", _f32p),
    ]


def _declare(L: ctypes.CDLL) -> None:
    sig = {
        "orc_gauss_project": (None, [_i64, _f32p, _f32p, _f32p, _f32p, _int, _int, _f32p, _f32p, _f32p]),
        "orc_circle_project": (None, [_i64, _f32p, _f32p, _int, _int, ctypes.c_float, _f32p, _f32p]),
        "orc_circle_aabb": (None, [_i64, _f32p, _f32p, _f32p]),
        "orc_tile2pnt_count": (ctypes.c_uint64, [_i64, _f32p, _int, _int, _int, _u32p]),
        "orc_tile2pnt_fill": (None, [_i64, _f32p, _f32p, _int, _int, _int, _u32p, _u32p, _u64p]),
        "orc_gauss_rasterize_tiled": (None, [_int, _int, _int, _u32p, _u32p, _f32p, _f32p, _f32p, _f32p, _f32p,
                                             _f32p, _f32p, _i32p, _int]),
        "orc_gauss_rasterize_tiled_mode": (None, [_int, _int, _int, _u32p, _u32p, _f32p, _f32p, _f32p, _f32p,
                                                  _f32p, _f32p, _f32p, _i32p, _int, _int]),
        "orc_gauss_render_naive": (None, [_i64, _f32p, _f32p, _f32p, _f32p, _f32p, _int, _int, _f32p]),
        "orc_gauss_render_naive_mode": (None, [_i64, _f32p, _f32p, _f32p, _f32p, _f32p, _int, _int, _f32p, _int]),
        "orc_circle_splat_tiled": (None, [_int, _int, _int, _u32p, _u32p, _f32p, _f32p, _i32p]),
        "orc_point_render_sort_depth": (None, [_i64, _f32p, _int, _int, _i32p]),
        "orc_fused_project": (None, [_i64, _f32p, _f32p, _f32p, _f32p, _int, _f32p, _f32p, _int, _int,
                                     _f32p, _f32p, _f32p, _f32p]),
        "orc_sh_eval": (None, [_i64, _f32p, _f32p, _int, _f32p, _f32p]),
        "orc_expf_cr": (None, [_i64, _f32p, _f32p]),
        "orc64_loss": (ctypes.c_double, [ctypes.POINTER(Scene64), _u8p, _f64p]),
        "orc64_backward": (ctypes.c_double, [ctypes.POINTER(Scene64), _f64p, _f64p, _f64p, _f64p, _f64p]),
        "orc64_fd": (ctypes.c_double, [ctypes.POINTER(Scene64), _int, _i64, _int, ctypes.c_double]),
        "orc_cpu_fwd_bwd": (ctypes.c_uint64, [ctypes.POINTER(Scene64), _int, _f32p, _f32p, _f32p, _f32p, _f32p, _f32p]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args


def _p(a: Optional[np.ndarray], ct):
    if a is None:
        return ctypes.cast(None, ct)
    assert a.flags["C_CONTIGUOUS"], "oracle arrays must be C-contiguous"
    return a.ctypes.data_as(ct)


def f32(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.float32)


def expf_cr(x):
    """exp(x) correctly rounded to float32, elementwise (threaded)."""
    x = f32(x).ravel()
    out = np.empty_like(x)
    lib().orc_expf_cr(x.size, _p(x, _f32p), _p(out, _f32p))
    return out


def tile_shape(w: int, h: int, ts: int):
    return (w + ts - 1) // ts, (h + ts - 1) // ts


# ---------------------------------------------------------------- forward
def gauss_project(xyz, quat, scale, mvp, w, h):
    xyz, quat, scale, mvp = f32(xyz), f32(quat), f32(scale), f32(mvp).reshape(16)
    n = xyz.shape[0]
    xyd = np.zeros((n, 3), np.float32)
    conic = np.zeros((n, 3), np.float32)
    aabb = np.zeros((n, 4), np.float32)
    lib().orc_gauss_project(n, _p(xyz, _f32p), _p(quat, _f32p), _p(scale, _f32p), _p(mvp, _f32p), w, h,
                            _p(xyd, _f32p), _p(conic, _f32p), _p(aabb, _f32p))
    return xyd, conic, aabb


def fused_project(means, log_scales, quats, colors, sh_deg, mvp, campos, w, h):
    means, log_scales, quats = f32(means), f32(log_scales), f32(quats)
    colors, mvp, campos = f32(colors), f32(mvp).reshape(16), f32(campos).reshape(3)
    n = means.shape[0]
    xyd = np.zeros((n, 3), np.float32)
    conic = np.zeros((n, 3), np.float32)
    aabb = np.zeros((n, 4), np.float32)
    rgb = np.zeros((n, 3), np.float32)
    lib().orc_fused_project(n, _p(means, _f32p), _p(log_scales, _f32p), _p(quats, _f32p), _p(colors, _f32p),
                            sh_deg, _p(mvp, _f32p), _p(campos, _f32p), w, h,
                            _p(xyd, _f32p), _p(conic, _f32p), _p(aabb, _f32p), _p(rgb, _f32p))
    return xyd, conic, aabb, rgb


def circle_project(xyz, mvp, w, h, radius):
    xyz, mvp = f32(xyz), f32(mvp).reshape(16)
    n = xyz.shape[0]
    xyd = np.zeros((n, 3), np.float32)
    rad = np.zeros((n,), np.float32)
    lib().orc_circle_project(n, _p(xyz, _f32p), _p(mvp, _f32p), w, h, float(radius), _p(xyd, _f32p), _p(rad, _f32p))
    return xyd, rad


def circle_aabb(xyd, rad):
    xyd, rad = f32(xyd), f32(rad)
    aabb = np.zeros((xyd.shape[0], 4), np.float32)
    lib().orc_circle_aabb(xyd.shape[0], _p(xyd, _f32p), _p(rad, _f32p), _p(aabb, _f32p))
    return aabb


def tile2pnt(xyd, aabb, w, h, ts, with_keys=True):
    """tile_acceleration.rs:3-58 -> (tile2idx[T+1] u32, idx2pnt[P] u32, keys[P] u64)."""
    xyd, aabb = f32(xyd), f32(aabb)
    tw, th = tile_shape(w, h, ts)
    n = xyd.shape[0]
    tile2idx = np.zeros(tw * th + 1, np.uint32)
    P = lib().orc_tile2pnt_count(n, _p(aabb, _f32p), tw, th, ts, _p(tile2idx, _u32p))
    idx2pnt = np.zeros(P, np.uint32)
    keys = np.zeros(P, np.uint64) if with_keys else None
    lib().orc_tile2pnt_fill(n, _p(aabb, _f32p), _p(xyd, _f32p), tw, th, ts, _p(tile2idx, _u32p),
                            _p(idx2pnt, _u32p), _p(keys, _u64p))
    return tile2idx, idx2pnt, keys


def gauss_rasterize_tiled(w, h, ts, tile2idx, idx2pnt, xyd, conic, aabb, opacity, rgb, nthreads=1, mode=0):
    """Tiled front-to-back blend -> (image [H,W,3], final T [H,W], stop position [H,W])."""
    pix = np.zeros((h, w, 3), np.float32)
    T = np.zeros((h, w), np.float32)
    last = np.zeros((h, w), np.int32)
    tile2idx = np.ascontiguousarray(tile2idx, np.uint32)
    idx2pnt = np.ascontiguousarray(idx2pnt, np.uint32)
    xyd, conic, aabb, opacity, rgb = f32(xyd), f32(conic), f32(aabb), f32(opacity), f32(rgb)
    lib().orc_gauss_rasterize_tiled_mode(w, h, ts, _p(tile2idx, _u32p), _p(idx2pnt, _u32p), _p(xyd, _f32p),
                                         _p(conic, _f32p), _p(aabb, _f32p), _p(opacity, _f32p), _p(rgb, _f32p),
                                         _p(pix, _f32p), _p(T, _f32p), _p(last, _i32p), nthreads, int(mode))
    return pix, T, last


def gauss_render_naive(xyd, conic, aabb, opacity, rgb, w, h, mode=0):
    """pnt2pixxyndcz.rs:42-100 (untiled, global depth order)."""
    xyd, conic, aabb, opacity, rgb = f32(xyd), f32(conic), f32(aabb), f32(opacity), f32(rgb)
    pix = np.zeros((h, w, 3), np.float32)
    lib().orc_gauss_render_naive_mode(xyd.shape[0], _p(xyd, _f32p), _p(conic, _f32p), _p(aabb, _f32p),
                                      _p(opacity, _f32p), _p(rgb, _f32p), w, h, _p(pix, _f32p), int(mode))
    return pix


def circle_splat_tiled(w, h, ts, tile2idx, idx2pnt, xyd, rad):
    win = np.zeros((h, w), np.int32)
    tile2idx = np.ascontiguousarray(tile2idx, np.uint32)
    idx2pnt = np.ascontiguousarray(idx2pnt, np.uint32)
    xyd, rad = f32(xyd), f32(rad)
    lib().orc_circle_splat_tiled(w, h, ts, _p(tile2idx, _u32p), _p(idx2pnt, _u32p), _p(xyd, _f32p),
                                 _p(rad, _f32p), _p(win, _i32p))
    return win


def point_render_sort_depth(xyd, w, h):
    xyd = f32(xyd)
    win = np.zeros((h, w), np.int32)
    lib().orc_point_render_sort_depth(xyd.shape[0], _p(xyd, _f32p), w, h, _p(win, _i32p))
    return win


def point_unitdepth(ndcz: np.ndarray) -> np.ndarray:
    """splat_point.cu:66 -- `1.0-(ndcz + 1.)*0.5` evaluated in double, stored as float."""
    return (1.0 - (np.asarray(ndcz, np.float64) + 1.0) * 0.5).astype(np.float32)


# ---------------------------------------------------------------- FP64 gradient oracle
class Scene:
    """Keeps the numpy buffers alive for a Scene64 struct."""

    def __init__(self, means, log_scales, quats, opacity, colors, sh_deg, mvp, campos, w, h, ts,
                 tile2idx, idx2pnt, pix_last, aabb, target):
        if int(ts) <= 0 or int(w) <= 0 or int(h) <= 0:
            raise ValueError(f"oracle Scene: tile size and image size must be positive (ts={ts}, {w}x{h})")
        self.a = dict(
            means=f32(means), log_scales=f32(log_scales), quats=f32(quats), opacity=f32(opacity).reshape(-1),
            colors=f32(colors), mvp=f32(mvp).reshape(16), campos=f32(campos).reshape(3),
            tile2idx=np.ascontiguousarray(tile2idx, np.uint32), idx2pnt=np.ascontiguousarray(idx2pnt, np.uint32),
            pix_last=np.ascontiguousarray(pix_last, np.int32), aabb=f32(aabb), target=f32(target))
        a = self.a
        self.n = a["means"].shape[0]
        self.sh_deg = sh_deg
        self.K = 1 if sh_deg < 0 else (sh_deg + 1) ** 2
        self.s = Scene64(self.n, sh_deg, _p(a["means"], _f32p), _p(a["log_scales"], _f32p), _p(a["quats"], _f32p),
                         _p(a["opacity"], _f32p), _p(a["colors"], _f32p), _p(a["mvp"], _f32p),
                         _p(a["campos"], _f32p), w, h, ts, _p(a["tile2idx"], _u32p), _p(a["idx2pnt"], _u32p),
                         _p(a["pix_last"], _i32p), _p(a["aabb"], _f32p), _p(a["target"], _f32p))
        self.w, self.h = w, h

    def loss(self, with_image=False):
        img = np.zeros((self.h, self.w, 3), np.float64) if with_image else None
        L = lib().orc64_loss(ctypes.byref(self.s), _p(None, _u8p), _p(img, _f64p))
        return (L, img) if with_image else L

    def backward(self):
        n, K = self.n, self.K
        g = dict(means=np.zeros((n, 3)), log_scales=np.zeros((n, 3)), quats=np.zeros((n, 4)),
                 opacity=np.zeros(n), colors=np.zeros((n, K * 3)))
        L = lib().orc64_backward(ctypes.byref(self.s), _p(g["means"], _f64p), _p(g["log_scales"], _f64p),
                                 _p(g["quats"], _f64p), _p(g["opacity"], _f64p), _p(g["colors"], _f64p))
        return L, g

    KINDS = {"means": 0, "log_scales": 1, "quats": 2, "opacity": 3, "colors": 4}

    def fd(self, kind: str, gauss: int, comp: int, h: float = 1e-4) -> float:
        return lib().orc64_fd(ctypes.byref(self.s), self.KINDS[kind], int(gauss), int(comp), float(h))

    def cpu_fwd_bwd(self, nthreads: int):
        n, K = self.n, self.K
        img = np.zeros((self.h, self.w, 3), np.float32)
        g = [np.zeros((n, 3), np.float32), np.zeros((n, 3), np.float32), np.zeros((n, 4), np.float32),
             np.zeros(n, np.float32), np.zeros((n, K * 3), np.float32)]
        P = lib().orc_cpu_fwd_bwd(ctypes.byref(self.s), nthreads, _p(img, _f32p), *[_p(x, _f32p) for x in g])
        return P, img, g


# ---------------------------------------------------------------- reference pin (_ref)
def ref_tile2pnt(xyd, aabb, w, h, ts):
    xyd, aabb = f32(xyd), f32(aabb)
    tw, th = tile_shape(w, h, ts)
    tile2idx = np.zeros(tw * th + 1, np.uint32)
    n = xyd.shape[0]
    P = ref().ref_tiles_count(n, _p(aabb, _f32p), tw, th, ts, _p(tile2idx, _u32p))
    idx2pnt = np.zeros(P, np.uint32)
    keys = np.zeros(P, np.uint64)
    ref().ref_tiles_fill(n, _p(aabb, _f32p), _p(xyd, _f32p), tw, th, ts, _p(idx2pnt, _u32p), _p(keys, _u64p))
    return tile2idx, idx2pnt, keys


def ref_point_zbuffer(xyd, rgb, w, h):
    xyd, rgb = f32(xyd), f32(rgb)
    depth = np.full((h, w), np.finfo(np.float32).max, np.float32)
    img = np.zeros((h, w, 3), np.float32)
    ref().ref_point_zbuffer(xyd.shape[0], _p(xyd, _f32p), _p(rgb, _f32p), _p(depth, _f32p), _p(img, _f32p), w, h)
    return depth, img


def ref_gauss_project(xyz, quat, scale, mvp, w, h):
    """The reference's splat_gauss.cu:10-53 run on the CPU (del-geo restated)."""
    xyz, quat, scale, mvp = f32(xyz), f32(quat), f32(scale), f32(mvp).reshape(16)
    n = xyz.shape[0]
    xyd = np.zeros((n, 3), np.float32)
    conic = np.zeros((n, 3), np.float32)
    aabb = np.zeros((n, 4), np.float32)
    ref().ref_gauss_project(n, _p(xyz, _f32p), _p(quat, _f32p), _p(scale, _f32p), _p(mvp, _f32p), w, h,
                            _p(xyd, _f32p), _p(conic, _f32p), _p(aabb, _f32p))
    return xyd, conic, aabb


def ref_gauss_rasterize(w, h, ts, tile2idx, idx2pnt, xyd, conic, aabb, opacity, rgb):
    """The reference's splat_gauss.cu:56-109 run on the CPU -> image [H,W,3]."""
    pix = np.zeros((h, w, 3), np.float32)
    tile2idx = np.ascontiguousarray(tile2idx, np.uint32)
    idx2pnt = np.ascontiguousarray(idx2pnt, np.uint32)
    xyd, conic, aabb, opacity, rgb = f32(xyd), f32(conic), f32(aabb), f32(opacity), f32(rgb)
    ref().ref_gauss_rasterize(w, h, _p(pix, _f32p), _p(xyd, _f32p), _p(conic, _f32p), _p(aabb, _f32p),
                              _p(opacity, _f32p), _p(rgb, _f32p), ts, _p(tile2idx, _u32p), _p(idx2pnt, _u32p))
    return pix


def ref_circle_project(xyz, mvp, w, h, radius):
    """The reference's splat_circle.cu:7-41 run on the CPU."""
    xyz, mvp = f32(xyz), f32(mvp).reshape(16)
    n = xyz.shape[0]
    xyd = np.zeros((n, 3), np.float32)
    rad = np.zeros((n,), np.float32)
    ref().ref_circle_project(n, _p(xyz, _f32p), _p(mvp, _f32p), w, h, float(radius), _p(xyd, _f32p),
                             _p(rad, _f32p))
    return xyd, rad


def ref_circle_rasterize(w, h, ts, tile2idx, idx2pnt, xyd, rad, rgb):
    """The reference's splat_circle.cu:93-132 run on the CPU -> image [H,W,3]."""
    pix = np.zeros((h, w, 3), np.float32)
    tile2idx = np.ascontiguousarray(tile2idx, np.uint32)
    idx2pnt = np.ascontiguousarray(idx2pnt, np.uint32)
    xyd, rad, rgb = f32(xyd), f32(rad), f32(rgb)
    ref().ref_circle_rasterize(w, h, _p(pix, _f32p), ts, _p(tile2idx, _u32p), _p(idx2pnt, _u32p),
                               _p(xyd, _f32p), _p(rad, _f32p), _p(rgb, _f32p))
    return pix
