"""ctypes binding of libdsplat.so (the C ABI in include/dsplat.h).

The library is the only compute path: if it is missing or fails to load,
every call raises -- there is no CPU fallback.
"""
from __future__ import annotations

import ctypes
import os
from typing import Optional

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(os.path.dirname(_HERE), "lib", "libdsplat.so")

DSPLAT_OK = 0
STOP_CPU = 0   # del-splat-cpu's stop test, alpha_sum > 0.999f
STOP_CUDA = 1  # the reference CUDA kernel's, alpha_sum > 0.999 in double
ERRORS = {1: "invalid argument", 2: "pair capacity exceeded", 3: "CUDA error", 4: "workspace too small",
          5: "unsupported"}

_lib: Optional[ctypes.CDLL] = None

c_void_p = ctypes.c_void_p
c_u32 = ctypes.c_uint32
c_i32 = ctypes.c_int32
c_u64 = ctypes.c_uint64
c_i64 = ctypes.c_int64
c_f32 = ctypes.c_float
c_size = ctypes.c_size_t


class DsplatError(RuntimeError):
    def __init__(self, code: int, where: str):
        msg = lib().dsplat_last_error().decode(errors="replace") if _lib is not None else ""
        super().__init__(f"{where}: {ERRORS.get(code, code)} ({msg})")
        self.code = code


class View(ctypes.Structure):
    _fields_ = [("mvp", c_f32 * 16), ("campos", c_f32 * 3), ("width", c_i32), ("height", c_i32)]


class GaussParams(ctypes.Structure):
    _fields_ = [("num_pnt", c_i64), ("sh_degree", c_i32), ("means", c_void_p), ("log_scales", c_void_p),
                ("quats", c_void_p), ("opacity", c_void_p), ("colors", c_void_p)]


class GaussGrads(ctypes.Structure):
    _fields_ = [("means", c_void_p), ("log_scales", c_void_p), ("quats", c_void_p), ("opacity", c_void_p),
                ("colors", c_void_p)]


class GaussTensors(ctypes.Structure):
    _fields_ = [("means", c_void_p), ("log_scales", c_void_p), ("quats", c_void_p), ("opacity", c_void_p),
                ("colors", c_void_p)]


class BatchLayout(ctypes.Structure):
    _fields_ = [("total_bytes", c_size), ("num_items", c_u32), ("num_pix", c_u32), ("npad", c_u32),
                ("slabs_per_tile", c_u32), ("num_sb", c_u32), ("sb_chunks", c_u32),
                ("off_flags", c_size), ("off_rec", c_size), ("off_rect", c_size), ("off_cnt", c_size),
                ("off_order", c_size), ("off_sb_start", c_size), ("off_sb_list", c_size),
                ("off_pix_T", c_size), ("off_pix_stop", c_size), ("off_grad_pix", c_size),
                ("off_slab_loss", c_size), ("off_grad2d", c_size), ("sb_log2", c_i32 * 32)]


_P = c_void_p  # every pointer is passed as an integer address
SIGNATURES = {
    "dsplat_version": (ctypes.c_char_p, []),
    "dsplat_last_error": (ctypes.c_char_p, []),
    "dsplat_launch_count": (c_u64, []),
    "dsplat_gauss_pnt2splat3_to_pnt2splat2": (c_i32, [_P, c_u32, _P, _P, _P, _P, _P, _P, _P, c_u32, c_u32]),
    "dsplat_tile2idx_workspace_size": (c_size, [c_u32, c_u32, c_u32, c_u64]),
    "dsplat_gauss_tile2idx_count": (c_i32, [_P, c_u32, _P, c_u32, c_u32, c_u32, _P, c_size, ctypes.POINTER(c_u64)]),
    "dsplat_gauss_tile2idx_idx2pnt": (c_i32, [_P, c_u32, _P, _P, c_u32, c_u32, c_u32, _P, _P, c_u64, _P, _P, c_size]),
    "dsplat_gauss_rasterize_pnt2splat2": (c_i32, [_P, c_u32, c_u32, _P, _P, _P, _P, _P, _P, c_u32, _P, _P, _P, _P]),
    "dsplat_gauss_rasterize_pnt2splat2_stop": (c_i32, [_P, c_u32, c_u32, _P, _P, _P, _P, _P, _P, c_u32, _P, _P, _P,
                                                       _P, c_i32]),
    "dsplat_expf_cr": (c_i32, [_P, c_u64, _P, _P]),
    "dsplat_circle_pnt2splat3_to_pnt2splat2": (c_i32, [_P, c_u32, _P, _P, _P, _P, c_u32, c_u32, c_f32]),
    "dsplat_circle_tile2idx_count": (c_i32, [_P, c_u32, _P, _P, c_u32, c_u32, c_u32, _P, c_size,
                                             ctypes.POINTER(c_u64)]),
    "dsplat_circle_tile2idx_idx2pnt": (c_i32, [_P, c_u32, _P, _P, c_u32, c_u32, c_u32, _P, _P, c_u64, _P, _P,
                                               c_size]),
    "dsplat_circle_splat": (c_i32, [_P, c_u32, c_u32, _P, _P, _P, _P, c_u32, _P, _P]),
    "dsplat_circle_splat_zbuffer": (c_i32, [_P, c_u32, _P, _P, _P, c_i32, _P, _P, c_u32, c_u32, c_u32, _P]),
    "dsplat_point_rasterize_pix_zbuffer": (c_i32, [_P, c_u32, _P, _P, _P, _P, _P, c_u32, c_u32, _P]),
    "dsplat_point_rasterize_pix": (c_i32, [_P, c_u32, _P, _P, _P, c_u32, c_u32, _P]),
    "dsplat_point_rasterize_pix_zbuffer_noalloc": (c_i32, [_P, c_u32, _P, _P, _P, _P, _P, c_u32, c_u32]),
    "dsplat_gauss_batch_layout": (c_i32, [c_i64, c_i32, ctypes.POINTER(View), c_i32, c_i32, c_u64,
                                          ctypes.POINTER(BatchLayout)]),
    "dsplat_gauss_batch_forward": (c_i32, [_P, ctypes.POINTER(GaussParams), c_i32, ctypes.POINTER(View), c_i32,
                                           c_i32, c_u64, _P, c_size, _P, _P, _P]),
    "dsplat_gauss_batch_backward": (c_i32, [_P, ctypes.POINTER(GaussParams), c_i32, ctypes.POINTER(View), c_i32,
                                            c_i32, c_u64, _P, c_size, _P, ctypes.POINTER(GaussGrads)]),
    "dsplat_gauss_batch_status": (c_i32, [_P, _P, ctypes.POINTER(c_u32), ctypes.POINTER(c_u64),
                                          ctypes.POINTER(c_u64)]),
    "dsplat_set_stage_events": (c_i32, [ctypes.POINTER(c_void_p), c_i32]),
    "dsplat_adam_step": (c_i32, [_P, c_i64, _P, _P, _P, _P, c_f32, c_f32, c_f32, c_f32, c_i32]),
    "dsplat_gauss_adam_step": (c_i32, [_P, c_i64, c_i32, ctypes.POINTER(GaussTensors), ctypes.POINTER(GaussGrads),
                                       ctypes.POINTER(GaussTensors), ctypes.POINTER(GaussTensors),
                                       ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_double, _P]),
}


def lib() -> ctypes.CDLL:
    """Load libdsplat.so (raises if it was not built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"libdsplat.so not built: expected {LIB_PATH} "
                               "(run `python del-splat_b200/build.py`)")
        L = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def check(code: int, where: str) -> None:
    if code != DSPLAT_OK:
        raise DsplatError(code, where)
