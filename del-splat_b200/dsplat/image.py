"""Image output for rendered views: 8-bit RGB / RGBA PNG files.

The reference's examples save every render as a PNG; this writes the same
kind of file from an [H, W, 3] (or [H, W, 4]) array -- float in [0, 1]
(clamped, rounded) or uint8 -- or from a CUDA tensor (copied to the host),
and from a [H, W] u32 RGBA array as the circle/point z-buffer produces it
(byte 0 = red).  Plain zlib-compressed PNG (filter type 0 on every row), so
no imaging library is needed.
"""
from __future__ import annotations

import struct
import zlib

import numpy as np


def _chunk(kind: bytes, data: bytes) -> bytes:
    return struct.pack(">I", len(data)) + kind + data + struct.pack(">I", zlib.crc32(kind + data) & 0xffffffff)


def to_u8(img) -> np.ndarray:
    """[H, W, C] uint8 from a float image in [0, 1], a uint8 image, a
    [H, W] u32 RGBA image, or a torch tensor of any of those."""
    if hasattr(img, "detach"):
        img = img.detach().cpu().numpy()
    a = np.asarray(img)
    if a.ndim == 2 and a.dtype in (np.uint32, np.int32):
        a = a.astype(np.uint32).view(np.uint8).reshape(a.shape[0], a.shape[1], 4)
    if a.ndim != 3 or a.shape[2] not in (3, 4):
        raise ValueError(f"expected [H, W, 3|4] (or [H, W] u32 RGBA), got {a.shape}")
    if a.dtype == np.uint8:
        return np.ascontiguousarray(a)
    return np.ascontiguousarray(np.clip(np.rint(a.astype(np.float64) * 255.0), 0, 255).astype(np.uint8))


def encode_png(img) -> bytes:
    a = to_u8(img)
    h, w, c = a.shape
    raw = b"".join(b"\x00" + a[y].tobytes() for y in range(h))
    ihdr = struct.pack(">IIBBBBB", w, h, 8, 6 if c == 4 else 2, 0, 0, 0)
    return b"\x89PNG\r\n\x1a\n" + _chunk(b"IHDR", ihdr) + _chunk(b"IDAT", zlib.compress(raw, 6)) + \
        _chunk(b"IEND", b"")


def save_png(path, img) -> None:
    with open(path, "wb") as f:
        f.write(encode_png(img))


def decode_png(data: bytes) -> np.ndarray:
    """Inverse of encode_png for the files it writes (8-bit RGB/RGBA, filter 0)."""
    if data[:8] != b"\x89PNG\r\n\x1a\n":
        raise ValueError("not a PNG")
    o, idat = 8, b""
    w = h = c = None
    while o < len(data):
        (n,) = struct.unpack(">I", data[o:o + 4])
        kind, body = data[o + 4:o + 8], data[o + 8:o + 8 + n]
        o += 12 + n
        if kind == b"IHDR":
            w, h, depth, ctype = struct.unpack(">IIBB", body[:10])
            if depth != 8 or ctype not in (2, 6):
                raise ValueError("only 8-bit RGB/RGBA")
            c = 4 if ctype == 6 else 3
        elif kind == b"IDAT":
            idat += body
    raw = zlib.decompress(idat)
    rows = np.frombuffer(raw, np.uint8).reshape(h, 1 + w * c)
    if (rows[:, 0] != 0).any():
        raise ValueError("only filter type 0")
    return rows[:, 1:].reshape(h, w, c).copy()
