"""PLY readers restating del-splat-cpu/src/io_ply.rs (host-side file I/O).

* ``read_xyzrgb`` (io_ply.rs:30-104): binary little-endian vertices of
  (f64 x, y, z, u8 r, g, b) -> xyz f32 [N,3], rgb f32 [N,3] = u8 / 255.
* ``read_3d_gauss_splat`` (io_ply.rs:128-227): the 62-float 3DGS layout
  (x,y,z, nx,ny,nz, f_dc[3], f_rest[45], opacity, scale[3], rot[4]) with the
  reference's conversions: rgb = (f_dc + 0.5) * 0.5, quaternion (w,x,y,z) ->
  (x,y,z,w) normalised, scale = exp(scale), opacity = sigmoid(opacity).
  f_rest is returned as stored (channel-major, 3 x 15) like the reference,
  plus ``sh_coeffs`` in the [N,16,3] layout the SH kernels take (DC = f_dc).
"""
from __future__ import annotations

import numpy as np


def _header(f):
    lines = []
    while True:
        line = f.readline()
        if not line:
            raise ValueError("unexpected end of PLY header")
        s = line.decode("ascii", errors="replace")
        lines.append(s)
        if s == "end_header\n":
            return lines


def read_xyzrgb(path: str):
    with open(path, "rb") as f:
        hdr = _header(f)
        if hdr[0] != "ply\n":
            raise ValueError("not a PLY file")
        fmt = hdr[1].split()
        if fmt[0] != "format" or fmt[1] != "binary_little_endian":
            raise ValueError("only binary_little_endian is supported (as in the reference)")
        n = next(int(l.split()[2]) for l in hdr if l.startswith("element"))
        dt = np.dtype([("x", "<f8"), ("y", "<f8"), ("z", "<f8"), ("r", "u1"), ("g", "u1"), ("b", "u1")])
        data = np.frombuffer(f.read(n * dt.itemsize), dtype=dt, count=n)
    xyz = np.stack([data["x"], data["y"], data["z"]], 1).astype(np.float32)
    rgb = (np.stack([data["r"], data["g"], data["b"]], 1).astype(np.float32) / np.float32(255.0))
    return np.ascontiguousarray(xyz), np.ascontiguousarray(rgb)


def read_3d_gauss_splat(path: str):
    """Returns dict(xyz, rgb, sh_rest, opacity, scale, quat, sh_coeffs, log_scale)."""
    with open(path, "rb") as f:
        hdr = _header(f)
        if hdr[0] != "ply\n" or not hdr[1].startswith("format"):
            raise ValueError("not a PLY file")
        n = next(int(l.split()[2]) for l in hdr if l.startswith("element vertex"))
        props = [l for l in hdr if l.startswith("property")]
        if len(props) != 62 or any(p.split()[1] != "float" for p in props):
            raise ValueError("expected 62 float properties (3DGS layout)")
        buf = f.read()
    if len(buf) != 62 * n * 4:
        raise ValueError("payload size mismatch")
    a = np.frombuffer(buf, dtype="<f4").reshape(n, 62)
    xyz = a[:, 0:3]
    f_dc = a[:, 6:9]
    rest = a[:, 9:54]
    op = a[:, 54]
    sc = a[:, 55:58]
    rot = a[:, 58:62]
    rgb = (f_dc + np.float32(0.5)) * np.float32(0.5)
    q = np.stack([rot[:, 1], rot[:, 2], rot[:, 3], rot[:, 0]], 1)
    q = q / np.sqrt((q * q).sum(1, keepdims=True))
    scale = np.exp(sc)
    opacity = np.float32(1.0) / (np.float32(1.0) + np.exp(-op))
    sh = np.empty((n, 16, 3), np.float32)
    sh[:, 0, :] = f_dc
    sh[:, 1:, :] = rest.reshape(n, 3, 15).transpose(0, 2, 1)
    c = lambda x: np.ascontiguousarray(x, np.float32)  # noqa: E731
    return dict(xyz=c(xyz), rgb=c(rgb), sh_rest=c(rest), opacity=c(opacity), scale=c(scale), quat=c(q),
                sh_coeffs=c(sh), log_scale=c(sc))
