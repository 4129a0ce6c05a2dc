"""COLMAP sparse-model reader (binary cameras.bin / images.bin / points3D.bin)
and conversion of its cameras to batched views.

Mirrors del-splat-cpu/src/colmap.rs (read_cameras :16-51, read_images
:74-116, read_points3d :126-162): the same little-endian binary layout of
COLMAP's model files and the same fields.  As there, only the PINHOLE model
(model id 1: fx, fy, cx, cy) is accepted.  Poses follow COLMAP's convention:
x_cam = R(qvec) x_world + tvec with qvec = (w, x, y, z) and the camera
looking down +z, x right, y down.

`views_from_model` turns (camera, image) pairs into dsplat.scenes.Camera
objects in this library's convention (column-major world -> NDC matrix, NDC
y up, pixel y down, larger ndc_z = nearer, near plane -> +1, far -> -1), so
a COLMAP reconstruction can drive GaussBatch directly.
"""
from __future__ import annotations

import dataclasses
import struct
from typing import Dict, List, Sequence, Tuple

import numpy as np

PINHOLE = 1


@dataclasses.dataclass
class ColmapCamera:
    camera_id: int
    width: int
    height: int
    params: Tuple[float, float, float, float]  # fx, fy, cx, cy


@dataclasses.dataclass
class ColmapImage:
    image_id: int
    qvec: np.ndarray     # (w, x, y, z), world -> camera rotation
    tvec: np.ndarray     # world -> camera translation
    camera_id: int
    name: str
    xys: np.ndarray      # [K, 2] f64 keypoints
    point3d_ids: np.ndarray  # [K] i64 (-1: none)


@dataclasses.dataclass
class ColmapPoint:
    point3d_id: int
    xyz: np.ndarray      # f64[3]
    rgb: np.ndarray      # u8[3]
    error: float
    track: np.ndarray    # [T, 2] i32 (image_id, point2d_idx)


class _Reader:
    def __init__(self, data: bytes):
        self.d, self.o = data, 0

    def take(self, fmt: str):
        v = struct.unpack_from("<" + fmt, self.d, self.o)
        self.o += struct.calcsize("<" + fmt)
        return v

    def array(self, dtype, count: int) -> np.ndarray:
        a = np.frombuffer(self.d, dtype=np.dtype(dtype).newbyteorder("<"), count=count, offset=self.o)
        self.o += a.nbytes
        return a.copy()

    def cstring(self) -> str:
        end = self.d.index(b"\x00", self.o)
        s = self.d[self.o:end].decode("utf-8")
        self.o = end + 1
        return s


def read_cameras(path) -> List[ColmapCamera]:
    with open(path, "rb") as f:
        r = _Reader(f.read())
    (n,) = r.take("Q")
    cams = []
    for _ in range(n):
        camera_id, model_id, width, height = r.take("iIQQ")
        if model_id != PINHOLE:
            raise ValueError(f"camera {camera_id}: model {model_id} not supported (PINHOLE only)")
        cams.append(ColmapCamera(camera_id, int(width), int(height), tuple(float(x) for x in r.take("4d"))))
    return cams


def read_images(path) -> List[ColmapImage]:
    with open(path, "rb") as f:
        r = _Reader(f.read())
    (n,) = r.take("Q")
    images = []
    for _ in range(n):
        (image_id,) = r.take("i")
        q = np.array(r.take("4d"))
        t = np.array(r.take("3d"))
        (camera_id,) = r.take("i")
        name = r.cstring()
        (k,) = r.take("Q")
        rec = r.array(np.dtype([("x", "<f8"), ("y", "<f8"), ("id", "<i8")]), k)
        images.append(ColmapImage(image_id, q, t, camera_id, name, np.stack([rec["x"], rec["y"]], 1),
                                  rec["id"].astype(np.int64)))
    return images


def read_points3d(path) -> List[ColmapPoint]:
    with open(path, "rb") as f:
        r = _Reader(f.read())
    (n,) = r.take("Q")
    pts = []
    for _ in range(n):
        (pid,) = r.take("Q")
        xyz = np.array(r.take("3d"))
        rgb = np.array(r.take("3B"), np.uint8)
        (err,) = r.take("d")
        (tl,) = r.take("Q")
        track = r.array("<i4", 2 * tl).reshape(tl, 2)
        pts.append(ColmapPoint(int(pid), xyz, rgb, float(err), track))
    return pts


def qvec_to_rotation(q: Sequence[float]) -> np.ndarray:
    """Unit quaternion (w, x, y, z) -> 3x3 rotation (row-major numpy)."""
    w, x, y, z = (float(v) for v in q)
    n = np.sqrt(w * w + x * x + y * y + z * z)
    w, x, y, z = w / n, x / n, y / n, z / n
    return np.array([[1 - 2 * (y * y + z * z), 2 * (x * y - w * z), 2 * (x * z + w * y)],
                     [2 * (x * y + w * z), 1 - 2 * (x * x + z * z), 2 * (y * z - w * x)],
                     [2 * (x * z - w * y), 2 * (y * z + w * x), 1 - 2 * (x * x + y * y)]])


def world_to_ndc(cam: ColmapCamera, img: ColmapImage, near: float, far: float) -> np.ndarray:
    """4x4 world -> clip matrix (row-major numpy) of a PINHOLE view:
    ndc_x = (u - W/2) / (W/2), ndc_y = (H/2 - v) / (H/2) for the pinhole pixel
    (u, v) = (fx x/z + cx, fy y/z + cy), and ndc_z = a + b/z with ndc_z(near)
    = +1, ndc_z(far) = -1 (larger = nearer); w_clip = z."""
    fx, fy, cx, cy = cam.params
    W, H = float(cam.width), float(cam.height)
    b = 2.0 * near * far / (far - near)
    a = -(far + near) / (far - near)
    proj = np.array([[2 * fx / W, 0.0, 2 * cx / W - 1.0, 0.0],
                     [0.0, -2 * fy / H, 1.0 - 2 * cy / H, 0.0],
                     [0.0, 0.0, a, b],
                     [0.0, 0.0, 1.0, 0.0]])
    view = np.eye(4)
    view[:3, :3] = qvec_to_rotation(img.qvec)
    view[:3, 3] = img.tvec
    return proj @ view


def camera_centre(img: ColmapImage) -> np.ndarray:
    R = qvec_to_rotation(img.qvec)
    return -R.T @ np.asarray(img.tvec, np.float64)


def views_from_model(cameras: Sequence[ColmapCamera], images: Sequence[ColmapImage], near: float = 0.1,
                     far: float = 100.0):
    """dsplat.scenes.Camera per image (in the order given)."""
    from .scenes import Camera
    by_id: Dict[int, ColmapCamera] = {c.camera_id: c for c in cameras}
    out = []
    for img in images:
        cam = by_id[img.camera_id]
        m = world_to_ndc(cam, img, near, far)
        out.append(Camera(mvp=np.ascontiguousarray(m.T.reshape(-1), np.float32),
                          campos=camera_centre(img).astype(np.float32), width=cam.width, height=cam.height))
    return out
