"""Cameras and seeded synthetic scenes for the splatting workloads.

Random numbers come from numpy's PCG64 generator (``np.random.default_rng``)
seeded per scene; all arrays are float32 and C-contiguous.

Camera convention (the reference's): world -> NDC matrix stored column-major
(16 floats), NDC y up, pixel y down, and *larger ndc_z = nearer* -- the
OpenGL perspective with its depth row negated, so the near plane maps to +1
and the far plane to -1.
"""
from __future__ import annotations

import dataclasses
from typing import List, Tuple

import numpy as np


def look_at(eye, target=(0.0, 0.0, 0.0), up=(0.0, 1.0, 0.0)) -> np.ndarray:
    eye = np.asarray(eye, np.float64)
    f = np.asarray(target, np.float64) - eye
    f /= np.linalg.norm(f)
    up = np.asarray(up, np.float64)
    if abs(np.dot(f, up)) > 0.999:
        up = np.array([1.0, 0.0, 0.0]) if abs(f[0]) < 0.9 else np.array([0.0, 0.0, 1.0])
    r = np.cross(f, up)
    r /= np.linalg.norm(r)
    u = np.cross(r, f)
    m = np.eye(4)
    m[0, :3], m[1, :3], m[2, :3] = r, u, -f
    m[0, 3], m[1, 3], m[2, 3] = -r @ eye, -u @ eye, f @ eye
    return m


def perspective_reversed_z(fovy_deg: float, aspect: float, near: float, far: float) -> np.ndarray:
    t = 1.0 / np.tan(np.radians(fovy_deg) / 2.0)
    p = np.zeros((4, 4))
    p[0, 0] = t / aspect
    p[1, 1] = t
    p[2, 2] = -(far + near) / (near - far)
    p[2, 3] = -(2.0 * far * near) / (near - far)
    p[3, 2] = -1.0
    return p


@dataclasses.dataclass
class Camera:
    width: int
    height: int
    mvp: np.ndarray      # [16] float32, column-major
    campos: np.ndarray   # [3] float32

    @staticmethod
    def look_at_origin(eye, width, height, fovy_deg=60.0, near=0.1, far=10.0) -> "Camera":
        m = perspective_reversed_z(fovy_deg, width / height, near, far) @ look_at(eye)
        return Camera(width, height, np.ascontiguousarray(m.T.reshape(16), np.float32),
                      np.asarray(eye, np.float32))


@dataclasses.dataclass
class GaussScene:
    means: np.ndarray        # [N,3]
    log_scales: np.ndarray   # [N,3]
    quats: np.ndarray        # [N,4] (x,y,z,w), unit
    opacity: np.ndarray      # [N]
    colors: np.ndarray       # [N,3] RGB (sh_degree -1) or [N,K,3] SH
    sh_degree: int
    cameras: List[Camera]
    tile_size: int = 16

    @property
    def n(self) -> int:
        return self.means.shape[0]

    @property
    def scales(self) -> np.ndarray:
        """Linear standard deviations, the reference's pnt2scale."""
        return np.exp(self.log_scales.astype(np.float64)).astype(np.float32)


def _gauss_common(rng, n):
    means = rng.uniform(-1.0, 1.0, (n, 3)).astype(np.float32)
    log_scales = rng.uniform(-4.5, -2.5, (n, 3)).astype(np.float32)
    q = rng.standard_normal((n, 4))
    q /= np.linalg.norm(q, axis=1, keepdims=True)
    quats = q.astype(np.float32)
    op = 1.0 / (1.0 + np.exp(-rng.standard_normal(n)))
    opacity = np.clip(op, 0.01, 0.99).astype(np.float32)
    return means, log_scales, quats, opacity


def _sh_colors(rng, n, deg):
    k = (deg + 1) ** 2
    c = np.empty((n, k, 3), np.float32)
    c[:, 0, :] = rng.uniform(0.0, 1.0, (n, 3))
    if k > 1:
        c[:, 1:, :] = rng.normal(0.0, 0.1, (n, k - 1, 3))
    return c


def sphere_cameras(rng, count, radius, resolutions) -> List[Camera]:
    cams = []
    for _ in range(count):
        d = rng.standard_normal(3)
        d /= np.linalg.norm(d)
        w, h = resolutions[rng.integers(0, len(resolutions))]
        cams.append(Camera.look_at_origin(d * radius, int(w), int(h)))
    return cams


def config0(seed: int = 0, n: int = 16384, size: Tuple[int, int] = (256, 256)) -> GaussScene:
    """16,384 Gaussians, 256x256, 16x16 tiles, RGB colours, camera at (0,0,-3)."""
    rng = np.random.default_rng(seed)
    means, ls, quats, op = _gauss_common(rng, n)
    rgb = rng.uniform(0.0, 1.0, (n, 3)).astype(np.float32)
    cam = Camera.look_at_origin((0.0, 0.0, -3.0), size[0], size[1])
    return GaussScene(means, ls, quats, op, rgb, -1, [cam], 16)


@dataclasses.dataclass
class PointScene:
    xyz: np.ndarray       # [N,3]
    radius_px: np.ndarray  # [N] pixel radius
    rgba: np.ndarray      # [N] u32
    camera: Camera


def config1(seed: int = 1, n: int = 1 << 20, size: Tuple[int, int] = (1024, 1024)) -> PointScene:
    """1,048,576 points in [-1,1]^3, 1024x1024, pixel radius 1..4, u32 RGBA."""
    rng = np.random.default_rng(seed)
    xyz = rng.uniform(-1.0, 1.0, (n, 3)).astype(np.float32)
    rad = rng.integers(1, 5, n).astype(np.float32)
    rgba = rng.integers(0, 2 ** 32, n, dtype=np.uint64).astype(np.uint32)
    return PointScene(xyz, rad, rgba, Camera.look_at_origin((0.0, 0.0, -3.0), size[0], size[1]))


def config2(seed: int = 2, n: int = 262144, size: Tuple[int, int] = (1280, 720)) -> Tuple[GaussScene, np.ndarray]:
    """262,144 Gaussians, 1280x720, SH degree 3, with a U[0,1] target image."""
    rng = np.random.default_rng(seed)
    means, ls, quats, op = _gauss_common(rng, n)
    sh = _sh_colors(rng, n, 3)
    cam = Camera.look_at_origin((0.0, 0.0, -3.0), size[0], size[1])
    target = rng.uniform(0.0, 1.0, (size[1], size[0], 3)).astype(np.float32)
    return GaussScene(means, ls, quats, op, sh, 3, [cam], 16), target


CONFIG3_RESOLUTIONS = [(320, 240), (640, 480), (1280, 720), (1920, 1080)]


def config3(seed: int = 3, n: int = 1 << 20, views: int = 16, tile_size: int = 16) -> GaussScene:
    """1,048,576 Gaussians, SH 3, 16 cameras on a radius-3 sphere, mixed resolutions."""
    rng = np.random.default_rng(seed)
    means, ls, quats, op = _gauss_common(rng, n)
    sh = _sh_colors(rng, n, 3)
    cams = sphere_cameras(rng, views, 3.0, CONFIG3_RESOLUTIONS)
    return GaussScene(means, ls, quats, op, sh, 3, cams, tile_size)


def config4(seed: int = 4, n: int = 1 << 22, views: int = 8) -> GaussScene:
    """4,194,304 Gaussians, SH 3, 8 views at 1920x1080."""
    rng = np.random.default_rng(seed)
    means, ls, quats, op = _gauss_common(rng, n)
    sh = _sh_colors(rng, n, 3)
    cams = sphere_cameras(rng, views, 3.0, [(1920, 1080)])
    return GaussScene(means, ls, quats, op, sh, 3, cams, 16)


def targets_for(scene: GaussScene, seed: int = 99) -> List[np.ndarray]:
    rng = np.random.default_rng(seed)
    return [rng.uniform(0.0, 1.0, (c.height, c.width, 3)).astype(np.float32) for c in scene.cameras]
