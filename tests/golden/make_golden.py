"""Generates the small reference fixtures under tests/golden/ (run here, where
the del-splat sources exist; the outputs are committed).

The expected values come from the reference's own CUDA sources compiled as
host C++ (oracle/ref/: tile_acceleration.h for tile lists and keys,
splat_point.cu for the point z-buffer); the inputs are seeded synthetic
projections.  bulba_subset.ply is a seeded 3,000-row subset of the
reference's 3DGS capture asset/bulba.ply (header kept, vertex count
adjusted), the real-data input of the PLY reader and render tests.
Usage: python tests/golden/make_golden.py [del-splat checkout]
(default: $DSPLAT_REFERENCE_ROOT, else /root/reference)
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path[:0] = [ROOT, os.path.join(ROOT, "del-splat_b200")]

import oracle  # noqa: E402
from dsplat import scenes  # noqa: E402


def reference_root() -> str:
    if len(sys.argv) > 1:
        return sys.argv[1]
    return os.environ.get("DSPLAT_REFERENCE_ROOT", "/root/reference")


def bulba_subset(rows: int = 3000, seed: int = 17) -> None:
    src = os.path.join(reference_root(), "asset", "bulba.ply")
    with open(src, "rb") as f:
        head = []
        while True:
            line = f.readline()
            head.append(line)
            if line == b"end_header\n":
                break
        body = f.read()
    n = next(int(l.split()[2]) for l in head if l.startswith(b"element vertex"))
    rec = np.frombuffer(body, dtype="<f4").reshape(n, -1)
    keep = np.sort(np.random.default_rng(seed).choice(n, rows, replace=False))
    head = [b"element vertex %d\n" % rows if l.startswith(b"element vertex") else l for l in head]
    with open(os.path.join(HERE, "bulba_subset.ply"), "wb") as f:
        f.write(b"".join(head))
        f.write(np.ascontiguousarray(rec[keep]).tobytes())


def main():
    oracle.build(reference_root())
    bulba_subset()
    assert oracle.ref_available(), "oracle/_ref missing: needs the del-splat tree"
    # Gaussians: 2048 points, 120x72 image, 8-pixel tiles
    sc = scenes.config0(seed=11, n=2048, size=(120, 72))
    cam = sc.cameras[0]
    xyd, conic, aabb = oracle.gauss_project(sc.means, sc.quats, sc.scales, cam.mvp, cam.width, cam.height)
    t2i, i2p, keys = oracle.ref_tile2pnt(xyd, aabb, 120, 72, 8)
    np.savez_compressed(os.path.join(HERE, "tiles_gauss_small.npz"), shape=np.array([120, 72, 8]), xyd=xyd,
                        aabb=aabb, tile2idx=t2i, idx2pnt=i2p, keys=keys)
    # circles: 3000 points, 100x60 image, 16-pixel tiles, a few exact depth ties
    pts = scenes.config1(seed=12, n=3000, size=(100, 60))
    xyd_c, rad = oracle.circle_project(pts.xyz, pts.camera.mvp, 100, 60, 0.02)
    xyd_c[100:110, 2] = xyd_c[0, 2]
    aabb_c = oracle.circle_aabb(xyd_c, rad)
    t2i, i2p, keys = oracle.ref_tile2pnt(xyd_c, aabb_c, 100, 60, 16)
    np.savez_compressed(os.path.join(HERE, "tiles_circle_small.npz"), shape=np.array([100, 60, 16]), xyd=xyd_c,
                        aabb=aabb_c, rad=rad, tile2idx=t2i, idx2pnt=i2p, keys=keys)
    # points: serial run of splat_point.cu (coordinates >= -1, no ties)
    rng = np.random.default_rng(13)
    n, w, h = 4000, 48, 32
    xyd_p = np.stack([rng.uniform(-0.9, w + 2, n), rng.uniform(-0.9, h + 2, n), rng.uniform(-0.999, 0.999, n)],
                     1).astype(np.float32)
    rgb = rng.uniform(0, 1, (n, 3)).astype(np.float32)
    depth, img = oracle.ref_point_zbuffer(xyd_p, rgb, w, h)
    np.savez_compressed(os.path.join(HERE, "point_zbuffer_small.npz"), shape=np.array([w, h]), xyd=xyd_p, rgb=rgb,
                        depth=depth, rgb_out=img)
    print("fixtures written to", HERE)


if __name__ == "__main__":
    main()
