"""Host-side logic that needs no GPU: cameras, scenes, PLY I/O, DLPack layer."""
import os
import struct
import tempfile

import numpy as np
import pytest

from dsplat import ply, scenes


def _ndc(cam, p):
    m = cam.mvp.reshape(4, 4).T.astype(np.float64)
    q = m @ np.append(p, 1.0)
    return q[:3] / q[3]


def test_camera_convention_larger_ndc_z_is_nearer():
    cam = scenes.Camera.look_at_origin((0, 0, -3), 256, 256)
    near, far = _ndc(cam, np.array([0, 0, -1.0])), _ndc(cam, np.array([0, 0, 1.0]))
    assert near[2] > far[2]
    # near plane -> +1, far plane -> -1
    assert abs(_ndc(cam, np.array([0, 0, -3 + 0.1]))[2] - 1.0) < 1e-5
    assert abs(_ndc(cam, np.array([0, 0, -3 + 10.0]))[2] + 1.0) < 1e-5
    # 60 degree vertical FOV: a point at the top edge maps to ndc_y = 1
    top = np.array([0, 3 * np.tan(np.radians(30)), 0.0])
    assert abs(_ndc(cam, top)[1] - 1.0) < 1e-5


def test_synthetic_scenes_match_stated_distributions():
    sc = scenes.config0()
    assert sc.means.shape == (16384, 3) and sc.means.dtype == np.float32
    assert sc.log_scales.min() >= -4.5 and sc.log_scales.max() <= -2.5
    assert np.allclose(np.linalg.norm(sc.quats, axis=1), 1, atol=1e-6)
    assert sc.opacity.min() >= 0.01 and sc.opacity.max() <= 0.99
    s3 = scenes.config3(n=1000)
    assert len(s3.cameras) == 16 and s3.colors.shape == (1000, 16, 3)
    for c in s3.cameras:
        assert (c.width, c.height) in scenes.CONFIG3_RESOLUTIONS
        assert abs(np.linalg.norm(c.campos) - 3.0) < 1e-5
    p = scenes.config1(n=1000)
    assert set(np.unique(p.radius_px)) <= {1.0, 2.0, 3.0, 4.0} and p.rgba.dtype == np.uint32


def test_ply_xyzrgb_roundtrip():
    rng = np.random.default_rng(0)
    xyz = rng.normal(size=(50, 3))
    rgb = rng.integers(0, 256, (50, 3)).astype(np.uint8)
    with tempfile.NamedTemporaryFile(suffix=".ply", delete=False) as f:
        f.write(b"ply\nformat binary_little_endian 1.0\ncomment t\nelement vertex 50\n")
        for p in ("double x", "double y", "double z", "uchar red", "uchar green", "uchar blue"):
            f.write(f"property {p}\n".encode())
        f.write(b"end_header\n")
        for i in range(50):
            f.write(struct.pack("<3d3B", *xyz[i], *rgb[i]))
        path = f.name
    a, b = ply.read_xyzrgb(path)
    os.unlink(path)
    assert np.array_equal(a, xyz.astype(np.float32))
    assert np.array_equal(b, rgb.astype(np.float32) / np.float32(255.0))


def test_gauss_ply_reader_on_reference_asset():
    """A 3,000-row subset of the reference's own capture (asset/bulba.ply,
    written by tests/golden/make_golden.py)."""
    path = os.path.join(os.path.dirname(__file__), "golden", "bulba_subset.ply")
    d = ply.read_3d_gauss_splat(path)
    assert d["xyz"].shape == (3000, 3) and d["sh_coeffs"].shape == (3000, 16, 3)
    assert np.allclose(np.linalg.norm(d["quat"], axis=1), 1, atol=1e-5)
    assert (d["opacity"] >= 0).all() and (d["opacity"] <= 1).all() and (d["scale"] > 0).all()


def test_dlpack_layer_rejects_cpu_tensors():
    import torch
    from del_splat_dlpack import del_splat_dlpack as L3
    x = torch.zeros((4, 3))
    with pytest.raises(NotImplementedError):
        L3.circle_splat_from_project_spheres(x, 0.1, torch.zeros(16), (8, 8), torch.zeros((4, 3)),
                                             torch.zeros(4), 0)
    with pytest.raises(ValueError):
        L3.circle_splat_from_project_spheres(x, 0.1, torch.zeros(15), (8, 8), torch.zeros((4, 3)),
                                             torch.zeros(4), 0)


def test_png_roundtrip_float_u8_and_rgba_u32():
    from dsplat.image import decode_png, encode_png
    rng = np.random.default_rng(5)
    f = rng.uniform(-0.1, 1.1, (7, 11, 3)).astype(np.float32)
    back = decode_png(encode_png(f))
    assert np.array_equal(back, np.clip(np.rint(f.astype(np.float64) * 255), 0, 255).astype(np.uint8))
    u = rng.integers(0, 256, (5, 4, 4), dtype=np.uint8)
    assert np.array_equal(decode_png(encode_png(u)), u)
    rgba = rng.integers(0, 2 ** 32, (3, 6), dtype=np.uint64).astype(np.uint32)
    assert np.array_equal(decode_png(encode_png(rgba)), rgba.view(np.uint8).reshape(3, 6, 4))


def _colmap_files(tmp_path):
    import struct
    cams = struct.pack("<Q", 2)
    cams += struct.pack("<iIQQ4d", 1, 1, 640, 480, 500.0, 510.0, 320.5, 239.5)
    cams += struct.pack("<iIQQ4d", 7, 1, 320, 200, 250.0, 250.0, 160.0, 100.0)
    imgs = struct.pack("<Q", 2)
    q0, t0 = (0.9238795, 0.0, 0.3826834, 0.0), (0.1, -0.2, 4.0)
    imgs += struct.pack("<i4d3di", 3, *q0, *t0, 1) + b"view_a.png\x00" + struct.pack("<Q", 2)
    imgs += struct.pack("<ddq", 10.5, 20.25, 5) + struct.pack("<ddq", 1.0, 2.0, -1)
    imgs += struct.pack("<i4d3di", 4, 1.0, 0.0, 0.0, 0.0, 0.0, 0.0, 3.0, 7) + b"b.jpg\x00" + struct.pack("<Q", 0)
    pts = struct.pack("<Q", 1) + struct.pack("<Q3d3BdQ", 5, 0.1, 0.2, 0.3, 10, 20, 30, 0.5, 2)
    pts += struct.pack("<4i", 3, 0, 4, 1)
    for name, data in (("cameras.bin", cams), ("images.bin", imgs), ("points3D.bin", pts)):
        (tmp_path / name).write_bytes(data)
    return tmp_path


def test_colmap_binary_model_and_views(tmp_path):
    from dsplat import colmap
    d = _colmap_files(tmp_path)
    cams = colmap.read_cameras(d / "cameras.bin")
    imgs = colmap.read_images(d / "images.bin")
    pts = colmap.read_points3d(d / "points3D.bin")
    assert [c.camera_id for c in cams] == [1, 7] and cams[0].params == (500.0, 510.0, 320.5, 239.5)
    assert imgs[0].name == "view_a.png" and imgs[1].name == "b.jpg" and imgs[1].camera_id == 7
    assert np.array_equal(imgs[0].point3d_ids, [5, -1]) and np.allclose(imgs[0].xys, [[10.5, 20.25], [1.0, 2.0]])
    assert pts[0].point3d_id == 5 and list(pts[0].rgb) == [10, 20, 30] and pts[0].track.tolist() == [[3, 0], [4, 1]]
    views = colmap.views_from_model(cams, imgs, near=0.5, far=50.0)
    rng = np.random.default_rng(3)
    for img, view in zip(imgs, views):
        cam = next(c for c in cams if c.camera_id == img.camera_id)
        R = colmap.qvec_to_rotation(img.qvec)
        M = view.mvp.astype(np.float64).reshape(4, 4).T  # column-major -> row-major
        # points in front of the camera land on the pinhole pixel, nearer -> larger ndc_z
        xc = np.c_[rng.uniform(-1, 1, (20, 2)), rng.uniform(1.0, 20.0, 20)]
        xw = (xc - img.tvec) @ R  # R^T (x_c - t)
        h = np.c_[xw, np.ones(20)] @ M.T
        ndc = h[:, :3] / h[:, 3:]
        fx, fy, cx, cy = cam.params
        u, v = fx * xc[:, 0] / xc[:, 2] + cx, fy * xc[:, 1] / xc[:, 2] + cy
        px = 0.5 * cam.width * ndc[:, 0] + 0.5 * cam.width
        py = -0.5 * cam.height * ndc[:, 1] + 0.5 * cam.height
        assert np.allclose(px, u, atol=1e-3) and np.allclose(py, v, atol=1e-3)
        order = np.argsort(xc[:, 2])
        assert np.all(np.diff(ndc[order, 2]) < 0)
        assert np.allclose(view.campos, -R.T @ img.tvec, atol=1e-5)
    # near plane -> +1, far plane -> -1
    R = colmap.qvec_to_rotation(imgs[1].qvec)
    M = views[1].mvp.astype(np.float64).reshape(4, 4).T
    for z, want in ((0.5, 1.0), (50.0, -1.0)):
        xw = (np.array([0.0, 0.0, z]) - imgs[1].tvec) @ R
        hh = M @ np.r_[xw, 1.0]
        assert abs(hh[2] / hh[3] - want) < 1e-6
