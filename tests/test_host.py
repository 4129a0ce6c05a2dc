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
    path = "/root/reference/asset/bulba.ply"
    if not os.path.exists(path):
        pytest.skip("reference asset not present")
    d = ply.read_3d_gauss_splat(path)
    assert d["xyz"].shape == (11982, 3) and d["sh_coeffs"].shape == (11982, 16, 3)
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
