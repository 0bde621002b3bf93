"""Workload generators: sizes and determinism (no GPU)."""
import numpy as np

from rtb200 import scenes


def test_primary_scene_size_and_determinism():
    a = scenes.scene_spheres_100k(0)
    b = scenes.scene_spheres_100k(0)
    assert a.shape == (100002, 9) and a.dtype == np.float32
    assert np.array_equal(a, b)
    assert not np.array_equal(a, scenes.scene_spheres_100k(1))
    assert np.abs(a[2:]).max() < 60.0


def test_mesh_scene_exact_count():
    t = scenes.scene_meshes(3, 50000)
    assert t.shape == (50000, 9)
    assert np.array_equal(t, scenes.scene_meshes(3, 50000))


def test_camera_rays():
    r = scenes.pinhole_rays(64, 36, scenes.CAM_EYE, scenes.CAM_TARGET)
    assert r.shape == (64 * 36,)
    n = np.linalg.norm(r["dir"], axis=1)
    assert np.allclose(n, 1, atol=1e-6)


def test_diffuse_rays_in_hemisphere():
    pts = np.zeros((100, 3), np.float32)
    nrm = np.tile(np.array([[0, 0, 1]], np.float32), (100, 1))
    r = scenes.diffuse_rays(pts, nrm, 5000, seed=1)
    assert np.all(r["dir"][:, 2] >= 0)
    assert np.allclose(np.linalg.norm(r["dir"], axis=1), 1, atol=1e-5)
    # cosine-weighted: E[cos] = 2/3
    assert abs(r["dir"][:, 2].mean() - 2 / 3) < 0.02
    assert np.allclose(r["org"][:, 2], 1e-3)


def test_shadow_rays_stop_short_of_light():
    pts = np.zeros((10, 3), np.float32)
    nrm = np.tile(np.array([[0, 1, 0]], np.float32), (10, 1))
    r = scenes.shadow_rays(pts, nrm, 100, seed=2)
    end = r["org"] + r["tmax"][:, None] * r["dir"]
    assert np.all(end[:, 1] < scenes.LIGHT_CENTER[1])
    assert np.all(np.abs(end[:, 0]) <= 0.51) and np.all(np.abs(end[:, 2]) <= 0.51)
