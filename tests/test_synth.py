"""Seeded synthetic inputs: deterministic, with the stated noise model (CPU only)."""
import numpy as np

from oglfusionkinectv2_b200 import synth


def test_frames_are_deterministic_and_corrupted_as_specified():
    w = synth.plain_c1(3)
    a, b = w.frame(1), w.frame(1)
    np.testing.assert_array_equal(a, b)
    assert a.dtype == np.uint16 and a.shape == (424, 512)
    z = w.clean_depth(1)
    seen = np.isfinite(z) & (z >= 0.55) & (z <= 4.4)
    dropped = (a == 0) & seen
    assert 0.01 < dropped.sum() / seen.sum() < 0.03  # 2% seeded dropouts
    ok = seen & (a > 0)
    err = a[ok] / 1000.0 - z[ok]
    sigma = 0.0012 + 0.0019 * (z[ok] - 0.4) ** 2
    assert abs(np.std(err / np.sqrt(sigma ** 2 + (0.001 ** 2) / 12)) - 1.0) < 0.1
    assert np.all(a[a > 0] >= 500) and np.all(a <= 4500)


def test_orbit_geometry():
    w = synth.plain_c1(10)
    c = np.array([0.75, 0.75, 0.75])
    for T in w.poses:
        R = T[:3, :3]
        np.testing.assert_allclose(R.T @ R, np.eye(3), atol=1e-12)
        horiz = np.hypot(T[0, 3] - c[0], T[2, 3] - c[2])
        assert abs(horiz - 1.2) < 1e-9
    step = np.linalg.norm(w.poses[1][:3, 3] - w.poses[0][:3, 3])
    assert 0.009 < step < 0.014  # 0.5 deg at 1.2 m plus 2 mm drift


def test_scene_objects_inside_volume():
    for w in (synth.plain_c1(1), synth.precision_c2(1, size=64)):
        dim = w.config.volumeDimensions[0]
        for c, r in w.scene.spheres:
            assert all(r <= v <= dim - r for v in c)
