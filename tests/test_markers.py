"""Marker geometry of the sphere-drag and many-rod workloads (host only)."""
import numpy as np

from couplb_b200.markers import fibonacci_sphere, random_rods


def test_fibonacci_sphere():
    x = fibonacci_sphere(12.0, (96, 96, 96))
    assert x.shape == (1810, 3)                  # round(4 pi R^2)
    r = np.linalg.norm(x - 96.0, axis=1)
    np.testing.assert_allclose(r, 12.0, rtol=1e-12)
    assert np.abs(x.mean(0) - 96.0).max() < 0.05  # evenly spread
    d = np.linalg.norm(x[:, None] - x[None], axis=2) + np.eye(len(x)) * 1e9
    assert 0.7 < d.min(1).mean() < 1.1            # about one marker per unit area


def test_random_rods():
    box = (512, 256, 256)
    x = random_rods(1000, 200, box, seed=5, wall_margin=3.0)
    assert x.shape == (200000, 3)
    assert x[:, 1].min() >= 3.0 and x[:, 1].max() <= 253.0
    assert (x >= 0).all() and (x < np.array(box)).all()
    rods = x.reshape(1000, 200, 3)
    step = np.diff(rods, axis=1)
    step = step - np.round(step / np.array(box)) * np.array(box)   # undo periodic wrap
    np.testing.assert_allclose(np.linalg.norm(step, axis=2), 1.0, rtol=1e-9)
    np.testing.assert_array_equal(x, random_rods(1000, 200, box, seed=5, wall_margin=3.0))
