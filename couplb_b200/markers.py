"""Lagrangian marker sets of the sphere-drag and many-rod workloads
(synthetic geometry, seeded)."""
import numpy as np


def fibonacci_sphere(radius, center, n=None):
    """Markers on a sphere by the golden-angle (Fibonacci) spiral; n defaults
    to the sphere area in lattice units (about one marker per unit area)."""
    if n is None:
        n = int(round(4.0 * np.pi * radius * radius))
    i = np.arange(n, dtype=np.float64) + 0.5
    phi = np.arccos(1.0 - 2.0 * i / n)
    theta = np.pi * (1.0 + 5.0 ** 0.5) * i
    c = np.asarray(center, dtype=np.float64)
    return np.stack([c[0] + radius * np.cos(theta) * np.sin(phi),
                     c[1] + radius * np.sin(theta) * np.sin(phi),
                     c[2] + radius * np.cos(phi)], axis=1)


def random_rods(n_rods, per_rod, box, seed, spacing=1.0, wall_margin=None):
    """n_rods straight rods of per_rod markers at unit spacing, random centre
    (uniform in the box) and orientation (uniform on the sphere), from
    numpy's PCG64 with the given seed.  With wall_margin, rods whose markers
    come within that distance of the y faces are redrawn.  Returns
    (n_rods * per_rod, 3) positions wrapped into the periodic box."""
    rng = np.random.default_rng(seed)
    box = np.asarray(box, dtype=np.float64)
    s = (np.arange(per_rod) - 0.5 * (per_rod - 1)) * spacing
    out = []
    while len(out) < n_rods:
        c = rng.random(3) * box
        d = rng.normal(size=3)
        d /= np.linalg.norm(d)
        pts = c[None, :] + s[:, None] * d[None, :]
        if wall_margin is not None and (pts[:, 1].min() < wall_margin or
                                        pts[:, 1].max() > box[1] - wall_margin):
            continue
        out.append(pts)
    x = np.concatenate(out)
    return np.mod(x, box)
