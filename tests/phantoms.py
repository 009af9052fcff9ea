"""Seeded synthetic volumes: a sum of randomly rotated solid ellipsoids plus
Gaussian noise (the stand-in for the phantoms of the measurement plan)."""

import numpy as np


def _rotation(q):
    a, b, c, d = q / np.linalg.norm(q)
    return np.array([[a * a + b * b - c * c - d * d, 2 * (b * c - a * d), 2 * (b * d + a * c)],
                     [2 * (b * c + a * d), a * a - b * b + c * c - d * d, 2 * (c * d - a * b)],
                     [2 * (b * d - a * c), 2 * (c * d + a * b), a * a - b * b - c * c + d * d]])


def ellipsoid_phantom(dims, count=12, seed=0, noise=0.05, dtype=np.float32):
    """count ellipsoids with semi-axes U[8, 40] voxels (scaled by min(dims)/128),
    uniform random rotations (random unit quaternions), centres U[0.25 n, 0.75 n]
    per axis and intensities U(0.2, 1), plus N(0, noise^2)."""
    rng = np.random.default_rng(seed)
    dims = tuple(int(n) for n in dims)
    s = min(dims) / 128.0
    g = np.stack(np.meshgrid(*[np.arange(n, dtype=np.float64) for n in dims], indexing="ij"), axis=-1)
    vol = np.zeros(dims, dtype=np.float64)
    for _ in range(count):
        semi = rng.uniform(8, 40, 3) * s
        R = _rotation(rng.standard_normal(4))
        ctr = np.array([rng.uniform(0.25 * n, 0.75 * n) for n in dims])
        u = (g - ctr) @ R
        vol[np.sum((u / semi) ** 2, axis=-1) <= 1.0] += rng.uniform(0.2, 1.0)
    vol += noise * rng.standard_normal(dims)
    return vol.astype(dtype)
