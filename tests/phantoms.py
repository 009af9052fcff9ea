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
    per axis and intensities U(0.2, 1), plus N(0, noise^2).  Each ellipsoid is
    evaluated inside its axis-aligned bounding box only."""
    rng = np.random.default_rng(seed)
    dims = tuple(int(n) for n in dims)
    s = min(dims) / 128.0
    vol = np.zeros(dims, dtype=np.float64)
    for _ in range(count):
        semi = rng.uniform(8, 40, 3) * s
        R = _rotation(rng.standard_normal(4))
        ctr = np.array([rng.uniform(0.25 * n, 0.75 * n) for n in dims])
        # half-widths of the rotated ellipsoid's bounding box along each axis
        half = np.sqrt(((R * semi[None, :]) ** 2).sum(axis=1))
        lo = [max(0, int(np.floor(ctr[k] - half[k]))) for k in range(3)]
        hi = [min(dims[k], int(np.ceil(ctr[k] + half[k])) + 1) for k in range(3)]
        d = [np.arange(lo[k], hi[k], dtype=np.float64) - ctr[k] for k in range(3)]
        q = np.zeros((hi[0] - lo[0], hi[1] - lo[1], hi[2] - lo[2]))
        for j in range(3):
            u = d[0][:, None, None] * R[0, j] + d[1][None, :, None] * R[1, j] + d[2][None, None, :] * R[2, j]
            q += (u / semi[j]) ** 2
        vol[lo[0]:hi[0], lo[1]:hi[1], lo[2]:hi[2]][q <= 1.0] += rng.uniform(0.2, 1.0)
    vol += noise * rng.standard_normal(dims)
    return vol.astype(dtype)
