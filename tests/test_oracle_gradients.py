"""The float64 oracle gradient of the compressed-sensing loss against
central differences (h = 1e-4, 32 random unit directions), directly in c and
through analyze (x -> L(analyze(x)))."""

import numpy as np

from cs_problem import analyze_c, analyze_t_c, make_problem, oracle_grad, oracle_loss
from oracle import ns as N


def test_oracle_gradient_by_central_differences():
    dims = (32, 32, 32)
    T = N.make_tables(N.NSParams.make(scales=3, direction_levels=[2, 2, 3]), dims)
    ph, M, y, rng = make_problem(dims, 3)
    c0 = analyze_c(T, ph)
    c = c0 + 0.1 * (rng.standard_normal(c0.shape) + 1j * rng.standard_normal(c0.shape))
    g = oracle_grad(T, c, M, y)
    h = 1e-4
    for _ in range(32):
        d = rng.standard_normal(c.shape) + 1j * rng.standard_normal(c.shape)
        d /= np.linalg.norm(d)
        fd = (oracle_loss(T, c + h * d, M, y) - oracle_loss(T, c - h * d, M, y)) / (2 * h)
        an = float(np.sum((np.conj(g) * d).real))
        assert abs(fd - an) <= 1e-6 * abs(an) + 1e-9 * np.linalg.norm(g), (fd, an)


def test_oracle_gradient_through_analyze_by_central_differences():
    dims = (24, 20, 16)
    T = N.make_tables(N.NSParams.make(scales=2, direction_levels=[1, 2], bernstein_order=6), dims)
    ph, M, y, rng = make_problem(dims, 5)
    x = ph + 0.1 * (rng.standard_normal(dims) + 1j * rng.standard_normal(dims))
    gx = analyze_t_c(T, oracle_grad(T, analyze_c(T, x), M, y))
    h = 1e-4
    for _ in range(8):
        d = rng.standard_normal(dims) + 1j * rng.standard_normal(dims)
        d /= np.linalg.norm(d)
        fd = (oracle_loss(T, analyze_c(T, x + h * d), M, y) - oracle_loss(T, analyze_c(T, x - h * d), M, y)) / (2 * h)
        an = float(np.sum((np.conj(gx) * d).real))
        assert abs(fd - an) <= 1e-6 * abs(an) + 1e-9 * np.linalg.norm(gx), (fd, an)
