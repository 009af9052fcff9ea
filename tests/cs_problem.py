"""The compressed-sensing problem of the complex workload, in float64 on the
oracle (test infrastructure):

    L(c) = 0.5 || M o FFT3(synthesize(c)) - y ||^2 + lam sum sqrt(|c|^2 + eps^2)

M a seeded Bernoulli(0.25) k-space mask with a fully sampled 16^3 centre
(DC-centred, wrap-around indexing), y = M o FFT3(phantom), lam = 1e-3,
eps = 1e-6.  Complex volumes and coefficients go through the real oracle
channel by channel; gradients pack d/dRe + i d/dIm."""

import numpy as np

from oracle import ns as N
from phantoms import ellipsoid_phantom

LAM, EPS = 1e-3, 1e-6


def synthesize_c(T, c):
    return N.synthesize(T, c.real) + 1j * N.synthesize(T, c.imag)


def synthesize_t_c(T, g):
    return N.adjoint_synthesize(T, g.real) + 1j * N.adjoint_synthesize(T, g.imag)


def analyze_c(T, x):
    return N.analyze(T, x.real) + 1j * N.analyze(T, x.imag)


def analyze_t_c(T, g):
    return N.adjoint_analyze(T, g.real) + 1j * N.adjoint_analyze(T, g.imag)


def oracle_loss(T, c, M, y):
    r = M * np.fft.fftn(synthesize_c(T, c)) - y
    return 0.5 * np.sum(np.abs(r) ** 2) + LAM * np.sum(np.sqrt(np.abs(c) ** 2 + EPS ** 2))


def oracle_grad(T, c, M, y):
    x = synthesize_c(T, c)
    r = M * np.fft.fftn(x) - y
    gx = np.fft.ifftn(M * r) * x.size
    return synthesize_t_c(T, gx) + LAM * c / np.sqrt(np.abs(c) ** 2 + EPS ** 2)


def make_problem(dims, seed):
    rng = np.random.default_rng(seed)
    ph = ellipsoid_phantom(dims, seed=seed).astype(np.float64)
    ph = ph + 1j * ellipsoid_phantom(dims, seed=seed + 1)
    M = (rng.random(dims) < 0.25).astype(np.float64)
    c = [np.r_[0:min(8, n), max(n - 8, min(8, n)):n] for n in dims]   # |k| < 8 on every axis, wrapped
    M[np.ix_(*c)] = 1.0
    y = M * np.fft.fftn(ph)
    return ph, M, y, rng


