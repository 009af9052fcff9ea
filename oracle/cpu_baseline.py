"""Timed CPU baseline: the oracle's NSSurfacelet and Surfacelet restatements
run multithreaded on the host (scipy.fft with `workers`), float32 or float64.

Test/measurement infrastructure only: bench.py times it as the reference arm
and as `cpu_baseline`; the product never calls it.  The reference's own CPU
path (multithreaded Julia + FFTW) cannot run on this image (no Julia
toolchain, and its MultiscaleFilterBanks / AbstractMultiscaleTransforms
dependencies are not vendored), so this port of the same algorithms stands
in for it.  The masks are the oracle's (src/transforms/ns_surfacelet.jl
cascade: one rfft, 49 masked irffts; synthesis mirrored).
"""

import os

import numpy as np
import scipy.fft as sfft

from . import decimated as D
from . import ns as N


class NSBaseline:
    """analyze / synthesize of NSSurfacelet with precomputed float masks."""

    def __init__(self, p, dims, dtype=np.float32, workers=None):
        self.T = N.make_tables(p, dims)
        self.dims = tuple(dims)
        self.dtype = dtype
        self.workers = workers or os.cpu_count()
        ct = np.complex64 if dtype == np.float32 else np.complex128
        self.masks_a = [(s, M.astype(dtype)) for s, M in N.subband_masks(self.T, analysis=True)]
        self.masks_s = [(s, M.astype(dtype)) for s, M in N.subband_masks(self.T, analysis=False)]
        self.ct = ct

    def rfft3(self, x):
        return sfft.rfftn(x, axes=(1, 2, 0), workers=self.workers)

    def irfft3(self, X):
        d = self.dims
        return sfft.irfftn(X, s=(d[1], d[2], d[0]), axes=(1, 2, 0), workers=self.workers)

    def analyze(self, x, synth_masks=False):
        X = self.rfft3(x.astype(self.dtype, copy=False))
        c = np.empty(self.dims + (len(self.masks_a),), dtype=self.dtype)
        for s, M in (self.masks_s if synth_masks else self.masks_a):
            c[..., s - 1] = self.irfft3(X * M)
        return c

    def synthesize(self, c, analysis_masks=False):
        acc = None
        for s, M in (self.masks_a if analysis_masks else self.masks_s):
            F = self.rfft3(c[..., s - 1]) * M
            acc = F if acc is None else acc + F
        return self.irfft3(acc)


class SurfBaseline:
    """analyze / synthesize of the decimated Surfacelet (the oracle's float64
    restatement; numpy FFTs)."""

    def __init__(self, p, dims):
        self.T = D.make_tables(p, dims)

    def analyze(self, x):
        return D.analyze(self.T, x)

    def synthesize(self, c):
        return D.synthesize(self.T, c)
