"""The large streaming workload against the float64 oracle over every subband:
NSSurfacelet(scales = 4, direction_levels = [2, 2, 3, 3]) on a 256^3 phantom
(24 seeded ellipsoids plus N(0, 0.05^2) noise), S = 73.

One streamed pass (src/transforms/ns_surfacelet.jl:474-500, 583-641): the
device analyses the phantom one subband at a time while the oracle produces
the same subband in float64, and
- the float32 coefficients, and the bfloat16 coefficients with their
  per-subband float32 scales, are measured against the oracle's (rel. L2 over
  all 73 subbands: <= 1e-5 for float32, <= 4e-3 for bfloat16's 8-bit
  significand);
- the oracle's coefficients, rounded to float32, are pushed into the device's
  streaming synthesis, whose Kahan-compensated accumulation of the 73
  subbands must match the oracle's float64 synthesis of the same values to
  rel. L2 <= 1e-5.
The oracle holds one subband and one accumulator at a time (float64 FFTs on
the host's threads).
"""

import os

import numpy as np
import pytest
import torch

from conftest import gpu_available
from oracle import ns as N
from phantoms import ellipsoid_phantom

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not gpu_available(), reason="needs a CUDA device")]

KW = dict(scales=4, direction_levels=[2, 2, 3, 3])


def host64(b):
    return np.asfortranarray(b.permute(2, 1, 0).cpu().numpy().transpose()).astype(np.float64)


def test_stream_256_every_subband_and_synthesis_against_oracle(sfl):
    dims = (256, 256, 256)
    N.set_fft_workers(os.cpu_count() or 1)
    try:
        x = ellipsoid_phantom(dims, count=24, seed=5)
        t = sfl.NSSurfacelet(**KW)
        wa, ws = sfl.make_workspace(t, "float32", dims), sfl.make_workspace(t, "float32", dims)
        assert wa.nsubbands == 73
        xd = sfl.to_device(x)
        c16, sc16 = sfl.analyze_bf16(wa, xd)
        T = N.make_tables(N.NSParams.make(**KW), dims)
        bands = N.analyze_stream(T, x.astype(np.float64))
        masks = N.subband_masks(T, analysis=False)
        acc = np.zeros((dims[0] // 2 + 1,) + dims[1:], dtype=np.complex128)
        e32, e16, ref, order = [0.0], [0.0], [0.0], []

        def f(i, b):
            s, band = next(bands)
            assert s == i
            order.append(i)
            e32[0] += float(np.sum((host64(b) - band) ** 2))
            b16 = c16[..., i - 1].float() * sc16[i - 1]
            e16[0] += float(np.sum((host64(b16) - band) ** 2))
            ref[0] += float(np.sum(band ** 2))
            # the oracle's coefficients, as float32, into the device synthesis and the oracle's
            b32 = band.astype(np.float32)
            sm, M = next(masks)
            assert sm == i
            acc[...] += N.rfft3(b32.astype(np.float64)) * M
            return sfl.to_device(b32)

        y = sfl.volume_like(dims)
        sfl.analyze_synthesize_stream(f, y, xd, wa, ws)
        assert order == list(range(2, 74)) + [1]
        r32 = np.sqrt(e32[0] / ref[0])
        r16 = np.sqrt(e16[0] / ref[0])
        assert r32 <= 1e-5, r32
        assert r16 <= 4e-3, r16
        yref = N.irfft3(acc, dims)
        rs = np.linalg.norm(host64(y) - yref) / np.linalg.norm(yref)
        assert rs <= 1e-5, rs
        print(f"\n256^3 S=73 vs float64: float32 coefficients {r32:.3e}, bfloat16 {r16:.3e}, "
              f"synthesis of oracle coefficients {rs:.3e}")
    finally:
        N.set_fft_workers(1)
