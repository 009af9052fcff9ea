"""The fused soft-threshold denoiser against the three separate calls
(analyze, threshold, synthesize) of the same pipeline, bit for bit, and
against the float64 oracle; per-subband thresholds; the NDFB bank."""

import numpy as np
import pytest
import torch

from conftest import gpu_available
from oracle import ns as N
from phantoms import ellipsoid_phantom

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not gpu_available(), reason="needs a CUDA device")]


def soft(c, tau):
    return torch.sign(c) * torch.clamp(c.abs() - tau, min=0)


@pytest.mark.parametrize("dims,pipeline,kw", [
    ((64, 64, 64), "slabs", dict(scales=3, direction_levels=[2, 2, 3])),
    ((64, 64, 64), "lines", dict(scales=3, direction_levels=[2, 2, 3])),
    ((128, 96, 64), "slabs", dict(scales=2, direction_levels=[2, 3], bernstein_order=8)),
    ((40, 36, 48), "lines", dict(scales=2, direction_levels=[1, 2], bernstein_order=6, tight=False)),
    # fused axis-1 kernel on the line pipeline, an odd number of axis-1 lines (the last pair is one line)
    ((64, 33, 35), "lines", dict(scales=2, direction_levels=[2, 1], bernstein_order=6)),
    ((256, 32, 33), "lines", dict(scales=1, direction_levels=[2], bernstein_order=6, tight=False)),
    ((96, 40, 24), "lines", dict(scales=2, direction_levels=[1, 1], bernstein_order=6)),
])
def test_denoise_equals_three_calls(sfl, dims, pipeline, kw):
    ws = sfl.make_workspace(sfl.NSSurfacelet(**kw), "float32", dims)
    ws.set_pipeline(pipeline)
    x = ellipsoid_phantom(dims, seed=4, noise=0.2)
    xd = sfl.to_device(x)
    rng = np.random.default_rng(1)
    tau = torch.from_numpy(rng.uniform(0.0, 0.3, ws.nsubbands).astype(np.float32)).cuda()
    y = sfl.denoise(ws, xd, tau)
    c = sfl.analyze(ws, xd)
    ref = sfl.synthesize(ws, sfl.as_colmajor(soft(c, tau)))
    assert torch.equal(y, ref)
    if dims == (64, 64, 64) and pipeline == "slabs":
        T = N.make_tables(N.NSParams.make(**kw), dims)
        c64 = N.analyze(T, x.astype(np.float64))
        t64 = tau.cpu().numpy().astype(np.float64)
        y64 = N.synthesize(T, np.sign(c64) * np.maximum(np.abs(c64) - t64, 0))
        assert np.linalg.norm(sfl.to_host(y) - y64) / np.linalg.norm(y64) <= 1e-5
        # the scalar form keeps the lowpass
        y1 = sfl.denoise(ws, xd, 0.1)
        t1 = torch.full((ws.nsubbands,), 0.1, device="cuda")
        t1[0] = 0
        assert torch.equal(y1, sfl.synthesize(ws, sfl.as_colmajor(soft(c, t1))))


def test_denoise_ndfb_and_errors(sfl):
    dims = (64, 64, 64)
    ws = sfl.make_workspace(sfl.NDFB(levels=2, bernstein_order=6), "float32", dims)
    xd = sfl.to_device(ellipsoid_phantom(dims, seed=6, noise=0.2))
    y = sfl.denoise(ws, xd, 0.05)
    c = sfl.analyze(ws, xd)
    assert torch.equal(y, sfl.synthesize(ws, sfl.as_colmajor(soft(c, 0.05))))
    with pytest.raises(sfl.DimensionMismatch):
        sfl.denoise(ws, xd, torch.zeros(3, device="cuda"))
    wz = sfl.make_workspace(sfl.NDFB(levels=1, bernstein_order=6), "complex64", (16, 16, 16))
    with pytest.raises(sfl.ArgumentError):
        sfl.denoise(wz, sfl.volume_like((16, 16, 16), "complex64"), 0.1)
