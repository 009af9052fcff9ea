"""The large-volume workload: NSSurfacelet(scales=4, direction_levels=[2,2,3,3])
on a 256^3 phantom (S = 73, 4.9 GB of float32 coefficients if materialized),
streamed one subband at a time through analyze -> f -> synthesize; and the
bfloat16 coefficient format (per-subband float32 scales) against float32 and
the float64 oracle."""

import numpy as np
import pytest
import torch

from conftest import gpu_available
from oracle import ns as N
from phantoms import ellipsoid_phantom

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not gpu_available(), reason="needs a CUDA device")]


def rel(a, b):
    d = torch.complex128 if a.is_complex() or b.is_complex() else torch.float64
    return float(torch.linalg.vector_norm((a - b).to(d)) / torch.linalg.vector_norm(b.to(d)))


def soft(b, tau):
    return torch.sign(b) * torch.clamp(b.abs() - tau, min=0)


def test_stream_256_j4_parseval_reconstruction_and_shrinkage(sfl):
    dims = (256, 256, 256)
    kw = dict(scales=4, direction_levels=[2, 2, 3, 3])
    x = ellipsoid_phantom(dims, count=24, seed=5)
    t = sfl.NSSurfacelet(**kw)
    wa, ws = sfl.make_workspace(t, "float32", dims), sfl.make_workspace(t, "float32", dims)
    assert wa.nsubbands == 73
    xd = sfl.to_device(x)
    y = sfl.volume_like(dims)
    energy, firsts = [0.0], {}

    def keep(i, b):
        energy[0] += float((b.double() ** 2).sum())
        if len(firsts) < 2:
            firsts[i] = sfl.to_host(b)
        return b

    sfl.analyze_synthesize_stream(keep, y, xd, wa, ws)
    e0 = float(np.sum(x.astype(np.float64) ** 2))
    assert abs(energy[0] - e0) / e0 <= 2e-6            # Parseval (tight frame)
    assert rel(y, xd) <= 1e-5                            # perfect reconstruction
    # the first two streamed subbands against the float64 oracle
    T = N.make_tables(N.NSParams.make(**kw), dims)
    for i, band in N.analyze_stream(T, x.astype(np.float64)):
        if i in firsts:
            r = np.linalg.norm(firsts[i] - band) / np.linalg.norm(band)
            assert r <= 1e-5, (i, r)
            del firsts[i]
        if not firsts:
            break
    # shrinkage streamed subband by subband = shrinkage of the materialized set
    tau = 0.05
    y2 = sfl.volume_like(dims)
    sfl.analyze_synthesize_stream(lambda i, b: sfl.as_colmajor(soft(b, tau)), y2, xd, wa, ws)
    c = sfl.analyze(wa, xd)
    y3 = sfl.synthesize(ws, sfl.as_colmajor(soft(c, tau)))
    assert torch.equal(y2, y3)


@pytest.mark.parametrize("dims,pipeline", [((64, 64, 64), "slabs"), ((64, 64, 64), "lines"),
                                           ((128, 128, 128), "slabs")])
def test_bf16_coefficients(sfl, dims, pipeline):
    kw = dict(scales=3, direction_levels=[2, 2, 3])
    ws = sfl.make_workspace(sfl.NSSurfacelet(**kw), "float32", dims)
    ws.set_pipeline(pipeline)
    x = ellipsoid_phantom(dims, seed=2)
    xd = sfl.to_device(x)
    c16, s = sfl.analyze_bf16(ws, xd)
    c32 = sfl.analyze(ws, xd)
    # scales are powers of two, stored values within [-1, 1]
    assert bool(torch.all(torch.log2(s) == torch.round(torch.log2(s))))
    assert float(c16.float().abs().max()) <= 1.0
    ce = sfl.as_colmajor(c16.float() * s)
    r16 = rel(ce, c32)
    assert 1e-4 <= r16 <= 4e-3, r16                      # bfloat16 accuracy, not float32
    # synthesis from bfloat16 = float32 synthesis of the expanded values
    y16 = sfl.synthesize_bf16(ws, c16, s)
    assert torch.equal(y16, sfl.synthesize(ws, ce))
    assert rel(y16, xd) <= 4e-3
    if dims == (64, 64, 64) and pipeline == "slabs":
        cref = torch.from_numpy(N.analyze(N.make_tables(N.NSParams.make(**kw), dims), x.astype(np.float64)))
        cref = cref.cuda()
        assert rel(c32, cref) <= 1e-5 and rel(ce, cref) <= 4e-3
    with pytest.raises(sfl.ArgumentError):
        sfl.synthesize_bf16(ws, c16.float(), s)
