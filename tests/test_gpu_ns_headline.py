"""NSSurfacelet(scales = 3, direction_levels = [2, 2, 3]) with the default
bank (Bernstein order 12, halfband order 1, transition 1, tight) at the sizes
the throughput figures are quoted on, against the float64 oracle through the C
ABI: 96^3 (one volume analysed and synthesised, output 96^3 x 49) and 128^3
(the fused batch workload).

Tolerances (float32 against float64):
- rel. L2 <= 1e-5 over all 49 subbands, and per subband rel. L2 <= 1e-5 and
  max |.| < 1e-4 (the reference's own device-vs-host bound,
  test/items/test_gpu.jl:51-218);
- synthesis of arbitrary coefficients and the adjoints at rel. L2 <= 1e-5;
- perfect reconstruction and Parseval energy within 1e-5
  (test/items/test_ns_surfacelet.jl:1-60, 218-237).

The oracle streams one subband at a time (src/transforms/ns_surfacelet.jl:
474-500), so the float64 coefficient set (822 MB at 128^3) is never held.
"""

import numpy as np
import pytest
import torch

from conftest import gpu_available
from oracle import ns as N

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not gpu_available(), reason="needs a CUDA device")]

KW = dict(scales=3, direction_levels=[2, 2, 3])
REL = 1e-5
SIZES = [(96, 96, 96), (128, 128, 128)]


def band_host(c, s):
    """Subband s (1-based) of a column-major device coefficient array, float64 on the host."""
    b = c[..., s - 1]
    return np.asfortranarray(b.permute(2, 1, 0).cpu().numpy().transpose()).astype(np.float64)


@pytest.fixture(scope="module", params=SIZES, ids=lambda d: "x".join(map(str, d)))
def case(request, sfl):
    dims = request.param
    t = sfl.NSSurfacelet(**KW)
    ws = sfl.make_workspace(t, "float32", dims)
    T = N.make_tables(N.NSParams.make(**KW), dims)
    x = np.random.default_rng(96 if dims[0] == 96 else 128).standard_normal(dims).astype(np.float32)
    yield dims, t, ws, T, x
    ws.close()
    torch.cuda.empty_cache()


def test_analyze_every_subband_matches_oracle(sfl, case):
    dims, t, ws, T, x = case
    assert ws.nsubbands == 49
    c = sfl.analyze(t, sfl.to_device(x), workspace=ws)
    err2 = ref2 = 0.0
    worst = []
    for s, band in N.analyze_stream(T, x.astype(np.float64)):
        got = band_host(c, s)
        e2 = float(np.sum((got - band) ** 2))
        r2 = float(np.sum(band ** 2))
        err2 += e2
        ref2 += r2
        worst.append((np.sqrt(e2 / r2), float(np.abs(got - band).max()), s))
    assert np.sqrt(err2 / ref2) <= REL
    for rel, mx, s in worst:
        assert rel <= REL, (s, rel)
        assert mx < 1e-4, (s, mx)
    # Parseval: the tight bank preserves energy (test_ns_surfacelet.jl:218-237)
    e_c = float((c.double() ** 2).sum())
    e_x = float(np.sum(x.astype(np.float64) ** 2))
    assert abs(e_c - e_x) <= 1e-5 * e_x
    # perfect reconstruction
    y = sfl.to_host(sfl.synthesize(t, c, workspace=ws)).astype(np.float64)
    assert np.linalg.norm(y - x) / np.linalg.norm(x) <= REL


def test_synthesize_arbitrary_coefficients_matches_oracle(sfl, case):
    dims, t, ws, T, x = case
    rng = np.random.default_rng(7)
    cd = sfl.volume_like(dims + (49,))
    host = {}
    for s in range(1, 50):
        b = rng.standard_normal(dims).astype(np.float32)
        host[s] = b
        cd[..., s - 1].copy_(sfl.to_device(b))
    y = sfl.to_host(sfl.synthesize(t, cd, workspace=ws)).astype(np.float64)
    ref = N.synthesize_stream(T, lambda s: host[s].astype(np.float64))
    assert np.linalg.norm(y - ref) / np.linalg.norm(ref) <= REL
    # the adjoint of analysis equals synthesis for the tight bank; against the oracle's A^T
    ya = sfl.to_host(sfl.adjoint_analyze(ws, cd)).astype(np.float64)
    assert np.linalg.norm(ya - ref) / np.linalg.norm(ref) <= REL


def test_adjoint_synthesize_matches_oracle(sfl, case):
    dims, t, ws, T, x = case
    g = sfl.adjoint_synthesize(ws, sfl.to_device(x))
    err2 = ref2 = 0.0
    X = N.rfft3(x.astype(np.float64))
    for s, M in N.subband_masks(T, analysis=False):
        band = N.irfft3(X * M, dims)
        got = band_host(g, s)
        err2 += float(np.sum((got - band) ** 2))
        ref2 += float(np.sum(band ** 2))
    assert np.sqrt(err2 / ref2) <= REL
