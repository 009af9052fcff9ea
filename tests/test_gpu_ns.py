"""NSSurfacelet on the B200 through the C ABI, against the float64 oracle.

Tolerances: rel. L2 <= 1e-5 of the whole coefficient set or volume against
float64 (the float32 bar), the reference's own GPU-vs-CPU bound max|.| < 1e-4
per subband (test/items/test_gpu.jl:51-218), and exact equality where the
reference asserts it (complex = real + i imag, streaming = materialized).
"""

import numpy as np
import pytest
import torch

from conftest import gpu_available
from oracle import ns as N

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not gpu_available(), reason="needs a CUDA device")]

REL = 1e-5


def rel_l2(a, b):
    a = np.asarray(a, dtype=np.complex128 if np.iscomplexobj(a) else np.float64)
    return float(np.linalg.norm((a - b).ravel()) / max(np.linalg.norm(np.asarray(b).ravel()), 1e-300))


def oracle_tables(dims, **kw):
    return N.make_tables(N.NSParams.make(**kw), dims)


CASES = [
    ((16, 16, 16), dict(scales=2, direction_levels=[1, 2], bernstein_order=6)),
    ((12, 20, 8), dict(scales=3, direction_levels=[1, 1, 2], bernstein_order=6)),
    ((15, 20, 8), dict(scales=3, direction_levels=[1, 1, 2], bernstein_order=6)),
    ((9, 7, 5), dict(scales=2, direction_levels=[1, 2], bernstein_order=6)),
    ((32, 32, 32), dict(scales=3, direction_levels=[2, 2, 3])),
    ((26, 30, 12), dict(scales=1, direction_levels=[3], bernstein_order=6, transition=0.5)),
    ((16, 12, 20), dict(scales=2, direction_levels=[1, 2], bernstein_order=6, tight=False)),
    # sizes the slab and plane-major pipelines also support
    ((64, 64, 64), dict(scales=3, direction_levels=[2, 2, 3])),
    ((96, 64, 128), dict(scales=2, direction_levels=[1, 3], bernstein_order=6)),
    ((128, 128, 64), dict(scales=2, direction_levels=[2, 2], bernstein_order=8, tight=False)),
    ((64, 96, 32), dict(scales=3, direction_levels=[1, 2, 2], bernstein_order=8)),
]
PIPELINE_CASES = [(d, k, "lines") for d, k in CASES] + [(d, k, "slabs") for d, k in CASES[-4:]]


@pytest.mark.parametrize("dims,kw,pipeline", PIPELINE_CASES)
def test_analyze_synthesize_match_oracle(sfl, dims, kw, pipeline):
    rng = np.random.default_rng(202)
    x = rng.standard_normal(dims).astype(np.float32)
    t = sfl.NSSurfacelet(**kw)
    T = oracle_tables(dims, **kw)
    ws = sfl.make_workspace(t, "float32", dims)
    ws.set_pipeline(pipeline)
    xd = sfl.to_device(x)
    c = sfl.analyze(t, xd, workspace=ws)
    ch = sfl.to_host(c)
    cref = N.analyze(T, x.astype(np.float64))
    assert rel_l2(ch, cref) <= REL
    for i in range(cref.shape[-1]):
        assert np.abs(ch[..., i] - cref[..., i]).max() < 1e-4
    r = sfl.to_host(sfl.synthesize(t, c, workspace=ws))
    assert rel_l2(r, x) <= REL       # perfect reconstruction in float32
    # synthesis of arbitrary coefficients against the oracle
    cr = rng.standard_normal(cref.shape).astype(np.float32)
    y = sfl.to_host(sfl.synthesize(t, sfl.to_device(cr), workspace=ws))
    assert rel_l2(y, N.synthesize(T, cr.astype(np.float64))) <= REL
    # no bounded wait of the kernels ran out
    import ctypes as C
    st = C.c_int32(-1)
    assert sfl.lib.sfl_plan_status(ws._h, C.byref(st), 0) == 0 and st.value == 0


@pytest.mark.parametrize("dims,kw", [CASES[0], CASES[2], CASES[6]])
def test_adjoints(sfl, dims, kw):
    rng = np.random.default_rng(7)
    t = sfl.NSSurfacelet(**kw)
    T = oracle_tables(dims, **kw)
    ws = sfl.make_workspace(t, "float32", dims)
    x = rng.standard_normal(dims).astype(np.float32)
    c = rng.standard_normal(dims + (ws.nsubbands,)).astype(np.float32)
    ax = sfl.to_host(sfl.adjoint_analyze(ws, sfl.to_device(c)))
    assert rel_l2(ax, N.adjoint_analyze(T, c.astype(np.float64))) <= REL
    sx = sfl.to_host(sfl.adjoint_synthesize(ws, sfl.to_device(x)))
    assert rel_l2(sx, N.adjoint_synthesize(T, x.astype(np.float64))) <= REL
    # <A x, c> = <x, A^T c>
    Ax = sfl.to_host(sfl.analyze(ws, sfl.to_device(x))).astype(np.float64)
    assert np.sum(Ax * c) == pytest.approx(np.sum(x.astype(np.float64) * ax), rel=1e-5)


def test_parseval_and_constant(sfl):
    # test/items/test_ns_surfacelet.jl:69-77, 218-237
    dims = (16, 16, 16)
    t = sfl.NSSurfacelet(scales=2, direction_levels=[1, 1], bernstein_order=6)
    x = np.random.default_rng(98).standard_normal(dims).astype(np.float32)
    c = sfl.to_host(sfl.analyze(t, sfl.to_device(x))).astype(np.float64)
    assert np.sum(c * c) == pytest.approx(np.sum(x.astype(np.float64) ** 2), rel=1e-5)
    k = sfl.to_host(sfl.analyze(t, sfl.to_device(np.full(dims, 1.75, np.float32))))
    assert np.abs(k[..., 0] - 1.75).max() < 1e-5
    assert np.abs(k[..., 1:]).max() < 1e-5


def test_complex_equals_real_plus_i_imag_bit_for_bit(sfl):
    # test/items/test_ns_surfacelet.jl:140-152
    dims = (16, 16, 16)
    rng = np.random.default_rng(94)
    xr = rng.standard_normal(dims).astype(np.float32)
    xi = rng.standard_normal(dims).astype(np.float32)
    t = sfl.NSSurfacelet(scales=2, direction_levels=[1, 1], bernstein_order=6)
    cc = sfl.to_host(sfl.analyze(t, sfl.to_device(xr + 1j * xi)))
    cr = sfl.to_host(sfl.analyze(t, sfl.to_device(xr)))
    ci = sfl.to_host(sfl.analyze(t, sfl.to_device(xi)))
    assert np.array_equal(cc.real, cr) and np.array_equal(cc.imag, ci)
    z = sfl.to_host(sfl.synthesize(t, sfl.to_device(cc)))
    assert rel_l2(z, xr + 1j * xi) <= REL
    yr = sfl.to_host(sfl.synthesize(t, sfl.to_device(cr)))
    assert np.array_equal(z.real, yr)


def test_streaming_matches_materialized(sfl):
    # test/items/test_ns_surfacelet.jl:79-106
    dims = (16, 16, 16)
    t = sfl.NSSurfacelet(scales=2, direction_levels=[1, 2], bernstein_order=6)
    x = np.random.default_rng(92).standard_normal(dims).astype(np.float32)
    ws = sfl.make_workspace(t, "float32", dims)
    xd = sfl.to_device(x)
    ref = sfl.analyze(ws, xd)
    seen = []

    def f(i, band):
        seen.append(i)
        assert bool((band == ref[..., i - 1]).all())

    assert sfl.analyze(f, ws, xd) is None
    assert seen == list(range(2, ws.nsubbands + 1)) + [1]
    y = sfl.volume_like(dims)
    assert sfl.synthesize_(lambda i: ref[..., i - 1], y, ws) is y
    ym = sfl.synthesize(ws, ref)
    assert bool((y == ym).all())
    assert rel_l2(sfl.to_host(y), x) <= REL
    with pytest.raises(sfl.DimensionMismatch):
        sfl.synthesize_(lambda i: sfl.volume_like((4, 4, 4)), sfl.volume_like(dims), ws)


@pytest.mark.parametrize("dims,pipeline", [((64, 64, 64), "slabs"), ((64, 64, 64), "lines"),
                                           ((16, 16, 16), "lines")])
@pytest.mark.parametrize("dtype", ["float32", "complex64"])
def test_streaming_equals_materialized_bit_for_bit(sfl, dims, pipeline, dtype):
    # test/items/test_ns_surfacelet.jl:79-106, 108-138
    import torch
    t = sfl.NSSurfacelet(scales=2, direction_levels=[1, 2], bernstein_order=6)
    rng = np.random.default_rng(96)
    x = rng.standard_normal(dims).astype(np.float32)
    if dtype == "complex64":
        x = (x + 1j * rng.standard_normal(dims)).astype(np.complex64)
    ws = sfl.make_workspace(t, dtype, dims)
    ws.set_pipeline(pipeline)
    xd = sfl.to_device(x)
    ref = sfl.analyze(ws, xd)
    got = {}
    sfl.analyze(lambda i, b: got.__setitem__(i, b.clone()), ws, xd)
    for i in range(1, ws.nsubbands + 1):
        assert torch.equal(got[i], ref[..., i - 1]), i
    y = sfl.volume_like(dims, dtype)
    sfl.synthesize_(lambda i: ref[..., i - 1], y, ws)
    assert torch.equal(y, sfl.synthesize(ws, ref))
    assert rel_l2(sfl.to_host(y), x) <= REL


@pytest.mark.parametrize("pipeline,dims", [("lines", (20, 16, 12)), ("slabs", (64, 64, 32))])
def test_streaming_synthesis_stages_mask_groups(sfl, pipeline, dims):
    """Streaming synthesis stages each pushed subband and accumulates once per
    mask group; equal bit for bit to synthesize at group sizes 1, 3 and 8."""
    import torch
    t = sfl.NSSurfacelet(scales=2, direction_levels=[2, 3], bernstein_order=6)
    x = sfl.to_device(np.random.default_rng(6).standard_normal(dims).astype(np.float32))
    for g in (1, 3, 8):
        ws = sfl.make_workspace(t, "float32", dims, group=g)
        ws.set_pipeline(pipeline)
        c = sfl.analyze(ws, x)
        y = sfl.volume_like(dims)
        sfl.synthesize_(lambda i: c[..., i - 1], y, ws)
        assert torch.equal(y, sfl.synthesize(ws, c)), g
        wa = sfl.make_workspace(t, "float32", dims, group=g)
        wa.set_pipeline(pipeline)
        y2 = sfl.volume_like(dims)
        sfl.analyze_synthesize_stream(lambda i, b: b, y2, x, wa, ws)
        assert torch.equal(y2, y), g


@pytest.mark.parametrize("dims,pipeline", [((20, 16, 12), "lines"), ((64, 64, 32), "slabs")])
def test_group_size_does_not_change_results(sfl, dims, pipeline):
    """Analysis is the same bit for bit at every group size.  Synthesis on the
    slab pipeline combines the subbands that share a plane-b wedge before their
    axis-3 FFT when a chunk holds whole rows of them, so other chunkings round
    differently (float32 rounding level)."""
    t = sfl.NSSurfacelet(scales=2, direction_levels=[2, 3], bernstein_order=6)
    x = sfl.to_device(np.random.default_rng(5).standard_normal(dims).astype(np.float32))
    a = sfl.make_workspace(t, "float32", dims)
    b = sfl.make_workspace(t, "float32", dims, group=3)
    a.set_pipeline(pipeline)
    b.set_pipeline(pipeline)
    ca, cb = sfl.analyze(a, x), sfl.analyze(b, x)
    assert bool((ca == cb).all())
    ya, yb = sfl.synthesize(a, ca), sfl.synthesize(b, ca)
    if pipeline == "lines":
        assert bool((ya == yb).all())
    else:
        assert float(torch.linalg.vector_norm(ya - yb) / torch.linalg.vector_norm(ya)) <= 1e-6


def test_pipeline_selection_is_validated(sfl):
    ws = sfl.make_workspace(sfl.NSSurfacelet(scales=1, direction_levels=[1], bernstein_order=4), "float32", (12, 10, 8))
    with pytest.raises(sfl.ArgumentError, match="plane-major pipeline was retired"):
        ws.set_pipeline("planes")
    with pytest.raises(sfl.ArgumentError, match="slab pipeline does not support"):
        ws.set_pipeline("slabs")
    with pytest.raises(sfl.ArgumentError, match="unknown pipeline"):
        ws.set_pipeline("pencils")
    ws.set_pipeline("lines")


def test_workspace_validation(sfl):
    # test/items/test_ns_surfacelet.jl:165-196
    dims = (16, 16, 16)
    t = sfl.NSSurfacelet(scales=2, direction_levels=[1, 2], bernstein_order=6)
    ws = sfl.make_workspace(t, "float32", dims)
    x = sfl.to_device(np.zeros(dims, np.float32))
    with pytest.raises(sfl.DimensionMismatch):
        sfl.analyze(t, sfl.to_device(np.zeros((8, 8, 8), np.float32)), workspace=ws)
    with pytest.raises(sfl.ArgumentError, match="element type"):
        sfl.analyze(t, sfl.to_device(np.zeros(dims, np.complex64)), workspace=ws)
    with pytest.raises(sfl.ArgumentError, match="the workspace was built for NSSurfacelet\\(scales = 1"):
        sfl.analyze(t, x, workspace=sfl.make_workspace(sfl.NSSurfacelet(scales=1, direction_levels=[1]), "float32", dims))
    with pytest.raises(sfl.DimensionMismatch):
        sfl.analyze_(sfl.volume_like(dims + (5,)), t, x, workspace=ws)


def test_host_arrays_round_trip(sfl):
    # host (NumPy) arrays go through the same device path: the e2e form
    dims = (12, 16, 10)
    t = sfl.NSSurfacelet(scales=2, direction_levels=[1, 2], bernstein_order=6)
    x = np.asfortranarray(np.random.default_rng(13).standard_normal(dims).astype(np.float32))
    c = sfl.analyze(t, x)
    assert isinstance(c, np.ndarray) and c.shape == dims + (sfl.nsubbands(t, dims),)
    assert rel_l2(sfl.synthesize(t, c), x) <= REL
