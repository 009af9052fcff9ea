"""The slab pipeline with a 256-point axis: at 256 x 256 (x n3) one slab
(130 x 256 complex bins) is split over the two CTAs of a thread-block
cluster; with the other axis of 64 to 160 points a slab fits one CTA's
shared memory.  Analysis and synthesis against the float64 oracle, the line
pipeline, the fused denoiser and streaming (bit for bit), complex data and
the adjoints."""

import numpy as np
import pytest

from conftest import gpu_available
from oracle import ns as N

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not gpu_available(), reason="needs a CUDA device")]

REL = 1e-5


def rel_l2(a, b):
    a = np.asarray(a, dtype=np.complex128 if np.iscomplexobj(a) else np.float64)
    return float(np.linalg.norm((a - b).ravel()) / max(np.linalg.norm(np.asarray(b).ravel()), 1e-300))


@pytest.mark.parametrize("dims,kw", [
    ((256, 256, 32), dict(scales=2, direction_levels=[1, 2], bernstein_order=6)),
    ((256, 256, 16), dict(scales=3, direction_levels=[1, 1, 2], bernstein_order=8, tight=False)),
])
def test_cluster_slabs_match_oracle(sfl, dims, kw):
    rng = np.random.default_rng(256)
    x = rng.standard_normal(dims).astype(np.float32)
    t = sfl.NSSurfacelet(**kw)
    ws = sfl.make_workspace(t, "float32", dims)
    assert ws.tuning()[0] == "slabs"
    T = N.make_tables(N.NSParams.make(**kw), dims)
    xd = sfl.to_device(x)
    c = sfl.analyze(ws, xd)
    ch = sfl.to_host(c)
    cref = N.analyze(T, x.astype(np.float64))
    assert rel_l2(ch, cref) <= REL
    for i in range(cref.shape[-1]):
        assert np.abs(ch[..., i] - cref[..., i]).max() < 1e-4
    assert rel_l2(sfl.to_host(sfl.synthesize(ws, c)), x) <= REL
    cr = rng.standard_normal(cref.shape).astype(np.float32)
    y = sfl.to_host(sfl.synthesize(ws, sfl.to_device(cr)))
    assert rel_l2(y, N.synthesize(T, cr.astype(np.float64))) <= REL
    # the line pipeline agrees to float32 rounding
    wl = sfl.make_workspace(t, "float32", dims)
    wl.set_pipeline("lines")
    assert rel_l2(ch, sfl.to_host(sfl.analyze(wl, xd))) <= 2e-6
    import ctypes as C
    st = C.c_int32(-1)
    assert sfl.lib.sfl_plan_status(ws._h, C.byref(st), 0) == 0 and st.value == 0


def test_cluster_slabs_complex_and_adjoint(sfl):
    import torch
    dims = (256, 256, 16)
    kw = dict(scales=2, direction_levels=[1, 2], bernstein_order=6, tight=False)
    rng = np.random.default_rng(57)
    xr = rng.standard_normal(dims).astype(np.float32)
    xi = rng.standard_normal(dims).astype(np.float32)
    t = sfl.NSSurfacelet(**kw)
    wc = sfl.make_workspace(t, "complex64", dims)
    wr = sfl.make_workspace(t, "float32", dims)
    assert wc.tuning()[0] == "slabs" and wr.tuning()[0] == "slabs"
    cc = sfl.to_host(sfl.analyze(wc, sfl.to_device(xr + 1j * xi)))
    cr = sfl.to_host(sfl.analyze(wr, sfl.to_device(xr)))
    ci = sfl.to_host(sfl.analyze(wr, sfl.to_device(xi)))
    assert np.array_equal(cc.real, cr) and np.array_equal(cc.imag, ci)
    z = sfl.to_host(sfl.synthesize(wc, sfl.to_device(cc)))
    assert rel_l2(z, xr + 1j * xi) <= REL
    T = N.make_tables(N.NSParams.make(**kw), dims)
    c = rng.standard_normal(dims + (wr.nsubbands,)).astype(np.float32)
    ax = sfl.to_host(sfl.adjoint_analyze(wr, sfl.to_device(c)))
    assert rel_l2(ax, N.adjoint_analyze(T, c.astype(np.float64))) <= REL
    sx = sfl.to_host(sfl.adjoint_synthesize(wr, sfl.to_device(xr)))
    assert rel_l2(sx, N.adjoint_synthesize(T, xr.astype(np.float64))) <= REL


def test_cluster_slabs_denoise_and_stream_bit_for_bit(sfl):
    import torch
    dims = (256, 256, 16)
    t = sfl.NSSurfacelet(scales=2, direction_levels=[2, 2], bernstein_order=6)
    ws = sfl.make_workspace(t, "float32", dims, group=3)
    assert ws.tuning()[0] == "slabs"
    x = sfl.to_device(np.random.default_rng(3).standard_normal(dims).astype(np.float32))
    tau = torch.from_numpy(np.random.default_rng(4).uniform(0, 0.2, ws.nsubbands).astype(np.float32)).cuda()
    c = sfl.analyze(ws, x)
    y = sfl.denoise(ws, x, tau)
    ref = sfl.synthesize(ws, sfl.as_colmajor(torch.sign(c) * torch.clamp(c.abs() - tau, min=0)))
    assert torch.equal(y, ref)
    got = {}
    sfl.analyze(lambda i, b: got.__setitem__(i, b.clone()), ws, x)
    for i in range(1, ws.nsubbands + 1):
        assert torch.equal(got[i], c[..., i - 1]), i
    ys = sfl.volume_like(dims)
    sfl.synthesize_(lambda i: c[..., i - 1], ys, ws)
    assert torch.equal(ys, sfl.synthesize(ws, c))


@pytest.mark.parametrize("dims", [(256, 128, 32), (128, 256, 16), (256, 160, 16), (96, 256, 16), (256, 64, 32)])
def test_one_cta_slabs_with_a_256_axis(sfl, dims):
    import torch
    kw = dict(scales=2, direction_levels=[1, 2], bernstein_order=6)
    rng = np.random.default_rng(sum(dims))
    x = rng.standard_normal(dims).astype(np.float32)
    t = sfl.NSSurfacelet(**kw)
    ws = sfl.make_workspace(t, "float32", dims)
    assert ws.tuning()[0] == "slabs"
    T = N.make_tables(N.NSParams.make(**kw), dims)
    xd = sfl.to_device(x)
    c = sfl.analyze(ws, xd)
    ch = sfl.to_host(c)
    assert rel_l2(ch, N.analyze(T, x.astype(np.float64))) <= REL
    assert rel_l2(sfl.to_host(sfl.synthesize(ws, c)), x) <= REL
    cr = rng.standard_normal(ch.shape).astype(np.float32)
    y = sfl.to_host(sfl.synthesize(ws, sfl.to_device(cr)))
    assert rel_l2(y, N.synthesize(T, cr.astype(np.float64))) <= REL
    tau = torch.full((ws.nsubbands,), 0.1, device="cuda")
    ref = sfl.synthesize(ws, sfl.as_colmajor(torch.sign(c) * torch.clamp(c.abs() - tau, min=0)))
    assert torch.equal(sfl.denoise(ws, xd, tau), ref)
    import ctypes as C
    st = C.c_int32(-1)
    assert sfl.lib.sfl_plan_status(ws._h, C.byref(st), 0) == 0 and st.value == 0
