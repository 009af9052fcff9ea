"""Gradients through the transforms (torch autograd over the C ABI) for the
compressed-sensing loss of the complex workload

    L(c) = 0.5 || M o FFT3(synthesize(c)) - y ||^2 + lam sum sqrt(|c|^2 + eps^2)

with M a seeded Bernoulli(0.25) sampling mask with a fully sampled 16^3 centre
and y = M o FFT3(phantom):
the device gradient is held against the float64 oracle gradient (itself
pinned by central differences in test_oracle_gradients.py), and the same for
the gradient through analyze, x -> L(analyze(x)).  At 128^3 (the workload's
size) the device gradient is held against the float64 oracle's gradient and
the oracle's float64 central differences (h = 1e-4, 32 directions), and by
central differences of the device loss."""

import numpy as np
import pytest
import torch

from conftest import gpu_available
from oracle import ns as N

from cs_problem import EPS, LAM, analyze_c, analyze_t_c, make_problem, oracle_grad

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not gpu_available(), reason="needs a CUDA device")]


def device_loss(sfl, ws, c, M, y):
    x = sfl.synthesize_ad(ws, c)
    r = M * torch.fft.fftn(x) - y
    return 0.5 * (r.abs() ** 2).sum() + LAM * torch.sqrt(c.abs() ** 2 + EPS ** 2).sum()


def test_gradients_match_the_float64_oracle(sfl):
    dims = (32, 32, 32)
    kw = dict(scales=3, direction_levels=[2, 2, 3])
    T = N.make_tables(N.NSParams.make(**kw), dims)
    ph, M, y, rng = make_problem(dims, 3)
    c0 = analyze_c(T, ph)
    c = c0 + 0.1 * (rng.standard_normal(c0.shape) + 1j * rng.standard_normal(c0.shape))
    g = oracle_grad(T, c, M, y)
    # the device gradient (float32) against the oracle's
    ws = sfl.make_workspace(sfl.NSSurfacelet(**kw), "complex64", dims)
    cd = sfl.to_device(c.astype(np.complex64)).requires_grad_(True)
    L = device_loss(sfl, ws, cd, torch.from_numpy(M.astype(np.float32)).cuda(),
                    torch.from_numpy(y.astype(np.complex64)).cuda())
    L.backward()
    gd = sfl.to_host(sfl.as_colmajor(cd.grad))
    assert np.linalg.norm(gd - g) / np.linalg.norm(g) <= 1e-5
    # through analyze: x -> L(analyze(x)), gradient A^T grad_c, away from the
    # data (x = phantom + noise), so that the data term carries the gradient
    x = (ph + 0.1 * (rng.standard_normal(dims) + 1j * rng.standard_normal(dims))).astype(np.complex64)
    xd = sfl.to_device(x).requires_grad_(True)
    ca = sfl.analyze_ad(ws, xd)
    La = device_loss(sfl, ws, ca, torch.from_numpy(M.astype(np.float32)).cuda(),
                     torch.from_numpy(y.astype(np.complex64)).cuda())
    La.backward()
    gx = analyze_t_c(T, oracle_grad(T, analyze_c(T, x.astype(np.complex128)), M, y))
    gxd = sfl.to_host(sfl.as_colmajor(xd.grad))
    assert np.linalg.norm(gxd - gx) / np.linalg.norm(gx) <= 1e-4


def test_device_gradient_by_central_differences_at_128(sfl):
    dims = (128, 128, 128)
    ws = sfl.make_workspace(sfl.NSSurfacelet(scales=3, direction_levels=[2, 2, 3]), "complex64", dims)
    ph, M, y, rng = make_problem(dims, 4)
    Md = torch.from_numpy(M.astype(np.float32)).cuda()
    yd = torch.from_numpy(y.astype(np.complex64)).cuda()
    c0 = sfl.analyze(ws, sfl.to_device(ph.astype(np.complex64)))
    g = torch.Generator(device="cuda").manual_seed(8)
    c = (c0 + 0.1 * torch.randn(c0.shape, dtype=torch.complex64, generator=g, device="cuda")).detach()
    c = sfl.as_colmajor(c).requires_grad_(True)
    device_loss(sfl, ws, c, Md, yd).backward()
    grad = c.grad.detach()

    def loss64(cc):
        x = sfl.synthesize(ws, sfl.as_colmajor(cc)).to(torch.complex128)
        r = Md.double() * torch.fft.fftn(x) - yd.to(torch.complex128)
        cd = cc.to(torch.complex128)
        return float(0.5 * (r.abs() ** 2).sum() + LAM * torch.sqrt(cd.abs() ** 2 + EPS ** 2).sum())

    # directions with a component along the gradient, so that the directional
    # derivative stands well above the float32 rounding of the loss
    h = 0.05
    ghat = grad / torch.linalg.vector_norm(grad)
    for _ in range(4):
        d = torch.randn(c.shape, dtype=torch.complex64, generator=g, device="cuda")
        d = ghat + 0.5 * d / torch.linalg.vector_norm(d)
        fd = (loss64(c.detach() + h * d) - loss64(c.detach() - h * d)) / (2 * h)
        an = float((grad.conj() * d).real.double().sum())
        assert abs(fd - an) <= 2e-3 * abs(an), (fd, an)


def test_gradients_at_128_against_the_float64_oracle_and_its_central_differences(sfl):
    """The complex workload as stated: ComplexF32 128^3, NSSurfacelet(3, [2, 2, 3]).
    The device gradient in c, and through analyze, against the float64
    oracle's gradient (the reference's CPU gradient: synthesis' adjoint is
    analysis, test/items/test_ns_surfacelet.jl:218-237); and the oracle's
    float64 central differences, h = 1e-4 along 32 random unit directions,
    against both the oracle gradient and the device gradient.  Synthesis is
    linear, so L(c +- h d) is evaluated from synthesize(c) +- h synthesize(d),
    all in float64 (one oracle synthesis per direction; the loss's FFT and
    sums in float64 on the device)."""
    import os

    from cs_problem import synthesize_c
    dims = (128, 128, 128)
    kw = dict(scales=3, direction_levels=[2, 2, 3])
    N.set_fft_workers(os.cpu_count() or 1)
    try:
        T = N.make_tables(N.NSParams.make(**kw), dims)
        ph, M, y, rng = make_problem(dims, 4)
        ws = sfl.make_workspace(sfl.NSSurfacelet(**kw), "complex64", dims)
        Md = torch.from_numpy(M.astype(np.float32)).cuda()
        yd = torch.from_numpy(y.astype(np.complex64)).cuda()
        gen = torch.Generator(device="cuda").manual_seed(9)
        c0 = sfl.analyze(ws, sfl.to_device(ph.astype(np.complex64)))
        cd = sfl.as_colmajor(c0 + 0.1 * torch.randn(c0.shape, dtype=torch.complex64, generator=gen,
                                                    device="cuda")).detach()
        c = sfl.to_host(cd).astype(np.complex128)          # the same point, in float64
        cd.requires_grad_(True)
        device_loss(sfl, ws, cd, Md, yd).backward()
        gd = sfl.to_host(sfl.as_colmajor(cd.grad)).astype(np.complex128)
        g = oracle_grad(T, c, M, y)
        assert np.linalg.norm(gd - g) / np.linalg.norm(g) <= 1e-5
        # central differences of the float64 loss; the oracle synthesizes each direction on the host, the
        # loss sums run in float64 on the device (same arithmetic, faster)
        x = synthesize_c(T, c)
        Mg = torch.from_numpy(M).cuda()
        yg = torch.from_numpy(y).cuda()
        cg = torch.from_numpy(c).cuda()
        xg = torch.from_numpy(x).cuda()
        gen64 = torch.Generator(device="cuda").manual_seed(10)

        def loss(xx, cc):
            r = Mg * torch.fft.fftn(xx) - yg
            return float(0.5 * (r.real ** 2 + r.imag ** 2).sum()
                         + LAM * torch.sqrt(cc.real ** 2 + cc.imag ** 2 + EPS ** 2).sum())

        h = 1e-4
        for k in range(32):
            dg = torch.randn(c.shape, dtype=torch.complex128, generator=gen64, device="cuda")
            dg /= torch.linalg.vector_norm(dg)
            d = dg.cpu().numpy()
            sdg = torch.from_numpy(synthesize_c(T, d)).cuda()
            fd = (loss(xg + h * sdg, cg + h * dg) - loss(xg - h * sdg, cg - h * dg)) / (2 * h)
            an = float(np.sum((np.conj(g) * d).real))
            an_dev = float(np.sum((np.conj(gd) * d).real))
            assert abs(fd - an) <= 1e-6 * abs(an) + 1e-9 * np.linalg.norm(g), (k, fd, an)
            assert abs(fd - an_dev) <= 1e-4 * abs(an) + 1e-5 * np.linalg.norm(g) / np.sqrt(d.size), (k, fd, an_dev)
            del dg, sdg
        del cg, Mg, yg, xg
        del cd, c0
        # through analyze: x -> L(analyze(x)), away from the data
        xa = (ph + 0.1 * (rng.standard_normal(dims) + 1j * rng.standard_normal(dims))).astype(np.complex64)
        xd = sfl.to_device(xa).requires_grad_(True)
        ca = sfl.analyze_ad(ws, xd)
        device_loss(sfl, ws, ca, Md, yd).backward()
        gx = analyze_t_c(T, oracle_grad(T, analyze_c(T, xa.astype(np.complex128)), M, y))
        gxd = sfl.to_host(sfl.as_colmajor(xd.grad))
        assert np.linalg.norm(gxd - gx) / np.linalg.norm(gx) <= 1e-4
    finally:
        N.set_fft_workers(1)
