"""The decimated Surfacelet on the B200 through the C ABI: the SurfBox golden
fingerprints (in float32), the float64 oracle, perfect reconstruction and
exact real-linearity."""

import numpy as np
import pytest

from conftest import gpu_available
from oracle import decimated as D
from oracle import golden as G

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not gpu_available(), reason="needs a CUDA device")]

REL = 1e-5
L111 = np.array([[-1, 1, 1], [1, -1, 1], [1, 1, -1]])
L212 = np.array([[-1, 2, 1], [1, -1, 2], [2, 1, -1]])
GOLD = G.load()


def rel_l2(a, b):
    a = np.asarray(a, dtype=np.complex128 if np.iscomplexobj(a) else np.float64)
    return float(np.linalg.norm((a - b).ravel()) / max(np.linalg.norm(np.asarray(b).ravel()), 1e-300))


def fp_rel(A, ref):
    return G.fp_error(np.asarray(A, dtype=np.float64), ref)


@pytest.mark.parametrize("tag,n,mode,lev_array,bo", [
    ("m15", 48, 1.5, [L111, L111], 8),
    ("m2", 64, 2, [L212, L111], 4),
])
def test_matches_surfbox_golden(sfl, tag, n, mode, lev_array, bo):
    # test/items/test_irc.jl:163-184, in float32
    x = G.testvol(n).astype(np.float32)
    t = sfl.Surfacelet(direction_levels=list(reversed(lev_array)), pyramid_ratio=mode, checkerboard_order=bo)
    dims = x.shape
    ws = sfl.make_workspace(t, "float32", dims)
    c = sfl.analyze(ws, sfl.to_device(x))
    for i, d in enumerate(sfl.subband_layout(t, dims), start=1):
        sb = sfl.to_host(sfl.subband(t, c, i, dims))
        key = f"surf_{tag}_low" if i == 1 else f"surf_{tag}_{t.scales - d['scale'] + 1}_{d['hourglass']}_{d['wedge']}"
        assert fp_rel(sb, GOLD[key]) < 1e-5, key
    r = sfl.to_host(sfl.synthesize(ws, c))
    assert fp_rel(r, GOLD[f"surfrec_{tag}"]) < 1e-5
    assert np.abs(r - x).max() < 1e-5


CASES = [
    ((48, 48, 48), 1.5, 2, [1, 2], 12),
    ((48, 24, 36), 1.5, 1, [2], 8),
    ((32, 32, 32), 1, 2, [1, 1], 4),
    ((64, 32, 32), 2, 2, [1, 3], 18),
    ((32, 32, 32), 2, 1, [np.array([[-1, 2, 0], [1, -1, 1], [0, 3, -1]])], 6),
    ((24, 24, 24), 1.5, 1, [0], 12),
    ((128, 128, 128), 2, 3, [2, 2, 3], 12),
    # hourglass 3's finest plane (256 x 128 complex, 256 KB) exceeds shared memory and takes the
    # per-stage IRC kernels; every other plane takes the fused plane pass
    ((256, 128, 32), 2, 2, [1, 2], 8),
]


@pytest.mark.parametrize("dims,mode,J,L,bo", CASES)
def test_analyze_synthesize_match_oracle(sfl, dims, mode, J, L, bo):
    # test/items/test_surfacelet.jl:43-63 cases, plus the 128^3 mode-2 workload
    rng = np.random.default_rng(100)
    x = rng.standard_normal(dims).astype(np.float32)
    t = sfl.Surfacelet(scales=J, direction_levels=L, pyramid_ratio=mode, checkerboard_order=bo)
    p = D.SurfParams.make(scales=J, direction_levels=L, pyramid_ratio=mode, checkerboard_order=bo)
    T = D.make_tables(p, dims)
    ws = sfl.make_workspace(t, "float32", dims)
    assert ws.ncoeffs == round(sfl.surfacelet_redundancy(t, dims) * np.prod(dims))
    c = sfl.analyze(ws, sfl.to_device(x))
    ch = c.cpu().numpy()
    cref = D.analyze(T, x.astype(np.float64))
    assert rel_l2(ch, cref) <= REL
    r = sfl.to_host(sfl.synthesize(ws, c))
    assert rel_l2(r, x) <= REL
    cr = rng.standard_normal(cref.shape).astype(np.float32)
    y = sfl.to_host(sfl.synthesize(ws, sfl.to_device(cr)))
    assert rel_l2(y, D.synthesize(T, cr.astype(np.float64))) <= REL


def test_complex_equals_real_plus_i_imag_bit_for_bit(sfl):
    # test/items/test_surfacelet.jl:91-111
    dims = (48, 24, 36)
    rng = np.random.default_rng(102)
    xr = rng.standard_normal(dims).astype(np.float32)
    xi = rng.standard_normal(dims).astype(np.float32)
    t = sfl.Surfacelet(scales=2, direction_levels=[1, 2])
    cc = sfl.analyze(t, sfl.to_device(xr + 1j * xi)).cpu().numpy()
    cr = sfl.analyze(t, sfl.to_device(xr)).cpu().numpy()
    ci = sfl.analyze(t, sfl.to_device(xi)).cpu().numpy()
    assert np.array_equal(cc.real, cr) and np.array_equal(cc.imag, ci)
    ws = sfl.make_workspace(t, "complex64", dims)
    import torch
    z = sfl.to_host(sfl.synthesize(ws, torch.from_numpy(cc).cuda()))
    assert rel_l2(z, xr + 1j * xi) <= REL


def test_constant_lands_in_coarse_subband(sfl):
    # test/items/test_surfacelet.jl:152-162
    dims = (48, 48, 48)
    t = sfl.Surfacelet(scales=2, direction_levels=[1, 1])
    ws = sfl.make_workspace(t, "float32", dims)
    c = sfl.analyze(ws, sfl.to_device(np.full(dims, 0.5, np.float32)))
    for i in range(2, ws.nsubbands + 1):
        assert float(sfl.subband(t, c, i, dims).abs().max()) < 1e-5
    assert np.abs(sfl.to_host(sfl.synthesize(ws, c)) - 0.5).max() < 1e-5


def test_plane_wave_lands_in_its_hourglass(sfl):
    # test/items/test_surfacelet.jl:134-150
    n = 48
    t = sfl.Surfacelet(scales=1, direction_levels=[2])
    ws = sfl.make_workspace(t, "float32", (n, n, n))
    I = np.indices((n, n, n))
    for k, K in (((14, 3, 2), 1), ((2, 15, 4), 2), ((3, -2, 13), 3)):
        v = np.cos(np.pi * 2 * (k[0] * I[0] + k[1] * I[1] + k[2] * I[2]) / n).astype(np.float32)
        c = sfl.analyze(ws, sfl.to_device(v))
        e = np.array([float((sfl.subband(t, c, i, (n, n, n)).double() ** 2).sum()) for i in range(2, 14)])
        assert (int(np.argmax(e))) // 4 + 1 == K
        assert e.max() / e[4 * K - 4:4 * K].sum() > 0.6


ADJ_CASES = [CASES[0], CASES[1], CASES[2], CASES[3], CASES[5]]


@pytest.mark.parametrize("dims,mode,J,L,bo", ADJ_CASES)
def test_adjoints_against_the_oracle_forward(sfl, dims, mode, J, L, bo):
    # <A x, c> = <x, A^T c> and <S c, x> = <c, S^T x>, with A and S the float64
    # oracle and the transposes from the device.  c (x) is correlated with A x
    # (S c) so that the products are large and the test is relative.
    t = sfl.Surfacelet(scales=J, direction_levels=L, pyramid_ratio=mode, checkerboard_order=bo)
    T = D.make_tables(D.SurfParams.make(scales=J, direction_levels=L, pyramid_ratio=mode, checkerboard_order=bo), dims)
    ws = sfl.make_workspace(t, "float32", dims)
    rng = np.random.default_rng(7)
    for _ in range(3):
        x = rng.standard_normal(dims).astype(np.float32)
        Ax = D.analyze(T, x.astype(np.float64))
        c = (Ax + rng.standard_normal(Ax.shape)).astype(np.float32)
        Atc = sfl.to_host(sfl.adjoint_analyze(ws, sfl.to_device(c), dims=dims)).astype(np.float64)
        lhs, rhs = float(np.dot(Ax, c)), float(np.sum(x * Atc))
        assert abs(lhs - rhs) <= 2e-5 * abs(lhs), (lhs, rhs)
        cc = rng.standard_normal(Ax.shape).astype(np.float32)
        Sc = D.synthesize(T, cc.astype(np.float64))
        y = (Sc + rng.standard_normal(dims)).astype(np.float32)
        Sty = sfl.adjoint_synthesize(ws, sfl.to_device(y)).cpu().numpy().astype(np.float64)
        lhs, rhs = float(np.sum(Sc * y)), float(np.dot(cc, Sty))
        assert abs(lhs - rhs) <= 2e-5 * abs(lhs), (lhs, rhs)


def test_adjoints_at_128_mode_2_and_complex_linearity(sfl):
    # the device transposes against the device transforms at the 128^3 workload,
    # and complex data = real + i imag exactly
    dims = (128, 128, 128)
    t = sfl.Surfacelet(scales=3, direction_levels=[2, 2, 3], pyramid_ratio=2)
    ws = sfl.make_workspace(t, "float32", dims)
    import torch
    g = torch.Generator(device="cuda").manual_seed(5)
    x = sfl.volume_like(dims)
    x.copy_(torch.randn(dims, generator=g, device="cuda"))
    Ax = sfl.analyze(ws, x)
    c = Ax + torch.randn(Ax.shape, generator=g, device="cuda")
    lhs = float((Ax.double() * c.double()).sum())
    rhs = float((x.double() * sfl.adjoint_analyze(ws, c, dims=dims).double()).sum())
    assert abs(lhs - rhs) <= 2e-5 * abs(lhs)
    Sc = sfl.synthesize(ws, c)
    y = Sc + x
    lhs = float((Sc.double() * y.double()).sum())
    rhs = float((c.double() * sfl.adjoint_synthesize(ws, y).double()).sum())
    assert abs(lhs - rhs) <= 2e-5 * abs(lhs)
    dz = (48, 24, 36)
    tz = sfl.Surfacelet(scales=2, direction_levels=[1, 2])
    wz = sfl.make_workspace(tz, "complex64", dz)
    wr = sfl.make_workspace(tz, "float32", dz)
    rng = np.random.default_rng(9)
    cr = rng.standard_normal(wz.ncoeffs).astype(np.float32)
    ci = rng.standard_normal(wz.ncoeffs).astype(np.float32)
    zc = sfl.to_host(sfl.adjoint_analyze(wz, torch.from_numpy((cr + 1j * ci).astype(np.complex64)).cuda(), dims=dz))
    zr = sfl.to_host(sfl.adjoint_analyze(wr, torch.from_numpy(cr).cuda(), dims=dz))
    zi = sfl.to_host(sfl.adjoint_analyze(wr, torch.from_numpy(ci).cuda(), dims=dz))
    assert np.array_equal(zc.real, zr) and np.array_equal(zc.imag, zi)


@pytest.mark.parametrize("dims,mode,red", [((128, 128, 128), 2, 3.4238), ((96, 96, 96), 1.5, 4.0046)])
def test_phantom_workload_against_oracle(sfl, dims, mode, red):
    # the decimated workload: Surfacelet(scales=3, direction_levels=[2,2,3]) on the
    # 12-ellipsoid phantom plus N(0, 0.05^2) noise, about 3.4 / 4 coefficients a voxel
    from phantoms import ellipsoid_phantom
    x = ellipsoid_phantom(dims, count=12, seed=21, noise=0.05)
    t = sfl.Surfacelet(scales=3, direction_levels=[2, 2, 3], pyramid_ratio=mode)
    assert abs(sfl.surfacelet_redundancy(t, dims) - red) < 1e-4
    T = D.make_tables(D.SurfParams.make(scales=3, direction_levels=[2, 2, 3], pyramid_ratio=mode), dims)
    ws = sfl.make_workspace(t, "float32", dims)
    c = sfl.analyze(ws, sfl.to_device(x))
    assert rel_l2(c.cpu().numpy(), D.analyze(T, x.astype(np.float64))) <= REL
    assert rel_l2(sfl.to_host(sfl.synthesize(ws, c)), x) <= REL
