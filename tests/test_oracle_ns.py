"""The NSSurfacelet oracle against the reference's component and property
tests (test/items/test_hourglass.jl, test_ndfb.jl, test_ns_surfacelet.jl,
test_literature.jl).  The reference ships no NS golden coefficients, so these
properties are what pins the restatement."""

import numpy as np
import pytest

from oracle import filters as F
from oracle import ns as N


def test_bernstein_partition_of_unity():
    # test/items/test_hourglass.jl:1-18
    w = np.linspace(0, 2 * np.pi, 33)
    for order in (1, 4, 12):
        tbl = F.bernstein_table(order, w)
        assert tbl.shape == (order + 1, 33)
        assert np.abs(tbl.sum(0) - 1).max() < 1e-12
        assert tbl.min() >= -1e-15
    t0 = F.bernstein_table(6, [0.0])
    assert t0[0, 0] == pytest.approx(1.0) and np.abs(t0[1:, 0]).max() < 1e-14
    assert F.bernstein_table(6, [np.pi])[-1, 0] == pytest.approx(1.0)


def test_mapping_coefficients_sign_pattern():
    # test/items/test_hourglass.jl:20-33
    c = F.mapping_coefficients(4, 2, (1,))
    for j1 in range(5):
        for j2 in range(5):
            assert c[j1, j2] == (1 if j1 > j2 else (-1 if j1 < j2 else 0))
    c3 = F.mapping_coefficients(3, 3, (1,))
    assert c3[3, 0, 0] == 1 and c3[0, 3, 0] == -1 and c3[1, 1, 1] == 0


def test_halfband_split_complementarity():
    # test/items/test_hourglass.jl:35-57
    for m in range(4):
        assert F.halfband_split(1.0, m) == pytest.approx(1.0)
        assert F.halfband_split(-1.0, m) == pytest.approx(0.0)
        assert F.halfband_split(0.0, m) == pytest.approx(0.5)
        x = np.linspace(-1, 1, 21)
        f = F.halfband_split(x, m)
        assert np.abs(f + F.halfband_split(-x, m) - 1).max() < 1e-12
    f = [float(F.halfband_split(0.5, m)) for m in range(61)]
    assert f == sorted(f) and all(0 <= v <= 1 for v in f)
    for m in (31, 45, 60):
        x = np.linspace(-1, 1, 9)
        assert np.abs(F.halfband_split(x, m) + F.halfband_split(-x, m) - 1).max() < 1e-12


def test_hourglass_partition_and_parseval():
    # test/items/test_hourglass.jl:59-96
    dims = (12, 14, 10)
    m1, m2 = N.hourglass_tables(dims, 6, 1)
    w = [N.hourglass_weight(m1, m2, i) for i in (1, 2, 3)]
    assert np.abs(w[0] + w[1] + w[2] - 1).max() < 1e-14
    m = [N.hourglass_mask(m1, m2, i) for i in (1, 2, 3)]
    assert np.abs(m[0] ** 2 + m[1] ** 2 + m[2] ** 2 - 1).max() < 1e-14
    x = np.random.default_rng(71).standard_normal(dims)
    s = N.hourglass_decompose(x, dims, 6, 1)
    assert abs(sum(np.sum(b ** 2) for b in s) / np.sum(x ** 2) - 1) < 1e-12


def test_hourglass_sharpness_figures():
    # test/items/test_hourglass.jl:147-175
    n = 24

    def mae(order, tight=True):
        m1, m2 = N.hourglass_tables((n, n, n), order, 1)
        m = N.hourglass_mask(m1, m2, 1, tight)
        fold = lambda k: np.minimum(k * 2 * np.pi / n, 2 * np.pi - k * 2 * np.pi / n)
        w1 = fold(np.arange(m.shape[0]))[:, None, None]
        w2 = fold(np.arange(n))[None, :, None]
        w3 = fold(np.arange(n))[None, None, :]
        mx = np.maximum(w2, w3)
        sel = np.broadcast_to(np.abs(w1 - mx) > 1e-9, m.shape)
        return np.sum(np.abs(m - (w1 > mx))[sel]) / np.sum(sel)

    assert mae(12) < mae(4) and mae(20) < mae(12)
    assert mae(4, tight=False) == pytest.approx(0.095, abs=0.001)
    assert mae(20, tight=False) == pytest.approx(0.024, abs=0.001)


def test_hourglass_plane_waves():
    # test/items/test_hourglass.jl:113-145
    n = 16
    I = np.indices((n, n, n))
    for ax in range(3):
        v = np.cos(np.pi * 2 * 6 * I[ax] / n)
        e = np.array([np.sum(b ** 2) for b in N.hourglass_decompose(v, (n, n, n), 8, 1)])
        e /= e.sum()
        assert e[ax] > 0.999
    v = np.cos(np.pi * 2 * 5 * (I[0] + I[1]) / n)
    e = np.array([np.sum(b ** 2) for b in N.hourglass_decompose(v, (n, n, n), 8, 1)])
    e /= e.sum()
    assert abs(e[0] - e[1]) < 1e-6 and e[2] < 1e-6


@pytest.mark.parametrize("n", [12, 26, 30])
def test_ndfb_masks_even_in_frequency(n):
    # test/items/test_ndfb.jl:51-71
    neg = (-np.arange(n)) % n
    for m in N.ndfb_masks((n, n, n), 2, order=6):
        for i1 in (0, n // 2):
            assert np.abs(m[i1] - m[i1][np.ix_(neg, neg)]).max() <= 1e-13


def test_ndfb_partition_of_unity():
    # test/items/test_ndfb.jl:23-33
    for L in range(4):
        ms = N.ndfb_masks((10, 12, 8), L, order=6, tight=False)
        assert np.abs(sum(ms) - 1).max() < 1e-13
        ms = N.ndfb_masks((10, 12, 8), L, order=6)
        assert np.abs(sum(m ** 2 for m in ms) - 1).max() < 1e-13


def test_ndfb_plane_waves_land_in_predicted_wedge():
    # test/items/test_ndfb.jl:118-147
    n = 32
    L = 4
    la, lb = N.wedge_levels(L)

    def predict(k):
        i = int(np.argmax(np.abs(k)))
        a, b = N.transverse_axes(i + 1)
        p = min(max(int(np.floor((k[a - 1] / k[i] + 1) / (2 / (1 << la)))) + 1, 1), 1 << la)
        q = min(max(int(np.floor((k[b - 1] / k[i] + 1) / (2 / (1 << lb)))) + 1, 1), 1 << lb)
        return (i * (1 << la) + (p - 1)) * (1 << lb) + q

    I = np.indices((n, n, n))
    for k in ([2, 5, 9], [5, 9, -12], [-2, 3, -13], [-13, -9, 7], [9, 7, -12], [3, 11, -7]):
        v = np.cos(np.pi * 2 * (k[0] * I[0] + k[1] * I[1] + k[2] * I[2]) / n)
        e = np.array([np.sum(b ** 2) for b in N.ndfb_decompose(v, (n, n, n), L, order=12, transition=0.5)])
        assert int(np.argmax(e)) + 1 == predict(k)
        assert e.max() / e.sum() > 0.3


def test_wedge_centre_energy_follows_transition():
    # test/items/test_literature.jl:5-33
    n = 32
    I = np.indices((n, n, n))
    v = np.cos(np.pi * 2 * (8 * I[0] + 4 * I[1] + 4 * I[2]) / n)

    def share(tr):
        e = np.array([np.sum(b ** 2) for b in N.ndfb_decompose(v, (n, n, n), 2, transition=tr)])
        assert int(np.argmax(e)) + 1 == 4    # ndfb_subband_index(fb, 1, 2, 2)
        return e.max() / e.sum()

    assert share(1.0) == pytest.approx(0.71, abs=0.01)
    assert share(0.5) > 0.99
    assert share(0.0) == pytest.approx(share(0.5), abs=1e-3)


@pytest.mark.parametrize("dims", [(16, 16, 16), (12, 20, 8)])
@pytest.mark.parametrize("J,L", [(1, [0]), (2, [1, 2]), (3, [1, 1, 2])])
def test_ns_perfect_reconstruction(dims, J, L):
    # test/items/test_ns_surfacelet.jl:40-54
    x = np.random.default_rng(90).standard_normal(dims)
    p = N.NSParams.make(scales=J, direction_levels=L, bernstein_order=6)
    T = N.make_tables(p, dims)
    c = N.analyze(T, x)
    assert c.shape[-1] == N.nsubbands(p) == 1 + sum(3 * 2 ** l for l in L)
    assert np.abs(N.synthesize(T, c) - x).max() < 1e-12


@pytest.mark.parametrize("dims", [(16, 16, 16), (15, 20, 8)])
@pytest.mark.parametrize("J,L", [(1, [1]), (3, [1, 1, 2])])
def test_ns_parseval_inverse_is_adjoint(dims, J, L):
    # test/items/test_ns_surfacelet.jl:218-237
    rng = np.random.default_rng(98)
    p = N.NSParams.make(scales=J, direction_levels=L, bernstein_order=6)
    T = N.make_tables(p, dims)
    x = rng.standard_normal(dims)
    c = N.analyze(T, x)
    assert np.sum(c * c) == pytest.approx(np.sum(x * x), rel=1e-12)
    r = rng.standard_normal(c.shape)
    assert np.sum(c * r) == pytest.approx(np.sum(x * N.synthesize(T, r)), rel=1e-12)


def test_ns_not_tight_and_adjoints():
    rng = np.random.default_rng(7)
    for tight in (False, True):
        p = N.NSParams.make(scales=2, direction_levels=[1, 2], bernstein_order=6, tight=tight)
        T = N.make_tables(p, (16, 12, 20))
        x = rng.standard_normal((16, 12, 20))
        c = N.analyze(T, x)
        assert np.abs(N.synthesize(T, c) - x).max() < 1e-12
        r = rng.standard_normal(c.shape)
        assert np.sum(c * r) == pytest.approx(np.sum(x * N.adjoint_analyze(T, r)), rel=1e-12)
        y = N.synthesize(T, r)
        assert np.sum(y * x) == pytest.approx(np.sum(r * N.adjoint_synthesize(T, x)), rel=1e-12)


def test_ns_shift_invariance_and_constant():
    # test/items/test_ns_surfacelet.jl:56-77
    rng = np.random.default_rng(91)
    p = N.NSParams.make(scales=2, direction_levels=[1, 2], bernstein_order=6)
    T = N.make_tables(p, (16, 16, 16))
    x = rng.standard_normal((16, 16, 16))
    s = (3, -2, 5)
    a = N.analyze(T, x)
    b = N.analyze(T, np.roll(x, s, axis=(0, 1, 2)))
    assert np.abs(b - np.roll(a, s, axis=(0, 1, 2))).max() < 1e-10
    p = N.NSParams.make(scales=2, direction_levels=[1, 1], bernstein_order=6)
    T = N.make_tables(p, (16, 16, 16))
    c = N.analyze(T, np.full((16, 16, 16), 1.75))
    assert np.abs(c[..., 0] - 1.75).max() < 1e-12 and np.abs(c[..., 1:]).max() < 1e-12


def test_ns_streaming_order_and_empty_scale():
    # test/items/test_ns_surfacelet.jl:79-94, 239-252
    p = N.NSParams.make(scales=2, direction_levels=[1, 2], bernstein_order=6)
    T = N.make_tables(p, (16, 16, 16))
    seen = [i for i, _ in N.analyze_stream(T, np.zeros((16, 16, 16)))]
    assert seen == list(range(2, N.nsubbands(p) + 1)) + [1]
    with pytest.raises(N.ArgumentError, match="too small for 4 scales"):
        N.make_tables(N.NSParams.make(scales=4, direction_levels=[0, 0, 0, 0], bernstein_order=4), (8, 8, 8))
    N.make_tables(N.NSParams.make(scales=3, direction_levels=[0, 1, 1], bernstein_order=4), (32, 32, 8))


def test_ns_layout():
    # test/items/test_ns_surfacelet.jl:14-18
    p = N.NSParams.make(scales=3, direction_levels=[1, 2, 2])
    lay = N.subband_layout(p)
    assert len(lay) == N.nsubbands(p) == 1 + 6 + 12 + 12
    assert lay[0] == (0, 0) and lay[1] == (1, 1) and lay[7] == (2, 1)
    assert N.NSParams.make(scales=4).direction_levels == (1, 1, 2, 2)
