"""The oracle against the SurfBox golden data the reference's suite carries
(test/items/test_irc.jl), at the reference's own tolerances."""

import numpy as np
import pytest

from oracle import decimated as D
from oracle import filters as F
from oracle import golden as G

GOLD = G.load()
L111 = np.array([[-1, 1, 1], [1, -1, 1], [1, 1, -1]])
L212 = np.array([[-1, 2, 1], [1, -1, 2], [2, 1, -1]])


def _dtft(H, c, w1, w2):
    i = np.arange(1, H.shape[0] + 1)[:, None]
    j = np.arange(1, H.shape[1] + 1)[None, :]
    return np.sum(H * np.exp(-1j * (w1 * (i - c[0, 0]) + w2 * (j - c[0, 1]))))


@pytest.mark.parametrize("bo", [4, 8, 12])
def test_checkerboard_filters_match_surfbox(bo):
    # test/items/test_irc.jl:68-90
    t = F.cbd_ladder(bo)
    ws = np.linspace(0, 2 * np.pi, 13)[:12]
    worst = 0.0
    for a in ws:
        for b in ws:
            for ch, tag in ((0, "0"), (1, "1")):
                hd = _dtft(GOLD[f"cbd_{bo}_dec_H{tag}"]["data"], GOLD[f"cbd_{bo}_dec_c{tag}"]["data"], a, b)
                hr = _dtft(GOLD[f"cbd_{bo}_rec_H{tag}"]["data"], GOLD[f"cbd_{bo}_rec_c{tag}"]["data"], a, b)
                worst = max(worst, abs(F.cbd_analysis(t, ch, a, b) - hd), abs(F.cbd_synthesis(t, ch, a, b) - hr))
    assert worst < 1e-13


def test_ritf_hourglass_and_irc_stages_match_surfbox():
    # test/items/test_irc.jl:92-115
    x = G.testvol(32)
    X = np.fft.fftn(x.astype(complex))
    V = D.ritf_masks(x.shape)
    for K in (1, 2, 3):
        half = tuple(slice(0, 17) if d == K - 1 else slice(None) for d in range(3))
        hg = X[half] * V[K - 1]
        assert G.fp_match(hg, GOLD[f"hg_{K}"], rtol=1e-10)
        for nm, L in (("l111", L111), ("l212", L212)):
            levels = tuple(0 if d == K - 1 else int(L[K - 1, d]) for d in range(3))
            st = D.irc_stages(hg.shape, 32, K, levels, 4)
            Sk = hg.copy()
            D.irc_analysis(Sk, st)
            assert G.fp_match(Sk, GOLD[f"irc_{nm}_{K}"], rtol=1e-10)
            D.irc_synthesis(Sk, st)
            assert np.abs(Sk - hg).max() < 1e-12 * np.abs(hg).max()
    Vf = D.ritf_masks((16, 20, 12))
    s = Vf[0][:9, :11, :7] ** 2 + Vf[1][:9, :11, :7] ** 2 + Vf[2][:9, :11, :7] ** 2
    assert np.abs(s - 3).max() < 1e-12


@pytest.mark.parametrize("nm,L", [("l111", L111), ("l212", L212)])
def test_ndfb_subbands_match_surfbox(nm, L):
    # test/items/test_irc.jl:117-137
    x = G.testvol(32)
    lv = D.surf_levels(L)
    sc = D.scale_tables(x.shape, lv, 4)
    bands = D.surf_scale_forward(np.fft.fftn(x.astype(complex)), sc)
    i = 0
    for K in (1, 2, 3):
        for w in range(1, (1 << sum(lv[K - 1])) + 1):
            assert G.fp_match(bands[i], GOLD[f"ndfb_{nm}_{K}_{w}"])
            i += 1
    rec = np.fft.ifftn(D.surf_scale_inverse(bands, sc)).real
    assert G.fp_match(rec, GOLD[f"ndfbrec_{nm}"])
    assert np.abs(rec - x).max() < 1e-13


@pytest.mark.parametrize("tag,n,mode", [("m15", 48, 1.5), ("m1", 32, 1), ("m2", 32, 2)])
def test_fourier_pyramid_matches_surfbox(tag, n, mode):
    # test/items/test_irc.jl:139-161
    x = G.testvol(n)
    levels = D.fourier_pyramid(x.shape, 2, mode)
    X = np.fft.fftn(x.astype(complex))
    orig = X.copy()
    highs = []
    for lv in levels:
        low = D.pyramid_split(X, lv)
        highs.append(X)
        X = low
    assert G.fp_match(highs[0], GOLD[f"pyr_{tag}_1"])
    assert G.fp_match(highs[1], GOLD[f"pyr_{tag}_2"])
    assert G.fp_match(X, GOLD[f"pyr_{tag}_3"])
    for k in (1, 0):
        X = D.pyramid_merge(highs[k], X, levels[k])
    assert np.abs(X - orig).max() < 1e-12 * np.abs(orig).max()


@pytest.mark.parametrize("tag,n,mode,lev_array,bo", [
    ("m15", 48, 1.5, [L111, L111], 8),
    ("m2", 64, 2, [L212, L111], 4),
])
def test_whole_transform_matches_surfdec_surfrec(tag, n, mode, lev_array, bo):
    # test/items/test_irc.jl:163-184
    x = G.testvol(n)
    p = D.SurfParams.make(direction_levels=list(reversed(lev_array)), pyramid_ratio=mode, checkerboard_order=bo)
    T = D.make_tables(p, x.shape)
    c = D.analyze(T, x)
    for i, d in enumerate(D.subband_layout(p, x.shape), start=1):
        if i == 1:
            continue
        key = f"surf_{tag}_{p.scales - d[0] + 1}_{d[1]}_{d[2]}"
        assert G.fp_match(D.subband(T, c, i), GOLD[key]), key
    assert G.fp_match(D.subband(T, c, 1), GOLD[f"surf_{tag}_low"])
    r = D.synthesize(T, c)
    assert G.fp_match(r, GOLD[f"surfrec_{tag}"])
    assert np.abs(r - x).max() < 1e-13


@pytest.mark.parametrize("nm,Lm,J", [
    ("d24", [[-1, 1, 2], [2, -1, 1], [1, 2, -1]], 3),
    ("d96", [[-1, 2, 3], [3, -1, 2], [2, 3, -1]], 2),
])
def test_redundancy_matches_surfbox(nm, Lm, J):
    # test/items/test_irc.jl:186-193
    p = D.SurfParams.make(scales=J, direction_levels=[np.array(Lm)] * J, checkerboard_order=4)
    assert D.redundancy(p, (96, 96, 96)) == pytest.approx(float(GOLD[f"red_96_{nm}"]["data"].ravel()[0]))
