"""The C-ABI library on the host (no GPU needed): it loads, exports every
symbol the header declares, and its float64 design tables, layouts and
validation agree with the oracle and the reference's messages."""

import ctypes as C
import os
import re

import numpy as np
import pytest

from oracle import decimated as D
from oracle import ns as N

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_library_exports_every_declared_symbol(sfl):
    hdr = open(os.path.join(ROOT, "include", "surfacelets_b200.h")).read()
    names = sorted(set(re.findall(r"\b(sfl_[a-z0-9_]+)\s*\(", hdr)))
    assert len(names) >= 25
    lib = C.CDLL(sfl.LIB_PATH)
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def _ns_table(sfl, t, dims, name, index=0):
    lib = sfl.lib
    cnt = C.c_int64()
    d = (C.c_int32 * 3)(*dims)
    p = t._params()
    sfl._lib.check(lib.sfl_ns_design_table(C.byref(p), d, name.encode(), index, None, C.byref(cnt)))
    out = (C.c_double * cnt.value)()
    sfl._lib.check(lib.sfl_ns_design_table(C.byref(p), d, name.encode(), index, out, C.byref(cnt)))
    return np.frombuffer(out, dtype=np.float64).copy()


def _surf_table(sfl, t, dims, name, index=0):
    lib = sfl.lib
    cnt = C.c_int64()
    d = (C.c_int32 * 3)(*dims)
    p = t._params()
    sfl._lib.check(lib.sfl_surf_design_table(C.byref(p), d, name.encode(), index, None, C.byref(cnt)))
    out = (C.c_double * cnt.value)()
    sfl._lib.check(lib.sfl_surf_design_table(C.byref(p), d, name.encode(), index, out, C.byref(cnt)))
    return np.frombuffer(out, dtype=np.float64).copy()


@pytest.mark.parametrize("dims,L,order,tr,tight", [
    ((16, 12, 20), [1, 2], 6, 1.0, True),
    ((15, 20, 8), [1, 1, 2], 12, 0.5, False),
    ((26, 26, 26), [3], 6, 1.0, True),
])
def test_ns_design_tables_match_oracle(sfl, dims, L, order, tr, tight):
    t = sfl.NSSurfacelet(direction_levels=L, bernstein_order=order, transition=tr, tight=tight)
    p = N.NSParams.make(direction_levels=L, bernstein_order=order, transition=tr, tight=tight)
    T = N.make_tables(p, dims)
    h1 = dims[0] // 2 + 1
    m1 = _ns_table(sfl, t, dims, "m1").reshape((h1, dims[1], dims[2]), order="F")
    assert np.abs(m1 - T.m1).max() < 1e-12
    m2 = _ns_table(sfl, t, dims, "m2").reshape((dims[1], dims[2]), order="F")
    assert np.abs(m2 - T.m2).max() < 1e-12
    for j in range(len(L)):
        for i in (1, 2, 3):
            pa, pb = T.wedges[j][i - 1]
            for plane, lst in ((0, pa), (1, pb)):
                ref = i
                tr_ax = N.transverse_axes(i)[plane]
                for w, W in enumerate(lst):
                    got = _ns_table(sfl, t, dims, "wedge", ((j * 3 + i - 1) * 2 + plane) * 64 + w)
                    exp = W if ref < tr_ax else W.T       # stored (lo axis, hi axis), lo fastest
                    assert np.abs(got - exp.ravel(order="F")).max() < 1e-12
    for lv in range(len(L) + 1):
        for ax in range(3):
            assert np.abs(_ns_table(sfl, t, dims, "pa", lv * 3 + ax) - T.pa[lv][ax]).max() < 1e-15
    for lv in range(len(L)):
        for ax in range(3):
            assert np.abs(_ns_table(sfl, t, dims, "pl", lv * 3 + ax) - T.pl[lv][ax]).max() < 1e-15


@pytest.mark.parametrize("dims,L,order,tr,tight", [
    ((16, 12, 20), [1, 2], 6, 1.0, True),
    ((15, 20, 8), [1, 1, 2], 12, 0.5, False),
])
def test_ns_group_tables_match_oracle(sfl, dims, L, order, tr, tight):
    """The float64 group tables B_j hg_i, the bandpasses B_j and the hourglass
    masks the plans round to float32 (src/transforms/ns_surfacelet.jl:265-272,
    src/directional/hourglass.jl:264-289)."""
    t = sfl.NSSurfacelet(direction_levels=L, bernstein_order=order, transition=tr, tight=tight)
    p = N.NSParams.make(direction_levels=L, bernstein_order=order, transition=tr, tight=tight)
    T = N.make_tables(p, dims)
    h1 = dims[0] // 2 + 1
    J = len(L)
    shape = (h1, dims[1], dims[2])
    for j in range(1, J + 1):
        for i in (1, 2, 3):
            got = _ns_table(sfl, t, dims, "group", 3 * (j - 1) + i - 1).reshape(shape, order="F")
            exp = T.band[J - j] * N.hg_factor(T.m1, T.m2, i, tight)
            assert np.abs(got - exp).max() < 1e-12
    for lv in range(J):
        got = _ns_table(sfl, t, dims, "bandpass", lv).reshape(shape, order="F")
        assert np.abs(got - T.band[lv]).max() < 1e-12
    for i in (1, 2, 3):
        got = _ns_table(sfl, t, dims, "hourglass", i - 1).reshape(shape, order="F")
        assert np.abs(got - N.hourglass_mask(T.m1, T.m2, i, tight)).max() < 1e-12
    with pytest.raises(ValueError, match="out of range"):
        _ns_table(sfl, t, dims, "group", 3 * J)


@pytest.mark.parametrize("dims,L,mode,bo", [
    ((48, 48, 48), [[[-1, 1, 1], [1, -1, 1], [1, 1, -1]]] * 2, 1.5, 8),
    ((32, 32, 32), [[[-1, 2, 0], [1, -1, 1], [0, 3, -1]]], 2, 6),
])
def test_surf_design_tables_match_oracle(sfl, dims, L, mode, bo):
    Lm = [np.array(m) for m in L]
    t = sfl.Surfacelet(direction_levels=Lm, pyramid_ratio=mode, checkerboard_order=bo)
    p = D.SurfParams.make(direction_levels=Lm, pyramid_ratio=mode, checkerboard_order=bo)
    T = D.make_tables(p, dims)
    for lv, sc in enumerate(T.scales):
        for K in range(3):
            got = _surf_table(sfl, t, dims, "ritf", lv * 3 + K)
            assert np.abs(got - sc.masks[K].ravel(order="F")).max() < 1e-12
            for s, st in enumerate(sc.stages[K]):
                for which, plane in enumerate([st.ana[0], st.ana[1], st.syn[0], st.syn[1]]):
                    got = _surf_table(sfl, t, dims, "irc", ((lv * 3 + K) * 32 + s) * 4 + which)
                    got = got[0::2] + 1j * got[1::2]
                    # oracle planes are oriented 3-D; the library stores (K-half, m), K fastest
                    P = np.squeeze(plane)
                    if K + 1 > st.m:
                        P = P.T
                    assert np.abs(got - P.ravel(order="F")).max() < 1e-12
        for ax in range(3):
            got = _surf_table(sfl, t, dims, "pyr_prof", lv * 3 + ax)
            assert np.abs(got - T.pyramid[lv].prof[ax]).max() < 1e-15


def test_ns_layout_and_validation(sfl):
    # test/items/test_ns_surfacelet.jl:1-38, 316-324
    t = sfl.NSSurfacelet(scales=3, direction_levels=[1, 2, 2])
    lay = sfl.subband_layout(t, (16, 16, 16))
    assert sfl.nsubbands(t, (16, 16, 16)) == len(lay) == 1 + 6 + 12 + 12
    assert lay[0] == {"scale": 0, "direction": 0}
    assert lay[1] == {"scale": 1, "direction": 1}
    assert lay[7] == {"scale": 2, "direction": 1}
    assert t == sfl.NSSurfacelet(scales=3, direction_levels=[1, 2, 2])
    assert hash(sfl.NSSurfacelet(scales=1, transition=-0.0)) == hash(sfl.NSSurfacelet(scales=1, transition=0.0))
    assert t != sfl.NSSurfacelet(scales=3, direction_levels=[1, 2, 2], tight=False)
    assert repr(t) == ("NSSurfacelet(scales = 3, direction_levels = [1, 2, 2], bernstein_order = 12, "
                       "halfband_order = 1, transition = 1.0, tight = true)")
    assert sfl.NSSurfacelet(scales=4).direction_levels == [1, 1, 2, 2]
    assert sfl.NSSurfacelet(direction_levels=[1, 2]).scales == 2
    assert sfl.supports_streaming(t)
    with pytest.raises(sfl.ArgumentError, match="three axes"):
        sfl.subband_layout(t, (16, 16))
    for kw, msg in [
        (dict(scales=0, direction_levels=[]), "scales must be ≥ 1"),
        (dict(scales=2, direction_levels=[1]), "length\\(direction_levels\\) must equal scales"),
        (dict(scales=1, direction_levels=[-1]), "direction_levels entries must be ≥ 0"),
        (dict(scales=1, direction_levels=[1], bernstein_order=0), "bernstein_order must be ≥ 1"),
        (dict(scales=1, direction_levels=[1], halfband_order=-1), "halfband_order must be ≥ 0"),
        (dict(scales=1, direction_levels=[1], transition=-1), "transition must be ≥ 0"),
        (dict(), "give `scales`, `direction_levels` or both"),
    ]:
        with pytest.raises(sfl.ArgumentError, match=msg):
            sfl.NSSurfacelet(**kw)
    # src/transforms/ns_surfacelet.jl:109-115: an empty scale is refused at workspace time
    q = sfl.NSSurfacelet(scales=4, direction_levels=[0, 0, 0, 0], bernstein_order=4)
    with pytest.raises(sfl.ArgumentError, match="too small for 4 scales"):
        sfl.make_workspace(q, "float32", (8, 8, 8))


def test_surf_layout_and_validation(sfl):
    # test/items/test_surfacelet.jl:1-41, 175-207; test_literature.jl:47-58
    t = sfl.Surfacelet(scales=2, direction_levels=[1, 2])
    assert repr(t) == ("Surfacelet(scales = 2, direction_levels = [1, 2], pyramid_ratio = 1.5, "
                       "checkerboard_order = 12, diamond_length = 15, kaiser_beta = 2.5, diamond_power = 4)")
    lay = sfl.subband_layout(t, (48, 48, 48))
    assert lay[0] == {"scale": 0, "hourglass": 0, "wedge": 0}
    assert lay[1] == {"scale": 1, "hourglass": 1, "wedge": 1}
    assert sum(d["scale"] == 1 for d in lay) == 6 and sum(d["scale"] == 2 for d in lay) == 12
    assert sfl.nsubbands(t, (48, 48, 48)) == 19
    assert not sfl.supports_streaming(t)
    q = sfl.Surfacelet(scales=1, direction_levels=[[[-1, 2, 1], [1, -1, 2], [2, 1, -1]]])
    assert q.levels[0] == [[0, 2, 1], [1, 0, 2], [2, 1, 0]]
    assert sfl.nsubbands(q, (96, 96, 96)) == 25
    assert sfl.checkerboard_orders() == list(range(4, 19, 2))
    for kw, msg in [
        (dict(scales=0, direction_levels=[]), "scales must be ≥ 1"),
        (dict(scales=2, direction_levels=[1]), "length\\(direction_levels\\) must equal scales"),
        (dict(scales=1, direction_levels=[-1]), "directional levels must be ≥ 0"),
        (dict(scales=1, direction_levels=[np.ones((2, 2), int)]), "3 × 3"),
        (dict(scales=1, direction_levels=[1.5]), "integer or a 3 × 3"),
        (dict(scales=1, direction_levels=[1], pyramid_ratio=3), "pyramid_ratio"),
        (dict(scales=1, direction_levels=[1], checkerboard_order=5), "checkerboard_order must be one of"),
        (dict(scales=1, direction_levels=[1], diamond_length=14), "diamond_length"),
        (dict(scales=1, direction_levels=[1], kaiser_beta=0), "kaiser_beta"),
        (dict(scales=1, direction_levels=[1], diamond_power=3), "diamond_power"),
    ]:
        with pytest.raises(sfl.ArgumentError, match=msg):
            sfl.Surfacelet(**kw)
    t2 = sfl.Surfacelet(scales=1, direction_levels=[0], pyramid_ratio=2)
    msg = ("axis 1: at scale 1 of 1 (1 the coarsest) the length is 10, too small for the pyramid's lowpass; "
           "the nearest length that fits is 8")
    for f in (sfl.subband_layout, sfl.surfacelet_redundancy, sfl.nsubbands):
        with pytest.raises(sfl.ArgumentError, match="too small for the pyramid's lowpass"):
            f(t2, (10, 10, 10))
    with pytest.raises(sfl.ArgumentError) as e:
        sfl.make_workspace(t2, "float32", (10, 10, 10))
    assert msg in str(e.value)
    with pytest.raises(sfl.ArgumentError, match="axis 1: at scale 3 of 3 \\(1 the coarsest\\) the length is 20"):
        sfl.make_workspace(sfl.Surfacelet(scales=3), "float32", (20, 24, 24))
    with pytest.raises(sfl.ArgumentError, match="resampling by 3/2 needs to be a multiple of 3"):
        sfl.make_workspace(sfl.Surfacelet(scales=1, direction_levels=[0]), "float32", (20, 24, 24))
    # redundancy: the paper's figures (test/items/test_literature.jl:47-58) and the oracle
    for mode, r in ((1, 6.4), (1.5, 4.0), (2, 3.4)):
        for L in ([1, 1, 1], [3, 3, 3]):
            u = sfl.Surfacelet(scales=3, direction_levels=L, pyramid_ratio=mode, checkerboard_order=4)
            assert abs(sfl.surfacelet_redundancy(u, (192, 192, 192)) - r) <= 0.1
    u = sfl.Surfacelet(scales=3, direction_levels=[2, 2, 3], pyramid_ratio=2)
    p = D.SurfParams.make(scales=3, direction_levels=[2, 2, 3], pyramid_ratio=2)
    assert sfl.subband_sizes(u, (128, 128, 128)) == [tuple(s) for s in D.layout_sizes(p, (128, 128, 128))]
    assert sfl.surfacelet_redundancy(u, (128, 128, 128)) == pytest.approx(D.redundancy(p, (128, 128, 128)))
