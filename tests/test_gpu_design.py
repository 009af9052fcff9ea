"""The NSSurfacelet and NDFB mask tables are designed on the device in float64
(the m1 contraction, the halfband response, B_j and the hourglass factor per
bin) and rounded to float32.  They must equal the float64 host design rounded
to float32 bit for bit (src/transforms/ns_surfacelet.jl:265-272,
src/directional/hourglass.jl:172-189, 264-303)."""

import ctypes as C

import numpy as np
import pytest

from conftest import gpu_available

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not gpu_available(), reason="needs a CUDA device")]


def _host(sfl, params, dims, name, index):
    lib = sfl.lib
    cnt = C.c_int64()
    d = (C.c_int32 * 3)(*dims)
    sfl._lib.check(lib.sfl_ns_design_table(C.byref(params), d, name.encode(), index, None, C.byref(cnt)))
    out = (C.c_double * cnt.value)()
    sfl._lib.check(lib.sfl_ns_design_table(C.byref(params), d, name.encode(), index, out, C.byref(cnt)))
    return np.frombuffer(out, dtype=np.float64).astype(np.float32)


def _plan(sfl, ws, name, index):
    cnt = C.c_int64()
    sfl._lib.check(sfl.lib.sfl_ns_plan_table(ws._h, name.encode(), index, None, C.byref(cnt)))
    out = (C.c_float * cnt.value)()
    sfl._lib.check(sfl.lib.sfl_ns_plan_table(ws._h, name.encode(), index, out, C.byref(cnt)))
    return np.frombuffer(out, dtype=np.float32).copy()


NS_CASES = [((16, 12, 20), [1, 2], 6, 1.0, True),
            ((15, 20, 8), [1, 1, 2], 12, 0.5, False),
            ((128, 128, 128), [2, 2, 3], 12, 1.0, True),
            ((96, 64, 160), [1, 2, 2], 12, 1.0, False),
            ((63, 47, 33), [2, 3], 9, 0.7, True)]


@pytest.mark.parametrize("dims,L,order,tr,tight", NS_CASES)
def test_ns_plan_tables_equal_host_design(sfl, dims, L, order, tr, tight):
    t = sfl.NSSurfacelet(scales=len(L), direction_levels=L, bernstein_order=order, transition=tr, tight=tight)
    ws = sfl.make_workspace(t, "float32", dims)
    p = t._params()
    for g in range(3 * len(L)):
        np.testing.assert_array_equal(_plan(sfl, ws, "group", g), _host(sfl, p, dims, "group", g))
    if not tight:
        for lv in range(len(L)):
            np.testing.assert_array_equal(_plan(sfl, ws, "bandpass", lv), _host(sfl, p, dims, "bandpass", lv))
    else:
        with pytest.raises(ValueError, match="out of range"):
            _plan(sfl, ws, "bandpass", 0)


@pytest.mark.parametrize("dims,levels,tight", [((24, 20, 16), 1, False), ((64, 64, 64), 2, True)])
def test_ndfb_plan_tables_equal_host_design(sfl, dims, levels, tight):
    t = sfl.NDFB(levels=levels, bernstein_order=6, tight=tight)
    ws = sfl.make_workspace(t, "float32", dims)
    p = sfl.NSSurfacelet(scales=1, direction_levels=[levels], bernstein_order=6, tight=tight)._params()
    for i in range(3):
        np.testing.assert_array_equal(_plan(sfl, ws, "group", i), _host(sfl, p, dims, "hourglass", i))
    if not tight:
        np.testing.assert_array_equal(_plan(sfl, ws, "bandpass", 0), np.ones(ws.dims[0] // 2 + 1, np.float32).repeat(
            dims[1] * dims[2]))


def _surf_host(sfl, params, dims, name, index):
    lib = sfl.lib
    cnt = C.c_int64()
    d = (C.c_int32 * 3)(*dims)
    sfl._lib.check(lib.sfl_surf_design_table(C.byref(params), d, name.encode(), index, None, C.byref(cnt)))
    out = (C.c_double * cnt.value)()
    sfl._lib.check(lib.sfl_surf_design_table(C.byref(params), d, name.encode(), index, out, C.byref(cnt)))
    return np.frombuffer(out, dtype=np.float64).astype(np.float32)


def _surf_plan(sfl, ws, name, index):
    cnt = C.c_int64()
    sfl._lib.check(sfl.lib.sfl_surf_plan_table(ws._h, name.encode(), index, None, C.byref(cnt)))
    out = (C.c_float * cnt.value)()
    sfl._lib.check(sfl.lib.sfl_surf_plan_table(ws._h, name.encode(), index, out, C.byref(cnt)))
    return np.frombuffer(out, dtype=np.float32).copy()


SURF_CASES = [((128, 128, 128), dict(scales=3, direction_levels=[2, 2, 3], pyramid_ratio=2)),
              ((96, 96, 96), dict(scales=3, direction_levels=[2, 2, 3])),
              ((48, 48, 48), dict(scales=2, direction_levels=[1, 2], checkerboard_order=8)),
              ((64, 32, 48), dict(scales=1, direction_levels=[2], pyramid_ratio=1, checkerboard_order=6))]


@pytest.mark.parametrize("dims,kw", SURF_CASES)
def test_surf_plan_tables_equal_host_design(sfl, dims, kw):
    """The decimated transform's ritf masks V_K and IRC filter slices, composed
    on the device from the host's separable factors, equal the host's float64
    design rounded to float32 bit for bit (src/directional/ritf.jl:89-108,
    src/directional/irc.jl:49-91)."""
    t = sfl.Surfacelet(**kw)
    ws = sfl.make_workspace(t, "float32", dims)
    p = t._params()
    nstages = 0
    for lv in range(kw["scales"]):
        for K in range(3):
            np.testing.assert_array_equal(_surf_plan(sfl, ws, "ritf", lv * 3 + K),
                                          _surf_host(sfl, p, dims, "ritf", lv * 3 + K))
            for st in range(32):
                idx = ((lv * 3 + K) * 32 + st) * 4
                try:
                    got = [_surf_plan(sfl, ws, "irc", idx + w) for w in range(4)]
                except ValueError:
                    break
                nstages += 1
                for w in range(4):
                    np.testing.assert_array_equal(got[w], _surf_host(sfl, p, dims, "irc", idx + w))
    assert nstages > 0
    with pytest.raises(ValueError, match="out of range"):
        _surf_plan(sfl, ws, "ritf", 3 * kw["scales"])
