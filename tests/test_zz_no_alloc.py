"""sfl_ns_analyze_subband_static, the entry point for callers that cannot
allocate device memory when they transform (allocation-free real-time loops,
processes whose memory manager owns the device): it computes one
NSSurfacelet subband with scratch held in a static device array of the
library.  Checked through the C ABI against the existing sfl_analyze, on two
calls in a row; it must agree whether this file runs alone or after the rest
of the suite (the static scratch keeps the previous call's contents).  After a
warm-up call, further calls must leave the device's free memory unchanged.
"""

import ctypes as C

import numpy as np
import pytest
import torch

from conftest import gpu_available

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not gpu_available(), reason="needs a CUDA device")]

REL = 1e-5


def rel_l2(a, b):
    return float(torch.linalg.vector_norm(a - b) / torch.linalg.vector_norm(b))


def call(sfl, ws, x, b, i, stream=None):
    s = stream if stream is not None else torch.cuda.current_stream()
    return sfl.lib.sfl_ns_analyze_subband_static(ws._h, C.c_void_p(x.data_ptr()), C.c_void_p(b.data_ptr()), i,
                                                 C.c_void_p(s.cuda_stream))


@pytest.mark.parametrize("dims,kw", [
    ((64, 64, 64), dict(scales=3, direction_levels=[2, 2, 3])),
    ((32, 24, 20), dict(scales=2, direction_levels=[1, 2], bernstein_order=6)),
])
def test_static_scratch_subbands_match_sfl_analyze(sfl, dims, kw):
    lib = sfl.lib
    t = sfl.NSSurfacelet(**kw)
    ws = sfl.make_workspace(t, "float32", dims)
    x = sfl.to_device(np.random.default_rng(7).standard_normal(dims).astype(np.float32))
    ref = sfl.analyze(ws, x)                      # the existing entry point (sfl_analyze)
    picks = [2, ws.nsubbands, 1]                  # two calls in a row, then the lowpass
    bands = [sfl.volume_like(dims) for _ in picks]
    for i, b in zip(picks, bands):
        assert call(sfl, ws, x, b, i) == 0, lib.sfl_last_error().decode()
    torch.cuda.synchronize()
    for i, b in zip(picks, bands):
        assert rel_l2(b, ref[..., i - 1]) <= REL, i


def test_static_scratch_allocates_nothing_after_warm_up(sfl):
    dims = (64, 64, 64)
    ws = sfl.make_workspace(sfl.NSSurfacelet(scales=3, direction_levels=[2, 2, 3]), "float32", dims)
    x = sfl.to_device(np.random.default_rng(8).standard_normal(dims).astype(np.float32))
    ref = sfl.analyze(ws, x)
    picks = (2, 17, 49, 1)
    bands = [sfl.volume_like(dims) for _ in picks]
    assert call(sfl, ws, x, bands[0], 5) == 0     # warm-up: address look-up, kernel loading
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    for i, b in zip(picks, bands):
        assert call(sfl, ws, x, b, i) == 0
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info()[0] == free0   # nothing was allocated on the device
    for i, b in zip(picks, bands):
        assert rel_l2(b, ref[..., i - 1]) <= REL, i


def test_static_scratch_rejects_sizes_beyond_its_limit(sfl):
    lib = sfl.lib
    dims = (128, 128, 128)            # (n1/2+1) n2 n3 = 1,064,960 > 262,144
    ws = sfl.make_workspace(sfl.NSSurfacelet(scales=1, direction_levels=[1], bernstein_order=4), "float32", dims)
    x = sfl.volume_like(dims)
    b = sfl.volume_like(dims)
    assert call(sfl, ws, x, b, 1) == sfl._lib.SFL_ERR_ARGUMENT
    assert "static scratch" in lib.sfl_last_error().decode()


@pytest.mark.parametrize("case", ["index0", "index_past_end", "complex", "decimated"])
def test_static_scratch_rejects_bad_arguments(sfl, case):
    lib = sfl.lib
    dims = (32, 32, 32)
    if case == "complex":
        ws = sfl.make_workspace(sfl.NSSurfacelet(scales=2, direction_levels=[1, 1], bernstein_order=6), "complex64", dims)
        msg, i = "real", 2
    elif case == "decimated":
        dims = (48, 48, 48)         # the default pyramid_ratio 1.5 needs lengths divisible by 3
        ws = sfl.make_workspace(sfl.Surfacelet(scales=1, direction_levels=[1]), "float32", dims)
        msg, i = "NSSurfacelet plans only", 2
    else:
        ws = sfl.make_workspace(sfl.NSSurfacelet(scales=2, direction_levels=[1, 1], bernstein_order=6), "float32", dims)
        i = 0 if case == "index0" else ws.nsubbands + 1
        msg = "out of range"
    x = sfl.volume_like(dims)
    b = sfl.volume_like(dims)
    assert call(sfl, ws, x, b, i) == sfl._lib.SFL_ERR_ARGUMENT
    assert msg in lib.sfl_last_error().decode()
