"""sfl_ns_analyze_subband_static, the entry point for callers that cannot
allocate device memory when they transform (host functions on a stream,
allocation-free real-time loops, processes whose memory manager owns the
device): it computes one NSSurfacelet subband with scratch held in a static
device array of the library.  Checked through the C ABI against the existing
sfl_analyze, on two calls in a row; it must agree whether this file runs
alone or after the rest of the suite (the static scratch keeps the previous
call's contents).
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
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    picks = [2, ws.nsubbands, 1]                  # two calls in a row, then the lowpass
    bands = [sfl.volume_like(dims) for _ in picks]
    for i, b in zip(picks, bands):
        st = lib.sfl_ns_analyze_subband_static(ws._h, C.c_void_p(x.data_ptr()), C.c_void_p(b.data_ptr()), i, stream)
        assert st == 0, lib.sfl_last_error().decode()
    torch.cuda.synchronize()
    for i, b in zip(picks, bands):
        assert rel_l2(b, ref[..., i - 1]) <= REL, i


def test_static_scratch_rejects_sizes_beyond_its_limit(sfl):
    lib = sfl.lib
    dims = (128, 128, 128)            # (n1/2+1) n2 n3 = 1,064,960 > 262,144
    ws = sfl.make_workspace(sfl.NSSurfacelet(scales=1, direction_levels=[1], bernstein_order=4), "float32", dims)
    x = sfl.volume_like(dims)
    b = sfl.volume_like(dims)
    st = lib.sfl_ns_analyze_subband_static(ws._h, C.c_void_p(x.data_ptr()), C.c_void_p(b.data_ptr()), 1,
                                           C.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert st == -1
    assert "static scratch" in lib.sfl_last_error().decode()
