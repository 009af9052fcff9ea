"""The item-range entry points behind subband sharding, on one B200: ranges
reproduce analyze bit for bit, partial spectra add up to the synthesis, and
analyze_sharded / synthesize_sharded over NCCL with a group of one equal the
plain calls.  (The multi-rank host logic runs on CPU ranks in
test_sharded_gloo.py; several ranks on one GPU are not emulated.)"""

import datetime
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist

from conftest import gpu_available

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not gpu_available(), reason="needs a CUDA device")]


def rel(a, b):
    d = torch.complex128 if a.is_complex() or b.is_complex() else torch.float64
    return float(torch.linalg.vector_norm((a - b).to(d)) / torch.linalg.vector_norm(b.to(d)))


@pytest.mark.parametrize("dims,pipeline,dtype", [((64, 64, 64), "slabs", "float32"), ((64, 64, 64), "lines", "float32"),
                                                 ((40, 36, 48), "lines", "complex64"),
                                                 ((96, 64, 128), "slabs", "complex64")])
def test_ranges_reproduce_the_transforms(sfl, dims, pipeline, dtype):
    t = sfl.NSSurfacelet(scales=3, direction_levels=[2, 2, 3]) if dims[0] == 64 else \
        sfl.NSSurfacelet(scales=2, direction_levels=[1, 3], bernstein_order=6)
    ws = sfl.make_workspace(t, dtype, dims)
    ws.set_pipeline(pipeline)
    ops = sfl.LibRanges(ws)
    rng = np.random.default_rng(4)
    x = rng.standard_normal(dims).astype(np.float32)
    if dtype == "complex64":
        x = (x + 1j * rng.standard_normal(dims)).astype(np.complex64)
    xd = sfl.to_device(x)
    cf = sfl.analyze(ws, xd)
    X = ops.new_spectrum()
    ops.forward_spectrum(xd, X)
    S, order = ws.nsubbands, ops.stream_order
    assert sorted(order) == list(range(1, S + 1))
    As, cs = [], []
    for r in range(3):                      # three shares, one after another
        f, n = sfl.shard(S, 3, r)
        c = ops.new_subbands(n)
        ops.analyze_range(X, f, n, c)
        for q in range(n):
            assert torch.equal(c[..., q], cf[..., order[f + q] - 1]), (r, q)
        A = ops.new_spectrum()
        ops.accumulate_range(c, f, n, A, True)
        As.append(A)
        cs.append(c)
    y = ops.new_volume()
    ops.inverse_spectrum(As[0] + As[1] + As[2], y)
    yf = sfl.synthesize(ws, cf)
    assert rel(y, yf) <= 1e-6
    # one share holding everything is the plain synthesis, bit for bit
    call = torch.cat(cs, dim=-1)
    call = sfl.as_colmajor(call)
    A = ops.new_spectrum()
    ops.accumulate_range(call, 0, S, A, True)
    ops.inverse_spectrum(A, y)
    assert torch.equal(y, yf)
    with pytest.raises(sfl.ArgumentError):
        ops.analyze_range(X, S - 1, 2, ops.new_subbands(2))
    # spectra move in 16-byte blocks: a spectrum one bin off a 16-byte boundary is refused
    Xb = torch.empty(ops.nch * ops.spectrum_elems + 1, dtype=torch.complex64, device="cuda")[1:]
    c1 = sfl.as_colmajor(call[..., :1])
    for fn in (lambda: ops.forward_spectrum(xd, Xb), lambda: ops.analyze_range(Xb, 0, 1, ops.new_subbands(1)),
               lambda: ops.accumulate_range(c1, 0, 1, Xb, True), lambda: ops.inverse_spectrum(Xb, y)):
        with pytest.raises(sfl.ArgumentError, match="16-byte aligned"):
            fn()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_sharded_over_nccl_with_a_group_of_one(sfl):
    dims = (128, 128, 128)
    ws = sfl.make_workspace(sfl.NSSurfacelet(scales=3, direction_levels=[2, 2, 3]), "float32", dims)
    ops = sfl.LibRanges(ws)
    xd = sfl.to_device(np.random.default_rng(6).standard_normal(dims).astype(np.float32))
    dist.init_process_group("nccl", init_method=f"tcp://127.0.0.1:{_free_port()}", rank=0, world_size=1,
                            timeout=datetime.timedelta(seconds=60), device_id=torch.device("cuda", 0))
    try:
        c, first = sfl.analyze_sharded(ops, xd)
        cf = sfl.analyze(ws, xd)
        assert first == 0 and c.shape[-1] == ws.nsubbands
        for q, s in enumerate(ops.stream_order):
            assert torch.equal(c[..., q], cf[..., s - 1])
        y = sfl.synthesize_sharded(ops, c, first)
        assert torch.equal(y, sfl.synthesize(ws, cf))
    finally:
        dist.destroy_process_group()
