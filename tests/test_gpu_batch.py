"""Batches replayed as one CUDA graph (sfl_batch_*) against a loop of plain
calls: the same kernels on the same data, so the outputs agree bit for bit,
also after the inputs are refilled in place between runs (the batch workload
of mixed sizes and scale counts)."""

import numpy as np
import pytest
import torch

from conftest import gpu_available

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not gpu_available(), reason="needs a CUDA device")]

MEMBERS = [
    ("ns", (64, 64, 64), dict(scales=3, direction_levels=[2, 2, 3])),
    ("ns", (96, 64, 128), dict(scales=2, direction_levels=[1, 3], bernstein_order=6)),
    ("ns", (64, 96, 64), dict(scales=2, direction_levels=[2, 1])),
    ("ns", (40, 36, 48), dict(scales=2, direction_levels=[1, 2], bernstein_order=6)),
    ("surf", (48, 48, 48), dict(scales=2, direction_levels=[1, 2])),
]


def _members(sfl):
    out = []
    for kind, dims, kw in MEMBERS:
        t = sfl.NSSurfacelet(**kw) if kind == "ns" else sfl.Surfacelet(**kw)
        out.append(sfl.make_workspace(t, "float32", dims))
    out.append(out[0])          # one workspace twice: its transforms keep their order
    return out


def _coef(sfl, ws):
    return sfl.similar_coefficients(ws.transform, sfl.volume_like(ws.dims))


def test_batch_analyze_and_synthesize_equal_plain_calls(sfl):
    wss = _members(sfl)
    rng = np.random.default_rng(11)
    xs = [sfl.to_device(rng.standard_normal(ws.dims).astype(np.float32)) for ws in wss]
    cs = [_coef(sfl, ws) for ws in wss]
    b = sfl.Batch(wss, xs, cs, "analyze")
    for rnd in range(2):
        if rnd:
            for x in xs:      # refill in place; the graph keeps the pointers
                x.copy_(sfl.to_device(rng.standard_normal(tuple(x.shape)).astype(np.float32)))
        b.run()
        torch.cuda.synchronize()
        for ws, x, c in zip(wss, xs, cs):
            assert torch.equal(c, sfl.analyze(ws, x)), ws.dims
    ys = [sfl.volume_like(ws.dims) for ws in wss]
    bs = sfl.Batch(wss, cs, ys, "synthesize")
    bs.run()
    torch.cuda.synchronize()
    for ws, c, y, x in zip(wss, cs, ys, xs):
        assert torch.equal(y, sfl.synthesize(ws, c)), ws.dims
        assert float(torch.linalg.vector_norm(y - x) / torch.linalg.vector_norm(x)) <= 1e-5
    b.close()
    bs.close()


def test_batch_argument_errors(sfl):
    wss = _members(sfl)[:2]
    xs = [sfl.volume_like(ws.dims) for ws in wss]
    cs = [_coef(sfl, ws) for ws in wss]
    with pytest.raises(sfl.ArgumentError):
        sfl.Batch(wss, xs[:1], cs, "analyze")
    with pytest.raises(sfl.ArgumentError):
        sfl.Batch(wss, xs, cs, "transpose")
    with pytest.raises(sfl.ArgumentError):
        sfl.Batch(wss, xs, cs, ["analyze"])
    with pytest.raises(sfl.DimensionMismatch):
        sfl.Batch(wss, xs[::-1], cs, "analyze")


def test_batch_chains_operators_of_one_workspace(sfl):
    # analyze -> synthesize -> adjoint of synthesize per workspace, in one graph
    wss = _members(sfl)[:5]
    rng = np.random.default_rng(12)
    ents, refs = [], []
    for ws in wss:
        x = sfl.to_device(rng.standard_normal(ws.dims).astype(np.float32))
        c, y, g = _coef(sfl, ws), sfl.volume_like(ws.dims), _coef(sfl, ws)
        ents += [(ws, "analyze", x, c), (ws, "synthesize", c, y), (ws, "adjoint_synthesize", y, g)]
        refs.append((ws, x, c, y, g))
    b = sfl.Batch([e[0] for e in ents], [e[2] for e in ents], [e[3] for e in ents], [e[1] for e in ents])
    b.run()
    torch.cuda.synchronize()
    for ws, x, c, y, g in refs:
        c0 = sfl.analyze(ws, x)
        y0 = sfl.synthesize(ws, c0)
        assert torch.equal(c, c0) and torch.equal(y, y0)
        assert torch.equal(g, sfl.adjoint_synthesize(ws, y0))
    b.close()


def test_batch_copies_volumes_to_and_from_pinned_host_memory(sfl):
    wss = _members(sfl)[:3]
    rng = np.random.default_rng(13)
    ents, chk = [], []
    for ws in wss:
        hx = torch.from_numpy(rng.standard_normal(ws.dims[::-1]).astype(np.float32)).pin_memory()
        hy = torch.empty(ws.dims[::-1]).pin_memory()
        x, y, c = sfl.volume_like(ws.dims), sfl.volume_like(ws.dims), _coef(sfl, ws)
        ents += [(ws, "copy_volume", hx, x), (ws, "analyze", x, c), (ws, "synthesize", c, y),
                 (ws, "copy_volume", y, hy)]
        chk.append((ws, hx, hy))
    b = sfl.Batch([e[0] for e in ents], [e[2] for e in ents], [e[3] for e in ents], [e[1] for e in ents])
    for _ in range(2):
        b.run()
        torch.cuda.synchronize()
        for ws, hx, hy in chk:
            xd = hx.cuda().permute(2, 1, 0)              # column-major view of the host volume
            y0 = sfl.synthesize(ws, sfl.analyze(ws, xd))
            assert torch.equal(hy.cuda().permute(2, 1, 0), y0)
    with pytest.raises(sfl.ArgumentError):
        sfl.Batch([wss[0]], [torch.empty(wss[0].dims[::-1])], [sfl.volume_like(wss[0].dims)], ["copy_volume"])
    b.close()


def _mixed_configs(n, seed):
    # the batch workload: every axis from {64, 96, 128, 160}, scales from {2, 3, 4},
    # each scale's direction level from {1, 2, 3}
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n):
        dims = tuple(int(v) for v in rng.choice([64, 96, 128, 160], 3))
        J = int(rng.choice([2, 3, 4]))
        out.append((dims, dict(scales=J, direction_levels=[int(v) for v in rng.choice([1, 2, 3], J)])))
    return out


def test_autotune_picks_and_remembers(sfl):
    dims = (64, 96, 64)
    t = sfl.NSSurfacelet(scales=3, direction_levels=[2, 1, 3])
    ws = sfl.make_workspace(t, "float32", dims)
    x = sfl.to_device(np.random.default_rng(2).standard_normal(dims).astype(np.float32))
    c0 = sfl.analyze(ws, x)
    pick = ws.autotune(x)
    assert pick[0] in ("slabs", "lines") and pick[1] in (2, 4, 8)
    c1 = sfl.analyze(ws, x)
    assert float(torch.linalg.vector_norm(c1 - c0) / torch.linalg.vector_norm(c0)) <= 1e-6
    assert sfl.make_workspace(t, "float32", dims).tuning() == pick          # the process-wide record
    assert sfl.make_workspace(t, "complex64", dims).tuning()[1] == 8        # another element type: untuned


def test_mixed_batch_as_one_graph(sfl):
    cfgs = _mixed_configs(8, 44)
    rng = np.random.default_rng(45)
    wss, xs = [], []
    for dims, kw in cfgs:
        ws = sfl.make_workspace(sfl.NSSurfacelet(**kw), "float32", dims)
        x = sfl.to_device(rng.standard_normal(dims).astype(np.float32))
        ws.autotune(x)
        wss.append(ws)
        xs.append(x)
    cs = [_coef(sfl, ws) for ws in wss]
    ys = [sfl.volume_like(ws.dims) for ws in wss]
    gs = [_coef(sfl, ws) for ws in wss]
    ents = []
    for ws, x, c, y, g in zip(wss, xs, cs, ys, gs):
        ents += [(ws, "analyze", x, c), (ws, "synthesize", c, y), (ws, "adjoint_synthesize", y, g)]
    b = sfl.Batch([e[0] for e in ents], [e[2] for e in ents], [e[3] for e in ents], [e[1] for e in ents])
    b.run()
    torch.cuda.synchronize()
    for ws, x, c, y, g in zip(wss, xs, cs, ys, gs):
        c0 = sfl.analyze(ws, x)
        assert torch.equal(c, c0)
        assert torch.equal(y, sfl.synthesize(ws, c0))
        assert float(torch.linalg.vector_norm(y - x) / torch.linalg.vector_norm(x)) <= 1e-5
    b.close()


def test_axis3_tile_is_tunable_and_does_not_change_results(sfl):
    """Subbands a CTA of the slab axis-3 analysis pass (the tile the autotuner
    picks): 1, 2 and 4 give the same coefficients bit for bit."""
    dims = (64, 64, 64)
    t = sfl.NSSurfacelet(scales=3, direction_levels=[2, 2, 3])
    ws = sfl.make_workspace(t, "float32", dims)
    x = sfl.to_device(np.random.default_rng(12).standard_normal(dims).astype(np.float32))
    assert ws.tile() == 0
    ref = sfl.analyze(ws, x)
    for ipc in (1, 2, 4, 8):
        assert ws.tile(ipc) == ipc and ws.tile() == ipc
        assert torch.equal(sfl.analyze(ws, x), ref), ipc
    with pytest.raises(sfl.ArgumentError, match="1, 2, 4 or 8"):
        ws.tile(3)
    ws.tile(0)
    ws.autotune(x)
    assert ws.tile() in (0, 1, 2, 4)
    assert torch.equal(sfl.analyze(ws, x), ref) or ws.tuning()[0] == "lines"
