"""Subband sharding (analyze_sharded / synthesize_sharded) on two CPU ranks
over gloo, with the float64 oracle standing in for the library's item-range
operations: the partition, the broadcast of the spectrum and the reduction
of the partial spectra are the product's host logic."""

import datetime
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from conftest import load_package
from oracle import ns as N

KW = dict(scales=2, direction_levels=[1, 2], bernstein_order=6)
DIMS = (12, 10, 8)


class OracleRanges:
    """The item-range operations of sharded.LibRanges, in float64 on the host."""

    def __init__(self, kw, dims):
        self.T = N.make_tables(N.NSParams.make(**kw), dims)
        self.dims = dims
        ana = list(N.subband_masks(self.T, analysis=True))
        self.stream_order = [s for s, _ in ana]
        self.amasks = [m for _, m in ana]
        self.smasks = [m for _, m in N.subband_masks(self.T, analysis=False)]
        self.nsubbands = len(ana)
        self.grid = self.amasks[0].shape
        self.spectrum_elems = int(np.prod(self.grid))

    def new_spectrum(self, device):
        return torch.zeros(self.spectrum_elems, dtype=torch.complex128)

    def new_volume(self, device):
        return torch.empty(self.dims, dtype=torch.float64)

    def new_subbands(self, count, device):
        return torch.empty(self.dims + (count,), dtype=torch.float64)

    def forward_spectrum(self, x, X):
        X.copy_(torch.from_numpy(N.rfft3(x.numpy()).ravel()))

    def analyze_range(self, X, first, count, c):
        Xn = X.numpy().reshape(self.grid)
        for q in range(count):
            c[..., q] = torch.from_numpy(N.irfft3(Xn * self.amasks[first + q], self.dims))

    def accumulate_range(self, c, first, count, A, clear):
        if clear:
            A.zero_()
        acc = sum(self.smasks[first + q] * N.rfft3(c[..., q].numpy()) for q in range(count))
        A += torch.from_numpy(acc.ravel())

    def inverse_spectrum(self, A, x):
        x.copy_(torch.from_numpy(N.irfft3(A.numpy().reshape(self.grid), self.dims)))


def _worker(rank, world, port, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        sfl = load_package()
        ops = OracleRanges(KW, DIMS)
        x = np.random.default_rng(0).standard_normal(DIMS)
        c, first = sfl.analyze_sharded(ops, torch.from_numpy(x) if rank == 0 else None, device="cpu")
        ref = N.analyze(ops.T, x)
        err = 0.0
        for q in range(c.shape[-1]):
            s = ops.stream_order[first + q]
            err = max(err, float(np.abs(c[..., q].numpy() - ref[..., s - 1]).max()))
        y = sfl.synthesize_sharded(ops, c, first, device="cpu")
        pr = float(np.abs(y.numpy() - x).max()) if rank == 0 else 0.0
        out.put((rank, first, c.shape[-1], err, pr, y is None))
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_shard_partitions_positions():
    sfl = load_package()
    for S in (1, 7, 49, 73):
        for world in (1, 2, 3, 8):
            got = [sfl.shard(S, world, r) for r in range(world)]
            assert sum(n for _, n in got) == S
            assert [f for f, _ in got] == [sum(n for _, n in got[:r]) for r in range(world)]
            assert max(n for _, n in got) - min(n for _, n in got) <= 1
    with pytest.raises(sfl.ArgumentError):
        sfl.shard(5, 2, 2)


def test_sharded_analysis_and_synthesis_on_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(out.get(timeout=180) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    S = N.nsubbands(N.NSParams.make(**KW))
    assert [(r[1], r[2]) for r in res] == [(0, (S + 1) // 2), ((S + 1) // 2, S // 2)]
    for rank, first, count, err, pr, none in res:
        assert err < 1e-12
        assert none == (rank != 0)
    assert res[0][4] < 1e-12      # perfect reconstruction on the root
