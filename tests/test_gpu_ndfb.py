"""The standalone directional banks (NDFB, HourglassFB) on the B200 against
the float64 oracle (src/directional/ndfb.jl, hourglass.jl): decomposition,
reconstruction, Parseval when tight, the bare-sum reconstruction when not,
streaming and complex data."""

import numpy as np
import pytest
import torch

from conftest import gpu_available
from oracle import ns as N

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not gpu_available(), reason="needs a CUDA device")]

REL = 1e-5


def rel(a, b):
    a = np.asarray(a, dtype=np.complex128 if np.iscomplexobj(a) else np.float64)
    return float(np.linalg.norm((a - b).ravel()) / np.linalg.norm(np.asarray(b).ravel()))


CASES = [((16, 16, 16), 2, True, 1.0), ((20, 12, 18), 3, True, 0.5), ((24, 20, 16), 1, False, 1.0),
         ((64, 64, 64), 2, True, 1.0), ((128, 96, 64), 3, False, 1.0)]


@pytest.mark.parametrize("dims,levels,tight,transition", CASES)
def test_ndfb_matches_oracle(sfl, dims, levels, tight, transition):
    t = sfl.NDFB(levels=levels, bernstein_order=6, tight=tight, transition=transition)
    ws = sfl.make_workspace(t, "float32", dims)
    assert ws.nsubbands == 3 * 2 ** levels
    x = np.random.default_rng(17).standard_normal(dims).astype(np.float32)
    c = sfl.to_host(sfl.ndfb_decompose(ws, sfl.to_device(x)))
    ref = N.ndfb_decompose(x.astype(np.float64), dims, levels, order=6, tight=tight, transition=transition)
    for idx in range(1, ws.nsubbands + 1):
        assert rel(c[..., idx - 1], ref[idx - 1]) <= REL, idx
    y = sfl.to_host(sfl.ndfb_reconstruct(ws, sfl.to_device(c)))
    assert rel(y, x) <= REL                                   # perfect reconstruction
    if tight:
        e = float(np.sum(c.astype(np.float64) ** 2))
        assert abs(e - float(np.sum(x.astype(np.float64) ** 2))) <= 1e-5 * e   # Parseval
    else:
        assert rel(np.sum(c.astype(np.float64), axis=-1), x) <= REL        # a bare sum


def test_hourglass_bank(sfl):
    dims = (24, 16, 20)
    ws = sfl.make_workspace(sfl.HourglassFB(bernstein_order=6), "float32", dims)
    x = np.random.default_rng(3).standard_normal(dims).astype(np.float32)
    s = sfl.hourglass_decompose(ws, sfl.to_device(x))
    ref = N.hourglass_decompose(x.astype(np.float64), dims, 6, 1)
    for i in range(3):
        assert rel(sfl.to_host(s[i]), ref[i]) <= REL
    assert rel(sfl.to_host(sfl.hourglass_reconstruct(ws, s)), x) <= REL
    with pytest.raises(sfl.DimensionMismatch):
        sfl.hourglass_reconstruct(ws, (s[0], s[1], sfl.volume_like((4, 4, 4))))


def test_ndfb_streaming_and_complex(sfl):
    dims = (64, 64, 64)
    t = sfl.NDFB(levels=2, bernstein_order=6)
    rng = np.random.default_rng(8)
    xr = rng.standard_normal(dims).astype(np.float32)
    xi = rng.standard_normal(dims).astype(np.float32)
    ws = sfl.make_workspace(t, "float32", dims)
    xd = sfl.to_device(xr)
    c = sfl.ndfb_decompose(ws, xd)
    got = {}
    sfl.analyze(lambda i, b: got.__setitem__(i, b.clone()), ws, xd)
    assert sorted(got) == list(range(1, ws.nsubbands + 1))   # stream order = index order
    for i, b in got.items():
        assert torch.equal(b, c[..., i - 1])
    wz = sfl.make_workspace(t, "complex64", dims)
    cz = sfl.to_host(sfl.ndfb_decompose(wz, sfl.to_device(xr + 1j * xi)))
    ci = sfl.to_host(sfl.ndfb_decompose(ws, sfl.to_device(xi)))
    assert np.array_equal(cz.real, sfl.to_host(c)) and np.array_equal(cz.imag, ci)
