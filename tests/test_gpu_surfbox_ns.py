"""The device hourglass and NDFB banks against SurfBox's golden data for the
nonsubsampled transform (test/items/test_surfbox_reference.jl:17-156), through
the C ABI in float32.

The hourglass weights are read off the device transform itself: a unit impulse
at the origin has a flat spectrum, so the subbands of hourglass_decompose are
irfft(M_i) and their rfft gives back the analysis masks M_i = sqrt(W_i) to
float32 rounding.  The reference's geometric bounds then apply as stated, with
the dominant hourglass taken as the first of the weights within 1e-6 of the
maximum (float32 noise would otherwise break the exact ties where hourglasses
meet); the exact partition-of-unity bound (1e-12 in float64) becomes 1e-5.
"""

import numpy as np
import pytest

import surfbox_ns as SB
from conftest import gpu_available
from oracle import ns as N

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not gpu_available(), reason="needs a CUDA device")]


def test_device_hourglass_matches_surfbox_partition(sfl):
    octant, _, _ = SB.load()
    _, w_ref = SB.reference_weights(octant)
    dims = (32, 32, 32)
    ws = sfl.make_workspace(sfl.HourglassFB(), "float32", dims)   # order 12, halfband 1, tight
    delta = np.zeros(dims, np.float32)
    delta[0, 0, 0] = 1.0
    s = sfl.hourglass_decompose(ws, sfl.to_device(delta))
    masks = [N.rfft3(sfl.to_host(b).astype(np.float64)) for b in s]
    for M in masks:
        assert np.max(np.abs(M.imag)) <= 1e-6          # real, even masks
    w_mine = tuple(M.real ** 2 for M in masks)
    assert np.max(np.abs(sum(w_mine) - 1.0)) <= 1e-5   # partition of unity, float32
    # ties at 8 float32 ulps of 1 (the weights' rounding noise through the FFTs is ~1e-7)
    SB.assert_hourglass_statistics(SB.hourglass_statistics(w_mine, w_ref, tie_tol=1e-6))


def test_device_ndfb_matches_surfbox_wedge_partition(sfl):
    _, dirs, labels = SB.load()
    dims = (32, 32, 32)
    ws = sfl.make_workspace(sfl.NDFB(levels=2), "float32", dims)  # make_ndfb's defaults
    assert ws.nsubbands == 12
    energies = np.zeros((80, 12))
    for t in range(80):
        c = sfl.ndfb_decompose(ws, sfl.to_device(SB.plane_wave(dirs[:, t]).astype(np.float32)))
        energies[t] = (c.double() ** 2).sum(dim=(0, 1, 2)).cpu().numpy()
    SB.assert_direction_statistics(SB.direction_statistics(energies, labels))
