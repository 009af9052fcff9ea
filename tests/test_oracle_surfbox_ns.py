"""The float64 oracle's hourglass and NDFB banks against SurfBox's golden data
for the nonsubsampled transform (test/items/test_surfbox_reference.jl:17-156):
the 32^3 hourglass octant and the 80-direction wedge partition."""

import numpy as np

import surfbox_ns as SB
from oracle import ns as N


def test_fixture_shapes_and_surfbox_tightness():
    octant, dirs, labels = SB.load()
    assert octant.shape == (17, 17, 17) and dirs.shape == (3, 80) and labels.shape == (80,)
    assert np.unique(labels).size == 12                       # test_surfbox_reference.jl:121-122
    tight_dev, _ = SB.reference_weights(octant)
    assert tight_dev <= 1.0e-5                                 # sum_k V_k^2 == 3 (:34-36)


def test_hourglass_matches_surfbox_partition():
    octant, _, _ = SB.load()
    _, w_ref = SB.reference_weights(octant)
    dims = (32, 32, 32)
    m1, m2 = N.hourglass_tables(dims, 12, 1)
    w_mine = tuple(N.hourglass_weight(m1, m2, i) for i in (1, 2, 3))
    assert all(w.shape == (17, 32, 32) for w in w_mine)
    st = SB.hourglass_statistics(w_mine, w_ref)
    SB.assert_hourglass_statistics(st)
    # a partition of unity; the tight masks (square roots) are Parseval (:76-84)
    assert np.max(np.abs(sum(w_mine) - 1.0)) <= 1.0e-12
    masks = [N.hourglass_mask(m1, m2, i, tight=True) for i in (1, 2, 3)]
    assert np.max(np.abs(sum(m * m for m in masks) - 1.0)) <= 1.0e-12
    # loose masks are the weights, frame-bound ratio 3 (:86-90)
    energy = sum(N.hourglass_mask(m1, m2, i, tight=False) ** 2 for i in (1, 2, 3))
    assert abs(energy.min() - 1.0 / 3.0) <= 1.0e-3
    assert abs(energy.max() - 1.0) <= 1.0e-12


def test_ndfb_matches_surfbox_wedge_partition():
    _, dirs, labels = SB.load()
    dims = (32, 32, 32)
    masks = N.ndfb_masks(dims, 2)          # levels 2, order 12, tight: make_ndfb's defaults
    assert len(masks) == 12
    energies = np.zeros((80, 12))
    for t in range(80):
        X = N.rfft3(SB.plane_wave(dirs[:, t]))
        energies[t] = [float(np.sum(N.irfft3(X * M, dims) ** 2)) for M in masks]
    SB.assert_direction_statistics(SB.direction_statistics(energies, labels))
