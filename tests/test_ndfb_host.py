"""The standalone directional banks' host side (no GPU): parameter checks with
the reference's messages, subband counts and the index <-> triple map
(src/directional/ndfb.jl:91-104, 150-203)."""

import pytest

from conftest import load_package


def test_parameters_and_index_map():
    sfl = load_package()
    with pytest.raises(sfl.ArgumentError, match="levels must be ≥ 0"):
        sfl.NDFB(levels=-1)
    with pytest.raises(sfl.ArgumentError, match="transition must be ≥ 0"):
        sfl.NDFB(transition=-0.1)
    for L in range(0, 6):
        t = sfl.NDFB(levels=L, bernstein_order=6)
        S = sfl.nsubbands(t, (16, 16, 16))
        assert S == 3 * 2 ** L
        na, nb = t.wedge_counts()
        assert na * nb == 2 ** L and na == 2 ** ((L + 1) // 2)
        for idx in range(1, S + 1):
            assert sfl.ndfb_subband_index(t, *sfl.ndfb_subband_triple(t, idx)) == idx
    t = sfl.NDFB(levels=2, bernstein_order=6)
    assert sfl.ndfb_subband_index(t, 2, 1, 2) == 6          # the reference's doctest
    assert sfl.ndfb_subband_triple(t, 6) == (2, 1, 2)
    with pytest.raises(sfl.ArgumentError, match="hourglass index must be 1, 2 or 3"):
        sfl.ndfb_subband_index(t, 4, 1, 1)
    with pytest.raises(sfl.ArgumentError, match="wedge index p out of range 1:2"):
        sfl.ndfb_subband_index(t, 1, 3, 1)
    with pytest.raises(sfl.ArgumentError, match="subband index out of range"):
        sfl.ndfb_subband_triple(t, 13)
    assert sfl.nsubbands(sfl.HourglassFB(), (8, 8, 8)) == 3
