"""Checks of the nonsubsampled hourglass and NDFB banks against SurfBox's golden
data, as the reference's suite states them
(test/items/test_surfbox_reference.jl:17-156).  Shared by the oracle test
(float64, CPU) and the device test (float32 through the C ABI).

SurfBox (Lu and Do's MATLAB toolbox) builds its hourglasses from a Kaiser-
windowed diamond kernel and normalises them so that sum_k V_k^2 = 3; the
transforms here compose Bernstein mapping polynomials into a partition of
unity, so the comparable quantity is W_k = V_k^2 / 3 and the comparison is of
geometry (which hourglass, which wedge dominates), not of values.
"""

import json
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def load():
    """The re-encoded fixture (tests/golden/make_surfbox_ns_fixture.py)."""
    with open(os.path.join(HERE, "golden", "surfbox_ns.json")) as f:
        g = json.load(f)
    octant = np.asarray(g["hourglass_octant"]["data"], dtype=np.float32).reshape((17, 17, 17), order="F")
    dirs = np.asarray(g["directions"]["data"], dtype=np.float64).reshape((3, 80), order="F")
    return octant, dirs, np.asarray(g["labels"], dtype=np.int64)


def expand_even(octant, n=32):
    """The octant mirrored onto the full n^3 grid (the mask is even along every
    axis).  test/items/test_surfbox_reference.jl:24-29"""
    m = np.array([i if i <= n // 2 else n - i for i in range(n)])
    return octant.astype(np.float64)[np.ix_(m, m, m)]


def reference_weights(octant):
    """(tightness deviation, W_ref per hourglass on the 17 x 32 x 32 rfft grid).
    Masks 2 and 3 are axis permutations of mask 1.
    test/items/test_surfbox_reference.jl:31-40"""
    v1 = expand_even(octant)
    v = (v1, np.transpose(v1, (1, 0, 2)), np.transpose(v1, (2, 1, 0)))
    tight_dev = float(np.max(np.abs(v[0] ** 2 + v[1] ** 2 + v[2] ** 2 - 3.0)))
    return tight_dev, tuple(v[k][:17] ** 2 / 3.0 for k in range(3))


def hourglass_statistics(w_mine, w_ref, tie_tol=0.0):
    """The geometric figures the reference asserts on
    (test/items/test_surfbox_reference.jl:44-74): the cross-distance matrix
    d[k][m] = max |W_k - W_ref_m|, the dominant-hourglass agreement, the
    median and maximum of the reference's top-two gap over the disagreeing
    bins, the mean gap over all bins, and the mean |W - W_ref|.

    The dominant hourglass is the first maximum, as Julia's argmax.  tie_tol
    counts weights within tie_tol of the maximum as tied (first index wins):
    float32 weights carry rounding noise of a few ulps, which would otherwise
    decide the bins where the hourglasses meet with equal weight."""
    d = [[float(np.max(np.abs(w_mine[k] - w_ref[m]))) for m in range(3)] for k in range(3)]
    wm = np.stack([w.ravel() for w in w_mine])
    wr = np.stack([w.ravel() for w in w_ref])
    dom_m = np.argmax(wm >= wm.max(axis=0) - tie_tol, axis=0)
    dom_r = np.argmax(wr, axis=0)
    s = -np.sort(-wr, axis=0)
    gap = s[0] - s[1]
    dis = dom_m != dom_r
    gaps = np.sort(gap[dis])
    n = wm.shape[1]
    return {
        "cross": d,
        "agreement": 1.0 - dis.sum() / n,
        "gap_median": float(gaps[(gaps.size + 1) // 2 - 1]) if gaps.size else 0.0,   # gaps[cld(len, 2)]
        "gap_max": float(gaps[-1]) if gaps.size else 0.0,
        "gap_mean": float(gap.sum() / n),
        "mean_abs": float(sum(np.abs(w_mine[k] - w_ref[k]).sum() for k in range(3)) / (3 * n)),
    }


def assert_hourglass_statistics(st):
    """The reference's bounds (test/items/test_surfbox_reference.jl:49-74)."""
    for k in range(3):
        for m in range(3):
            if k == m:
                assert st["cross"][k][m] < 0.5, (k, m, st["cross"])
            else:
                assert st["cross"][k][m] > 0.9, (k, m, st["cross"])
    assert st["agreement"] > 0.94, st
    assert st["gap_median"] < 1.0e-6, st
    assert st["gap_max"] < 0.48, st
    assert abs(st["gap_mean"] - 0.887) <= 0.001, st
    assert st["mean_abs"] < 0.04, st


def plane_wave(dirvec, n=32):
    """cos(2 pi k.x / n) with k = round(0.6 (n/2) d), [1, 0, 0] when that rounds
    to zero.  test/items/test_surfbox_reference.jl:128-134 (Julia's round is
    half-to-even, as NumPy's rint)"""
    k = np.rint(dirvec * (0.6 * n / 2)).astype(np.int64)
    if not k.any():
        k = np.array([1, 0, 0])
    i, j, l = np.meshgrid(np.arange(n), np.arange(n), np.arange(n), indexing="ij")
    return np.cos(np.pi * 2 * (k[0] * i + k[1] * j + k[2] * l) / n)


def direction_statistics(energies, ref_label):
    """Partition agreement up to relabelling (test/items/test_surfbox_reference.jl:137-155).
    energies: (80, 12); ref_label: 1-based SurfBox subband per direction."""
    nd = energies.shape[0]
    my = np.argmax(energies, axis=1) + 1
    same = ((ref_label[:, None] == ref_label[None, :]) == (my[:, None] == my[None, :])).sum()
    conf = np.zeros((12, 12), dtype=np.int64)
    for t in range(nd):
        conf[my[t] - 1, ref_label[t] - 1] += 1
    relabel = np.argmax(conf, axis=1) + 1
    inverse = np.zeros(13, dtype=np.int64)
    for m in range(1, 13):
        inverse[relabel[m - 1]] = m
    runner_up = []
    for t in range(nd):
        top2 = np.argsort(-energies[t], kind="stable")[:2] + 1
        runner_up.append(bool(inverse[ref_label[t]] in top2))
    return {
        "my_unique": int(np.unique(my).size),
        "same": float(same / nd ** 2),
        "relabel_unique": int(np.unique(relabel).size),
        "relabel_agree": float(np.mean(relabel[my - 1] == ref_label)),
        "runner_up": runner_up,
    }


def assert_direction_statistics(st):
    assert st["my_unique"] == 12, st
    assert st["same"] > 0.93, st
    assert st["relabel_unique"] == 12, st
    assert st["relabel_agree"] > 0.8, st
    assert all(st["runner_up"]), st
