"""SurfBox golden data: the deterministic test volume, the fingerprint, and
the loader of the re-encoded fixture.

Test infrastructure (see the package docstring).  Follows
test/items/test_irc.jl:7-66 and test/reference/gen_surfbox_irc.m:8-24.
"""

import json
import os

import numpy as np


def testvol(n):
    """Exact broadband test volume.  test/items/test_irc.jl:39-44"""
    i, j, k = np.meshgrid(np.arange(1, n + 1), np.arange(1, n + 1), np.arange(1, n + 1), indexing="ij")
    q = 73 * i ** 2 + 179 * j ** 2 + 283 * k ** 2 + 31 * i * j + 47 * j * k + 61 * k * i
    return np.mod(q, 1031) / 1031 - 0.5


def fingerprint(A):
    """[sum A W1, sum A W2, sum |A|^2] (complex: re/im of the sums + energy).

    test/items/test_irc.jl:46-56
    """
    A = np.asarray(A)
    n1, n2, n3 = A.shape
    i, j, k = np.meshgrid(np.arange(1, n1 + 1), np.arange(1, n2 + 1), np.arange(1, n3 + 1), indexing="ij")
    W1 = np.cos(0.37 * i + 0.91 * j + 1.53 * k)
    W2 = np.sin(1.11 * i - 0.29 * j + 0.77 * k)
    s1 = np.sum(A * W1)
    s2 = np.sum(A * W2)
    e = float(np.sum(np.abs(A) ** 2))
    if np.iscomplexobj(A):
        return [s1.real, s1.imag, s2.real, s2.imag, e]
    return [float(s1), float(s2), e]


def fp_match(A, ref, rtol=1.0e-11):
    """Every entry agrees to rtol of the array's norm.  test/items/test_irc.jl:59-65"""
    if tuple(np.shape(A)) != tuple(ref["size"]):
        return False
    f = fingerprint(A)
    fp = ref["fp"]
    scale = np.sqrt(fp[-1])
    ok = all(abs(a - b) <= rtol * scale for a, b in zip(f[:-1], fp[:-1]))
    return ok and abs(f[-1] - fp[-1]) <= rtol * fp[-1]


def fp_error(A, ref):
    """Largest fingerprint deviation relative to the array norm (energy: relative)."""
    f = fingerprint(A)
    fp = ref["fp"]
    scale = np.sqrt(fp[-1])
    return max(max(abs(a - b) / scale for a, b in zip(f[:-1], fp[:-1])), abs(f[-1] - fp[-1]) / fp[-1])


def load(path=None):
    """The SurfBox records: name -> {"kind", "size", "fp" | "data"}."""
    if path is None:
        path = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))),
                            "tests", "golden", "surfbox_irc.json")
    with open(path) as f:
        recs = json.load(f)
    for r in recs.values():
        if r["kind"] == "full":
            r["data"] = np.asarray(r["data"], dtype=np.float64).reshape(r["size"], order="F")
    return recs
