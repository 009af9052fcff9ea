"""Filter design in float64: Bernstein mapping kernels, the halfband split
polynomial, soft steps, raised-cosine profiles and the checkerboard ladder.

Test infrastructure (see the package docstring).  Each function follows the
reference file:line given in its docstring.
"""

from fractions import Fraction
from math import comb, ceil, floor

import numpy as np


def dft_frequencies(n, half=False):
    """omega_k = 2*pi*(k-1)/n, k = 1..m (m = n//2+1 when half).

    src/filters/bernstein.jl:64-67
    """
    m = n // 2 + 1 if half else n
    k = np.arange(m, dtype=np.float64)
    return 2 * np.pi * k / n


def folded_frequencies(n, half=False):
    """DFT angular frequencies folded to (-pi, pi]; half = the rfft half.

    src/filters/bernstein.jl:72-79
    """
    if half:
        return dft_frequencies(n, half=True)
    w = 2 * np.pi * np.arange(n, dtype=np.float64) / n
    return np.where(w > np.pi, w - 2 * np.pi, w)


def bernstein_table(N, omega):
    """(N+1) x len(omega) table binom(N,j) x^j (1-x)^(N-j), x = sin(w/2)^2.

    src/filters/bernstein.jl:36-53
    """
    N = int(N)
    if N < 1:
        raise ValueError("Bernstein order must be ≥ 1")
    omega = np.asarray(omega, dtype=np.float64)
    x = np.clip(np.sin(omega / 2) ** 2, 0.0, 1.0)
    y = 1.0 - x
    tbl = np.empty((N + 1, omega.size))
    for j in range(N + 1):
        tbl[j] = float(comb(N, j)) * x ** j * y ** (N - j)
    return tbl


def mapping_coefficients(N, d, group):
    """Sign tensor of the passband max_{group}|w| >= max_{rest}|w| at j/N.

    src/filters/bernstein.jl:97-108
    """
    G = len(group)
    if not (1 <= G < d):
        raise ValueError("group must be a proper non-empty subset of 1:d")
    if not all(1 <= g <= d for g in group):
        raise ValueError("group indices out of range")
    idx = np.indices((N + 1,) * d)
    a = np.max(np.stack([idx[g - 1] for g in group]), axis=0)
    rest = [t for t in range(1, d + 1) if t not in group]
    b = np.max(np.stack([idx[t - 1] for t in rest]), axis=0)
    return np.sign(a - b).astype(np.int64)


def mapping_response(coeffs, tables):
    """M(w) = sum_j c_j prod_i table_i[j_i, k_i], by axis contractions.

    src/filters/bernstein.jl:123-151
    """
    c = np.asarray(coeffs, dtype=np.float64)
    if c.ndim == 1:
        return tables[0].T @ c
    if c.ndim == 2:
        b1, b2 = tables
        return b1.T @ (c @ b2)
    b1, b2, b3 = tables
    t = np.tensordot(c, b1, axes=([0], [0]))      # (j2, j3, k1)
    t = np.tensordot(t, b2, axes=([0], [0]))      # (j3, k1, k2)
    t = np.tensordot(t, b3, axes=([0], [0]))      # (k1, k2, k3)
    return t


def halfband_split(x, m):
    """f0(x) = ((1+x)/2)^(m+1) sum_k binom(m+k,k) ((1-x)/2)^k, sum first.

    src/filters/bernstein.jl:171-190 (the sum is formed first and scaled last;
    binom(m+k,k) by the recurrence c_{k+1} = c_k (m+k+1)/(k+1)).
    """
    m = int(m)
    if m < 0:
        raise ValueError("polynomial order must be ≥ 0")
    x = np.asarray(x, dtype=np.float64)
    u = (1.0 + x) / 2
    v = (1.0 - x) / 2
    s = np.zeros_like(x)
    c = 1.0
    for k in range(m + 1):
        s = s + c * v ** k
        c = c * (m + k + 1) / (k + 1)
    out = u ** (m + 1) * s
    return np.where(u == 0, 0.0, out)


def step(u, poly):
    """Soft step 0 -> 1 across [-1, 1]: halfband_split of the clamped argument.

    src/filters/bernstein.jl:196
    """
    return halfband_split(np.clip(u, -1.0, 1.0), poly)


def soft_step(s, b, w, poly):
    """The step placed at b with half-width w; w <= 0 is a hard step.

    src/filters/bernstein.jl:200-203
    """
    s = np.asarray(s, dtype=np.float64)
    if w <= 0:
        return np.where(s >= b, 1.0, 0.0)
    return step((s - b) / w, poly)


# ── Raised-cosine pyramid profiles ──────────────────────────────────────────


def rcos(x):
    """0 below 0, 1 above 1, (1 - cos(pi x))/2 between.

    src/pyramid/fourier_pyramid.jl:155 (numbered as in the file)
    """
    x = np.asarray(x, dtype=np.float64)
    mid = (1 - np.cos(np.pi * np.clip(x, 0.0, 1.0))) / 2
    return np.where(x <= 0, 0.0, np.where(x >= 1, 1.0, mid))


def rcos_edges(n, w, t):
    """(P, Q) = (ceil(n/2 (w+t)), floor(n/2 (w-t))) with exact rationals.

    src/pyramid/fourier_pyramid.jl:160
    """
    w = Fraction(w)
    t = Fraction(t)
    return ceil(Fraction(n, 2) * (w + t)), floor(Fraction(n, 2) * (w - t))


def rcos_axis(n, w, t):
    """The sqrt-rcos lowpass on a full n-point DFT axis, and its edge P.

    src/pyramid/fourier_pyramid.jl:163-174
    """
    P, Q = rcos_edges(n, w, t)
    k = np.arange(n)
    f = np.abs(np.where(k <= n // 2, k, k - n)).astype(np.float64)
    with np.errstate(invalid="ignore", divide="ignore"):
        prof = np.sqrt(rcos((P - f) / float(P - Q)))
    return np.where(f <= P, prof, 0.0), P


# ── Checkerboard ladder filters (SurfBox's cbd filters) ─────────────────────

# The 1-D odd ladder taps t_q (q = 1, 3, ..., bo-1) that define SurfBox's
# checkerboard filters of order bo.  These numbers are a table that must be
# identical to SurfBox's for coefficient parity (src/filters/checkerboard.jl:26-53);
# the decimated golden fingerprints pin them for bo = 4, 8, 12.
CBD_LADDER = {
    4: [-0.6262169131293146, -0.2391935764853579],
    6: [-0.6263429050738657, -0.18302382681237633, -0.10753046674888095],
    8: [-0.627819441355453, -0.1868110527281001, -0.08821345831338342, -0.05299463507171143],
    10: [-0.6290391996524649, -0.19023436487159193, -0.09316419099049718,
         -0.04787638089257991, -0.02729049477362672],
    12: [-0.6299909650161403, -0.19294788893803155, -0.09719811683520764,
         -0.05257765509290852, -0.027224347419537415, -0.014421093056370137],
    14: [-0.6307470366053054, -0.19509552613399547, -0.10042251574577052,
         -0.056418179282558024, -0.03113763249657735, -0.015819995468636647,
         -0.007750295209451851],
    16: [-0.631356163548133, -0.19683521105934682, -0.10304471724680653,
         -0.05956342644490844, -0.03441276144847804, -0.018849533868796398,
         -0.009297418074817033, -0.004215553479603451],
    18: [-0.6318535467876545, -0.19826135647461407, -0.10520738123671233,
         -0.06218709792109189, -0.037184557113685186, -0.021472356755448885,
         -0.011535270028700011, -0.00549634585408209, -0.0023119823375261405],
}


def checkerboard_orders():
    """src/filters/checkerboard.jl:61"""
    return sorted(CBD_LADDER)


def cbd_ladder(bo):
    """src/filters/checkerboard.jl:63-68"""
    if bo not in CBD_LADDER:
        raise ValueError(f"checkerboard_order must be one of {checkerboard_orders()}, got {bo}")
    return CBD_LADDER[bo]


def cbd_b(t, w):
    """b(w) = 2 sum_i t_i sin((2i-1) w).  src/filters/checkerboard.jl:71-77"""
    w = np.asarray(w, dtype=np.float64)
    s = np.zeros_like(w)
    for i, ti in enumerate(t, start=1):
        s = s + ti * np.sin((2 * i - 1) * w)
    return 2 * s


def cbd_analysis(t, chan, w1, w2):
    """H0 = (1+B)/sqrt2, H1 = e^{j w2}(2-B-B^2)/sqrt2, B = -b(w1) b(w2).

    src/filters/checkerboard.jl:80-84
    """
    B = -cbd_b(t, w1) * cbd_b(t, w2)
    r = 1 / np.sqrt(2.0)
    if chan == 0:
        return (r * (1 + B)).astype(np.complex128)
    return np.exp(1j * np.asarray(w2)) * (r * (2 - B - B ** 2))


def cbd_synthesis(t, chan, w1, w2):
    """G0 = (2+B-B^2)/sqrt2, G1 = e^{-j w2}(1-B)/sqrt2.

    src/filters/checkerboard.jl:87-91
    """
    B = -cbd_b(t, w1) * cbd_b(t, w2)
    r = 1 / np.sqrt(2.0)
    if chan == 0:
        return (r * (2 + B - B ** 2)).astype(np.complex128)
    return np.exp(-1j * np.asarray(w2)) * (r * (1 - B))
