"""Nonsubsampled surfacelet transform (NSSurfacelet) in float64.

Test infrastructure (see the package docstring).  Restates
src/transforms/ns_surfacelet.jl, src/directional/hourglass.jl,
src/directional/ndfb_wedges.jl and the nonsubsampled pyramid of
src/pyramid/fourier_pyramid.jl, plus the MaskBankEngine semantics described at
src/transforms/ns_surfacelet.jl:10-32 (group product once per group, one
inverse FFT per subband; synthesis is one forward FFT per subband, a
per-group sum and one inverse FFT; streaming order = directional subbands
ascending, then the lowpass).
"""

from dataclasses import dataclass, field
from fractions import Fraction

import numpy as np

from . import filters as F


# ── Parameters ──────────────────────────────────────────────────────────────


def parabolic_levels(scales):
    """src/types/transforms.jl:147"""
    return [1 + (j - 1) // 2 for j in range(1, scales + 1)]


@dataclass(frozen=True)
class NSParams:
    """NSSurfacelet parameters (src/types/transforms.jl:86-113)."""
    scales: int
    direction_levels: tuple
    bernstein_order: int = 12
    halfband_order: int = 1
    transition: float = 1.0
    tight: bool = True

    @staticmethod
    def make(scales=None, direction_levels=None, **kw):
        if direction_levels is None:
            if scales is None:
                raise ValueError("give `scales`, `direction_levels` or both")
            direction_levels = parabolic_levels(scales)
        if scales is None:
            scales = len(direction_levels)
        return NSParams(int(scales), tuple(int(v) for v in direction_levels), **kw)


def nbands(p, j):
    """Directional subbands of scale j (1 = coarsest).  src/types/transforms.jl:157"""
    return 3 * (1 << p.direction_levels[j - 1])


def nsubbands(p):
    """src/transforms/ns_surfacelet.jl:527"""
    return 1 + sum(nbands(p, j) for j in range(1, p.scales + 1))


def subband_layout(p):
    """[(scale, direction)], the lowpass (0, 0) first.  ns_surfacelet.jl:518-525"""
    out = [(0, 0)]
    for j in range(1, p.scales + 1):
        out += [(j, k) for k in range(1, nbands(p, j) + 1)]
    return out


# ── Tables ──────────────────────────────────────────────────────────────────


def hourglass_tables(dims, order, poly):
    """m1 = f0(M1) on the rfft grid (h1, n2, n3); m2 = f0(M2) on (n2, n3).

    src/directional/hourglass.jl:172-189
    """
    n1, n2, n3 = dims
    b1 = F.bernstein_table(order, F.dft_frequencies(n1, half=True))
    b2 = F.bernstein_table(order, F.dft_frequencies(n2))
    b3 = F.bernstein_table(order, F.dft_frequencies(n3))
    m1 = F.halfband_split(F.mapping_response(F.mapping_coefficients(order, 3, (1,)), (b1, b2, b3)), poly)
    m2 = F.halfband_split(F.mapping_response(F.mapping_coefficients(order, 2, (1,)), (b2, b3)), poly)
    return m1, m2


def stage1_weight(f0, i):
    """src/directional/hourglass.jl:296"""
    return f0 if i == 1 else 1.0 - f0


def stage2_weight(f0, i):
    """src/directional/hourglass.jl:300-303"""
    if i == 1:
        return np.ones_like(f0)
    return f0 if i == 2 else 1.0 - f0


def tight_sqrt(x):
    """src/directional/hourglass.jl:289"""
    return np.sqrt(np.maximum(x, 0.0))


def hourglass_weight(m1, m2, i):
    """W_i on the rfft grid.  src/directional/hourglass.jl:279-285"""
    return stage1_weight(m1, i) * stage2_weight(m2[None, :, :], i)


def hg_factor(m1, m2, i, tight):
    """sqrt(W) when tight, W otherwise.  src/transforms/ns_surfacelet.jl:265-268"""
    w = stage1_weight(m1, i) * stage2_weight(m2[None, :, :], i)
    return tight_sqrt(w) if tight else w


def transverse_axes(i):
    """src/directional/ndfb_wedges.jl:14"""
    return (2, 3) if i == 1 else ((1, 3) if i == 2 else (1, 2))


def wedge_levels(L):
    """(ceil(L/2), floor(L/2)).  src/directional/ndfb_wedges.jl:19"""
    return (-(-L // 2), L // 2)


def wedge_weight(s, idx, nw, transition, poly):
    """src/directional/ndfb_wedges.jl:25-32"""
    if nw == 1:
        return np.ones_like(s)
    delta = 2.0 / nw
    width = transition * delta
    lo = 1.0 if idx == 1 else F.soft_step(s, -1.0 + (idx - 1) * delta, width, poly)
    hi = 0.0 if idx == nw else F.soft_step(s, -1.0 + idx * delta, width, poly)
    return lo - hi


def self_conjugate_bin(k0, n):
    """Bin k0 (0-based) is its own negative.  src/directional/ndfb_wedges.jl:78"""
    return (2 * k0) % n == 0


def wedge_ratio(wr, wt, ref_self, tr_self):
    """Canonical signed slope w_tr / w_ref.  src/directional/ndfb_wedges.jl:97-106"""
    with np.errstate(divide="ignore", invalid="ignore"):
        r = np.where(ref_self, np.abs(wt) / np.abs(wr),
                     np.where(tr_self, wt / np.abs(wr), wt / wr))
    return np.where(wr == 0, 0.0, r)


def wedge_masks_plane(dims, ref, tr, l, poly, transition):
    """The 2^l wedge planes of one transverse axis, each indexed (ref, tr).

    src/directional/ndfb_wedges.jl:45-69 (returned as 2-D planes; the
    reference orients them into 3-D arrays with a singleton third axis)
    """
    nref, ntr = dims[ref - 1], dims[tr - 1]
    wref = F.folded_frequencies(nref, half=(ref == 1))
    wtr = F.folded_frequencies(ntr, half=(tr == 1))
    nw = 1 << l
    if l == 0:
        return [np.ones((wref.size, wtr.size))]
    pr = np.arange(wref.size)
    qt = np.arange(wtr.size)
    ref_self = np.array([self_conjugate_bin(p, nref) for p in pr])[:, None]
    tr_self = np.array([self_conjugate_bin(q, ntr) for q in qt])[None, :]
    WR = np.broadcast_to(wref[:, None], (wref.size, wtr.size))
    WT = np.broadcast_to(wtr[None, :], (wref.size, wtr.size))
    s = wedge_ratio(WR, WT, np.broadcast_to(ref_self, WR.shape), np.broadcast_to(tr_self, WR.shape))
    return [wedge_weight(s, k, nw, transition, poly) for k in range(1, nw + 1)]


def orient_plane(P, ref, tr, grid_shape):
    """Lay a (ref, tr) plane out as a 3-D array broadcastable on grid_shape.

    src/directional/ndfb_wedges.jl:112-113
    """
    shape = [1, 1, 1]
    shape[ref - 1] = grid_shape[ref - 1]
    shape[tr - 1] = grid_shape[tr - 1]
    M = P if ref < tr else P.T
    return M.reshape(shape)


def ns_wedge_factors(dims, L, poly, transition, tight):
    """Per hourglass i: (planes_a, planes_b), square-rooted when tight.

    src/transforms/ns_surfacelet.jl:178-185
    """
    la, lb = wedge_levels(L)
    out = []
    for i in (1, 2, 3):
        a, b = transverse_axes(i)
        pa = wedge_masks_plane(dims, i, a, la, poly, transition)
        pb = wedge_masks_plane(dims, i, b, lb, poly, transition)
        if tight:
            pa = [tight_sqrt(w) for w in pa]
            pb = [tight_sqrt(w) for w in pb]
        out.append((pa, pb))
    return out


def rc_responses(J, n, nbins):
    """Per-axis pyramid factors on the first nbins bins of an n-point axis:
    acc[j] = prod_{i<j} l_i (j = 0..J) and prof[j] = l_{j+1} (j = 0..J-1),
    with l_j the sqrt-rcos lowpass of cutoff 1/2^j and transition 1/(3 2^j).

    src/pyramid/fourier_pyramid.jl:256-263 (file numbering)
    """
    prof = [F.rcos_axis(n, Fraction(1, 2 ** j), Fraction(1, 3 * 2 ** j))[0][:nbins] for j in range(1, J + 1)]
    acc = [np.ones(nbins)]
    for j in range(J):
        acc.append(acc[-1] * prof[j])
    return acc, prof


class ArgumentError(ValueError):
    pass


def fmt_dims(dims):
    return "(" + ", ".join(str(d) for d in dims) + ")"


@dataclass
class NSTables:
    dims: tuple
    p: NSParams
    m1: np.ndarray
    m2: np.ndarray
    wedges: list          # [scale j-1][hourglass i-1] = (planes_a, planes_b)
    pa: list              # [level 0..J] of 3 per-axis vectors
    pl: list              # [level 0..J-1] of 3 per-axis vectors
    band: list = field(default_factory=list)   # [level] B_j on the rfft grid


def make_tables(p, dims):
    """Workspace tables.  src/transforms/ns_surfacelet.jl:98-123"""
    if len(dims) != 3:
        raise ArgumentError(f"the surfacelet transforms take volumes (three axes), got size {fmt_dims(dims)}")
    if not all(d >= 1 for d in dims):
        raise ArgumentError(f"volume size must be positive, got {fmt_dims(dims)}")
    n1, n2, n3 = dims
    m1, m2 = hourglass_tables(dims, p.bernstein_order, p.halfband_order)
    wedges = [ns_wedge_factors(dims, L, p.halfband_order, float(p.transition), p.tight) for L in p.direction_levels]
    nb = (n1 // 2 + 1, n2, n3)
    resp = [rc_responses(p.scales, dims[d], nb[d]) for d in range(3)]
    J = p.scales
    for j in range(J):
        empty = all(np.all((resp[d][0][j] == 0) | (resp[d][1][j] == 1)) for d in range(3))
        if empty:
            raise ArgumentError(
                f"size {fmt_dims(dims)} is too small for {J} scales: scale {J - j} would be empty")
    pa = [tuple(resp[d][0][j] for d in range(3)) for j in range(J + 1)]
    pl = [tuple(resp[d][1][j] for d in range(3)) for j in range(J)]
    band = [bandpass_grid(pa[j], pl[j]) for j in range(J)]
    return NSTables(tuple(dims), p, m1, m2, wedges, pa, pl, band)


def bandpass_grid(a, l):
    """B_j = a1 a2 a3 sqrt(max(1 - (l1 l2 l3)^2, 0)) on the rfft grid.

    src/transforms/ns_surfacelet.jl:271-272
    """
    a1, a2, a3 = a[0][:, None, None], a[1][None, :, None], a[2][None, None, :]
    l1, l2, l3 = l[0][:, None, None], l[1][None, :, None], l[2][None, None, :]
    return a1 * a2 * a3 * np.sqrt(np.maximum(1 - (l1 * l2 * l3) ** 2, 0.0))


def lowpass_grid(T):
    """pa_{J+1} = a1 a2 a3.  src/transforms/ns_surfacelet.jl:350-371"""
    a = T.pa[-1]
    return a[0][:, None, None] * a[1][None, :, None] * a[2][None, None, :]


def subband_index(p, j, i, a, b, na, nb):
    """1-based subband index of wedge (a, b) of hourglass i at scale j.

    src/transforms/ns_surfacelet.jl:222-242 (offsets) and :430 (_ns_index)
    """
    off = 1 + sum(nbands(p, jj) for jj in range(1, j))
    return off + ((i - 1) * na + (a - 1)) * nb + b


def group_items(T):
    """Yields (j, i, level_index, [(subband, plane_a, plane_b), ...]) in item order."""
    p = T.p
    J = p.scales
    for j in range(1, J + 1):
        lv = J - j   # 0-based pyramid level (0 = finest)
        for i in (1, 2, 3):
            pa_list, pb_list = T.wedges[j - 1][i - 1]
            na, nb = len(pa_list), len(pb_list)
            a_ax, b_ax = transverse_axes(i)
            items = []
            for a in range(1, na + 1):
                for b in range(1, nb + 1):
                    items.append((subband_index(p, j, i, a, b, na, nb),
                                  orient_plane(pa_list[a - 1], i, a_ax, (T.dims[0] // 2 + 1,) + T.dims[1:]),
                                  orient_plane(pb_list[b - 1], i, b_ax, (T.dims[0] // 2 + 1,) + T.dims[1:])))
            yield j, i, lv, items


# Threads of the float64 FFTs (scipy.fft's pocketfft) for the large checks;
# 1 keeps NumPy's FFT.
_FFT_WORKERS = 1


def set_fft_workers(n):
    """Run the oracle's float64 FFTs on n host threads (large volumes)."""
    global _FFT_WORKERS
    _FFT_WORKERS = max(1, int(n))


def rfft3(x):
    """Unnormalized rfft halving axis 0 (Julia's first axis)."""
    if _FFT_WORKERS > 1:
        import scipy.fft as sfft
        return sfft.rfftn(x, axes=(1, 2, 0), workers=_FFT_WORKERS)
    return np.fft.rfftn(x, axes=(1, 2, 0))


def irfft3(X, dims):
    """Normalized irfft restoring axis 0 of length dims[0]."""
    if _FFT_WORKERS > 1:
        import scipy.fft as sfft
        return sfft.irfftn(X, s=(dims[1], dims[2], dims[0]), axes=(1, 2, 0), workers=_FFT_WORKERS)
    return np.fft.irfftn(X, s=(dims[1], dims[2], dims[0]), axes=(1, 2, 0))


def subband_masks(T, analysis=True):
    """Yields (subband index, full mask on the rfft grid) in item order, the
    lowpass (index 1) last.  The analysis mask of a directional subband is
    B_j hg_i wa wb; the synthesis mask is the same when tight and B_j alone
    otherwise (src/transforms/ns_surfacelet.jl:226-227, 237-238)."""
    p = T.p
    for j, i, lv, items in group_items(T):
        if analysis or p.tight:
            G = T.band[lv] * hg_factor(T.m1, T.m2, i, p.tight)
        else:
            G = T.band[lv]
        for s, wa, wb in items:
            if analysis or p.tight:
                yield s, G * wa * wb
            else:
                yield s, G
    yield 1, lowpass_grid(T)


def analyze_stream(T, x):
    """Streaming analysis of a real volume: yields (subband index, band) with
    the directional subbands in increasing index, then the lowpass.

    src/transforms/ns_surfacelet.jl:474-479, 584-624
    """
    X = rfft3(np.asarray(x, dtype=np.float64))
    p = T.p
    for j, i, lv, items in group_items(T):
        Y = X * (T.band[lv] * hg_factor(T.m1, T.m2, i, p.tight))
        for s, wa, wb in items:
            yield s, irfft3(Y * wa * wb, T.dims)
    yield 1, irfft3(X * lowpass_grid(T), T.dims)


def analyze(T, x):
    """Coefficients (n1, n2, n3, S) of a real or complex volume.

    src/transforms/ns_surfacelet.jl:551-566; complex = two real channels (:208)
    """
    x = np.asarray(x)
    S = nsubbands(T.p)
    if np.iscomplexobj(x):
        return analyze(T, x.real) + 1j * analyze(T, x.imag)
    c = np.empty(T.dims + (S,))
    for s, band in analyze_stream(T, x):
        c[..., s - 1] = band
    return c


def synthesize(T, c):
    """Inverse from the stacked coefficients.  src/transforms/ns_surfacelet.jl:568-581"""
    c = np.asarray(c)
    if np.iscomplexobj(c):
        return synthesize(T, c.real) + 1j * synthesize(T, c.imag)
    return synthesize_stream(T, lambda s: c[..., s - 1])


def synthesize_stream(T, source):
    """Streaming synthesis: source(i) returns subband i, asked in the order
    directional ascending, then the lowpass.  src/transforms/ns_surfacelet.jl:483-500
    """
    p = T.p
    acc = np.zeros((T.dims[0] // 2 + 1,) + T.dims[1:], dtype=np.complex128)
    for j, i, lv, items in group_items(T):
        A = np.zeros_like(acc)
        for s, wa, wb in items:
            Fs = rfft3(np.asarray(source(s), dtype=np.float64))
            A += Fs * wa * wb if p.tight else Fs
        G = T.band[lv] * hg_factor(T.m1, T.m2, i, p.tight) if p.tight else T.band[lv]
        acc += A * G
    acc += rfft3(np.asarray(source(1), dtype=np.float64)) * lowpass_grid(T)
    return irfft3(acc, T.dims)


def adjoint_synthesize(T, x):
    """Adjoint of synthesize: c_s = irfft(X * synthesis mask_s).  For a tight
    transform it equals analyze (src/transforms/ns_surfacelet.jl:21-25)."""
    x = np.asarray(x)
    if np.iscomplexobj(x):
        return adjoint_synthesize(T, x.real) + 1j * adjoint_synthesize(T, x.imag)
    X = rfft3(x.astype(np.float64))
    c = np.empty(T.dims + (nsubbands(T.p),))
    for s, M in subband_masks(T, analysis=False):
        c[..., s - 1] = irfft3(X * M, T.dims)
    return c


def adjoint_analyze(T, c):
    """Adjoint of analyze: x = irfft(sum_s rfft(c_s) * analysis mask_s)."""
    c = np.asarray(c)
    if np.iscomplexobj(c):
        return adjoint_analyze(T, c.real) + 1j * adjoint_analyze(T, c.imag)
    acc = np.zeros((T.dims[0] // 2 + 1,) + T.dims[1:], dtype=np.complex128)
    for s, M in subband_masks(T, analysis=True):
        acc += rfft3(c[..., s - 1].astype(np.float64)) * M
    return irfft3(acc, T.dims)


# ── Standalone hourglass bank (src/directional/hourglass.jl) ────────────────


def hourglass_mask(m1, m2, i, tight=True):
    """src/directional/hourglass.jl:264-270, 400-412"""
    w = hourglass_weight(m1, m2, i)
    return tight_sqrt(w) if tight else w


def hourglass_decompose(x, dims, order, poly, tight=True):
    """src/directional/hourglass.jl:343-358"""
    m1, m2 = hourglass_tables(dims, order, poly)
    X = rfft3(np.asarray(x, dtype=np.float64))
    return [irfft3(X * hourglass_mask(m1, m2, i, tight), dims) for i in (1, 2, 3)]


# ── Standalone NDFB (src/directional/ndfb.jl) ───────────────────────────────


def ndfb_masks(dims, levels, order=12, poly=1, tight=True, transition=1.0):
    """All 3*2^levels analysis masks on the rfft grid, in ndfb_subband_index
    order ((i-1) na + (p-1)) nb + q.  src/directional/ndfb.jl:91-104, 184-190,
    and the mask kernel src/directional/hourglass.jl:400-412 with wedge planes.
    """
    m1, m2 = hourglass_tables(dims, order, poly)
    la, lb = wedge_levels(levels)
    grid = (dims[0] // 2 + 1,) + tuple(dims[1:])
    out = []
    for i in (1, 2, 3):
        a, b = transverse_axes(i)
        pa = wedge_masks_plane(dims, i, a, la, poly, transition)
        pb = wedge_masks_plane(dims, i, b, lb, poly, transition)
        W = hourglass_weight(m1, m2, i)
        for wa in pa:
            for wb in pb:
                w = W * orient_plane(wa, i, a, grid) * orient_plane(wb, i, b, grid)
                out.append(tight_sqrt(w) if tight else w)
    return out


def ndfb_decompose(x, dims, levels, **kw):
    """src/directional/ndfb.jl (decompose): irfft(X * mask) per subband."""
    X = rfft3(np.asarray(x, dtype=np.float64))
    return [irfft3(X * M, dims) for M in ndfb_masks(dims, levels, **kw)]
