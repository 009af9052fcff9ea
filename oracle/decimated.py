"""Decimated surfacelet transform (Surfacelet, SurfBox's construction) in
float64.

Test infrastructure (see the package docstring).  Restates
src/pyramid/fourier_pyramid.jl, src/directional/ritf.jl,
src/directional/irc.jl, src/directional/surfacelet_scale.jl,
src/transforms/surfacelet.jl and the parameter rules of
src/types/transforms.jl:222-315.
"""

from dataclasses import dataclass
from fractions import Fraction

import numpy as np

from . import filters as F
from .ns import ArgumentError, fmt_dims, transverse_axes, wedge_levels


class DimensionMismatch(ValueError):
    pass


# ── Parameters ──────────────────────────────────────────────────────────────


def surf_levels(L):
    """levels[K][m] for an integer L or a 3x3 level matrix (diagonal ignored).

    src/types/transforms.jl:270-284
    """
    if isinstance(L, (int, np.integer)):
        la, lb = wedge_levels(int(L))
        out = []
        for K in (1, 2, 3):
            a, b = transverse_axes(K)
            out.append(tuple(la if m == a else (lb if m == b else 0) for m in (1, 2, 3)))
        return tuple(out)
    M = np.asarray(L)
    if M.shape != (3, 3):
        raise ArgumentError(f"a level matrix must be 3 × 3, got size {M.shape}")
    return tuple(tuple(0 if m == K else int(M[K - 1, m - 1]) for m in (1, 2, 3)) for K in (1, 2, 3))


def nsubbands_scale(lv):
    """src/types/transforms.jl:315"""
    return sum(1 << sum(lv[K]) for K in range(3))


def pyramid_mode(mode):
    """(w, tbw, D) of the first and every later level.  src/pyramid/fourier_pyramid.jl:148-153"""
    if mode == 1:
        return (Fraction(1, 2), Fraction(1, 4)), (Fraction(1, 6), Fraction(1, 12)), (Fraction(1), Fraction(2))
    if mode == 1.5:
        return (Fraction(1, 2), Fraction(3, 8)), (Fraction(1, 7), Fraction(1, 9)), (Fraction(3, 2), Fraction(2))
    if mode == 2:
        return (Fraction(1, 3), Fraction(1, 3)), (Fraction(1, 7), Fraction(1, 7)), (Fraction(2), Fraction(2))
    raise ArgumentError(f"pyramid_ratio must be 1, 1.5 or 2, got {mode}")


@dataclass(frozen=True)
class SurfParams:
    """Surfacelet parameters (src/types/transforms.jl:222-261)."""
    scales: int
    levels: tuple            # [scale j-1 (coarse first)][K-1][m-1]
    pyramid_ratio: float = 1.5
    checkerboard_order: int = 12
    diamond_length: int = 15
    kaiser_beta: float = 2.5
    diamond_power: int = 4

    @staticmethod
    def make(scales=None, direction_levels=None, pyramid_ratio=1.5, checkerboard_order=12,
             diamond_length=15, kaiser_beta=2.5, diamond_power=4):
        if direction_levels is None:
            if scales is None:
                raise ArgumentError("give `scales`, `direction_levels` or both")
            direction_levels = [1 + (j - 1) // 2 for j in range(1, scales + 1)]
        if scales is None:
            scales = len(direction_levels)
        lv = tuple(surf_levels(L) for L in direction_levels)
        pyramid_mode(pyramid_ratio)
        F.cbd_ladder(checkerboard_order)
        return SurfParams(int(scales), lv, pyramid_ratio, checkerboard_order, diamond_length,
                          kaiser_beta, diamond_power)


# ── Pyramid ─────────────────────────────────────────────────────────────────


@dataclass
class PyramidLevel:
    n: tuple
    nlow: tuple
    D: Fraction
    idx: tuple        # per axis, 0-based bins of n inside the lowpass support
    idx_low: tuple    # where they land in nlow
    prof: tuple       # per axis, the 1-D profile on idx


def pyramid_level(n, w, tbw, D):
    """src/pyramid/fourier_pyramid.jl:181-198 (file numbering)"""
    if not all((d * D.denominator) % D.numerator == 0 for d in n):
        raise ArgumentError(f"a pyramid level with factor {D.numerator}//{D.denominator} cannot divide size {fmt_dims(n)}")
    nlow = tuple(d * D.denominator // D.numerator for d in n)
    idx, idx_low, prof = [], [], []
    for a in range(3):
        full, P = F.rcos_axis(n[a], w, tbw)
        if not 2 * P <= nlow[a]:
            raise ArgumentError(f"size {n[a]} is too small for the pyramid")
        ia = np.concatenate([np.arange(0, P + 1), np.arange(n[a] - P, n[a])])
        il = np.concatenate([np.arange(0, P + 1), np.arange(nlow[a] - P, nlow[a])])
        idx.append(ia)
        idx_low.append(il)
        prof.append(full[ia])
    return PyramidLevel(tuple(n), nlow, D, tuple(idx), tuple(idx_low), tuple(prof))


def fourier_pyramid(dims, J, mode):
    """src/pyramid/fourier_pyramid.jl:205-216 (file numbering)"""
    ws, tbws, Ds = pyramid_mode(mode)
    levels = []
    n = tuple(dims)
    for j in range(1, J + 1):
        k = 0 if j == 1 else 1
        lv = pyramid_level(n, ws[k], tbws[k], Ds[k])
        levels.append(lv)
        n = lv.nlow
    return levels


def _lowpass_box(lv):
    l1, l2, l3 = lv.prof
    return l1[:, None, None] * l2[None, :, None] * l3[None, None, :]


def pyramid_split(X, lv):
    """Returns the lowpass (size nlow); X becomes the highpass in place.

    src/pyramid/fourier_pyramid.jl:221-231 (file numbering)
    """
    L = _lowpass_box(lv)
    ix = np.ix_(*lv.idx)
    box = X[ix]
    low = np.zeros(lv.nlow, dtype=np.complex128)
    low[np.ix_(*lv.idx_low)] = (L * (1.0 / float(lv.D) ** 1.5)) * box
    X[ix] = box * np.sqrt(1 - L ** 2)
    return low


def pyramid_merge(X, low, lv):
    """X holds the highpass on entry and the merged spectrum on exit.

    src/pyramid/fourier_pyramid.jl:235-240 (file numbering)
    """
    L = _lowpass_box(lv)
    ix = np.ix_(*lv.idx)
    X[ix] = np.sqrt(1 - L ** 2) * X[ix] + (L * float(lv.D) ** 1.5) * low[np.ix_(*lv.idx_low)]
    return X


# ── ritf hourglass masks ────────────────────────────────────────────────────


def ritf_I0(x):
    """Modified Bessel I0 by SurfBox's truncated series.  src/directional/ritf.jl:24-37"""
    x = x / 2
    y = 1.0
    z = 1.0
    t = 1.0
    k = 1
    while t > 1.0e-10 * y:
        z = z * x / k
        k += 1
        t = z * z
        y += t
    return y


def ritf_window(n, beta):
    """Kaiser window times the half-band sinc.  src/directional/ritf.jl:40-52"""
    if n % 2 == 0:
        raise ArgumentError("msize must be odd")
    den = ritf_I0(float(beta))
    half = (n - 1) // 2
    val = [2.0 * i / (n - 1) - 1 for i in range(half + 1)]
    wh = [ritf_I0(beta * np.sqrt(1 - v * v)) / den for v in val]
    w = np.array(wh + wh[:-1][::-1])
    u = np.arange(-half, half + 1)
    return w * np.sinc(u / 2.0)


def ritf_diamond(w, a, b):
    """D(a, b) = Ce(al) Ce(be) + Co(al) Co(be).  src/directional/ritf.jl:58-73"""
    half = (len(w) - 1) // 2
    al = (a + b) / 2
    be = (a - b) / 2
    ce_a = ce_b = co_a = co_b = 0.0
    for i, u in enumerate(range(-half, half + 1)):
        if u % 2 == 0:
            ce_a = ce_a + w[i] * np.cos(u * al)
            ce_b = ce_b + w[i] * np.cos(u * be)
        else:
            co_a = co_a + w[i] * np.cos(u * al)
            co_b = co_b + w[i] * np.cos(u * be)
    return ce_a * ce_b + co_a * co_b


def ritf_plane(w, nK, nm, lam):
    """D(w_K + pi, w_m)^lambda on the nK x nm DFT grid.  src/directional/ritf.jl:76-84"""
    a = (2 * np.pi) * np.arange(nK) / nK + np.pi
    b = (2 * np.pi) * np.arange(nm) / nm
    return ritf_diamond(w, a[:, None], b[None, :]) ** lam


def ritf_masks(dims, msize=15, beta=2.5, lam=4):
    """V_K = sqrt(3 hg_K / sum hg) on the half-spectrum of axis K.

    src/directional/ritf.jl:89-108
    """
    if not (lam % 2 == 0 and lam > 0):
        raise ArgumentError("lambda must be a positive even integer")
    if not all(d % 2 == 0 for d in dims):
        raise ArgumentError(f"the hourglass stage needs even dimensions, got {fmt_dims(dims)}")
    w = ritf_window(msize, beta)
    hg = []
    for K in (1, 2, 3):
        acc = np.ones(dims)
        for m in (1, 2, 3):
            if m == K:
                continue
            P = ritf_plane(w, dims[K - 1], dims[m - 1], lam)
            shape = [1, 1, 1]
            shape[K - 1] = dims[K - 1]
            shape[m - 1] = dims[m - 1]
            acc = acc * (P if K < m else P.T).reshape(shape)
        hg.append(acc)
    total = hg[0] + hg[1] + hg[2]
    out = []
    for K in (1, 2, 3):
        sl = tuple(slice(0, dims[d] // 2 + 1) if d == K - 1 else slice(None) for d in range(3))
        out.append(np.sqrt(3 * hg[K - 1][sl] / total[sl]))
    return out


# ── IRC checkerboard stages ─────────────────────────────────────────────────


def half_dims(n, K):
    """src/directional/surfacelet_scale.jl:28"""
    return tuple(n[d] // 2 + 1 if d == K - 1 else n[d] for d in range(3))


def irc_slice(f, t, chan, hdims, nK, K, m, le, scale):
    """Filter slice of channel `chan` at stage `le` on axis m, as a (K, m)
    plane oriented to broadcast on the half-spectrum.

    src/directional/irc.jl:49-67
    """
    nKh = hdims[K - 1]
    nm = hdims[m - 1]
    W = nm >> (le - 1)
    c = np.arange(nm)
    g, l = np.divmod(c, W)
    sf = (1 << (le - 1)) - 1 - 2 * g
    wK = (2 * np.pi) * np.arange(nKh) / nK
    wm = (2 * np.pi) * l[None, :] / W + sf[None, :] * wK[:, None]
    S = scale * f(t, chan, np.broadcast_to(wK[:, None], wm.shape), wm)
    shape = [1, 1, 1]
    shape[K - 1] = nKh
    shape[m - 1] = nm
    return (S if K < m else S.T).reshape(shape)


@dataclass
class IRCStage:
    m: int
    b: int
    ana: tuple
    syn: tuple


def irc_stages(hdims, nK, K, levels, bo):
    """Analysis-order stages: axes m != K ascending, levels[m] stages each.

    src/directional/irc.jl:275-290 (file numbering)
    """
    t = F.cbd_ladder(bo)
    stages = []
    for m in (1, 2, 3):
        if m == K:
            continue
        lv = levels[m - 1]
        if lv < 0:
            raise ArgumentError("directional levels must be ≥ 0")
        if hdims[m - 1] % (1 << lv) != 0:
            raise ArgumentError(f"axis {m} of length {hdims[m - 1]} cannot be split {lv} times")
        for le in range(1, lv + 1):
            ana = tuple(irc_slice(F.cbd_analysis, t, c, hdims, nK, K, m, le, 0.5) for c in (0, 1))
            syn = tuple(irc_slice(F.cbd_synthesis, t, c, hdims, nK, K, m, le, 1.0) for c in (0, 1))
            stages.append(IRCStage(m, hdims[m - 1] >> le, ana, syn))
    return stages


def irc_halves(X, m, b):
    """Views (A, B) of the two halves of every 2b-bin group along axis m.

    src/directional/irc.jl:238-244, 295-299 (file numbering)
    """
    n = X.shape[m - 1]
    # column-major split (b fastest, then the pair, then the group) expressed
    # with index arrays, so that the halves keep axis m
    c = np.arange(n)
    r = c % (2 * b)
    A_idx = c[r < b]
    B_idx = c[r >= b]
    return A_idx, B_idx


def _take(X, ax, idx):
    return np.take(X, idx, axis=ax)


def _put(X, ax, idx, V):
    sl = [slice(None)] * X.ndim
    sl[ax] = idx
    X[tuple(sl)] = V


def irc_stage(S, m, b, W11, W12, W21, W22):
    """A <- W11 A + W12 B, B <- W21 A + W22 B.  src/directional/irc.jl:304-311"""
    ax = m - 1
    A_idx, B_idx = irc_halves(S, m, b)
    A = _take(S, ax, A_idx)
    B = _take(S, ax, B_idx)
    t = W11 * A + W12 * B
    Bn = W21 * A + W22 * B
    _put(S, ax, A_idx, t)
    _put(S, ax, B_idx, Bn)
    return S


def _filter_halves(Fs, m, b):
    ax = m - 1
    A_idx, B_idx = irc_halves(Fs, m, b) if Fs.shape[ax] > 1 else (None, None)
    return _take(Fs, ax, A_idx), _take(Fs, ax, B_idx)


def irc_analysis(S, stages):
    """src/directional/irc.jl:326-333 (file numbering)"""
    for st in stages:
        F0a, F0b = _filter_halves(st.ana[0], st.m, st.b)
        F1a, F1b = _filter_halves(st.ana[1], st.m, st.b)
        irc_stage(S, st.m, st.b, F0a, F0b, F1a, F1b)
    return S


def irc_synthesis(S, stages):
    """src/directional/irc.jl:338-345 (file numbering)"""
    for st in reversed(stages):
        G0a, G0b = _filter_halves(st.syn[0], st.m, st.b)
        G1a, G1b = _filter_halves(st.syn[1], st.m, st.b)
        irc_stage(S, st.m, st.b, G0a, G1a, G0b, G1b)
    return S


# ── One scale ───────────────────────────────────────────────────────────────


@dataclass
class SurfScale:
    dims: tuple
    levels: tuple
    masks: list
    stages: list


def surf_blocks(sc, K):
    """(counts, bsize) of hourglass K.  src/directional/surfacelet_scale.jl:32-37"""
    n = sc.dims
    counts = tuple(1 << sc.levels[K - 1][d] for d in range(3))
    bsize = tuple(n[d] // 2 + 1 if d == K - 1 else n[d] // counts[d] for d in range(3))
    return counts, bsize


def surf_subband_size(sc, K):
    """src/directional/surfacelet_scale.jl:40-43"""
    _, bsize = surf_blocks(sc, K)
    return tuple(sc.dims[d] if d == K - 1 else bsize[d] for d in range(3))


def block_ranges(counts, bsize, i):
    """Block i (0-based, column-major over block indices).  surfacelet_scale.jl:57-60"""
    v = np.unravel_index(i, counts, order="F")
    return tuple(slice(v[d] * bsize[d], (v[d] + 1) * bsize[d]) for d in range(3))


def _others(K):
    return [d for d in range(3) if d != K - 1]


def block_to_subband(blk, K, nK):
    """Unnormalized brfft halving axis K, complex along the others.

    src/directional/surfacelet_scale.jl:157-165
    """
    o = _others(K)
    s = [blk.shape[o[0]], blk.shape[o[1]], nK]
    return np.fft.irfftn(blk, s=s, axes=(o[0], o[1], K - 1)) * (nK * blk.shape[o[0]] * blk.shape[o[1]])


def subband_to_block(sb, K):
    """Unnormalized rfft halving axis K.  src/directional/surfacelet_scale.jl:168-176"""
    o = _others(K)
    return np.fft.rfftn(sb, axes=(o[0], o[1], K - 1))


def surf_scale_forward(X, sc):
    """Real subbands of one scale, in block order.  surfacelet_scale.jl:200-213"""
    out = []
    Ss = []
    for K in (1, 2, 3):
        s = 1.0 / float(np.prod(surf_subband_size(sc, K)))
        half = tuple(slice(0, sc.dims[d] // 2 + 1) if d == K - 1 else slice(None) for d in range(3))
        S = (X[half] * sc.masks[K - 1]) * s
        irc_analysis(S, sc.stages[K - 1])
        Ss.append(S)
    for K in (1, 2, 3):
        counts, bsize = surf_blocks(sc, K)
        for i in range(int(np.prod(counts))):
            out.append(block_to_subband(Ss[K - 1][block_ranges(counts, bsize, i)], K, sc.dims[K - 1]))
    return out


def hermitian_add(X, S, M, K, c):
    """X += c M S on the half of axis K and its conjugate mirror on the rest.

    src/directional/surfacelet_scale.jl:246-257
    """
    n = X.shape
    h = S.shape[K - 1]
    X[tuple(slice(0, s) for s in S.shape)] += c * M * S
    ax = K - 1
    nK = n[ax]
    # destination k_K = h .. nK-1 (0-based), source nK - k_K; other axes i -> (-i) mod n
    dst_k = np.arange(h, nK)
    src_k = nK - dst_k
    o1, o2 = _others(K)
    src1 = (-np.arange(n[o1])) % n[o1]
    src2 = (-np.arange(n[o2])) % n[o2]
    idx_src = [None, None, None]
    idx_src[ax] = src_k
    idx_src[o1] = src1
    idx_src[o2] = src2
    idx_dst = [None, None, None]
    idx_dst[ax] = dst_k
    idx_dst[o1] = np.arange(n[o1])
    idx_dst[o2] = np.arange(n[o2])
    Mm = M[np.ix_(*idx_src)]
    Sm = S[np.ix_(*idx_src)]
    X[np.ix_(*idx_dst)] += c * Mm * np.conj(Sm)
    return X


def surf_scale_inverse(subbands, sc):
    """Full spectrum of one scale from its subbands.  surfacelet_scale.jl:220-239"""
    X = np.zeros(sc.dims, dtype=np.complex128)
    it = iter(subbands)
    Ss = []
    for K in (1, 2, 3):
        counts, bsize = surf_blocks(sc, K)
        S = np.zeros(half_dims(sc.dims, K), dtype=np.complex128)
        for i in range(int(np.prod(counts))):
            sb = np.asarray(next(it), dtype=np.float64)
            if sb.shape != surf_subband_size(sc, K):
                raise DimensionMismatch(f"subband has size {sb.shape}, expected {surf_subband_size(sc, K)}")
            S[block_ranges(counts, bsize, i)] = subband_to_block(sb, K)
        Ss.append(S)
    for K in (1, 2, 3):
        irc_synthesis(Ss[K - 1], sc.stages[K - 1])
        hermitian_add(X, Ss[K - 1], sc.masks[K - 1], K, 1.0 / 3)
    return X


# ── Whole transform ─────────────────────────────────────────────────────────


def axis_problem(p, a, n):
    """First reason an axis of length n does not fit, or None.

    src/transforms/surfacelet.jl:230-249
    """
    J = p.scales
    ws, tbws, Ds = pyramid_mode(p.pyramid_ratio)
    for j in range(1, J + 1):
        s = J - j + 1
        where = f"at scale {s} of {J} (1 the coarsest) the length is {n}"
        if n % 2 != 0:
            return f"{where}, which must be even"
        c = 1 << max(p.levels[s - 1][K][a - 1] for K in range(3))
        if n % c != 0:
            return f"{where}, which the directional levels must split into {c} wedge blocks"
        k = 0 if j == 1 else 1
        D = Ds[k]
        if (n * D.denominator) % D.numerator != 0:
            return (f"{where}, which resampling by {D.numerator}/{D.denominator} needs to be a "
                    f"multiple of {D.numerator}")
        nlow = n * D.denominator // D.numerator
        P = F.rcos_edges(n, ws[k], tbws[k])[0]
        if not 2 * P <= nlow:
            return f"{where}, too small for the pyramid's lowpass"
        n = nlow
    return None


def fmt_ratio(r):
    return f"{float(r)}"


def check_size(p, dims):
    """src/transforms/surfacelet.jl:253-269"""
    for a in (1, 2, 3):
        problem = axis_problem(p, a, dims[a - 1])
        if problem is None:
            continue
        n = dims[a - 1]
        near = 0
        for d in range(1, 4 * n + 65):
            for m in (n - d, n + d):
                if m >= 1 and axis_problem(p, a, m) is None:
                    near = m
                    break
            if near > 0:
                break
        hint = f"; the nearest length that fits is {near}" if near > 0 else ""
        raise ArgumentError(
            f"a volume of size {fmt_dims(dims)} does not fit Surfacelet(scales = {p.scales}, "
            f"pyramid_ratio = {fmt_ratio(p.pyramid_ratio)}): axis {a}: {problem}{hint}")
    return dims


def layout_sizes(p, dims):
    """Subband sizes in layout order.  src/transforms/surfacelet.jl:275-290"""
    check_size(p, dims)
    pyr = fourier_pyramid(dims, p.scales, p.pyramid_ratio)
    sizes = [pyr[-1].nlow]
    for j in range(1, p.scales + 1):
        n = pyr[p.scales - j].n
        for K in (1, 2, 3):
            counts = tuple(1 << p.levels[j - 1][K - 1][d] for d in range(3))
            if not all(n[d] % counts[d] == 0 for d in range(3)):
                raise ArgumentError(
                    f"scale {j} of size {fmt_dims(n)} cannot be split into {fmt_dims(counts)} wedge blocks in hourglass {K}")
            sb = tuple(n[d] if d == K - 1 else n[d] // counts[d] for d in range(3))
            sizes += [sb] * int(np.prod(counts))
    return sizes


def subband_layout(p, dims):
    """[(scale, hourglass, wedge)], the lowpass (0, 0, 0) first.  surfacelet.jl:301-308"""
    layout_sizes(p, dims)
    out = [(0, 0, 0)]
    for j in range(1, p.scales + 1):
        for K in (1, 2, 3):
            for w in range(1, (1 << sum(p.levels[j - 1][K - 1])) + 1):
                out.append((j, K, w))
    return out


def redundancy(p, dims):
    """src/transforms/surfacelet.jl:220-222"""
    return sum(int(np.prod(s)) for s in layout_sizes(p, dims)) / float(np.prod(dims))


@dataclass
class SurfTables:
    dims: tuple
    p: SurfParams
    pyramid: list
    scales: list       # per pyramid level (finest first)
    sizes: list
    offsets: list      # 0-based element offsets of each subband in the flat vector
    level_offsets: list  # [level] index (0-based) of its first subband


def make_tables(p, dims):
    """src/transforms/surfacelet.jl:136-149 and :73-102"""
    check_size(p, dims)
    pyr = fourier_pyramid(dims, p.scales, p.pyramid_ratio)
    scales = []
    J = p.scales
    for j in range(1, J + 1):
        n = pyr[j - 1].n
        lv = p.levels[J - j]
        masks = ritf_masks(n, p.diamond_length, p.kaiser_beta, p.diamond_power)
        stages = [irc_stages(half_dims(n, K), n[K - 1], K, lv[K - 1], p.checkerboard_order) for K in (1, 2, 3)]
        scales.append(SurfScale(n, lv, masks, stages))
    sizes = layout_sizes(p, dims)
    offs = np.concatenate([[0], np.cumsum([int(np.prod(s)) for s in sizes])])
    counts = [nsubbands_scale(sc.levels) for sc in scales]
    level_offsets = [1 + sum(counts[j + 1:]) for j in range(J)]
    return SurfTables(tuple(dims), p, pyr, scales, sizes, [int(o) for o in offs], level_offsets)


def total_coefficients(T):
    return T.offsets[-1]


def subband(T, c, i):
    """View of subband i (1-based) of the flat coefficient vector, column-major."""
    a, b = T.offsets[i - 1], T.offsets[i]
    return c[a:b].reshape(T.sizes[i - 1], order="F")


def analyze(T, x):
    """Flat coefficient vector.  src/transforms/surfacelet.jl:369-381 (complex: 339-352)"""
    x = np.asarray(x)
    if np.iscomplexobj(x):
        return analyze(T, x.real) + 1j * analyze(T, x.imag)
    c = np.empty(total_coefficients(T))
    X = np.fft.fftn(x.astype(np.complex128))
    for j, lv in enumerate(T.pyramid):
        low = pyramid_split(X, lv)
        bands = surf_scale_forward(X, T.scales[j])
        for n, b in enumerate(bands):
            i = T.level_offsets[j] + n + 1
            c[T.offsets[i - 1]:T.offsets[i]] = b.ravel(order="F")
        X = low
    C = np.fft.ifftn(X) * X.size   # unnormalized inverse
    c[T.offsets[0]:T.offsets[1]] = (C.real / X.size).ravel(order="F")
    return c


def synthesize(T, c):
    """Volume from the flat coefficients.  src/transforms/surfacelet.jl:384-396"""
    c = np.asarray(c)
    if np.iscomplexobj(c):
        return synthesize(T, c.real) + 1j * synthesize(T, c.imag)
    C = np.fft.fftn(subband(T, c, 1).astype(np.complex128))
    for j in reversed(range(len(T.pyramid))):
        sc = T.scales[j]
        nb = nsubbands_scale(sc.levels)
        bands = [subband(T, c, T.level_offsets[j] + n + 1) for n in range(nb)]
        Xj = surf_scale_inverse(bands, sc)
        C = pyramid_merge(Xj, C, T.pyramid[j])
    x = np.fft.ifftn(C) * C.size
    return x.real / C.size


# ── SurfBox-style helpers used by the golden tests ──────────────────────────


def scale_tables(n, lv, bo, msize=15, beta=2.5, lam=4):
    """A standalone scale (the reference tests build these directly)."""
    masks = ritf_masks(n, msize, beta, lam)
    stages = [irc_stages(half_dims(n, K), n[K - 1], K, lv[K - 1], bo) for K in (1, 2, 3)]
    return SurfScale(tuple(n), lv, masks, stages)
