"""Python mirror of the reference's interface for the surfacelet transforms
(AbstractMultiscaleTransforms methods of Surfacelets.jl): transform objects,
workspaces, analyze / synthesize (and the in-place `analyze_` / `synthesize_`,
the reference's `analyze!` / `synthesize!`), the streaming forms, and the
layout queries.  Everything runs through libsurfacelets_b200.so.

Arrays follow the reference's memory layout: a volume of size (n1, n2, n3)
is column-major (axis 1 fastest).  Device data are torch CUDA tensors of
shape (n1, n2, n3) whose strides are column-major (`volume_like`,
`to_device` make them); host data are NumPy arrays, which the calls copy to
the device and back (the host arrays of the reference's CPU path).
NSSurfacelet coefficients are (n1, n2, n3, S), subband i the slice
[..., i-1]; Surfacelet coefficients are one flat vector (the reference's
SubbandVector) whose subbands `subband` views in place.
"""

import ctypes as C

import numpy as np

from . import _lib
from ._lib import ArgumentError, DimensionMismatch, check, lib

try:
    import torch
except ImportError:     # the host-only queries still work without torch
    torch = None


# ── transform objects ────────────────────────────────────────────────────────


def _parabolic_levels(scales):
    """src/types/transforms.jl:147"""
    return [1 + (j - 1) // 2 for j in range(1, scales + 1)]


def _scales_and_levels(scales, direction_levels):
    """src/types/transforms.jl:136-142"""
    if direction_levels is None:
        if scales is None:
            raise ArgumentError("give `scales`, `direction_levels` or both")
        return scales, _parabolic_levels(scales)
    return (len(direction_levels) if scales is None else scales), direction_levels


def _fmt_real(x):
    x = float(x)
    return repr(x) if x != int(x) or abs(x) >= 1e16 else f"{x:.1f}"


class NSSurfacelet:
    """The nonsubsampled surfacelet transform.  src/types/transforms.jl:86-113"""

    def __init__(self, scales=None, direction_levels=None, bernstein_order=12, halfband_order=1,
                 transition=1.0, tight=True):
        J, levels = _scales_and_levels(scales, direction_levels)
        if not isinstance(J, (int, np.integer)) or J < 1:
            raise ArgumentError(f"scales must be ≥ 1, got {J}")
        if len(levels) != J:
            raise ArgumentError(f"length(direction_levels) must equal scales = {J}, got {len(levels)}")
        self.scales = int(J)
        self.direction_levels = [int(v) for v in levels]
        self.bernstein_order = int(bernstein_order)
        self.halfband_order = int(halfband_order)
        self.transition = float(transition) + 0.0
        self.tight = bool(tight)
        check(lib.sfl_ns_check_params(C.byref(self._params())))

    def _params(self):
        p = _lib.NSParams()
        p.scales = self.scales
        for j, v in enumerate(self.direction_levels[:_lib.SFL_MAX_SCALES]):
            p.direction_levels[j] = v
        p.bernstein_order = self.bernstein_order
        p.halfband_order = self.halfband_order
        p.transition = self.transition
        p.tight = 1 if self.tight else 0
        return p

    def _key(self):
        return (self.scales, tuple(self.direction_levels), self.bernstein_order, self.halfband_order,
                self.transition, self.tight)

    def __eq__(self, other):
        return isinstance(other, NSSurfacelet) and self._key() == other._key()

    def __hash__(self):
        return hash(("NSSurfacelet",) + self._key())

    def __repr__(self):
        return (f"NSSurfacelet(scales = {self.scales}, direction_levels = [{', '.join(map(str, self.direction_levels))}], "
                f"bernstein_order = {self.bernstein_order}, halfband_order = {self.halfband_order}, "
                f"transition = {_fmt_real(self.transition)}, tight = {'true' if self.tight else 'false'})")


class NDFB(NSSurfacelet):
    """The standalone nonsubsampled directional filter bank (make_ndfb,
    src/directional/ndfb.jl:91-104): 3 * 2^levels full-size subbands, the
    hourglass bank refined into wedges, run on the NSSurfacelet kernels with
    no pyramid and no lowpass.  levels = 0 is the hourglass bank."""

    def __init__(self, levels=2, bernstein_order=12, halfband_order=1, tight=True, transition=1.0):
        if isinstance(levels, (bool, np.bool_)) or not isinstance(levels, (int, np.integer)):
            raise ArgumentError(f"levels must be an integer, got {levels!r}")
        self.levels = int(levels)
        self.scales = 1
        self.direction_levels = [self.levels]
        self.bernstein_order = int(bernstein_order)
        self.halfband_order = int(halfband_order)
        self.transition = float(transition) + 0.0
        self.tight = bool(tight)
        check(lib.sfl_ndfb_check_params(C.byref(self._ndfb_params())))

    def _ndfb_params(self):
        p = _lib.NDFBParams()
        p.levels = self.levels
        p.bernstein_order = self.bernstein_order
        p.halfband_order = self.halfband_order
        p.transition = self.transition
        p.tight = 1 if self.tight else 0
        return p

    def _key(self):
        return ("NDFB", self.levels, self.bernstein_order, self.halfband_order, self.transition, self.tight)

    def __eq__(self, other):
        return isinstance(other, NDFB) and self._key() == other._key()

    def __hash__(self):
        return hash(self._key())

    def wedge_counts(self):
        """(na, nb): wedges on the two transverse planes of a hourglass (src/directional/ndfb.jl:146)."""
        return 1 << ((self.levels + 1) // 2), 1 << (self.levels // 2)

    def __repr__(self):
        return (f"NDFB(levels = {self.levels}, bernstein_order = {self.bernstein_order}, "
                f"halfband_order = {self.halfband_order}, tight = {'true' if self.tight else 'false'}, "
                f"transition = {_fmt_real(self.transition)})")


class HourglassFB(NDFB):
    """The three-subband hourglass bank (make_hourglass, src/directional/hourglass.jl:149-170)."""

    def __init__(self, bernstein_order=12, halfband_order=1, tight=True):
        super().__init__(0, bernstein_order, halfband_order, tight, 1.0)

    def __repr__(self):
        return (f"HourglassFB(bernstein_order = {self.bernstein_order}, halfband_order = {self.halfband_order}, "
                f"tight = {'true' if self.tight else 'false'})")


def ndfb_subband_index(t, hourglass, p, q):
    """src/directional/ndfb.jl:184-190"""
    na, nb = t.wedge_counts()
    if not 1 <= hourglass <= 3:
        raise ArgumentError("hourglass index must be 1, 2 or 3")
    if not 1 <= p <= na:
        raise ArgumentError(f"wedge index p out of range 1:{na}")
    if not 1 <= q <= nb:
        raise ArgumentError(f"wedge index q out of range 1:{nb}")
    return ((hourglass - 1) * na + (p - 1)) * nb + q


def ndfb_subband_triple(t, idx):
    """(hourglass, p, q) of subband idx.  src/directional/ndfb.jl:199-203"""
    na, nb = t.wedge_counts()
    if not 1 <= idx <= 3 * na * nb:
        raise ArgumentError("subband index out of range")
    r, q = divmod(idx - 1, nb)
    i, p = divmod(r, na)
    return i + 1, p + 1, q + 1


def _level_matrix(L):
    """src/types/transforms.jl:263-284"""
    if isinstance(L, (bool, np.bool_)):
        raise ArgumentError(f"a directional level must be an integer or a 3 × 3 integer matrix, got {L!r}")
    if isinstance(L, (int, np.integer)):
        out = ((C.c_int32 * 3) * 3)()
        check(lib.sfl_surf_levels_from_int(int(L), out))
        return [[out[K][m] for m in range(3)] for K in range(3)]
    M = np.asarray(L)
    if M.dtype.kind not in "iu":
        raise ArgumentError(f"a directional level must be an integer or a 3 × 3 integer matrix, got {L!r}")
    if M.shape != (3, 3):
        raise ArgumentError(f"a level matrix must be 3 × 3, got size {M.shape}")
    return [[0 if m == K else int(M[K, m]) for m in range(3)] for K in range(3)]


class Surfacelet:
    """The decimated surfacelet transform (SurfBox's construction).
    src/types/transforms.jl:222-261"""

    def __init__(self, scales=None, direction_levels=None, pyramid_ratio=1.5, checkerboard_order=12,
                 diamond_length=15, kaiser_beta=2.5, diamond_power=4):
        J, levels = _scales_and_levels(scales, direction_levels)
        if not isinstance(J, (int, np.integer)) or J < 1:
            raise ArgumentError(f"scales must be ≥ 1, got {J}")
        if len(levels) != J:
            raise ArgumentError(f"length(direction_levels) must equal scales = {J}, got {len(levels)}")
        self.scales = int(J)
        self.direction_levels = [int(L) if isinstance(L, (int, np.integer)) else np.asarray(L).astype(int)
                                 for L in levels]
        self.levels = [_level_matrix(L) for L in levels]
        self.pyramid_ratio = float(pyramid_ratio)
        self.checkerboard_order = int(checkerboard_order)
        self.diamond_length = int(diamond_length)
        self.kaiser_beta = float(kaiser_beta)
        self.diamond_power = int(diamond_power)
        check(lib.sfl_surf_check_params(C.byref(self._params())))

    def _params(self):
        p = _lib.SurfParams()
        p.scales = self.scales
        for j, M in enumerate(self.levels[:_lib.SFL_MAX_SCALES]):
            for K in range(3):
                for m in range(3):
                    p.levels[j][K][m] = M[K][m]
        p.pyramid_ratio = self.pyramid_ratio
        p.checkerboard_order = self.checkerboard_order
        p.diamond_length = self.diamond_length
        p.kaiser_beta = self.kaiser_beta
        p.diamond_power = self.diamond_power
        return p

    def _key(self):
        return (self.scales, tuple(tuple(map(tuple, M)) for M in self.levels), self.pyramid_ratio,
                self.checkerboard_order, self.diamond_length, self.kaiser_beta, self.diamond_power)

    def __eq__(self, other):
        return isinstance(other, Surfacelet) and self._key() == other._key()

    def __hash__(self):
        return hash(("Surfacelet",) + self._key())

    def __repr__(self):
        def lev(L):
            if isinstance(L, int):
                return str(L)
            return "[" + "; ".join(" ".join(str(int(v)) for v in row) for row in np.asarray(L)) + "]"
        return (f"Surfacelet(scales = {self.scales}, direction_levels = [{', '.join(lev(L) for L in self.direction_levels)}], "
                f"pyramid_ratio = {self.pyramid_ratio}, checkerboard_order = {self.checkerboard_order}, "
                f"diamond_length = {self.diamond_length}, kaiser_beta = {self.kaiser_beta}, "
                f"diamond_power = {self.diamond_power})")


def checkerboard_orders():
    """src/filters/checkerboard.jl:61"""
    return [4, 6, 8, 10, 12, 14, 16, 18]


# ── layout queries (host only) ───────────────────────────────────────────────


def _dims3(dims):
    dims = tuple(int(d) for d in dims)
    if len(dims) != 3:
        raise ArgumentError(f"the surfacelet transforms take volumes (three axes), got size ({', '.join(map(str, dims))}{',' if len(dims) == 1 else ''})")
    return dims


def _cdims(dims):
    return _lib.Dims(*dims)


def nsubbands(t, dims):
    """src/transforms/ns_surfacelet.jl:527, src/transforms/surfacelet.jl:310"""
    dims = _dims3(dims)
    if isinstance(t, NDFB):
        return 3 << t.levels
    if isinstance(t, NSSurfacelet):
        n = C.c_int32()
        check(lib.sfl_ns_nsubbands(C.byref(t._params()), C.byref(n)))
        return n.value
    n = C.c_int32()
    check(lib.sfl_surf_layout(C.byref(t._params()), _cdims(dims), C.byref(n), None, None, None, None))
    return n.value


def subband_layout(t, dims):
    """What each subband is, the lowpass first.  src/transforms/ns_surfacelet.jl:518-525
    (dicts with `scale`, `direction`) and src/transforms/surfacelet.jl:301-308
    (dicts with `scale`, `hourglass`, `wedge`)."""
    dims = _dims3(dims)
    n = nsubbands(t, dims)
    if isinstance(t, NDFB):
        return [dict(zip(("hourglass", "wedge_a", "wedge_b"), ndfb_subband_triple(t, i))) for i in range(1, n + 1)]
    if isinstance(t, NSSurfacelet):
        sc = (C.c_int32 * n)()
        di = (C.c_int32 * n)()
        check(lib.sfl_ns_layout(C.byref(t._params()), sc, di))
        return [{"scale": sc[i], "direction": di[i]} for i in range(n)]
    sc, hg, we = (C.c_int32 * n)(), (C.c_int32 * n)(), (C.c_int32 * n)()
    check(lib.sfl_surf_layout(C.byref(t._params()), _cdims(dims), None, None, sc, hg, we))
    return [{"scale": sc[i], "hourglass": hg[i], "wedge": we[i]} for i in range(n)]


def subband_sizes(t, dims):
    """Shape of every subband, in layout order."""
    dims = _dims3(dims)
    if isinstance(t, NDFB):
        return [dims] * nsubbands(t, dims)
    if isinstance(t, NSSurfacelet):
        check(lib.sfl_ns_check_size(C.byref(t._params()), _cdims(dims)))
        return [dims] * nsubbands(t, dims)
    n = nsubbands(t, dims)
    sz = (C.c_int32 * (3 * n))()
    check(lib.sfl_surf_layout(C.byref(t._params()), _cdims(dims), None, sz, None, None, None))
    return [tuple(sz[3 * i:3 * i + 3]) for i in range(n)]


def surfacelet_redundancy(t, dims):
    """src/transforms/surfacelet.jl:220-222"""
    r = C.c_double()
    check(lib.sfl_surf_redundancy(C.byref(t._params()), _cdims(_dims3(dims)), C.byref(r)))
    return r.value


def supports_streaming(t):
    """src/transforms/ns_surfacelet.jl:504"""
    return isinstance(t, NSSurfacelet)


# ── arrays ───────────────────────────────────────────────────────────────────


def _need_torch():
    if torch is None:
        raise ImportError("torch is needed for device arrays")


def volume_like(dims, dtype="float32", device="cuda"):
    """Uninitialized column-major device array of shape dims (torch)."""
    _need_torch()
    td = {"complex64": torch.complex64, "torch.complex64": torch.complex64, "bfloat16": torch.bfloat16,
          "torch.bfloat16": torch.bfloat16}.get(str(dtype), torch.float32)
    return torch.empty(tuple(reversed(tuple(dims))), dtype=td, device=device).permute(*reversed(range(len(dims))))


def to_device(a, device="cuda"):
    """Column-major device copy of a NumPy array (float32 / complex64)."""
    _need_torch()
    a = np.asarray(a)
    dt = np.complex64 if np.iscomplexobj(a) else np.float32
    t = torch.from_numpy(np.ascontiguousarray(a.astype(dt, copy=False).transpose()))
    return t.to(device).permute(*reversed(range(a.ndim)))


def to_host(t):
    """NumPy copy (column-major, Fortran order) of a column-major device array."""
    _need_torch()
    return np.asfortranarray(t.permute(*reversed(range(t.dim()))).cpu().numpy().transpose())


def _is_colmajor(t):
    exp = 1
    for n, s in zip(t.shape, t.stride()):
        if n != 1 and s != exp:
            return False
        exp *= n
    return True


def _dtype_code(x):
    if torch is not None and isinstance(x, torch.Tensor):
        if x.dtype == torch.complex64:
            return _lib.SFL_COMPLEX64
        if x.dtype == torch.float32:
            return _lib.SFL_REAL32
        raise ArgumentError(f"element type {x.dtype} is not supported (float32 or complex64)")
    return _lib.SFL_COMPLEX64 if np.iscomplexobj(x) else _lib.SFL_REAL32


def _dtype_name(code):
    return "ComplexF32" if code == _lib.SFL_COMPLEX64 else "Float32"


def _ptr(t):
    return C.c_void_p(t.data_ptr())


def _stream(stream):
    if stream is not None:
        return C.c_void_p(int(stream))
    return C.c_void_p(torch.cuda.current_stream().cuda_stream)


# ── workspaces ───────────────────────────────────────────────────────────────


class Workspace:
    """A plan of libsurfacelets_b200: tables, scratch and FFT set-up for one
    transform, volume size and element type (the reference's
    NSSurfaceletWorkspace / SurfaceletWorkspace).  Not reentrant: one call at a
    time (src/transforms/ns_surfacelet.jl:51-53)."""

    def __init__(self, t, dtype_code, dims, group=None):
        self.transform = t
        self.dims = _dims3(dims)
        self.dtype = dtype_code
        h = C.c_void_p()
        if isinstance(t, NDFB):
            check(lib.sfl_ndfb_plan_create(C.byref(t._ndfb_params()), _cdims(self.dims), dtype_code, C.byref(h)))
        elif isinstance(t, NSSurfacelet):
            check(lib.sfl_ns_plan_create(C.byref(t._params()), _cdims(self.dims), dtype_code, C.byref(h)))
        else:
            check(lib.sfl_surf_plan_create(C.byref(t._params()), _cdims(self.dims), dtype_code, C.byref(h)))
        self._h = h
        kind, dd, dt, ns, nc = C.c_int32(), _lib.Dims(), C.c_int32(), C.c_int32(), C.c_int64()
        check(lib.sfl_plan_info(h, C.byref(kind), dd, C.byref(dt), C.byref(ns), C.byref(nc)))
        self.nsubbands = ns.value
        self.ncoeffs = nc.value
        self._info = []
        for i in range(1, self.nsubbands + 1):
            sh, off = _lib.Dims(), C.c_int64()
            check(lib.sfl_subband_info(h, i, sh, C.byref(off)))
            self._info.append((tuple(sh), off.value))
        if group is not None:
            self.set_group(group)

    def set_group(self, group):
        check(lib.sfl_plan_set_group(self._h, int(group)))

    PIPELINES = {"lines": 0, "planes": 1, "slabs": 2}

    def tuning(self):
        """(pipeline name, group) in use."""
        pi, g = C.c_int32(), C.c_int32()
        check(lib.sfl_plan_tuning(self._h, C.byref(pi), C.byref(g)))
        names = {v: k for k, v in self.PIPELINES.items()}
        return names.get(pi.value), g.value

    def tile(self, ipc=None):
        """Subbands a CTA of the slab pipeline's axis-3 analysis pass takes
        (1, 2, 4 or 8; 0 = the default): read, or set when ipc is given."""
        v = C.c_int32(0 if ipc is None else int(ipc))
        check(lib.sfl_plan_tile(self._h, 0 if ipc is None else 1, C.byref(v)))
        return v.value

    def autotune(self, x=None, stream=None):
        """Time analysis + synthesis under each pipeline and group size (and the
        slab pipeline's axis-3 tile), keep the fastest and remember it for later
        workspaces of the same transform, size and type.
        x: a device volume to time on (random when omitted)."""
        if not isinstance(self.transform, NSSurfacelet):
            return self.tuning()
        if x is None:
            x = volume_like(self.dims, "complex64" if self.dtype else "float32")
            x.copy_(torch.randn(x.shape, dtype=x.dtype, device=x.device))
        c = similar_coefficients(self.transform, x)
        check(lib.sfl_plan_autotune(self._h, _ptr(x), _ptr(c), _stream(stream)))
        return self.tuning()

    def set_pipeline(self, name):
        """NSSurfacelet kernel pipeline: "slabs" (the default where the size
        allows) or "lines" ("planes", the retired plane-major pipeline, is
        refused by the library)."""
        if name not in self.PIPELINES:
            raise ArgumentError(f"unknown pipeline {name!r}; expected one of {sorted(self.PIPELINES)}")
        check(lib.sfl_plan_set_pipeline(self._h, self.PIPELINES[name]))

    def subband_info(self, i):
        """(shape, element offset) of subband i (1-based)."""
        return self._info[i - 1]

    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            check(lib.sfl_plan_destroy(self._h))
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def eltype(self):
        return _dtype_name(self.dtype)

    def __repr__(self):
        name = ("NDFBWorkspace" if isinstance(self.transform, NDFB) else
                "NSSurfaceletWorkspace" if isinstance(self.transform, NSSurfacelet) else "SurfaceletWorkspace")
        return f"{name}{{{self.eltype}}}({'×'.join(map(str, self.dims))}, {self.transform})"


def make_workspace(t, T_or_x, dims=None, group=None):
    """make_workspace(t, T, dims) / make_workspace(t, x).
    src/transforms/ns_surfacelet.jl:88-95, 165-173; src/transforms/surfacelet.jl:126-133, 192-199.
    T is "float32" / "complex64" (a NumPy or torch dtype works too)."""
    if dims is None:
        x = T_or_x
        return Workspace(t, _dtype_code(x), tuple(x.shape), group)
    name = str(T_or_x)
    code = _lib.SFL_COMPLEX64 if "complex" in name else _lib.SFL_REAL32
    return Workspace(t, code, dims, group)


def _workspace_for(workspace, t, x_code, dims):
    """src/transforms/ns_surfacelet.jl:247-252, src/transforms/surfacelet.jl:327-334"""
    if workspace is None:
        return Workspace(t, x_code, dims)
    if not isinstance(workspace, Workspace):
        raise ArgumentError(f"a {type(t).__name__} needs a workspace, got {type(workspace).__name__}")
    if workspace.transform != t:
        raise ArgumentError(f"the workspace was built for {workspace.transform}, not {t}")
    if workspace.dtype != x_code:
        raise ArgumentError(f"element type {_dtype_name(x_code)}, the workspace is for {workspace.eltype}")
    if tuple(workspace.dims) != tuple(dims):
        raise DimensionMismatch(f"the workspace was built for size {workspace.dims}, got {tuple(dims)}")
    return workspace


def similar_coefficients(t, x):
    """Uninitialized coefficients for volumes like x.
    src/transforms/ns_surfacelet.jl:534-537, src/transforms/surfacelet.jl:439-442"""
    dims = _dims3(x.shape)
    code = _dtype_code(x)
    if isinstance(t, NSSurfacelet):
        shape = dims + (nsubbands(t, dims),)
        if torch is not None and isinstance(x, torch.Tensor):
            return volume_like(shape, "complex64" if code else "float32", x.device)
        return np.empty(shape, dtype=np.complex64 if code else np.float32, order="F")
    n = sum(int(np.prod(s)) for s in subband_sizes(t, dims))
    if torch is not None and isinstance(x, torch.Tensor):
        return torch.empty(n, dtype=torch.complex64 if code else torch.float32, device=x.device)
    return np.empty(n, dtype=np.complex64 if code else np.float32)


def subband(t, c, i, dims=None):
    """View of subband i (1-based).  NS: c[..., i-1]; decimated: the block of
    the flat vector, viewed column-major (dims = the volume size)."""
    if isinstance(t, NSSurfacelet):
        return c[..., i - 1]
    if dims is None:
        raise ArgumentError("the volume size is needed to locate a Surfacelet subband")
    sizes = subband_sizes(t, dims)
    off = sum(int(np.prod(s)) for s in sizes[:i - 1])
    sz = sizes[i - 1]
    n = int(np.prod(sz))
    blk = c[off:off + n]
    if torch is not None and isinstance(c, torch.Tensor):
        return blk.view(tuple(reversed(sz))).permute(2, 1, 0)
    return blk.reshape(sz, order="F")


# ── transforms ───────────────────────────────────────────────────────────────


def _check_device_array(a, what, shape, code):
    if tuple(a.shape) != tuple(shape):
        raise DimensionMismatch(f"{what} of size {tuple(a.shape)}, expected {tuple(shape)}")
    if _dtype_code(a) != code:
        raise ArgumentError(f"{what} of element type {_dtype_name(_dtype_code(a))}, the workspace is for {_dtype_name(code)}")
    if not a.is_cuda:
        raise ArgumentError(f"{what} must be a CUDA tensor")
    if a.dim() > 1 and not _is_colmajor(a):
        raise ArgumentError(f"{what} must be column-major (see volume_like / to_device)")


def _coef_shape(ws):
    if isinstance(ws.transform, NSSurfacelet):
        return ws.dims + (ws.nsubbands,)
    return (ws.ncoeffs,)


def _run(fn, ws, a, b, stream):
    check(fn(ws._h, _ptr(a), _ptr(b), _stream(stream)))


def analyze_(c, t, x, workspace=None, stream=None):
    """In-place analysis (the reference's analyze!(c, t, x; workspace)).
    src/transforms/ns_surfacelet.jl:551-566, src/transforms/surfacelet.jl:446-454"""
    if isinstance(t, Workspace):
        workspace, t = t, t.transform
    dims = _dims3(x.shape)
    ws = _workspace_for(workspace, t, _dtype_code(x), dims)
    if not (torch is not None and isinstance(x, torch.Tensor)):
        cd = analyze_(to_device_like(c, ws), t, to_device(x), ws, stream)
        _copy_back(c, cd)
        return c
    _check_device_array(x, "volume", dims, ws.dtype)
    _check_device_array(c, "coefficients", _coef_shape(ws), ws.dtype)
    _run(lib.sfl_analyze, ws, x, c, stream)
    return c


def synthesize_(x, t, c=None, workspace=None, stream=None):
    """In-place synthesis (the reference's synthesize!(x, t, c; workspace)).
    With a callable as first argument it is the streaming form
    synthesize!(f, x, t): f(i) returns subband i.
    src/transforms/ns_surfacelet.jl:568-581, 626-641; src/transforms/surfacelet.jl:456-464"""
    if callable(x) and not hasattr(x, "shape"):
        return _synthesize_stream(x, t, c, workspace, stream)
    if isinstance(t, Workspace):
        workspace, t = t, t.transform
    dims = _dims3(x.shape)
    ws = _workspace_for(workspace, t, _dtype_code(x), dims)
    if not (torch is not None and isinstance(x, torch.Tensor)):
        xd = synthesize_(volume_like(dims, "complex64" if ws.dtype else "float32"), t, to_device_like(c, ws, copy=True),
                         ws, stream)
        _copy_back(x, xd)
        return x
    _check_device_array(x, "volume", dims, ws.dtype)
    _check_device_array(c, "coefficients", _coef_shape(ws), ws.dtype)
    _run(lib.sfl_synthesize, ws, c, x, stream)
    return x


def adjoint_analyze_(x, t, c, workspace=None, stream=None):
    """x = A^T c (the adjoint of analysis; for a tight NSSurfacelet, synthesize)."""
    if isinstance(t, Workspace):
        workspace, t = t, t.transform
    dims = _dims3(x.shape)
    ws = _workspace_for(workspace, t, _dtype_code(x), dims)
    _check_device_array(x, "volume", dims, ws.dtype)
    _check_device_array(c, "coefficients", _coef_shape(ws), ws.dtype)
    _run(lib.sfl_adjoint_analyze, ws, c, x, stream)
    return x


def adjoint_synthesize_(c, t, x, workspace=None, stream=None):
    """c = S^T x (the adjoint of synthesis; for a tight NSSurfacelet, analyze)."""
    if isinstance(t, Workspace):
        workspace, t = t, t.transform
    dims = _dims3(x.shape)
    ws = _workspace_for(workspace, t, _dtype_code(x), dims)
    _check_device_array(x, "volume", dims, ws.dtype)
    _check_device_array(c, "coefficients", _coef_shape(ws), ws.dtype)
    _run(lib.sfl_adjoint_synthesize, ws, x, c, stream)
    return c


def to_device_like(c, ws, copy=False):
    """Device array for the coefficients of ws (a copy of c when asked)."""
    if torch is not None and isinstance(c, torch.Tensor):
        return c
    shape = _coef_shape(ws)
    if copy:
        if len(shape) == 1:
            return torch.from_numpy(np.ascontiguousarray(c)).cuda()
        return to_device(c)
    if len(shape) == 1:
        return torch.empty(shape[0], dtype=torch.complex64 if ws.dtype else torch.float32, device="cuda")
    return volume_like(shape, "complex64" if ws.dtype else "float32")


def _copy_back(dst, src):
    h = to_host(src) if src.dim() > 1 else src.cpu().numpy()
    dst[...] = h


def analyze(*args, workspace=None, stream=None):
    """analyze(t, x) / analyze(ws, x): new coefficients.  analyze(f, t, x):
    streaming, f(i, band) per subband, the directional subbands in increasing
    i and then the lowpass (i = 1); band is valid only until f returns.
    src/transforms/ns_surfacelet.jl:551-566, 583-624; src/transforms/surfacelet.jl:446-454"""
    if len(args) == 3 and callable(args[0]):
        return _analyze_stream(args[0], args[1], args[2], workspace, stream)
    t, x = args
    if isinstance(t, Workspace):
        workspace, t = t, t.transform
    c = similar_coefficients(t, x)
    return analyze_(c, t, x, workspace, stream)


def synthesize(t, c, workspace=None, stream=None, dims=None):
    """synthesize(t, c) / synthesize(ws, c): the volume.  For a Surfacelet
    without a workspace, pass dims."""
    if isinstance(t, Workspace):
        workspace, t = t, t.transform
    if workspace is not None:
        dims = workspace.dims
    elif isinstance(t, NSSurfacelet):
        dims = tuple(c.shape[:3])
    elif dims is None:
        raise ArgumentError("synthesize(t::Surfacelet, c) needs the volume size: pass dims or a workspace")
    code = _dtype_code(c)
    if torch is not None and isinstance(c, torch.Tensor):
        x = volume_like(dims, "complex64" if code else "float32", c.device)
    else:
        x = np.empty(dims, dtype=np.complex64 if code else np.float32, order="F")
    return synthesize_(x, t, c, workspace, stream)


def adjoint_analyze(t, c, workspace=None, stream=None, dims=None):
    if isinstance(t, Workspace):
        workspace, t = t, t.transform
    dims = workspace.dims if workspace is not None else (tuple(c.shape[:3]) if dims is None else dims)
    x = volume_like(dims, "complex64" if _dtype_code(c) else "float32", c.device)
    return adjoint_analyze_(x, t, c, workspace, stream)


def adjoint_synthesize(t, x, workspace=None, stream=None):
    if isinstance(t, Workspace):
        workspace, t = t, t.transform
    c = similar_coefficients(t, x)
    return adjoint_synthesize_(c, t, x, workspace, stream)


def _analyze_stream(f, t, x, workspace, stream):
    """src/transforms/ns_surfacelet.jl:620-624"""
    if isinstance(t, Workspace):
        workspace, t = t, t.transform
    if not isinstance(t, NSSurfacelet):
        raise ArgumentError(f"{type(t).__name__} does not stream")
    dims = _dims3(x.shape)
    ws = _workspace_for(workspace, t, _dtype_code(x), dims)
    host = not (torch is not None and isinstance(x, torch.Tensor))
    xd = to_device(x) if host else x
    _check_device_array(xd, "volume", dims, ws.dtype)
    band = volume_like(dims, "complex64" if ws.dtype else "float32", xd.device)
    st = _stream(stream)
    check(lib.sfl_stream_analyze_begin(ws._h, _ptr(xd), st))
    idx = C.c_int32()
    while True:
        r = check(lib.sfl_stream_analyze_next(ws._h, _ptr(band), C.byref(idx), st))
        if r == _lib.SFL_DONE:
            break
        f(idx.value, to_host(band) if host else band)
    return None


def _synthesize_stream(f, x, t, workspace, stream):
    """src/transforms/ns_surfacelet.jl:626-641"""
    if isinstance(t, Workspace):
        workspace, t = t, t.transform
    if not isinstance(t, NSSurfacelet):
        raise ArgumentError(f"{type(t).__name__} does not stream")
    dims = _dims3(x.shape)
    ws = _workspace_for(workspace, t, _dtype_code(x), dims)
    host = not (torch is not None and isinstance(x, torch.Tensor))
    st = _stream(stream)
    check(lib.sfl_stream_synthesize_begin(ws._h, st))
    idx = C.c_int32()
    keep = []
    while check(lib.sfl_stream_synthesize_next_index(ws._h, C.byref(idx))) != _lib.SFL_DONE:
        i = idx.value
        b = f(i)
        if tuple(b.shape) != dims:
            raise DimensionMismatch(f"subband {i} has size {tuple(b.shape)}, expected {dims}")
        bd = to_device(b) if not (torch is not None and isinstance(b, torch.Tensor)) else b
        _check_device_array(bd, f"subband {i}", dims, ws.dtype)
        check(lib.sfl_stream_synthesize_push(ws._h, _ptr(bd), st))
        keep.append(bd)       # the push is asynchronous: keep the buffer alive
        if len(keep) > 2:
            torch.cuda.current_stream().synchronize() if stream is None else torch.cuda.synchronize()
            keep = keep[-1:]
    xd = volume_like(dims, "complex64" if ws.dtype else "float32") if host else x
    check(lib.sfl_stream_synthesize_end(ws._h, _ptr(xd), st))
    if host:
        _copy_back(x, xd)
    return x


# ── bfloat16 coefficients ───────────────────────────────────────────────────


def analyze_bf16(ws, x, stream=None):
    """NSSurfacelet analysis into bfloat16 coefficients: returns (c, scales)
    with c (n1, n2, n3, S) bfloat16 and scales (S,) float32 on the device,
    subband s = scales[s-1] * c[..., s-1] (each scale a power of two, the
    stored values within [-1, 1]).  Float32 volumes; no counterpart in the
    reference."""
    if not isinstance(ws, Workspace) or not isinstance(ws.transform, NSSurfacelet):
        raise ArgumentError("bfloat16 coefficients need an NSSurfacelet workspace")
    _check_device_array(x, "volume", ws.dims, ws.dtype)
    c = volume_like(ws.dims + (ws.nsubbands,), "bfloat16", x.device)
    scales = torch.empty(ws.nsubbands, dtype=torch.float32, device=x.device)
    check(lib.sfl_ns_analyze_bf16(ws._h, _ptr(x), _ptr(c), _ptr(scales), _stream(stream)))
    return c, scales


def synthesize_bf16(ws, c, scales, stream=None):
    """Synthesis from analyze_bf16's (c, scales)."""
    if not isinstance(ws, Workspace) or not isinstance(ws.transform, NSSurfacelet):
        raise ArgumentError("bfloat16 coefficients need an NSSurfacelet workspace")
    shape = ws.dims + (ws.nsubbands,)
    if tuple(c.shape) != shape:
        raise DimensionMismatch(f"coefficients of size {tuple(c.shape)}, expected {shape}")
    if c.dtype != torch.bfloat16 or not c.is_cuda or not _is_colmajor(c):
        raise ArgumentError("coefficients must be a column-major bfloat16 CUDA tensor")
    if tuple(scales.shape) != (ws.nsubbands,) or scales.dtype != torch.float32 or not scales.is_cuda:
        raise ArgumentError(f"scales must be {ws.nsubbands} float32 values on the device")
    x = volume_like(ws.dims, "float32", c.device)
    check(lib.sfl_ns_synthesize_bf16(ws._h, _ptr(c), _ptr(scales), _ptr(x), _stream(stream)))
    return x


# ── analysis -> per-subband processing -> synthesis, one subband at a time ──


def analyze_synthesize_stream(f, y, x, analysis_workspace, synthesis_workspace, stream=None):
    """y = sum_i S_i f(i, A_i x): subband i of x, handed to f(i, band) on the
    device, goes straight into the synthesis, so only one subband is ever in
    memory (a per-subband recompute instead of a materialized coefficient
    set; f = a shrinkage gives a denoiser).  The two workspaces are two plans
    of the same NSSurfacelet, size and element type (one per direction).
    f may modify band in place and return it, or return a new tensor; it runs
    on the current stream.  Built from the reference's streaming analyze(f, t,
    x) and synthesize!(f, x, t), src/transforms/ns_surfacelet.jl:600-641."""
    wa, wsy = analysis_workspace, synthesis_workspace
    for w in (wa, wsy):
        if not isinstance(w, Workspace) or not isinstance(w.transform, NSSurfacelet):
            raise ArgumentError("analyze_synthesize_stream needs two NSSurfacelet workspaces")
    if wa is wsy or wa._h.value == wsy._h.value:
        raise ArgumentError("analysis and synthesis need two workspaces (a plan holds one open stream)")
    if (wa.dims, wa.dtype, wa.nsubbands) != (wsy.dims, wsy.dtype, wsy.nsubbands):
        raise ArgumentError("the two workspaces must match in size, element type and subbands")
    _check_device_array(x, "volume", wa.dims, wa.dtype)
    _check_device_array(y, "output volume", wa.dims, wa.dtype)
    st = _stream(stream)
    band = volume_like(wa.dims, "complex64" if wa.dtype else "float32", x.device)
    check(lib.sfl_stream_analyze_begin(wa._h, _ptr(x), st))
    check(lib.sfl_stream_synthesize_begin(wsy._h, st))
    i, j = C.c_int32(), C.c_int32()
    while check(lib.sfl_stream_analyze_next(wa._h, _ptr(band), C.byref(i), st)) != _lib.SFL_DONE:
        check(lib.sfl_stream_synthesize_next_index(wsy._h, C.byref(j)))
        out = f(i.value, band)
        out = band if out is None else out
        _check_device_array(out, f"processed subband {i.value}", wa.dims, wa.dtype)
        check(lib.sfl_stream_synthesize_push(wsy._h, _ptr(out), st))
    check(lib.sfl_stream_synthesize_end(wsy._h, _ptr(y), st))
    return y


# ── the standalone directional banks (src/directional/ndfb.jl, hourglass.jl) ─


def ndfb_decompose(ws, x, stream=None):
    """All 3 * 2^levels subbands of x, as one (n1, n2, n3, S) array (subband
    idx at [..., idx-1]).  src/directional/ndfb.jl:263-285"""
    if not isinstance(ws, Workspace) or not isinstance(ws.transform, NDFB):
        raise ArgumentError("ndfb_decompose needs an NDFB workspace")
    return analyze(ws, x, stream=stream)


def ndfb_reconstruct(ws, c, stream=None):
    """src/directional/ndfb.jl:384-410"""
    if not isinstance(ws, Workspace) or not isinstance(ws.transform, NDFB):
        raise ArgumentError("ndfb_reconstruct needs an NDFB workspace")
    return synthesize(ws, c, stream=stream)


def hourglass_decompose(ws, x, stream=None):
    """(s1, s2, s3).  src/directional/hourglass.jl:330-358"""
    if not isinstance(ws, Workspace) or not isinstance(ws.transform, NDFB) or ws.transform.levels != 0:
        raise ArgumentError("hourglass_decompose needs a HourglassFB workspace")
    c = analyze(ws, x, stream=stream)
    return tuple(c[..., i] for i in range(3))


def hourglass_reconstruct(ws, subbands, stream=None):
    """src/directional/hourglass.jl:435-459"""
    if not isinstance(ws, Workspace) or not isinstance(ws.transform, NDFB) or ws.transform.levels != 0:
        raise ArgumentError("hourglass_reconstruct needs a HourglassFB workspace")
    if len(subbands) != 3:
        raise ArgumentError(f"a hourglass bank has 3 subbands, got {len(subbands)}")
    for i, b in enumerate(subbands, start=1):
        if tuple(b.shape) != ws.dims:
            raise DimensionMismatch(f"subband {i} has size {tuple(b.shape)}, expected {ws.dims}")
    if torch is not None and isinstance(subbands[0], torch.Tensor):
        c = volume_like(ws.dims + (3,), "complex64" if ws.dtype else "float32", subbands[0].device)
        for i, b in enumerate(subbands):
            c[..., i].copy_(b)
    else:
        c = np.stack([np.asarray(b) for b in subbands], axis=-1)
        c = np.asfortranarray(c)
    return synthesize(ws, c, stream=stream)


# ── soft-threshold denoiser ─────────────────────────────────────────────────


def denoise(ws, x, tau, stream=None):
    """y = synthesize(soft(analyze(x), tau)) with soft(c) = sign(c) max(|c| - tau, 0)
    per subband: tau is one threshold for every directional subband (the
    lowpass kept), or S thresholds by subband index.  Float32 volumes of an
    NSSurfacelet or NDFB workspace; on the slab pipeline no coefficient is
    written to device memory.  Bit for bit the three separate calls."""
    if not isinstance(ws, Workspace) or not isinstance(ws.transform, NSSurfacelet):
        raise ArgumentError("the denoiser needs an NSSurfacelet or NDFB workspace")
    _check_device_array(x, "volume", ws.dims, ws.dtype)
    if np.ndim(tau) == 0 and not (torch is not None and isinstance(tau, torch.Tensor) and tau.dim() > 0):
        t = torch.full((ws.nsubbands,), float(tau), dtype=torch.float32, device=x.device)
        if not isinstance(ws.transform, NDFB):
            t[0] = 0.0                   # subband 1 is the lowpass
    else:
        t = torch.as_tensor(tau, dtype=torch.float32, device=x.device).contiguous()
        if tuple(t.shape) != (ws.nsubbands,):
            raise DimensionMismatch(f"{tuple(t.shape)} thresholds, expected ({ws.nsubbands},)")
    y = volume_like(ws.dims, "float32", x.device)
    check(lib.sfl_ns_denoise(ws._h, _ptr(x), _ptr(y), _ptr(t), _stream(stream)))
    return y
