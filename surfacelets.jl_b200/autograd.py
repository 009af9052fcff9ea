"""Differentiable analyze / synthesize for torch (the counterpart of
ChainRulesCore rrules on the Julia side).

The transforms are real-linear and act on complex data channel by channel
with real operators, so the vector-Jacobian product of analyze is the adjoint
of analysis and that of synthesize the adjoint of synthesis, channel by
channel, under torch's convention for complex gradients (the gradient of a
real loss packs d/dRe + i d/dIm).  For a tight NSSurfacelet the adjoints are
synthesize and analyze themselves.
"""

from .transforms import (Workspace, adjoint_analyze_, adjoint_synthesize_, analyze_, similar_coefficients,
                         synthesize_, volume_like)

try:
    import torch
except ImportError:     # pragma: no cover - the module needs torch
    torch = None


def as_colmajor(t):
    """The same values in the column-major layout the library expects."""
    if t.dim() <= 1:
        return t.contiguous()
    rev = tuple(reversed(range(t.dim())))
    return t.permute(*rev).contiguous().permute(*rev)


class _Analyze(torch.autograd.Function if torch is not None else object):
    @staticmethod
    def forward(ctx, x, ws):
        ctx.ws = ws
        x = as_colmajor(x.detach())
        c = similar_coefficients(ws.transform, x)
        return analyze_(c, ws, x)

    @staticmethod
    def backward(ctx, gc):
        ws = ctx.ws
        gx = volume_like(ws.dims, "complex64" if gc.is_complex() else "float32", gc.device)
        return adjoint_analyze_(gx, ws, as_colmajor(gc)), None


class _Synthesize(torch.autograd.Function if torch is not None else object):
    @staticmethod
    def forward(ctx, c, ws):
        ctx.ws = ws
        x = volume_like(ws.dims, "complex64" if c.is_complex() else "float32", c.device)
        return synthesize_(x, ws, as_colmajor(c.detach()))

    @staticmethod
    def backward(ctx, gx):
        ws = ctx.ws
        gx = as_colmajor(gx)
        gc = similar_coefficients(ws.transform, gx)
        return adjoint_synthesize_(gc, ws, gx), None


def analyze_ad(ws, x):
    """analyze(ws, x) recorded for torch autograd."""
    if not isinstance(ws, Workspace):
        raise TypeError("analyze_ad needs a workspace (make_workspace)")
    return _Analyze.apply(x, ws)


def synthesize_ad(ws, c):
    """synthesize(ws, c) recorded for torch autograd."""
    if not isinstance(ws, Workspace):
        raise TypeError("synthesize_ad needs a workspace (make_workspace)")
    return _Synthesize.apply(c, ws)
