"""Batches of transforms replayed as one CUDA graph (sfl_batch_*).

The reference runs a batch of volumes as a loop of plain analyze!/synthesize!
calls.  Here `Batch(workspaces, inputs, outputs, ops)` runs each entry once,
captures the whole sequence into a CUDA graph (distinct workspaces on up to
eight concurrent branches, dealt out largest first to the least-loaded branch;
the entries of one workspace keep their order, so one entry may consume
another's output) and `run()` replays it: one launch for the batch.  The tensors stay bound to the graph; refill the inputs in
place between runs.
"""

import ctypes as C

from . import _lib
import numpy as np

from ._lib import ArgumentError, DimensionMismatch, check, lib
from .transforms import (NSSurfacelet, Workspace, _check_device_array, _coef_shape, _dims3, _ptr, _stream)

OPS = {"analyze": 0, "synthesize": 1, "adjoint_analyze": 2, "adjoint_synthesize": 3, "copy_volume": 4}


class Batch:
    """ops: one operator name for every entry, or one per entry."""

    def __init__(self, workspaces, inputs, outputs, ops="analyze"):
        n = len(workspaces)
        ops = [ops] * n if isinstance(ops, str) else list(ops)
        if n < 1 or len(inputs) != n or len(outputs) != n or len(ops) != n:
            raise ArgumentError("a batch needs as many operators, inputs and outputs as workspaces (at least one)")
        for ws, op, a, b in zip(workspaces, ops, inputs, outputs):
            if op not in OPS:
                raise ArgumentError(f"unknown operator {op!r}; expected one of {sorted(OPS)}")
            if not isinstance(ws, Workspace):
                raise ArgumentError("batch members must be workspaces (make_workspace)")
            if op == "copy_volume":
                # a volume between device memory and pinned host memory (or device to device)
                for t in (a, b):
                    if t.numel() != int(np.prod(ws.dims)) or t.element_size() != (8 if ws.dtype else 4):
                        raise DimensionMismatch(f"copy_volume needs {ws.dims} volumes of the workspace's type")
                    if not t.is_cuda and not t.is_pinned():
                        raise ArgumentError("copy_volume needs pinned host memory")
                continue
            vol, coef = (a, b) if op in ("analyze", "adjoint_synthesize") else (b, a)
            _check_device_array(vol, "volume", ws.dims, ws.dtype)
            _check_device_array(coef, "coefficients", _coef_shape(ws), ws.dtype)
        self.workspaces, self.inputs, self.outputs, self.ops = list(workspaces), list(inputs), list(outputs), ops
        arr = C.c_void_p * n
        h = C.c_void_p()
        check(lib.sfl_batch_create(n, arr(*[w._h for w in workspaces]), (C.c_int32 * n)(*[OPS[o] for o in ops]),
                                   arr(*[_ptr(a) for a in inputs]), arr(*[_ptr(b) for b in outputs]), C.byref(h)))
        self._h = h

    def run(self, stream=None):
        check(lib.sfl_batch_run(self._h, _stream(stream)))
        return self.outputs

    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            check(lib.sfl_batch_destroy(self._h))
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
