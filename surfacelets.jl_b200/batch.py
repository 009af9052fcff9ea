"""Batches of transforms replayed as one CUDA graph (sfl_batch_*).

The reference runs a batch of volumes as a loop of plain analyze!/synthesize!
calls.  Here `Batch(workspaces, inputs, outputs, op)` runs each transform once,
captures the whole sequence into a CUDA graph (distinct workspaces on up to
four concurrent branches) and `run()` replays it: one launch for the batch.
The tensors stay bound to the graph; refill the inputs in place between runs.
"""

import ctypes as C

from . import _lib
from ._lib import ArgumentError, check, lib
from .transforms import (NSSurfacelet, Workspace, _check_device_array, _coef_shape, _dims3, _ptr, _stream)

OPS = {"analyze": 0, "synthesize": 1, "adjoint_analyze": 2, "adjoint_synthesize": 3}


class Batch:
    def __init__(self, workspaces, inputs, outputs, op="analyze"):
        if op not in OPS:
            raise ArgumentError(f"unknown operator {op!r}; expected one of {sorted(OPS)}")
        n = len(workspaces)
        if n < 1 or len(inputs) != n or len(outputs) != n:
            raise ArgumentError("a batch needs as many inputs and outputs as workspaces (at least one)")
        for ws, a, b in zip(workspaces, inputs, outputs):
            if not isinstance(ws, Workspace):
                raise ArgumentError("batch members must be workspaces (make_workspace)")
            vol, coef = (a, b) if op in ("analyze", "adjoint_synthesize") else (b, a)
            _check_device_array(vol, "volume", ws.dims, ws.dtype)
            _check_device_array(coef, "coefficients", _coef_shape(ws), ws.dtype)
        self.workspaces, self.inputs, self.outputs, self.op = list(workspaces), list(inputs), list(outputs), op
        arr = C.c_void_p * n
        h = C.c_void_p()
        check(lib.sfl_batch_create(n, arr(*[w._h for w in workspaces]), arr(*[_ptr(a) for a in inputs]),
                                   arr(*[_ptr(b) for b in outputs]), OPS[op], C.byref(h)))
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
