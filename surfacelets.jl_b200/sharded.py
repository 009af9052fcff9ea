"""NSSurfacelet subbands sharded across the ranks of a torch.distributed
process group: one process per GPU, NCCL over NVLink on B200s.

    analysis   the root computes the spectrum X of the volume once and
               broadcasts it (8 B a bin on the rfft grid, about 4 B a voxel);
               every rank analyzes its own contiguous range of subbands
               (stream positions) from it;
    synthesis  every rank accumulates its range into a partial spectrum; one
               sum-reduction to the root, whose inverse spectrum is the volume.

The transform runs through `LibRanges` (the item-range entry points of
libsurfacelets_b200); any object with the same methods can stand in for it,
which is how the host logic is tested on CPU ranks with the float64 oracle.
A batch of volumes needs none of this: ranks take whole volumes (replicas).
"""

import ctypes as C

from ._lib import ArgumentError, check, lib
from .transforms import NSSurfacelet, Workspace, _check_device_array, _ptr, _stream, volume_like

try:
    import torch
    import torch.distributed as dist
except ImportError:     # pragma: no cover
    torch = dist = None


def shard(nitems, world, rank):
    """(first, count) of rank's contiguous share of nitems positions; shares
    differ by at most one, lower ranks take the larger ones."""
    if world < 1 or not 0 <= rank < world:
        raise ArgumentError(f"rank {rank} outside a group of {world}")
    q, r = divmod(nitems, world)
    first = rank * q + min(rank, r)
    return first, q + (1 if rank < r else 0)


class LibRanges:
    """Item-range operations of one NSSurfacelet workspace (slab or line pipeline)."""

    def __init__(self, ws, stream=None):
        if not isinstance(ws, Workspace) or not isinstance(ws.transform, NSSurfacelet):
            raise ArgumentError("item ranges need an NSSurfacelet workspace")
        self.ws, self.stream = ws, stream
        e = C.c_int64()
        check(lib.sfl_ns_spectrum_elems(ws._h, C.byref(e)))
        self.spectrum_elems = e.value
        order = (C.c_int32 * ws.nsubbands)()
        check(lib.sfl_ns_stream_order(ws._h, order))
        self.stream_order = list(order)
        self.nsubbands, self.dims = ws.nsubbands, ws.dims
        self.nch = 2 if ws.dtype else 1

    def _dt(self):
        return "complex64" if self.nch == 2 else "float32"

    def new_spectrum(self, device="cuda"):
        return torch.empty(self.nch * self.spectrum_elems, dtype=torch.complex64, device=device)

    def new_volume(self, device="cuda"):
        return volume_like(self.dims, self._dt(), device)

    def new_subbands(self, count, device="cuda"):
        return volume_like(self.dims + (count,), self._dt(), device)

    def forward_spectrum(self, x, X):
        _check_device_array(x, "volume", self.dims, self.ws.dtype)
        check(lib.sfl_ns_forward_spectrum(self.ws._h, _ptr(x), _ptr(X), _stream(self.stream)))

    def analyze_range(self, X, first, count, c):
        check(lib.sfl_ns_analyze_range(self.ws._h, _ptr(X), first, count, _ptr(c), _stream(self.stream)))

    def accumulate_range(self, c, first, count, A, clear):
        check(lib.sfl_ns_accumulate_range(self.ws._h, _ptr(c), first, count, _ptr(A), 1 if clear else 0,
                                          _stream(self.stream)))

    def inverse_spectrum(self, A, x):
        check(lib.sfl_ns_inverse_spectrum(self.ws._h, _ptr(A), _ptr(x), _stream(self.stream)))


def _group(group):
    return dist.get_rank(group), dist.get_world_size(group)


def analyze_sharded(ops, x, group=None, root=0, device="cuda"):
    """This rank's subbands of x: returns (c_local, first), c_local holding the
    subbands at stream positions first, first + 1, ... (subband indices
    ops.stream_order[first:first + count]).  x is read on the root only."""
    rank, world = _group(group)
    X = ops.new_spectrum(device)
    if rank == root:
        ops.forward_spectrum(x, X)
    dist.broadcast(X, src=dist.get_global_rank(group, root) if group is not None else root, group=group)
    first, count = shard(ops.nsubbands, world, rank)
    c = ops.new_subbands(count, device)
    if count:
        ops.analyze_range(X, first, count, c)
    return c, first


def synthesize_sharded(ops, c_local, first, group=None, root=0, device="cuda"):
    """The volume from every rank's subbands (as analyze_sharded left them):
    returned on the root, None elsewhere."""
    rank, world = _group(group)
    f, count = shard(ops.nsubbands, world, rank)
    if f != first or tuple(c_local.shape[-1:]) != (count,):
        raise ArgumentError(f"rank {rank} holds subbands from {first} ({tuple(c_local.shape)}), "
                            f"its share is {count} from {f}")
    A = ops.new_spectrum(device)
    if count:
        ops.accumulate_range(c_local, first, count, A, True)
    else:
        A.zero_()
    dist.reduce(A, dst=dist.get_global_rank(group, root) if group is not None else root, op=dist.ReduceOp.SUM,
                group=group)
    if rank != root:
        return None
    x = ops.new_volume(device)
    ops.inverse_spectrum(A, x)
    return x
