"""surfacelets_b200 — B200 (sm_100a) analyze/synthesize for the 3-D
surfacelet transforms of Surfacelets.jl: the nonsubsampled, Parseval
`NSSurfacelet` and the decimated `Surfacelet` (SurfBox's construction).

The compute path is libsurfacelets_b200.so (hand-written CUDA kernels behind
a C ABI, include/surfacelets_b200.h); this package is the host mirror of the
reference's AbstractMultiscaleTransforms interface over it.  There is no CPU
fallback: importing the package fails if the library is missing.
"""

from .autograd import analyze_ad, as_colmajor, synthesize_ad  # noqa: F401
from .batch import Batch  # noqa: F401
from .sharded import LibRanges, analyze_sharded, shard, synthesize_sharded  # noqa: F401
from ._lib import ArgumentError, CudaError, DimensionMismatch, LIB_PATH, StateError, DeviceWaitTimeout, lib  # noqa: F401
from .transforms import (  # noqa: F401
    NDFB, HourglassFB, NSSurfacelet, Surfacelet, Workspace, adjoint_analyze, hourglass_decompose,
    hourglass_reconstruct, ndfb_decompose, ndfb_reconstruct, ndfb_subband_index, ndfb_subband_triple, adjoint_analyze_, adjoint_synthesize,
    adjoint_synthesize_, analyze, analyze_, analyze_bf16, denoise, analyze_synthesize_stream, synthesize_bf16, checkerboard_orders, make_workspace, nsubbands,
    similar_coefficients, subband, subband_layout, subband_sizes, supports_streaming, surfacelet_redundancy,
    synthesize, synthesize_, to_device, to_host, volume_like,
)


def version():
    return lib.sfl_version().decode()
