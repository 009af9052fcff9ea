"""FP64 CPU oracle for the surfacelet analyze/synthesize path.

TEST INFRASTRUCTURE ONLY.  This package is a NumPy restatement, in float64, of
the algorithms of hakkelt/Surfacelets.jl (a pure-Julia package) for the
`NSSurfacelet` and decimated `Surfacelet` transforms.  Every function cites the
reference file and line it follows.  Only `tests/`, `__graft_entry__.smoke()`
and `bench.py` (its `cpu_baseline` leg and its `--impl reference` arm) may
import it, and there only as the checker or as the timed CPU baseline; the
product path (the CUDA library and its Python host mirror) never calls it.

Pinning:
  * decimated transform: pinned coefficient-for-coefficient to the SurfBox
    golden fingerprints that the reference's own test suite carries
    (test/reference/surfbox_irc.{bin,txt}, re-encoded under tests/golden/);
  * nonsubsampled transform: the reference ships no golden coefficients; its
    hourglass and NDFB banks are pinned to the SurfBox golden data the
    reference's suite carries for them (test/reference/surfbox_hourglass_32.bin
    and surfbox_directions_32.bin: the hourglass partition and the 12-wedge
    direction partition, re-encoded under tests/golden/), and the whole
    transform through the reference's component and property tests
    (partition of unity, Parseval, perfect reconstruction, mask evenness,
    sharpness figures, plane-wave wedge predictions, wedge-centre share).

Julia's column-major axis order is kept: a volume is a NumPy array of shape
(n1, n2, n3) whose axis 0 is the reference's axis 1 (the fastest in memory).
"""

from . import filters, ns, decimated, golden  # noqa: F401
