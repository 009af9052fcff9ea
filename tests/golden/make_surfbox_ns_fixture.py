"""Re-encode the reference's SurfBox golden data for the nonsubsampled banks.

Reads two files of hakkelt/Surfacelets.jl's test/reference/ (MATLAB outputs of
SurfBox, written by the reference's gen_surfbox_golden.m and
gen_surfbox_directions.m) and writes tests/golden/surfbox_ns.json:

- surfbox_hourglass_32.bin: the first hourglass analysis mask of SurfBox's
  HourGlassDec on a 32^3 grid, restricted to the non-negative-frequency octant,
  17 x 17 x 17 little-endian float32, column-major
  (test/items/test_surfbox_reference.jl:17-22);
- surfbox_directions_32.bin: 80 unit direction vectors (3 x 80) followed by 80
  subband labels, little-endian float64, column-major: for each direction, the
  SurfBox NDFB subband (of 12, levels 2) holding the most energy of a plane
  wave along it (test/items/test_surfbox_reference.jl:106-115).

The values are kept exactly: float32 octant values and float64 directions are
written with repr (round-trip exact).  Run it where the reference checkout is
available:

    python tests/golden/make_surfbox_ns_fixture.py /path/to/Surfacelets.jl
"""

import json
import os
import sys

import numpy as np


def main(ref_root):
    d = os.path.join(ref_root, "test", "reference")
    oct_ = np.frombuffer(open(os.path.join(d, "surfbox_hourglass_32.bin"), "rb").read(), dtype="<f4")
    assert oct_.size == 17 ** 3, oct_.size
    raw = np.frombuffer(open(os.path.join(d, "surfbox_directions_32.bin"), "rb").read(), dtype="<f8")
    nd = 80
    assert raw.size == 4 * nd, raw.size
    out = {
        # column-major 17^3 octant, flattened in Julia's memory order
        "hourglass_octant": {"size": [17, 17, 17], "data": [float(v) for v in oct_]},
        # dirs[:, t] is direction t (column-major 3 x 80)
        "directions": {"size": [3, nd], "data": [float(v) for v in raw[:3 * nd]]},
        "labels": [int(v) for v in raw[3 * nd:]],
    }
    dst = os.path.join(os.path.dirname(os.path.abspath(__file__)), "surfbox_ns.json")
    with open(dst, "w") as f:
        json.dump(out, f, separators=(",", ":"))
    print(f"wrote {dst}")


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else "/root/reference")
