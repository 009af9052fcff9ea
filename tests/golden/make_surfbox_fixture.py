"""Re-encode the reference's SurfBox golden data as a JSON fixture.

Reads test/reference/surfbox_irc.{txt,bin} of hakkelt/Surfacelets.jl (MATLAB
outputs of SurfBox written by the reference's test/reference/gen_surfbox_irc.m:
little-endian float64 records, one index line `name kind ndims dims...` each)
and writes tests/golden/surfbox_irc.json with the same records.  Run it where
the reference checkout is available:

    python tests/golden/make_surfbox_fixture.py /path/to/Surfacelets.jl
"""

import json
import os
import sys

import numpy as np

COMPLEX_PREFIXES = ("hg_", "irc_", "pyr_")   # test/items/test_irc.jl:35


def main(ref_root):
    d = os.path.join(ref_root, "test", "reference")
    raw = open(os.path.join(d, "surfbox_irc.bin"), "rb").read()
    vals = np.frombuffer(raw, dtype="<f8")
    pos = 0
    out = {}
    for ln in open(os.path.join(d, "surfbox_irc.txt")):
        f = ln.split()
        if not f:
            continue
        name, kind, nd = f[0], f[1], int(f[2])
        size = [int(v) for v in f[3:3 + nd]]
        if kind == "full":
            cnt = int(np.prod(size))
            out[name] = {"kind": "full", "size": size, "data": vals[pos:pos + cnt].tolist()}
        else:
            cnt = 5 if name.startswith(COMPLEX_PREFIXES) else 3
            out[name] = {"kind": "fp", "size": size, "fp": vals[pos:pos + cnt].tolist()}
        pos += cnt
    assert pos == vals.size, (pos, vals.size)
    dst = os.path.join(os.path.dirname(os.path.abspath(__file__)), "surfbox_irc.json")
    with open(dst, "w") as f:
        json.dump(out, f, separators=(",", ":"))
    print(f"wrote {len(out)} records to {dst}")


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else "/root/reference")
