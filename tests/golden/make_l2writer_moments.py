"""Writes tests/golden/l2writer_moments.json from the reference's own Level II writer (l2writer.py:14-27).

Run in a container where the reference is mounted (it imports l2writer.py from there, read-only):
    python tests/golden/make_l2writer_moments.py <path to the reference checkout>
(or with the path in the OUTBREAKLAB_REF environment variable).
The radar kernels quantise each moment with code = round(value * scale + offset); l2writer.py decodes the same
bytes with the same table, so the two must agree exactly.
"""
import json
import os
import sys

ref = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("OUTBREAKLAB_REF")
if not ref or not os.path.isfile(os.path.join(ref, "l2writer.py")):
    sys.exit("usage: %s <path to the reference checkout holding l2writer.py> (or set OUTBREAKLAB_REF)" % sys.argv[0])
sys.path.insert(0, ref)
import l2writer  # noqa: E402

out = {"GATE_FIRST_M": l2writer.GATE_FIRST_M, "GATE_SIZE_M": l2writer.GATE_SIZE_M,
       "MOMENTS": {k: {"block": v[0], "scale": v[1], "offset": v[2]} for k, v in l2writer.MOMENTS.items()},
       "MOMENT_ORDER": l2writer.MOMENT_ORDER}
with open(os.path.join(os.path.dirname(os.path.abspath(__file__)), "l2writer_moments.json"), "w") as f:
    json.dump(out, f, indent=1, sort_keys=True)
