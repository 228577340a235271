"""Writes tests/golden/level2_volume.npz: a small synthetic radar volume (the /api/volume header and payload the
browser sends, app.js:1743-1758) and the Archive II bytes the reference's own writer makes from it
(l2writer.encode_volume, l2writer.py:161-182).

Run in a container where the reference is mounted (it imports l2writer.py from there, read-only):
    python tests/golden/make_level2_volume.py <path to the reference checkout>
(or with the path in the OUTBREAKLAB_REF environment variable).
Three sweeps cover the writer's cases: a super-resolution surveillance cut (REF, ZDR, PHI, RHO), its Doppler pair
(VEL, SW) and a legacy-resolution cut with all six moments; gate codes are seeded, mostly zero like real volumes.
"""
import json
import os
import sys

import numpy as np

ref = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("OUTBREAKLAB_REF")
if not ref or not os.path.isfile(os.path.join(ref, "l2writer.py")):
    sys.exit("usage: %s <path to the reference checkout holding l2writer.py> (or set OUTBREAKLAB_REF)" % sys.argv[0])
sys.path.insert(0, ref)
import l2writer  # noqa: E402

rng = np.random.default_rng(2024)
epoch_ms = 1714586400000 + 1234
sweeps_spec = [
    dict(angle=0.5, superRes=True, kind="surv", az0=12.25, nrad=72, nyquist=63.5, unamb_km=466,
         start_ms=epoch_ms, dur_ms=24999, moments=[("REF", 100), ("ZDR", 100), ("PHI", 100), ("RHO", 100)]),
    dict(angle=0.5, superRes=True, kind="dop", az0=12.25, nrad=72, nyquist=27.5, unamb_km=300,
         start_ms=epoch_ms + 25000, dur_ms=25003, moments=[("VEL", 60), ("SW", 60)]),
    dict(angle=1.45, superRes=False, kind="both", az0=200.5, nrad=36, nyquist=26.25, unamb_km=300,
         start_ms=epoch_ms + 50000, dur_ms=17000,
         moments=[("REF", 80), ("VEL", 50), ("SW", 50), ("ZDR", 80), ("PHI", 80), ("RHO", 80)]),
]
payload = bytearray()
header = {"run": "golden", "icao": "KTLX", "lat": 35.3331, "lon": -97.2778, "elev": 390.0, "vcp": 212,
          "epoch_ms": epoch_ms, "sweeps": []}
for s in sweeps_spec:
    hs = {k: v for k, v in s.items() if k != "moments"}
    hs["moments"] = []
    for name, ng in s["moments"]:
        codes = rng.integers(2, 256, size=s["nrad"] * ng).astype(np.uint8)
        codes[rng.random(codes.size) < 0.7] = 0
        hs["moments"].append({"name": name, "ngates": ng, "off": len(payload)})
        payload += codes.tobytes()
        while len(payload) % 4:
            payload += b"\0"
    header["sweeps"].append(hs)

# the server's unpacking of /api/volume (server.py:256-266), then the reference writer
sw = []
for s in header["sweeps"]:
    mom = {m["name"]: (bytes(payload[m["off"]:m["off"] + s["nrad"] * m["ngates"]]), m["ngates"]) for m in s["moments"]}
    d = dict(s)
    d["moments"] = mom
    sw.append(d)
archive = l2writer.encode_volume(header["icao"], header["lat"], header["lon"], header["elev"], header["epoch_ms"], sw,
                                 header["vcp"])
out = os.path.join(os.path.dirname(os.path.abspath(__file__)), "level2_volume.npz")
np.savez_compressed(out, header=np.frombuffer(json.dumps(header).encode(), np.uint8),
                    payload=np.frombuffer(bytes(payload), np.uint8), archive=np.frombuffer(archive, np.uint8))
print(out, len(payload), len(archive))
