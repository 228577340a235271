"""CPU restatement of the Archive II radial assembly (TEST INFRASTRUCTURE ONLY).

Only tests/ import this module: it checks the host half of the Level II path (outbreaklab_b200/level2.py: templates,
metadata, framing) against the reference's own bytes without a GPU, by doing on the CPU what the GPU kernel
(ob_radar_level2) does: each radial = its sweep's template with the codes dropped in and the per-radial fields
patched, following _sweep_block of l2writer.py:91-158 (sequence, Julian date and milliseconds of
t0 + round-half-even(dur * i / nrad), radial number, azimuth (az0 + i * 360/nrad) mod 360 as big-endian float32,
status 3/0 on the first radial of the first/other sweeps and 4/2 on the last radial of the last/other sweeps).
"""
from __future__ import annotations

import numpy as np


def radials(header, payload: bytes):
    from outbreaklab_b200 import level2 as L2
    tpl, descs, total = L2.plan(header)
    out = np.zeros(total, np.uint8)
    pay = np.frombuffer(payload, np.uint8)
    t = np.frombuffer(tpl, np.uint8)
    for d in descs:
        n, Lr = d.nrad, d.rec_len
        arr = np.tile(t[d.tpl_off:d.tpl_off + Lr], (n, 1))
        ri = np.arange(n)
        tms = int(d.t0_ms) + np.rint(d.dur_ms * ri / n).astype(np.int64)
        days = tms // 86400000
        jd = ((days + 1) & 0xFFFF).astype(">u2")
        jms = (tms - days * 86400000).astype(">u4")
        seq = ((d.seq0 + ri) & 0xFFFF).astype(">u2")
        az = ((d.az0 + ri * (360.0 / n)) % 360.0).astype(">f4")
        status = np.ones(n, np.uint8)
        status[0] = 3 if d.ei == 0 else 0
        status[-1] = 4 if d.ei == d.nsw - 1 else 2

        def put(off, v):
            v = np.ascontiguousarray(v)
            arr[:, off:off + v.itemsize] = v.view(np.uint8).reshape(n, v.itemsize)
        put(16, seq); put(18, jd); put(20, jms)
        put(32, jms); put(36, jd); put(38, (ri + 1).astype(">u2")); put(40, az)
        arr[:, 49] = status
        for m in range(d.nmom):
            ng, at, src = d.ngates[m], d.data_at[m], d.src_off[m]
            arr[:, at:at + ng] = pay[src:src + n * ng].reshape(n, ng)
        out[d.out_off:d.out_off + n * Lr] = arr.reshape(-1)
    return out.tobytes()
