"""NEXRAD Level II (Archive II, message 31) files from the GPU radar volume.

The reference turns the gate codes the browser uploads into Archive II on its server (l2writer.py:91-188, called from
server.py:249-284). Here the codes never leave the GPU until they are records: the radial records are assembled on
the device (ob_radar_level2: one block per radial fills the sweep's template, drops in the codes and patches the
per-radial fields), and this module builds what is shared per sweep or per file and finishes the file on the host:

  sweep_template   the radial template of one sweep (message header, message 31 data header with its block pointers,
                   volume / elevation / radial data blocks, one data-moment header per moment) and its layout
  metadata         the 134 metadata segments: 131 empty, message 3, message 5 (the VCP's tilts), message 2
  frame            bzip2 of the metadata record and of every 120-radial record, the AR2V volume header and the
                   control words (negative on the last record)

The byte layout is Archive II's (the reader, GR2Analyst, binds products to it), so the field values and their order
follow the reference's writer exactly; the output is byte-identical to l2writer.encode_volume on the same volume
(tests/test_level2.py, against the reference's own bytes in tests/golden/level2_volume.npz).
"""
from __future__ import annotations

import bz2
import ctypes as C
import os
import struct
from concurrent.futures import ThreadPoolExecutor

import numpy as np

GATE_FIRST_M, GATE_SIZE_M = 2125, 250
# data-block name, scale, offset of each moment's 8-bit code (code = value * scale + offset; 0 below threshold)
MOMENTS = {"REF": ("DREF", 2.0, 66.0), "VEL": ("DVEL", 2.0, 129.0), "SW": ("DSW ", 2.0, 129.0),
           "ZDR": ("DZDR", 16.0, 128.0), "PHI": ("DPHI", 253.0 / 360.0, 2.0), "RHO": ("DRHO", 300.0, -60.5)}
ORDER = ("REF", "VEL", "SW", "ZDR", "PHI", "RHO")
SEGMENT = 2432           # bytes of a metadata segment
RADIALS_PER_RECORD = 120
FIRST_SEQ = 10           # message sequence number of the first radial (after the metadata messages)

_POOL = ThreadPoolExecutor(max_workers=max(2, min(16, (os.cpu_count() or 4) - 2)))


def julian(epoch_ms: int):
    """(Julian day with 1970-01-01 = 1, milliseconds of the day)."""
    days = int(epoch_ms // 86400000)
    return days + 1, int(epoch_ms - days * 86400000)


def _header(buf, size_halfwords, mtype, seq, epoch_ms, nseg=1, seg=1):
    jd, jms = julian(epoch_ms)
    struct.pack_into(">HBBHHIHH", buf, 12, size_halfwords, 8, mtype, seq & 0xFFFF, jd, jms, nseg, seg)


def _ascii(s, n):
    return s.encode("ascii")[:n].ljust(n, b" ")


def _msg5(tilts, epoch_ms, seq, vcp):
    buf = bytearray(SEGMENT)
    n = len(tilts)
    data_len = 22 + 46 * n
    _header(buf, (16 + data_len) // 2, 5, seq, epoch_ms)
    struct.pack_into(">HHHHHBB", buf, 28, data_len // 2, 2, vcp, n, 1, 2, 2)
    o = 50
    for t in tilts:
        sr = bool(t.get("superRes"))
        chan, wave, sres = {"surv": (2, 1, 0x0B), "dop": (2, 2, 0x07)}.get(t.get("kind", "both"), (0, 4, 0x0E))
        struct.pack_into(">HBBBBHh", buf, o, int(round(t["angle"] * 65536 / 360)) & 0xFFFF, chan, wave, sres, 1,
                         15 if sr else 3, 15400 if sr else 17944)
        struct.pack_into(">6h", buf, o + 10, *([28] * 6))
        for k, edge in enumerate((0x1558, 0x9558, 0xEE38)):
            struct.pack_into(">HHH", buf, o + 22 + 8 * k, edge, 6, 0x1F)
        o += 46
    return bytes(buf)


def _msg2(epoch_ms, seq, vcp):
    buf = bytearray(SEGMENT)
    _header(buf, 48, 2, seq, epoch_ms)
    jd, _ = julian(epoch_ms)
    hw = (16, 2, 4, 2, 1402, 8, 28, vcp, 0, 1910, 4, 2, 63, 2, 0, 0, 0, 0, jd, 22, jd, 1308, 65512, 3)
    struct.pack_into(">%dH" % len(hw), buf, 28, *hw)
    return bytes(buf)


def metadata(tilts, epoch_ms, vcp):
    m3 = bytearray(SEGMENT)
    _header(m3, 488, 3, 1, epoch_ms)
    return bytes(SEGMENT) * 131 + bytes(m3) + _msg5(tilts, epoch_ms, 2, vcp) + _msg2(epoch_ms, 3, vcp)


def sweep_template(s, ei, icao, lat, lon, height_m, vcp, epoch_ms=0):
    """Radial template of one sweep: (bytes, [(moment, data offset, gates)]). The per-radial fields (sequence,
    Julian date and milliseconds in both headers, radial number, azimuth, status) are left for the GPU."""
    sr = bool(s.get("superRes"))
    present = [(m["name"], int(m["ngates"]), int(m["off"])) for m in sorted(s["moments"], key=lambda m: ORDER.index(m["name"]))]
    data_len = 68 + 44 + 12 + 28 + sum(28 + ng for _, ng, _ in present)
    rad_len = data_len + (data_len & 1)
    buf = bytearray(28 + rad_len)
    _header(buf, (16 + rad_len) // 2, 31, 0, int(s.get("start_ms", epoch_ms)))
    d = 28
    buf[d:d + 4] = _ascii(icao, 4)
    struct.pack_into(">IHHfBBHBBBBfBB", buf, d + 4, 0, 0, 1, 0.0, 0, 0, rad_len, 1 if sr else 2, 1, ei + 1, 1,
                     float(s["angle"]), 0, 25 if sr else 50)
    ptrs = []
    p = 68
    ptrs.append(p)
    buf[d + p:d + p + 4] = b"RVOL"
    struct.pack_into(">HBBffhHfffffHH", buf, d + p + 4, 44, 2, 0, lat, lon, int(round(height_m)), 20, -43.1, 267.0, 258.0,
                     0.44, 60.0, vcp, 1)
    p += 44
    ptrs.append(p)
    buf[d + p:d + p + 4] = b"RELV"
    struct.pack_into(">Hhf", buf, d + p + 4, 12, -12, -42.5)
    p += 12
    ptrs.append(p)
    buf[d + p:d + p + 4] = b"RRAD"
    struct.pack_into(">HhffhHff", buf, d + p + 4, 28, int(round(float(s.get("unamb_km", 466.0)) * 10)), -80.4, -80.8,
                     int(round(float(s.get("nyquist", 63.5)) * 100)), 0, -42.6, -42.3)
    p += 28
    layout = []
    for name, ng, off in present:
        block, scale, offset = MOMENTS[name]
        ptrs.append(p)
        buf[d + p:d + p + 4] = block.encode("ascii")
        struct.pack_into(">IHHHHhBBff", buf, d + p + 4, 0, ng, GATE_FIRST_M, GATE_SIZE_M, 50, 16, 0, 8, scale, offset)
        layout.append((name, d + p + 28, ng, off))
        p += 28 + ng
    struct.pack_into(">H", buf, d + 30, len(ptrs))
    for k, pp in enumerate(ptrs):
        struct.pack_into(">I", buf, d + 32 + 4 * k, pp)
    return bytes(buf), layout


def frame(icao, epoch_ms, records):
    """The Archive II file: AR2V volume header, then each record bzip2-compressed behind its control word (the last
    one negative)."""
    jd, jms = julian(epoch_ms)
    parts = [b"AR2V0006.001" + struct.pack(">ii", jd, jms) + _ascii(icao, 4)]
    comp = list(_POOL.map(lambda r: bz2.compress(r, 5), records))
    for i, c in enumerate(comp):
        parts.append(struct.pack(">i", -len(c) if i == len(comp) - 1 else len(c)))
        parts.append(c)
    return b"".join(parts)


class ObL2Sweep(C.Structure):
    _fields_ = [("tpl_off", C.c_uint64), ("out_off", C.c_uint64), ("rec_len", C.c_uint32), ("nrad", C.c_uint32),
                ("nmom", C.c_uint32), ("seq0", C.c_uint32), ("ei", C.c_uint32), ("nsw", C.c_uint32),
                ("t0_ms", C.c_double), ("dur_ms", C.c_double), ("az0", C.c_double), ("data_at", C.c_uint32 * 6),
                ("ngates", C.c_uint32 * 6), ("src_off", C.c_uint64 * 6)]


def plan(header):
    """Templates and sweep descriptors of a volume header (the /api/volume header, app.js:1743-1758)."""
    icao, lat, lon, elev, vcp = header["icao"], float(header["lat"]), float(header["lon"]), float(header["elev"]), int(header.get("vcp", 212))
    sweeps = header["sweeps"]
    tpls, descs = [], []
    tpl_off = out_off = 0
    seq = FIRST_SEQ
    for ei, s in enumerate(sweeps):
        tpl, layout = sweep_template(s, ei, icao, lat, lon, elev, vcp, int(header["epoch_ms"]))
        d = ObL2Sweep()
        d.tpl_off, d.out_off, d.rec_len, d.nrad, d.nmom = tpl_off, out_off, len(tpl), int(s["nrad"]), len(layout)
        d.seq0, d.ei, d.nsw = seq, ei, len(sweeps)
        d.t0_ms = float(int(s.get("start_ms", header["epoch_ms"])))
        d.dur_ms, d.az0 = float(s.get("dur_ms", 15000)), float(s.get("az0", 0.0))
        for m, (_, at, ng, off) in enumerate(layout):
            d.data_at[m], d.ngates[m], d.src_off[m] = at, ng, off
        tpls.append(tpl)
        descs.append(d)
        tpl_off += len(tpl)
        out_off += len(tpl) * int(s["nrad"])
        seq += int(s["nrad"])
    return b"".join(tpls), descs, out_off


def records_of(header, radials: bytes):
    """The uncompressed records of a volume: the metadata record, then the radials 120 at a time per sweep."""
    tilts = [{"angle": s["angle"], "superRes": bool(s.get("superRes")), "kind": s.get("kind", "both")} for s in header["sweeps"]]
    recs = [metadata(tilts, int(header["epoch_ms"]), int(header.get("vcp", 212)))]
    _, descs, _ = plan(header)
    for d in descs:
        for i in range(0, d.nrad, RADIALS_PER_RECORD):
            a = d.out_off + i * d.rec_len
            recs.append(radials[a:a + min(RADIALS_PER_RECORD, d.nrad - i) * d.rec_len])
    return recs


def encode_volume_gpu(radar_handle, header) -> bytes:
    """Archive II bytes of the volume held by a radar (ob_radar_*), whose sweeps and moment offsets the header
    lists: the radial records come from the GPU (ob_radar_level2), the framing from the host."""
    from . import _native as N
    tpl, descs, total = plan(header)
    arr = (ObL2Sweep * len(descs))(*descs)
    out = np.empty(total, np.uint8)
    t = np.frombuffer(tpl, np.uint8)
    N.check(N.lib().ob_radar_level2(radar_handle, arr, len(descs), t.ctypes.data, t.nbytes, out.ctypes.data, out.nbytes))
    return frame(header["icao"], int(header["epoch_ms"]), records_of(header, out.tobytes()))


def archive_name(icao, epoch_ms):
    """File name of a volume, as the server names them (l2writer.py:185-188)."""
    import datetime as dt
    t = dt.datetime.fromtimestamp(epoch_ms / 1000.0, dt.timezone.utc)
    return "%s%s_V06" % (icao.upper(), t.strftime("%Y%m%d_%H%M%S"))
