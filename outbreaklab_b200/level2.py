"""NEXRAD Level II (Archive II, message 31) files from the GPU radar volume.

The reference turns the gate codes the browser uploads into Archive II on its server (l2writer.py:91-188, called from
server.py:249-284). Here the codes never leave the GPU until they are records: the radial records are assembled on
the device (ob_radar_level2: one block per radial copies its sweep's template, drops in the codes and patches the
per-radial fields), and this module builds what is shared per sweep or per file and finishes the file on the host.

Every Archive II structure is written from a ``Layout``: a table of its fields in order, each a big-endian struct
code with either a constant or a value the caller supplies. The layouts are the format's (the reader, GR2Analyst,
binds to these offsets and to the reference writer's constants), and they are the single description that the sweep
templates for the GPU, the metadata messages and the file header are all packed from. The per-radial fields the GPU
patches (sequence, Julian date, milliseconds, radial number, azimuth, status) sit at the offsets these tables give;
``RADIAL_PATCH`` lists them, and the kernel writes them at the same places. The output is byte-identical to the
reference writer's on the same volume (tests/test_level2.py, against tests/golden/level2_volume.npz).

File structure: the 24-byte volume header, then records, each bzip2-compressed (level 5) behind a 4-byte length
(negative on the last record). The first record holds the 134 metadata segments of 2432 bytes (131 empty, then
messages 3, 5 and 2); the others hold up to 120 radials of one sweep each.
"""
from __future__ import annotations

import bz2
import ctypes as C
import os
import struct
import time

import numpy as np

# The moment code table (l2writer.py:19-27): data-block name, scale, offset (code = value * scale + offset; 0 means
# below threshold). The radar kernels quantise with the same table (radar.js:21).
GATE_FIRST_M, GATE_SIZE_M = 2125, 250
MOMENTS = {"REF": ("DREF", 2.0, 66.0), "VEL": ("DVEL", 2.0, 129.0), "SW": ("DSW ", 2.0, 129.0),
           "ZDR": ("DZDR", 16.0, 128.0), "PHI": ("DPHI", 253.0 / 360.0, 2.0), "RHO": ("DRHO", 300.0, -60.5)}
ORDER = ("REF", "VEL", "SW", "ZDR", "PHI", "RHO")
SEGMENT = 2432            # bytes of a metadata segment
METADATA_SEGMENTS = 134
RADIALS_PER_RECORD = 120
FIRST_SEQ = 10            # message sequence number of the first radial (after the metadata messages)
MAX_BLOCKS = 9            # data-block pointers of a message 31: volume, elevation, radial + six moments


class Layout:
    """A fixed binary structure: (field, struct code[, constant]) in order, big-endian."""

    def __init__(self, name, fields):
        self.name = name
        self.fields = [(f[0], f[1], f[2] if len(f) > 2 else None) for f in fields]
        self.fmt = ">" + "".join(code for _, code, _ in self.fields)
        self.size = struct.calcsize(self.fmt)
        self._offset = {}
        at = 0
        for fname, code, _ in self.fields:
            self._offset[fname] = at
            at += struct.calcsize(">" + code)

    def offset(self, field):
        return self._offset[field]

    def values(self, given):
        """The flat value list for the struct format: constants where the table has them, else the given value; an
        array field ("6h") takes a sequence, a text field ("4s") a str."""
        out = []
        for fname, code, const in self.fields:
            if code.endswith("x"):
                continue
            v = const if const is not None else given[fname]
            if code.endswith("s"):
                out.append(v.encode("ascii") if isinstance(v, str) else v)
            elif code[:-1].isdigit() and int(code[:-1]) > 1:
                out.extend(v)
            else:
                out.append(v)
        return out

    def pack_into(self, buf, at, **given):
        unknown = set(given) - set(self._offset)
        if unknown:
            raise KeyError("%s has no field %s" % (self.name, sorted(unknown)))
        struct.pack_into(self.fmt, buf, at, *self.values(given))
        return at + self.size


def text(s, n):
    """An n-byte ASCII field, space padded."""
    return s[:n].ljust(n, " ")


# ---- record and message headers ----
VOLUME_HEADER = Layout("volume header", [("tape", "12s", "AR2V0006.001"), ("jdate", "i"), ("jms", "i"), ("icao", "4s")])
MESSAGE_HEADER = Layout("message header", [
    ("ctm", "12x"), ("size_hw", "H"), ("channel", "B", 8), ("type", "B"), ("seq", "H"), ("jdate", "H"), ("jms", "I"),
    ("nseg", "H", 1), ("seg", "H", 1)])

# ---- message 31: data header, then the blocks its pointers name ----
M31_HEADER = Layout("message 31 header", [
    ("icao", "4s"), ("jms", "I"), ("jdate", "H"), ("radial", "H"), ("azimuth", "f"), ("compression", "B", 0),
    ("spare", "B", 0), ("radial_len", "H"), ("az_spacing", "B"), ("status", "B"), ("elev_num", "B"),
    ("cut_sector", "B", 1), ("elevation", "f"), ("spot_blank", "B", 0), ("az_index", "B"), ("nblocks", "H"),
    ("pointers", "%dI" % MAX_BLOCKS)])
VOLUME_BLOCK = Layout("volume block", [
    ("name", "4s", "RVOL"), ("size", "H", 44), ("major", "B", 2), ("minor", "B", 0), ("lat", "f"), ("lon", "f"),
    ("height", "h"), ("feedhorn", "H", 20), ("calibration", "f", -43.1), ("tx_h", "f", 267.0), ("tx_v", "f", 258.0),
    ("zdr_cal", "f", 0.44), ("phase", "f", 60.0), ("vcp", "H"), ("processing", "H", 1)])
ELEVATION_BLOCK = Layout("elevation block", [("name", "4s", "RELV"), ("size", "H", 12), ("atmos", "h", -12),
                                             ("calibration", "f", -42.5)])
RADIAL_BLOCK = Layout("radial block", [
    ("name", "4s", "RRAD"), ("size", "H", 28), ("unamb_range", "h"), ("noise_h", "f", -80.4),
    ("noise_v", "f", -80.8), ("nyquist", "h"), ("spare", "H", 0), ("cal_h", "f", -42.6), ("cal_v", "f", -42.3)])
MOMENT_BLOCK = Layout("moment block", [
    ("name", "4s"), ("reserved", "I", 0), ("ngates", "H"), ("first_gate", "H", GATE_FIRST_M),
    ("gate_size", "H", GATE_SIZE_M), ("threshold", "H", 50), ("snr_threshold", "h", 16), ("control", "B", 0),
    ("word_size", "B", 8), ("scale", "f"), ("offset", "f")])

# ---- metadata messages ----
M5_HEADER = Layout("message 5 header", [
    ("size_hw", "H"), ("pattern_type", "H", 2), ("vcp", "H"), ("ncuts", "H"), ("clutter_group", "H", 1),
    ("velocity_res", "B", 2), ("pulse_width", "B", 2), ("reserved", "10x")])
M5_CUT = Layout("message 5 elevation cut", [
    ("angle", "H"), ("channel", "B"), ("waveform", "B"), ("super_res", "B"), ("surv_prf", "B", 1),
    ("surv_pulses", "H"), ("az_rate", "h"), ("snr", "6h", (28,) * 6),
    ("edge1", "H", 0x1558), ("prf1", "H", 6), ("pulses1", "H", 0x1F), ("pad1", "2x"),
    ("edge2", "H", 0x9558), ("prf2", "H", 6), ("pulses2", "H", 0x1F), ("pad2", "2x"),
    ("edge3", "H", 0xEE38), ("prf3", "H", 6), ("pulses3", "H", 0x1F), ("pad3", "2x")])
# message 2 (RDA status) body: halfwords in order; the build and generation-date fields carry the volume's date
M2_BODY = Layout("message 2 body", [
    ("rda_status", "H", 16), ("op_status", "H", 2), ("control", "H", 4), ("aux_power", "H", 2),
    ("avg_power", "H", 1402), ("zdr_cal", "H", 8), ("ops_mode", "H", 28), ("vcp", "H"), ("control_auth", "H", 0),
    ("build", "H", 1910), ("op_mode", "H", 4), ("super_res", "H", 2), ("cmd", "H", 63), ("avset", "H", 2),
    ("alarm", "H", 0), ("command_ack", "H", 0), ("channel", "H", 0), ("spot_blank", "H", 0), ("bypass_date", "H"),
    ("bypass_time", "H", 22), ("clutter_date", "H"), ("clutter_time", "H", 1308), ("vertical_cal", "H", 65512),
    ("transition", "H", 3)])

# the per-cut waveform of message 5 (channel, waveform, super-resolution control byte) by kind of cut
CUT_KINDS = {"surv": (2, 1, 0x0B), "dop": (2, 2, 0x07)}
CUT_BATCH = (0, 4, 0x0E)

# (structure, field, offset in a radial record): what the GPU rewrites per radial (ob_level2.cu)
RADIAL_PATCH = [("message header", f, MESSAGE_HEADER.offset(f)) for f in ("seq", "jdate", "jms")] + \
               [("message 31 header", f, MESSAGE_HEADER.size + M31_HEADER.offset(f))
                for f in ("jms", "jdate", "radial", "azimuth", "status")]


def julian(epoch_ms: int):
    """(Julian day with 1970-01-01 = 1, milliseconds of the day)."""
    day = int(epoch_ms // 86400000)
    return day + 1, int(epoch_ms - day * 86400000)


def message(buf, mtype, seq, epoch_ms, body_bytes):
    """Writes the message header of a message whose body (after the header) is ``body_bytes`` long."""
    jd, jms = julian(epoch_ms)
    MESSAGE_HEADER.pack_into(buf, 0, size_hw=(16 + body_bytes) // 2, type=mtype, seq=seq & 0xFFFF, jdate=jd, jms=jms)


def vcp_message(tilts, epoch_ms, seq, vcp):
    """Message 5: the volume coverage pattern, one entry per elevation cut."""
    seg = bytearray(SEGMENT)
    body = M5_HEADER.size + M5_CUT.size * len(tilts)
    message(seg, 5, seq, epoch_ms, body)
    at = M5_HEADER.pack_into(seg, MESSAGE_HEADER.size, size_hw=body // 2, vcp=vcp, ncuts=len(tilts))
    for t in tilts:
        sr = bool(t.get("superRes"))
        chan, wave, ctl = CUT_KINDS.get(t.get("kind", "both"), CUT_BATCH)
        at = M5_CUT.pack_into(seg, at, angle=int(round(t["angle"] * 65536 / 360)) & 0xFFFF, channel=chan,
                              waveform=wave, super_res=ctl, surv_pulses=15 if sr else 3,
                              az_rate=15400 if sr else 17944)
    return bytes(seg)


def status_message(epoch_ms, seq, vcp):
    """Message 2: RDA status."""
    seg = bytearray(SEGMENT)
    message(seg, 2, seq, epoch_ms, 80)
    jd, _ = julian(epoch_ms)
    M2_BODY.pack_into(seg, MESSAGE_HEADER.size, vcp=vcp, bypass_date=jd, clutter_date=jd)
    return bytes(seg)


def metadata(tilts, epoch_ms, vcp):
    """The metadata record: 131 empty segments, message 3 (an empty performance message), message 5, message 2."""
    m3 = bytearray(SEGMENT)
    message(m3, 3, 1, epoch_ms, 960)
    return bytes(SEGMENT) * (METADATA_SEGMENTS - 3) + bytes(m3) + vcp_message(tilts, epoch_ms, 2, vcp) + \
        status_message(epoch_ms, 3, vcp)


def sweep_template(s, ei, icao, lat, lon, height_m, vcp, epoch_ms=0):
    """Radial template of one sweep: (bytes, [(moment, data offset, gates, source offset)]). The per-radial fields
    (RADIAL_PATCH) are left for the GPU: the template carries radial 1, azimuth 0 and status 1 there."""
    sr = bool(s.get("superRes"))
    present = sorted(((m["name"], int(m["ngates"]), int(m["off"])) for m in s["moments"]), key=lambda m: ORDER.index(m[0]))
    blocks = M31_HEADER.size + VOLUME_BLOCK.size + ELEVATION_BLOCK.size + RADIAL_BLOCK.size + \
        sum(MOMENT_BLOCK.size + ng for _, ng, _ in present)
    rad_len = blocks + (blocks & 1)     # a whole number of halfwords
    rec = bytearray(MESSAGE_HEADER.size + rad_len)
    message(rec, 31, 0, int(s.get("start_ms", epoch_ms)), rad_len)
    d = MESSAGE_HEADER.size
    ptrs = []
    at = M31_HEADER.size
    ptrs.append(at)
    at = VOLUME_BLOCK.pack_into(rec, d + at, lat=lat, lon=lon, height=int(round(height_m)), vcp=vcp) - d
    ptrs.append(at)
    at = ELEVATION_BLOCK.pack_into(rec, d + at) - d
    ptrs.append(at)
    at = RADIAL_BLOCK.pack_into(rec, d + at, unamb_range=int(round(float(s.get("unamb_km", 466.0)) * 10)),
                                nyquist=int(round(float(s.get("nyquist", 63.5)) * 100))) - d
    layout = []
    for name, ng, off in present:
        block, scale, offset = MOMENTS[name]
        ptrs.append(at)
        at = MOMENT_BLOCK.pack_into(rec, d + at, name=block, ngates=ng, scale=scale, offset=offset) - d
        layout.append((name, d + at, ng, off))
        at += ng
    hdr = {"icao": text(icao, 4), "jms": 0, "jdate": 0, "radial": 1, "azimuth": 0.0, "radial_len": rad_len,
           "az_spacing": 1 if sr else 2, "status": 1, "elev_num": ei + 1, "elevation": float(s["angle"]),
           "az_index": 25 if sr else 50, "nblocks": len(ptrs)}
    M31_HEADER.pack_into(rec, d, pointers=ptrs + [0] * (MAX_BLOCKS - len(ptrs)), **hdr)
    return bytes(rec), layout


_compress_pool = None


def _compress_all(records, level=5):
    """bzip2 of every record; bz2 releases the interpreter lock, so the records compress on host threads."""
    global _compress_pool
    if len(records) < 4:
        return [bz2.compress(r, level) for r in records]
    if _compress_pool is None:
        from concurrent.futures import ThreadPoolExecutor
        _compress_pool = ThreadPoolExecutor(max(2, min(16, (os.cpu_count() or 4) - 2)))
    return list(_compress_pool.map(lambda r: bz2.compress(r, level), records))


def frame(icao, epoch_ms, records):
    """The Archive II file: the volume header, then each record compressed behind its control word (the length of
    the compressed record, negative for the last one)."""
    jd, jms = julian(epoch_ms)
    head = bytearray(VOLUME_HEADER.size)
    VOLUME_HEADER.pack_into(head, 0, jdate=jd, jms=jms, icao=text(icao, 4))
    comp = _compress_all(records)
    out = [bytes(head)]
    last = len(comp) - 1
    for i, c in enumerate(comp):
        out.append(struct.pack(">i", -len(c) if i == last else len(c)))
        out.append(c)
    return b"".join(out)


class ObL2Sweep(C.Structure):
    _fields_ = [("tpl_off", C.c_uint64), ("out_off", C.c_uint64), ("rec_len", C.c_uint32), ("nrad", C.c_uint32),
                ("nmom", C.c_uint32), ("seq0", C.c_uint32), ("ei", C.c_uint32), ("nsw", C.c_uint32),
                ("t0_ms", C.c_double), ("dur_ms", C.c_double), ("az0", C.c_double), ("data_at", C.c_uint32 * 6),
                ("ngates", C.c_uint32 * 6), ("src_off", C.c_uint64 * 6)]


def plan(header):
    """Templates and sweep descriptors of a volume header (the /api/volume header, app.js:1743-1758)."""
    icao, vcp = header["icao"], int(header.get("vcp", 212))
    lat, lon, elev = float(header["lat"]), float(header["lon"]), float(header["elev"])
    sweeps = header["sweeps"]
    tpls, descs = [], []
    tpl_off = out_off = 0
    seq = FIRST_SEQ
    for ei, s in enumerate(sweeps):
        tpl, layout = sweep_template(s, ei, icao, lat, lon, elev, vcp, int(header["epoch_ms"]))
        nrad = int(s["nrad"])
        d = ObL2Sweep(tpl_off=tpl_off, out_off=out_off, rec_len=len(tpl), nrad=nrad, nmom=len(layout), seq0=seq,
                      ei=ei, nsw=len(sweeps), t0_ms=float(int(s.get("start_ms", header["epoch_ms"]))),
                      dur_ms=float(s.get("dur_ms", 15000)), az0=float(s.get("az0", 0.0)))
        for m, (_, at, ng, off) in enumerate(layout):
            d.data_at[m], d.ngates[m], d.src_off[m] = at, ng, off
        tpls.append(tpl)
        descs.append(d)
        tpl_off += len(tpl)
        out_off += len(tpl) * nrad
        seq += nrad
    return b"".join(tpls), descs, out_off


def records_of(header, radials: bytes):
    """The uncompressed records of a volume: the metadata record, then each sweep's radials 120 at a time."""
    tilts = [{"angle": s["angle"], "superRes": bool(s.get("superRes")), "kind": s.get("kind", "both")}
             for s in header["sweeps"]]
    recs = [metadata(tilts, int(header["epoch_ms"]), int(header.get("vcp", 212)))]
    for d in plan(header)[1]:
        for first in range(0, d.nrad, RADIALS_PER_RECORD):
            n = min(RADIALS_PER_RECORD, d.nrad - first)
            a = d.out_off + first * d.rec_len
            recs.append(radials[a:a + n * d.rec_len])
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
    """File name of a volume: ICAO + UTC date and time of its start to the second + _V06, the name the server gives
    (l2writer.py:185-188)."""
    return icao.upper() + time.strftime("%Y%m%d_%H%M%S", time.gmtime(epoch_ms // 1000)) + "_V06"
