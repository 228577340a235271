"""Host-side mirror of the reference's virtual radar (radar.js:271-413) and its projection (geo.js:6-29).

``RadarSim`` keeps the reference's method names and meaning: ``add_radar(site, opts)`` (VCP cut table, volume
layout, scan timing), ``set_tornadoes(list)``, ``enc_due(sim_t)`` (samples every cut whose scan time has come and
returns the volumes that completed), ``enc_cut``, ``collect(done, run, epoch0)`` (bytes + the JSON header the
browser uploads) and ``destroy``. The gate sampling and the PhiDP pass run in the CUDA library (ob_radar_cut) on the
model's stream; nothing here computes a gate.

The reference draws each radar's volume phase and each volume's first azimuth from ``Math.random``
(radar.js:323, 352); here they come from a ``random.Random(seed)`` so runs repeat.
"""
from __future__ import annotations

import ctypes as C
import math
import random

import numpy as np

from . import _native as N

DEG = math.pi / 180.0
EARTH_R = 6371000.0
RE_M, KE = 6371000.0, 4.0 / 3.0
GATE0, GATEDR, MAX_REF_GATES, MAX_DOP_GATES = 2125.0, 250.0, 1832, 1192
# Level II scale / offset per moment (radar.js:21): code = round(value * scale + offset), 0 = below threshold
L2_SCALE = {"REF": (2, 66), "VEL": (2, 129), "SW": (2, 129), "ZDR": (16, 128), "PHI": (253 / 360, 2), "RHO": (300, -60.5)}
CUT_MOMENTS = {"surv": ["REF", "ZDR", "PHI", "RHO"], "dop": ["REF", "VEL", "SW"],
               "both": ["REF", "VEL", "SW", "ZDR", "PHI", "RHO"]}
MOMENT_BITS = {"REF": 1, "VEL": 2, "SW": 4, "ZDR": 8, "PHI": 16, "RHO": 32}


def _split_vcp(split, rest, nyq_split, nyq_rest):
    """radar.js:24-29: split cuts (surveillance + Doppler) at the lowest angles, then combined cuts."""
    cuts = []
    for a in split:
        cuts.append({"angle": a, "kind": "surv", "superRes": True, "nyquist": 8.9})
        cuts.append({"angle": a, "kind": "dop", "superRes": True, "nyquist": nyq_split})
    for a in rest:
        cuts.append({"angle": a, "kind": "both", "superRes": False, "nyquist": nyq_rest if a < 7 else 32.3})
    return cuts


_HIGH = [1.8, 2.4, 3.1, 4.0, 5.1, 6.4, 8.0, 10.0, 12.5, 15.6, 19.5]
VCPS = {  # radar.js:30-35
    212: {"label": "VCP 212", "dur": 270, "cuts": _split_vcp([0.5, 0.9, 1.3], _HIGH, 28.4, 29.4)},
    12: {"label": "VCP 12", "dur": 250, "cuts": _split_vcp([0.5, 0.9, 1.3], _HIGH, 28.4, 29.4)},
    215: {"label": "VCP 215", "dur": 360,
          "cuts": _split_vcp([0.5, 0.9, 1.3], [1.8, 2.4, 3.1, 4.0, 5.1, 6.4, 8.0, 10.0, 12.0, 14.0, 16.7, 19.5], 28.4, 29.4)},
    35: {"label": "VCP 35", "dur": 420, "cuts": _split_vcp([0.5, 0.9, 1.3], [1.8, 2.4, 3.1, 4.0, 5.1, 6.4], 26.0, 27.0)},
}


class Geo:
    """Azimuthal-equidistant projection about the domain centre (geo.js:6-29)."""

    def __init__(self, lat0, lon0, Lx=0.0, Ly=0.0, ground_msl=0.0):
        self.lat0, self.lon0, self.Lx, self.Ly, self.groundMSL = lat0, lon0, Lx, Ly, ground_msl
        self.p0, self.l0 = lat0 * DEG, lon0 * DEG
        self.sp0, self.cp0 = math.sin(self.p0), math.cos(self.p0)

    def fwd(self, lat, lon):
        p, dl = lat * DEG, lon * DEG - self.l0
        sp, cp, cdl = math.sin(p), math.cos(p), math.cos(dl)
        cc = max(-1.0, min(1.0, self.sp0 * sp + self.cp0 * cp * cdl))
        c = math.acos(cc)
        k = 1.0 if c < 1e-9 else c / math.sin(c)
        return EARTH_R * k * cp * math.sin(dl), EARTH_R * k * (self.cp0 * sp - self.sp0 * cp * cdl)

    def inv(self, x, y):
        rho = math.hypot(x, y)
        if rho < 1e-6:
            return self.lat0, self.lon0
        c = rho / EARTH_R
        sc, ccs = math.sin(c), math.cos(c)
        p = math.asin(ccs * self.sp0 + y * sc * self.cp0 / rho)
        lon = self.l0 + math.atan2(x * sc, rho * self.cp0 * ccs - y * self.sp0 * sc)
        return p / DEG, ((lon / DEG + 540) % 360) - 180

    def to_model(self, lat, lon):
        x, y = self.fwd(lat, lon)
        return x + self.Lx / 2, y + self.Ly / 2

    def from_model(self, mx, my):
        return self.inv(mx - self.Lx / 2, my - self.Ly / 2)


class ObRadarCut(C.Structure):
    _fields_ = [(n, C.c_float * 4) for n in ("site", "geo", "cut", "gates", "nyq", "offA", "offB", "mdl", "mdl2",
                                                 "phys", "phys2")]

    def as_array(self):
        return np.array([list(getattr(self, n)) for n, _ in self._fields_], np.float32).reshape(-1)


def radar_layout(Lx, Ly, sx, sy, vcp):
    """addRadar's gate counts, per-cut moment offsets (bytes) and scan timing (radar.js:293-318).
    Returns (ngRef, ngDop, cuts, volume bytes)."""
    far = 0.0
    for cx, cy in ((0, 0), (Lx, 0), (0, Ly), (Lx, Ly)):
        far = max(far, math.hypot(cx - sx, cy - sy))
    rng = min(460000.0, far + 10000.0)
    ng_ref = min(MAX_REF_GATES, math.ceil((rng - GATE0) / GATEDR))
    ng_ref = max(64, math.ceil(ng_ref / 4) * 4)
    ng_dop = min(MAX_DOP_GATES, ng_ref)
    off = 0
    cuts = []
    for ci, c in enumerate(vcp["cuts"]):
        nrad = 720 if c["superRes"] else 360
        mom = []
        for name in CUT_MOMENTS[c["kind"]]:
            ng = ng_ref if name == "REF" else ng_dop
            mom.append({"name": name, "ngates": ng, "off": off})
            off += nrad * ng
        cuts.append(dict(c, index=ci, nrad=nrad, mom=mom))
    wsum = sum(2 if c["superRes"] else 1 for c in cuts)
    acc = 0
    for c in cuts:
        c["t0"] = acc / wsum * vcp["dur"]
        acc += 2 if c["superRes"] else 1
        c["dur"] = (2 if c["superRes"] else 1) / wsum * vcp["dur"]
    return ng_ref, ng_dop, cuts, off


class RadarSim:
    """The reference's RadarSim over the CUDA radar kernels (radar.js:271-413)."""

    def __init__(self, model, geo, seed=0):
        self.m, self.geo = model, geo
        self.radars = []
        self.tornadoes = np.zeros(N.RADAR_TORNADO_FLOATS, np.float32)
        self.nTor = 0
        self.rng = random.Random(seed)

    # ---- radar.js:280-286 ----
    def set_tornadoes(self, lst):
        act = list(lst)[:N.RADAR_MAX_TORNADOES]
        f = np.zeros(max(1, len(act)) * N.RADAR_TORNADO_FLOATS, np.float32)
        for i, t in enumerate(act):
            f[i * 8:(i + 1) * 8] = [t["x"], t["y"], t["R"], t["v"], t["debrisTop"], t["debrisDbz"], t["debris"], 0]
        self.tornadoes, self.nTor = f, len(act)
        for R in self.radars:
            N.check(N.lib().ob_radar_set_tornadoes(R["h"], N.fptr(f), self.nTor))

    # ---- radar.js:288-327 ----
    def add_radar(self, site, opts=None):
        opts = dict(opts or {})
        m, g = self.m, self.geo
        vcp = VCPS.get(opts.get("vcp"), VCPS[212])
        sx, sy = g.to_model(site["lat"], site["lon"])
        ng_ref, ng_dop, cuts, off = radar_layout(m.Lx, m.Ly, sx, sy, vcp)
        h = C.c_void_p()
        N.check(N.lib().ob_radar_create(m.h, off, ng_dop, C.byref(h)))
        R = {"site": site, "opts": opts, "vcp": vcp, "vcpId": int(opts.get("vcp") or 212), "cuts": cuts,
             "bytes": off, "ngRef": ng_ref, "ngDop": ng_dop, "sx": sx, "sy": sy, "h": h,
             "phase": self.rng.random() * vcp["dur"], "vol": -1, "next": 0, "volStart": 0.0, "az0": 0.0,
             "done": 0, "failed": 0, "pending": []}
        if self.nTor:
            N.check(N.lib().ob_radar_set_tornadoes(h, N.fptr(self.tornadoes), self.nTor))
        self.radars.append(R)
        return R

    def destroy(self):
        for R in self.radars:
            if R.get("h"):
                N.lib().ob_radar_destroy(R["h"])
                R["h"] = None
        self.radars = []

    def __del__(self):
        try:
            self.destroy()
        except Exception:
            pass

    # ---- radar.js:343-367 ----
    def enc_due(self, sim_t):
        """Samples every cut whose scan time has been reached; returns the volumes that completed. The library
        reads a volume only when asked (collect), so there are no readback slots to wait for."""
        done = []
        for R in self.radars:
            while True:
                if R["vol"] < 0 or R["next"] >= len(R["cuts"]):
                    vstart = R["phase"] if R["vol"] < 0 else R["volStart"] + R["vcp"]["dur"]
                    if sim_t < vstart:
                        break
                    R["vol"] += 1
                    R["volStart"] = vstart
                    R["next"] = 0
                    R["az0"] = self.rng.random()
                c = R["cuts"][R["next"]]
                if sim_t < R["volStart"] + c["t0"]:
                    break
                self.enc_cut(R, c, sim_t)
                R["next"] += 1
                if R["next"] >= len(R["cuts"]):
                    done.append({"R": R, "vol": R["vol"], "volStart": R["volStart"], "az0": R["az0"]})
        return done

    def cut_uniforms(self, R, c, sim_t):
        """encCut's uniform block (radar.js:369-384)."""
        m, g = self.m, self.geo
        off = {o["name"]: o["off"] // 4 for o in c["mom"]}
        mask = 0
        for name, bit in MOMENT_BITS.items():
            if name in off:
                mask |= bit
        z_ant = R["site"]["h"] + 20
        U = ObRadarCut()
        U.site[:] = [R["sx"], R["sy"], z_ant, KE * RE_M]
        U.geo[:] = [g.lat0 * DEG, g.lon0 * DEG, R["site"]["lat"] * DEG, R["site"]["lon"] * DEG]
        U.cut[:] = [c["angle"] * DEG, R["az0"], 360 / c["nrad"], c["nrad"]]
        U.gates[:] = [R["ngRef"], R["ngDop"], GATE0, GATEDR]
        nyq = 63.5 if R["opts"].get("aliasing") is False else c["nyquist"]
        U.nyq[:] = [nyq, sim_t, (R["vol"] * 97 + c["index"] * 13) % 100000, 25]
        U.offA[:] = [off.get("REF", 0), off.get("VEL", 0), off.get("SW", 0), off.get("ZDR", 0)]
        U.offB[:] = [off.get("PHI", 0), off.get("RHO", 0), 0, mask]
        U.mdl[:] = [m.nx, m.ny, m.nz, m.dx]
        U.mdl2[:] = [m.dz, g.groundMSL, -m.Lx / 2, -m.Ly / 2]
        U.phys[:] = [m.rho_sfc or 1.15, R["opts"].get("minDbz", 0) or 0,
                     1 if m.params.get("scheme") == "thompson" else 0, self.nTor]
        hur = getattr(m, "hurricane", None)   # hurricane mode's maritime graupel (radar.js:384)
        U.phys2[:] = [1 if hur is not None and hur.maritime > 0.5 else 0, 0, 0, 0]
        return U

    def enc_cut(self, R, c, sim_t):
        U = self.cut_uniforms(R, c, sim_t)
        N.check(N.lib().ob_radar_cut(R["h"], C.byref(U)))
        c["simT"] = sim_t
        return U

    # ---- radar.js:394-412 ----
    def _volume_header(self, d, run, epoch0):
        """The JSON header of a volume (radar.js:394-412): site, VCP, and per cut its timing and moment offsets."""
        R = d["R"]
        t0 = epoch0 + d["volStart"] * 1000
        nyq = lambda c: 63.5 if R["opts"].get("aliasing") is False else c["nyquist"]
        return {
            "run": run, "icao": R["site"]["id"], "lat": R["site"]["lat"], "lon": R["site"]["lon"],
            "elev": R["site"]["h"] + 20, "vcp": R["vcpId"], "epoch_ms": round(t0),
            "sweeps": [{"angle": c["angle"], "superRes": c["superRes"], "kind": c["kind"], "az0": d["az0"],
                        "nrad": c["nrad"], "nyquist": nyq(c), "unamb_km": 466 if c["kind"] == "surv" else 300,
                        "start_ms": round(t0 + c["t0"] * 1000), "dur_ms": round(c["dur"] * 1000),
                        "moments": [{"name": o["name"], "ngates": o["ngates"], "off": o["off"]} for o in c["mom"]]}
                       for c in R["cuts"]]}

    def collect(self, d, run, epoch0):
        R = d["R"]
        buf = np.empty(R["bytes"], np.uint8)
        try:
            N.check(N.lib().ob_radar_read(R["h"], buf.ctypes.data, buf.nbytes))
        except Exception:
            R["failed"] += 1
            raise
        header = self._volume_header(d, run, epoch0)
        R["done"] += 1
        return {"R": R, "header": header, "bytes": buf}

    def collect_level2(self, d, run, epoch0):
        """The finished volume as an Archive II file, as the server would write it from collect()'s upload
        (server.py:249-284, l2writer.py:161-188), with the radial records assembled on the GPU from the radar
        volume (no readback of the raw codes). Returns {"R", "header", "name", "bytes"}."""
        from . import level2 as L2
        R = d["R"]
        header = self._volume_header(d, run, epoch0)
        data = L2.encode_volume_gpu(R["h"], header)
        R["done"] += 1
        return {"R": R, "header": header, "name": L2.archive_name(header["icao"], header["epoch_ms"]), "bytes": data}

    # ---- diagnostics (no counterpart in the reference) ----
    def cut_moments(self, R, U):
        """Runs one cut and returns its per-gate moments, shape (nrad, ngRef, 6): dBZ, Vr, SW, ZDR, rho_hv, KDP."""
        nrad, ngr = int(U.cut[3]), int(U.gates[0])
        out = np.empty(nrad * ngr * 6, np.float32)
        N.check(N.lib().ob_radar_cut_moments(R["h"], C.byref(U), N.fptr(out), out.size))
        return out.reshape(nrad, ngr, 6)

    def read_volume(self, R):
        buf = np.empty(R["bytes"], np.uint8)
        N.check(N.lib().ob_radar_read(R["h"], buf.ctypes.data, buf.nbytes))
        return buf

    def read_kdp(self, R, nrad):
        out = np.empty(nrad * R["ngDop"], np.float32)
        N.check(N.lib().ob_radar_kdp(R["h"], N.fptr(out), out.size))
        return out.reshape(nrad, R["ngDop"])
