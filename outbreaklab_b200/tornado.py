"""The sub-grid tornado scheme (app.js:1435-1572) on the B200 model.

The km-scale model resolves the low-level mesocyclone but not the tornado. After each map readback the scheme finds
tornado candidates (a strong 1-km vortex that is the largest of its neighbourhood, under an updraft with strong 2-5 km
helicity) on the GPU, in the device copy of the maps (ob_model_tornado_candidates), tracks them as mesocyclones from
readback to readback (mesoUpdate), spawns tornadoes from mature mesocyclones at a rate scaled by the sounding's STP
(tornadoUpdate), and every step advances the active tornadoes and hands them to the radars (tornadoTick), which draw a
beam-smeared vortex and lofted debris into the radar data.

The random draws come from the run's own mulberry32 stream, seeded as app.js:1647, in the reference's order, so the
same candidates give the same tornadoes. The log names the place in model kilometres; the reference's nearest-city
name needs the map's city list, which belongs to the UI.
"""
from __future__ import annotations

import ctypes as C
import math

import numpy as np

from . import workloads as W

EF_V = (33, 44, 55, 68, 82, 96)      # app.js:1439, peak wind (m/s) of EF0..EF5
CAND_FLOATS = 7


def clamp(x, a, b):
    return max(a, min(b, x))


def lerp(a, b, t):
    return a + (b - a) * t


def smooth(a, b, x):
    """util.js smooth: smoothstep of x over [a, b]."""
    t = clamp((x - a) / (b - a), 0.0, 1.0)
    return t * t * (3 - 2 * t)


def js_round(x):
    """Math.round: halves go up."""
    return math.floor(x + 0.5)


def float_at_least(x):
    """The smallest float32 >= x: for a float32 z, z < x exactly when z < float_at_least(x)."""
    f = np.float32(x)
    if float(f) < x:
        f = np.nextafter(f, np.float32(np.inf))
    return f


def gpu_candidates(model, zmin, cap=4096):
    """Candidates of the maps of the model's last request_maps, from the GPU, in the reference's lattice order
    (rows j, then columns i): dicts {i, j, x, y, z1, uh, w}."""
    from . import _native as N
    out = np.empty(cap * CAND_FLOATS, np.float32)
    n = C.c_int(0)
    N.check(N.lib().ob_model_tornado_candidates(model.h, float(float_at_least(zmin)), N.fptr(out), cap, C.byref(n)))
    if n.value > cap:
        return gpu_candidates(model, zmin, n.value)
    a = out[:n.value * CAND_FLOATS].reshape(-1, CAND_FLOATS)
    rows = sorted(((int(r[1]), int(r[0]), float(r[4]), float(r[5]), float(r[6])) for r in a))
    dx = model.dx
    return [{"i": i, "j": j, "x": (i + 0.5) * dx, "y": (j + 0.5) * dx, "z1": z1, "uh": uh, "w": w} for j, i, z1, uh, w in rows]


class TornadoScheme:
    """TOR and MESO of app.js:1440, 1472, with tornadoUpdate / tornadoTick as update / tick.

    model: the RegionalModel (dx, nx, ny; its last request_maps is what update reads on the GPU); radar: a RadarSim or
    None; events: a callable giving the current storm-initiation events (RUN.events, for forcedNear); stp: the
    sounding's significant tornado parameter (1 when unknown); on / rate: CFG.tor; hurricane: the hurricane mode, in
    which the scheme is off (app.js:1511); candidates: the candidate search, maps -> list of dicts (default: the GPU)."""

    def __init__(self, model, radar=None, ci_seed=7, stp=None, rate=1.0, on=True, events=None, hurricane=False,
                 candidates=None, log=None, epoch0_ms=0):
        self.m, self.radar = model, radar
        self.on, self.rate, self.hurricane = bool(on), float(rate), bool(hurricane)
        self.stp = stp if stp is not None and math.isfinite(stp) else 1.0
        self.events = events or (lambda: [])
        self._cands = candidates
        self.log = log if log is not None else []
        self.epoch0 = epoch0_ms
        self.reset(ci_seed)

    def reset(self, ci_seed=7):
        """app.js:1647-1648."""
        self.list, self.last_t = [], 0.0
        self.rng = W.Mulberry32((int(ci_seed) | 0) * 104729 + 71)
        self.meso, self.meso_next = [], 1
        self.cands, self.mature = 0, 0

    # ---- app.js:1450-1452, 1511 ----
    def zeta_scale(self):
        return 1500.0 / self.m.dx

    def zeta_min(self):
        return 0.003 * self.zeta_scale()

    def active(self):
        return self.on and not self.hurricane and self.m.dx >= 400

    def candidates(self, maps):
        if self._cands is not None:
            return self._cands(maps, self.m.dx, self.zeta_min())
        return gpu_candidates(self.m, self.zeta_min())

    def gauss(self):
        """app.js:1467 (Box-Muller, two draws in this order)."""
        a = math.sqrt(-2 * math.log(max(self.rng(), 1e-9)))
        return a * math.cos(2 * math.pi * self.rng())

    # ---- app.js:1473-1483 ----
    def field_around(self, arr, ch, x, y, rad, fn, init):
        nx, ny, dx = self.m.nx, self.m.ny, self.m.dx
        r = math.ceil(rad / dx)
        i0, j0 = math.floor(x / dx), math.floor(y / dx)
        v = init
        for j in range(max(0, j0 - r), min(ny - 1, j0 + r) + 1, 2):
            for i in range(max(0, i0 - r), min(nx - 1, i0 + r) + 1, 2):
                if (i - i0) ** 2 + (j - j0) ** 2 > r * r:
                    continue
                v = fn(v, float(arr[j, i, ch]))
        return v

    # ---- app.js:1484-1485 ----
    @staticmethod
    def tower_pos(e, t):
        dt = max(0.0, min(t, e["t1"]) - e["t0"])
        return e["x"] + e.get("vx", 0.0) * dt, e["y"] + e.get("vy", 0.0) * dt

    def forced_near(self, x, y, t):
        for e in self.events():
            if t < e["t0"] or t > e["t1"]:
                continue
            ex, ey = self.tower_pos(e, t)
            if math.hypot(ex - x, ey - y) < 1.5 * e["rh"] + 8000:
                return True
        return False

    # ---- app.js:1486-1510 ----
    def meso_update(self, maps, t, dt):
        cands = self.candidates(maps)
        for M in self.meso:
            M["hit"] = None
        for c in cands:
            best, bd = None, 16000.0
            for M in self.meso:
                if M["hit"] is not None:
                    continue
                d = math.hypot(c["x"] - (M["x"] + M["vx"] * dt), c["y"] - (M["y"] + M["vy"] * dt))
                if d < bd:
                    bd, best = d, M
            forced = self.forced_near(c["x"], c["y"], t)
            if best is not None:
                k = 1 - math.exp(-dt / 300)
                best["vx"] = lerp(best["vx"], (c["x"] - best["x"]) / dt, 0.3)
                best["vy"] = lerp(best["vy"], (c["y"] - best["y"]) / dt, 0.3)
                best["x"], best["y"], best["seen"] = c["x"], c["y"], t
                best["z1"] = lerp(best["z1"], c["z1"], k)
                best["uh"] = lerp(best["uh"], c["uh"], k)
                best["hit"] = c
                c["meso"] = best["id"]
                best["strongFor"] = 0.0 if forced else best["strongFor"] + dt
                if forced:
                    best["freeSince"] = t
            else:
                M = {"id": self.meso_next, "x": c["x"], "y": c["y"], "vx": 0.0, "vy": 0.0, "born": t, "seen": t,
                     "z1": c["z1"], "uh": c["uh"], "strongFor": 0.0, "freeSince": t if forced else t - 1e9,
                     "lastTor": -1e9, "hit": c}
                self.meso_next += 1
                self.meso.append(M)
                c["meso"] = M["id"]
        self.meso = [M for M in self.meso if t - M["seen"] < 360]
        return cands

    # ---- app.js:1512-1556 ----
    def update(self, maps, t):
        if not self.active() or self.rng is None:
            return
        dt = max(1.0, t - self.last_t)
        self.last_t = t
        cands = self.meso_update(maps, t, dt)
        self.cands = len(cands)
        stp = self.stp
        f_stp = clamp(0.25 + stp / 3, 0.2, 2.5) * self.rate
        for T in self.list:
            if T["done"]:
                continue
            best, bd = None, 12000.0
            for c in cands:
                d = math.hypot(c["x"] - T["x"], c["y"] - T["y"])
                if d < bd:
                    bd, best = d, c
            if best is not None:
                k = min(1.0, dt / 120)
                T["vx"] = lerp(T["vx"], (best["x"] - T["mx"]) / max(dt, 1), 0.3)
                T["vy"] = lerp(T["vy"], (best["y"] - T["my"]) / max(dt, 1), 0.3)
                T["mx"], T["my"] = best["x"], best["y"]
                T["x"] = lerp(T["x"], best["x"], k * 0.5)
                T["y"] = lerp(T["y"], best["y"], k * 0.5)
                T["lost"] = 0.0
            else:
                T["lost"] += dt
            if T["lost"] > 300 and T["t1"] > t + 120:       # lost its mesocyclone: rope out
                T["t1"] = t + 120
            if t > T["t1"]:
                T["done"] = True
                self.log.append("tornado #%d (EF%d) lifted after %.0f min" % (T["id"], T["ef"], (T["t1"] - T["t0"]) / 60))
        self.mature = 0
        zs = self.zeta_scale()
        for M in self.meso:
            c = M["hit"]
            if c is None:
                continue
            if t - M["born"] < 900 or M["strongFor"] < 480 or t - M["freeSince"] < 600 or t - M["lastTor"] < 600:
                continue
            if any(not T["done"] and math.hypot(T["x"] - c["x"], T["y"] - c["y"]) < 20000 for T in self.list):
                continue
            core = self.field_around(maps["m0"], 1, c["x"], c["y"], 10000, max, -30.0)   # heavy rain reaching low levels
            cold = self.field_around(maps["m0"], 2, c["x"], c["y"], 12000, min, 99.0)    # storm outflow
            if core < 40 or cold > -1.0:
                continue
            self.mature += 1
            p = 0.08 * f_stp * smooth(0.003 * zs, 0.010 * zs, M["z1"]) * smooth(60, 400, M["uh"])
            if self.rng() >= p * dt / 60:
                continue
            M["lastTor"] = t
            f_i = clamp(0.3 + stp / 4, 0.3, 2.2)
            s = f_i * smooth(0.003 * zs, 0.010 * zs, M["z1"]) * smooth(80, 600, M["uh"])
            ef = int(clamp(js_round(0.2 + 1.8 * s + 1.0 * self.gauss()), 0, 5))
            life = (4 + 7 * ef + 15 * self.rng()) * 60
            T = {"id": len(self.list) + 1, "ef": ef, "x": c["x"], "y": c["y"], "mx": c["x"], "my": c["y"], "vx": 0.0,
                 "vy": 0.0, "t0": t, "t1": t + life, "R": 40 + 55 * ef + 50 * self.rng(), "lost": 0.0, "track": [],
                 "done": False}
            self.list.append(T)
            self.log.append("TORNADO #%d EF%d at (%.1f, %.1f) km, t+%.0f min" % (T["id"], ef, c["x"] / 1000, c["y"] / 1000, t / 60))

    # ---- app.js:1558-1572 ----
    def tick(self, t, dt):
        if not self.active():
            if self.radar is not None and self.radar.nTor:
                self.radar.set_tornadoes([])
            return []
        act = []
        for T in self.list:
            if T["done"]:
                continue
            T["x"] += T["vx"] * dt
            T["y"] += T["vy"] * dt
            age = (t - T["t0"]) / max(T["t1"] - T["t0"], 1)
            env = smooth(0, 0.15, age) * (1 - smooth(0.7, 1, age))
            v = EF_V[T["ef"]] * env * (0.92 + 0.08 * math.sin(t / 47 + T["id"]))
            lp = T["track"][-1] if T["track"] else None
            if lp is None or math.hypot(T["x"] - lp[0], T["y"] - lp[1]) > 1500:
                T["track"].append((T["x"], T["y"]))
            act.append({"x": T["x"], "y": T["y"], "R": T["R"] * (0.6 + 0.4 * env), "v": v, "debrisTop": 500 + 800 * T["ef"],
                        "debrisDbz": 40 + 4 * T["ef"], "debris": smooth(60, 240, t - T["t0"]) * env if T["ef"] >= 1 else 0.0})
        if self.radar is not None:
            self.radar.set_tornadoes(act)
        return act

    def counts(self):
        """(active tornadoes, all tornadoes): the status line's figures (app.js:1785)."""
        return sum(1 for T in self.list if not T["done"]), len(self.list)
