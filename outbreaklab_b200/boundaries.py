"""Air-mass boundaries of an outbreak run: the reference's host geometry that turns the boundaries drawn on the map
(lat/lon polylines of a type) into the per-boundary records the large-scale forcing pass reads.

- ``BND_TYPES``, ``mk_bound``: the five boundary types and their defaults (app.js:12-18, 61-65).
- ``default_bounds``: the example cold front, warm front and dryline that meet at a triple point over western
  Oklahoma (app.js:52-56).
- ``bnd_side``, ``bnd_motion`` (app.js:479-490), ``find_lows``, ``low_motion``, ``boundary_vels`` (app.js:495-525):
  which side holds the other air mass, each boundary's drift, and the surface lows where two or more boundaries meet
  (vertices within 8 km), whose vertices move together at the mean motion of the boundaries that meet there.
- ``bnd_model`` (app.js:527-541): one boundary in model metres with its air-mass parameters; ``boundary_models``
  builds the list startRun passes to setBoundaries (app.js:1617-1619).
- ``pack_boundaries`` (model.js:1371-1380): 148 float32 per boundary, the layout of OB_BOUNDARY_FLOATS.
- ``pts_at``, ``sdist``, ``other_weight`` (app.js:543-563): the scheduler's CPU copy of the forcing pass's signed
  distance, and how deep a point lies inside any boundary's air mass.

All arithmetic is Python float (IEEE double, as JavaScript numbers); the packed record is rounded to float32 once, as
a Float32Array.set does.
"""
from __future__ import annotations

import math

import numpy as np

DEG = math.pi / 180.0
MAX_BOUNDS = 8          # model.js MAX_BOUNDS
MAX_BPTS = 32           # model.js MAX_BPTS
BOUNDARY_FLOATS = 148   # 20 parameters + 32 points x (x, y, vx, vy)

# app.js:12-18
BND_TYPES = {
    "cold": {"label": "Cold front", "dT": -8, "depth": 1600, "slope": 0.012, "dq": 0.55, "windDir": 320, "windSpd": 11,
             "speed": 9, "dir": 120, "halfW": 7000, "nudge": True, "rate": 4.0, "otherAhead": False, "vary": 0.8},
    "warm": {"label": "Warm front", "dT": -5, "depth": 900, "slope": 0.005, "dq": 0.2, "windDir": 95, "windSpd": 8,
             "speed": 3, "dir": 10, "halfW": 12000, "nudge": True, "rate": 2.0, "otherAhead": True, "vary": 0.7},
    "dry": {"label": "Dryline", "dT": 2.5, "depth": 2800, "slope": 0.05, "dq": 0.72, "windDir": 245, "windSpd": 11,
            "speed": 3, "dir": 90, "halfW": 5000, "nudge": True, "rate": 3.0, "otherAhead": False, "vary": 0.8},
    "stat": {"label": "Stationary front", "dT": -6, "depth": 1200, "slope": 0.012, "dq": 0.35, "windDir": 60,
             "windSpd": 6, "speed": 0, "dir": 160, "halfW": 8000, "nudge": True, "rate": 2.0, "otherAhead": False,
             "vary": 0.7},
    "outflow": {"label": "Outflow boundary", "dT": -5, "depth": 700, "slope": 0.05, "dq": 0.1, "windDir": None,
                "windSpd": 8, "speed": 6, "dir": 150, "halfW": 4000, "nudge": False, "rate": 3.0, "otherAhead": False,
                "vary": 0.6},
}


def smooth(a, b, x):
    """util.js:9 (smoothstep)."""
    t = min(max((x - a) / (b - a), 0.0), 1.0)
    return t * t * (3 - 2 * t)


def mk_bound(kind, pts, bid=None):
    """A boundary of type ``kind`` through ``pts`` ([lat, lon] degrees) with its type's defaults (app.js:61-65).
    The reference gives each boundary a random six-character id, which seeds its along-front pattern; ``bid`` fixes
    it (default: none, so the seed comes from the type name, as bndModel does for a boundary without an id)."""
    T = BND_TYPES[kind]
    return {"id": bid, "type": kind, "pts": [list(p) for p in pts], "speed": T["speed"], "dir": T["dir"], "flip": False,
            "dT": T["dT"], "depth": T["depth"], "slope": T["slope"], "dq": T["dq"], "windDir": T["windDir"],
            "windSpd": T["windSpd"], "trigger": True, "rate": T["rate"], "nudge": T["nudge"], "vary": T["vary"]}


def default_bounds():
    """The example setup of a fresh configuration: a cold front + warm front + dryline triple point over Oklahoma
    (app.js:52-56)."""
    return [mk_bound("cold", [[39.4, -101.6], [37.4, -100.2], [36.3, -99.9]]),
            mk_bound("warm", [[36.3, -99.9], [36.9, -97.4], [37.4, -94.6]]),
            mk_bound("dry", [[36.3, -99.9], [34.8, -99.4], [33.0, -99.6]])]


def bnd_side(b, pts_xy):
    """+1 when the other air mass lies left of the drawing direction (app.js:479-489)."""
    T = BND_TYPES[b["type"]]
    md = (math.sin(b["dir"] * DEG), math.cos(b["dir"] * DEG))
    oth = md if T["otherAhead"] else (-md[0], -md[1])
    a, e = pts_xy[0], pts_xy[-1]
    ab = (e[0] - a[0], e[1] - a[1])
    left = (-ab[1], ab[0])
    s = 1 if (left[0] * oth[0] + left[1] * oth[1]) >= 0 else -1
    return -s if b.get("flip") else s


def bnd_motion(b):
    """app.js:490: (vx, vy) m/s from speed and the direction it moves toward."""
    return [b["speed"] * math.sin(b["dir"] * DEG), b["speed"] * math.cos(b["dir"] * DEG)]


def find_lows(bounds, geo):
    """Surface lows (app.js:495-515): groups of vertices of different boundaries within 8 km of a first vertex."""
    V = []
    for bi, b in enumerate(bounds):
        for i, p in enumerate(b["pts"]):
            x, y = geo.fwd(p[0], p[1])
            V.append({"bi": bi, "i": i, "x": x, "y": y})
    used = [False] * len(V)
    lows = []
    for a in range(len(V)):
        if used[a]:
            continue
        gi = [a]
        for c in range(a + 1, len(V)):
            if used[c] or any(V[k]["bi"] == V[c]["bi"] for k in gi):
                continue
            if math.hypot(V[c]["x"] - V[a]["x"], V[c]["y"] - V[a]["y"]) < 8000:
                gi.append(c)
        if len(gi) < 2:
            continue
        for k in gi:
            used[k] = True
        grp = [V[k] for k in gi]
        lows.append({"x": sum(g["x"] for g in grp) / len(grp), "y": sum(g["y"] for g in grp) / len(grp),
                     "members": grp,
                     "front": any(bounds[g["bi"]]["type"] in ("cold", "warm", "stat") for g in grp)})
    return lows


def low_motion(L, bounds, low=None):
    """app.js:516-521: a fixed motion when the configuration's low is not automatic, else the mean of the motions of
    the boundaries that meet there."""
    lm = low or {}
    if lm.get("auto") is False and math.isfinite(lm.get("speed", math.nan)) and math.isfinite(lm.get("dir", math.nan)):
        return [lm["speed"] * math.sin(lm["dir"] * DEG), lm["speed"] * math.cos(lm["dir"] * DEG)]
    ms = [bnd_motion(bounds[g["bi"]]) for g in L["members"]]
    return [sum(m[0] for m in ms) / len(ms), sum(m[1] for m in ms) / len(ms)]


def boundary_vels(bounds, geo, low=None):
    """Per-point velocities of every boundary (app.js:523-527)."""
    vel = [[bnd_motion(b) for _ in b["pts"]] for b in bounds]
    for L in find_lows(bounds, geo):
        m = low_motion(L, bounds, low)
        for g in L["members"]:
            vel[g["bi"]][g["i"]] = m
    return vel


def _seed(b):
    s = 0
    for ch in str(b.get("id") or b["type"]):
        s = (s * 31 + ord(ch)) % 9973
    return s


def bnd_model(b, geo, wind_sfc):
    """One boundary in model metres (app.js:527-541). ``wind_sfc`` is the sounding's wind 150 m above the ground
    (SND.A.windAt(0.15)); the air mass's wind anomaly is its own wind minus that."""
    pts = [list(geo.to_model(p[0], p[1])) for p in b["pts"]]
    T = BND_TYPES[b["type"]]
    side = bnd_side(b, pts)
    wd = b.get("windDir")
    if wd is None or wd == "" or not math.isfinite(wd):
        wd = (b["dir"] + 180) % 360
    wo = (-b["windSpd"] * math.sin(wd * DEG), -b["windSpd"] * math.cos(wd * DEG))
    Hmax = max(200, b["depth"])
    vary = b.get("vary")
    if vary is None:
        vary = T.get("vary", 0.7)
    return {"pts": pts, "motion": bnd_motion(b), "halfW": T["halfW"], "dT": b["dT"], "Hmax": Hmax,
            "slope": max(1e-4, b["slope"]), "Hmin": min(300, Hmax), "dq": min(max(b["dq"], 0), 0.9), "qRatio": 1.0,
            "du": wo[0] - wind_sfc[0], "dv": wo[1] - wind_sfc[1], "wRatio": 1.0, "nudge": bool(b["nudge"]),
            "dFree": 25000, "side": side, "vary": min(max(vary, 0), 1), "seed": _seed(b) * 0.731 + 11.3,
            "varyL": 50000}


def boundary_models(bounds, geo, wind_sfc, low=None):
    """startRun's RUN.mbs (app.js:1617-1618): every boundary with its per-point velocities and its drawn source, those
    with fewer than two points left out."""
    BV = boundary_vels(bounds, geo, low)
    out = []
    for b, v in zip(bounds, BV):
        mb = bnd_model(b, geo, wind_sfc)
        mb["vel"], mb["b"] = v, b
        if len(mb["pts"]) >= 2:
            out.append(mb)
    return out


def pack_boundaries(bnds):
    """setBoundaries' record (model.js:1371-1380): (MAX_BOUNDS * 148) float32 and the count. Per boundary:
    [npts, vx, vy, halfW, dT, Hmax, slope, Hmin, dq, qRatio, du, dv, wRatio, nudge, dFree, side, vary, seed, varyL, 0]
    then (x, y, vx, vy) per point, at most 32 points."""
    bnds = list(bnds)[:MAX_BOUNDS]
    f = np.zeros(MAX_BOUNDS * BOUNDARY_FLOATS, np.float32)
    for i, b in enumerate(bnds):
        o = i * BOUNDARY_FLOATS
        pts = list(b["pts"])[:MAX_BPTS]
        f[o:o + 20] = [len(pts), b["motion"][0], b["motion"][1], b["halfW"], b["dT"], b["Hmax"], b["slope"], b["Hmin"],
                       b["dq"], b["qRatio"], b["du"], b["dv"], b["wRatio"], 1 if b.get("nudge") else 0, b["dFree"],
                       b["side"], b.get("vary", 0) or 0, b.get("seed", 0) or 0, b.get("varyL", 60000) or 60000, 0]
        vel = b.get("vel") or []
        for k, p in enumerate(pts):
            v = (vel[k] if k < len(vel) else None) or b["motion"]
            f[o + 20 + 4 * k:o + 24 + 4 * k] = [p[0], p[1], v[0], v[1]]
    return f, len(bnds)


def pts_at(mb, t):
    """app.js:543: the boundary's points at model time t."""
    vel = mb.get("vel") or []
    out = []
    for i, p in enumerate(mb["pts"]):
        v = (vel[i] if i < len(vel) else None) or mb["motion"]
        out.append([p[0] + v[0] * t, p[1] + v[1] * t])
    return out


def sdist(mb, x, y, t):
    """app.js:544-557: signed distance (> 0 inside the boundary's air mass) and how far beyond its end points."""
    P = pts_at(mb, t)
    n = len(P)
    best, sg, over = 1e30, 1, 0.0
    for i in range(n - 1):
        ax, ay, bx, by = P[i][0], P[i][1], P[i + 1][0], P[i + 1][1]
        abx, aby = bx - ax, by - ay
        la = max(math.hypot(abx, aby), 1)
        t0 = ((x - ax) * abx + (y - ay) * aby) / (la * la)
        tt = t0
        if i > 0:
            tt = max(tt, 0)
        if i < n - 2:
            tt = min(tt, 1)
        d = math.hypot(x - (ax + tt * abx), y - (ay + tt * aby))
        if d < best:
            best = d
            sg = 1 if abx * (y - ay) - aby * (x - ax) > 0 else -1
            over = (max(-t0, 0) * la if i == 0 else 0) + (max(t0 - 1, 0) * la if i == n - 2 else 0)
    return best * sg * mb["side"], over


def other_weight(mbs, x, y, t):
    """app.js:559-563: the largest weight of any boundary's air mass at (x, y)."""
    w = 0.0
    for mb in mbs:
        d, over = sdist(mb, x, y, t)
        w = max(w, smooth(-mb["halfW"], mb["halfW"], d) * (1 - smooth(0, 60000, over)))
    return w
