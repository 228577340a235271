"""Soundings: SHARPpy parser, parcel/kinematic analysis and the hydrostatic base state of the cloud model.

Host-side mirror of the reference's ``Sounding`` module (sounding.js:7-200). JavaScript numbers are IEEE f64, so this
is plain Python float arithmetic in the same order; the base state is stored as float32 like the reference's
``Float32Array`` (sounding.js:160). The result feeds ``ob_model_set_base_state`` / ``RegionalModel.set_sounding``.
"""
from __future__ import annotations

import math
import re
from dataclasses import dataclass, field

import numpy as np

KT = 0.514444
RD, CP, LV, EPS, G, RV = 287.04, 1005.7, 2.501e6, 0.622, 9.80665, 461.5


@dataclass
class Level:
    p: float
    h: float
    t: float
    td: float
    wd: float
    ws: float


@dataclass
class SoundingData:
    title: str = ""
    station: str = ""
    levels: list = field(default_factory=list)


def _isfinite(v):
    return v is not None and math.isfinite(v)


def parse_sharppy(text: str) -> SoundingData:
    """sounding.js:10-32: %TITLE% / %RAW% rows of PRES, HGHT, TEMP, DWPT, WDIR, WSPD(kt), sorted by falling pressure."""
    out = SoundingData()
    mode = ""
    for raw in text.replace("\r", "").split("\n"):
        L = raw.strip()
        if not L:
            continue
        if re.match(r"^%TITLE%", L, re.I):
            mode = "title"
            continue
        if re.match(r"^%RAW%", L, re.I):
            mode = "raw"
            continue
        if re.match(r"^%END%", L, re.I):
            mode = ""
            continue
        if mode == "title":
            if not out.title:
                out.title = L
                out.station = L.split()[0]
            continue
        if mode == "raw" or (not mode and re.match(r"^-?\d", L)):
            parts = [x for x in re.split(r"[,\s]+", L) if x]
            try:
                f = [float(x) for x in parts]
            except ValueError:
                continue
            if len(f) < 6 or any(not math.isfinite(v) for v in f):
                continue
            p, h, t, td, wd, ws = f[:6]
            if p <= 0 or h < -1000 or h > 40000 or p == -9999:
                continue
            nan = float("nan")
            out.levels.append(Level(p, h, t if t > -9990 else nan, td if td > -9990 else nan,
                                    wd if wd > -9990 else nan, ws if ws > -9990 else nan))
    out.levels.sort(key=lambda lv: -lv.p)
    if len(out.levels) < 4:
        raise ValueError("Could not read at least 4 levels. Expected SHARPpy format: %RAW% rows of  "
                         "PRES, HGHT, TEMP, DWPT, WDIR, WSPD(kt)  ... %END%")
    return out


def es(t):  # sounding.js:34
    return 6.112 * math.exp(17.67 * t / (t + 243.5))


def mixr(p, t):  # sounding.js:35
    e = es(t)
    return EPS * e / max(p - e, 1e-3)


def tvK(tK, w):
    return tK * (1 + 0.61 * w)


def _interp_logp(levels, key, p):  # sounding.js:37-48
    for i in range(len(levels) - 1):
        a, b = levels[i], levels[i + 1]
        if a.p >= p >= b.p:
            va, vb = getattr(a, key), getattr(b, key)
            if not (_isfinite(va) and _isfinite(vb)):
                return va if _isfinite(va) else vb
            f = math.log(a.p / p) / math.log(a.p / b.p)
            return va + (vb - va) * f
    return float("nan")


def _moist_step(p, tK, dp):  # sounding.js:49-53 (RK4 on the moist adiabat)
    def f(pp, T):
        rs = mixr(pp, T - 273.15)
        return (1 / pp) * (RD * T + LV * rs) / (CP + LV * LV * rs * EPS / (RD * T * T))
    k1 = f(p, tK)
    k2 = f(p + dp / 2, tK + dp / 2 * k1)
    k3 = f(p + dp / 2, tK + dp / 2 * k2)
    k4 = f(p + dp, tK + dp * k3)
    return tK + dp / 6 * (k1 + 2 * k2 + 2 * k3 + k4)


def _lift_parcel(grid, p0, t0, td0):  # sounding.js:54-84
    T0, TD0 = t0 + 273.15, td0 + 273.15
    tl = 1 / (1 / (TD0 - 56) + math.log(T0 / TD0) / 800) + 56
    pl = p0 * math.pow(tl / T0, 1 / 0.2857)
    w0 = mixr(p0, td0)
    theta = T0 * math.pow(1000 / p0, 0.2857)
    cin, lfcH, elH, above, capeTot = 0.0, float("nan"), float("nan"), False, 0.0
    moistP, moistT = pl, tl
    pts = []
    for k, p in enumerate(grid["p"]):
        if p > p0:
            continue
        if p >= pl:
            tp, wp = theta * math.pow(p / 1000, 0.2857), w0
        else:
            while moistP > p + 1e-6:
                dp = max(-5, p - moistP)
                moistT = _moist_step(moistP, moistT, dp)
                moistP += dp
            tp, wp = moistT, mixr(p, moistT - 273.15)
        pts.append((p, grid["h"][k], tvK(tp, wp), grid["tv"][k]))
    lclH = grid["hAt"](pl)
    for k in range(1, len(pts)):
        a, b = pts[k - 1], pts[k]
        buoy = ((a[2] - a[3]) / a[3] + (b[2] - b[3]) / b[3]) / 2
        e = G * buoy * (b[1] - a[1])
        if buoy > 0:
            if not above and b[0] < pl + 1:
                above = True
                if not math.isfinite(lfcH):
                    lfcH = a[1]
            if above:
                capeTot += e
                elH = b[1]
        elif not above:
            cin += e
    return {"cape": max(0.0, capeTot), "cin": min(0.0, cin), "lclH": lclH, "lfcH": lfcH, "elH": elH, "pLcl": pl}


@dataclass
class Analysis:
    sfcH: float
    P: dict
    rm: tuple
    lm: tuple
    mean6: tuple
    wl: list

    def wind_at(self, z):  # sounding.js:118-123 (z in km AGL)
        wl = self.wl
        if z <= wl[0][0]:
            return wl[0][1], wl[0][2]
        for i in range(len(wl) - 1):
            if wl[i][0] <= z <= wl[i + 1][0]:
                f = (z - wl[i][0]) / max(1e-6, wl[i + 1][0] - wl[i][0])
                return wl[i][1] + (wl[i + 1][1] - wl[i][1]) * f, wl[i][2] + (wl[i + 1][2] - wl[i][2]) * f
        return wl[-1][1], wl[-1][2]

    def mean_wind(self, z0, z1):
        u = v = 0.0
        k = 0
        z = z0
        while z <= z1 + 1e-9:
            w = self.wind_at(z)
            u += w[0]
            v += w[1]
            k += 1
            z += 0.05
        return u / k, v / k


def analyze(snd: SoundingData, parcels: bool = True) -> Analysis:
    """sounding.js:86-137: SB/ML/MU parcels, Bunkers motion, SRH, shear, STP. ``parcels=False`` skips the parcel
    lifts (the base state only needs the wind profile)."""
    lv = [l for l in snd.levels if _isfinite(l.h)]
    sfc = lv[0]
    sfcH = sfc.h
    wl = []
    for l in lv:
        if _isfinite(l.wd) and _isfinite(l.ws):
            d = l.wd * math.pi / 180
            s = l.ws * KT
            wl.append(((l.h - sfcH) / 1000, -s * math.sin(d), -s * math.cos(d)))
    A = Analysis(sfcH, {}, (0, 0), (0, 0), (0, 0), wl)
    mean6 = A.mean_wind(0, 6)
    lo = A.mean_wind(0, 0.5)
    hi = A.mean_wind(5.5, 6)
    sh = (hi[0] - lo[0], hi[1] - lo[1])
    shm = math.hypot(*sh) or 1
    A.rm = (mean6[0] + 7.5 * sh[1] / shm, mean6[1] - 7.5 * sh[0] / shm)
    A.lm = (mean6[0] - 7.5 * sh[1] / shm, mean6[1] + 7.5 * sh[0] / shm)
    A.mean6 = mean6

    def srh(z1, cm):
        s = 0.0
        prev = A.wind_at(0)
        z = 0.02
        while z <= z1 + 1e-9:
            w = A.wind_at(z)
            s += (w[0] - cm[0]) * (prev[1] - cm[1]) - (prev[0] - cm[0]) * (w[1] - cm[1])
            prev = w
            z += 0.02
        return s

    def shear(z0, z1):
        a, b = A.wind_at(z0), A.wind_at(z1)
        return math.hypot(b[0] - a[0], b[1] - a[1])

    P = {"srh05": srh(0.5, A.rm), "srh1": srh(1, A.rm), "srh3": srh(3, A.rm), "shr1": shear(0, 1), "shr6": shear(0, 6)}
    if parcels:
        grid = {"p": [], "h": [], "tv": []}
        p = sfc.p
        pmin = max(100, lv[-1].p)
        while p >= pmin:
            t, td, h = _interp_logp(lv, "t", p), _interp_logp(lv, "td", p), _interp_logp(lv, "h", p)
            if math.isfinite(t) and math.isfinite(h):
                grid["p"].append(p)
                grid["h"].append(h - sfcH)
                grid["tv"].append(tvK(t + 273.15, mixr(p, td) if math.isfinite(td) else 0))
            p -= 2

        def hAt(pp):
            gp, gh = grid["p"], grid["h"]
            for k in range(len(gp) - 1):
                if gp[k] >= pp >= gp[k + 1]:
                    f = math.log(gp[k] / pp) / math.log(gp[k] / gp[k + 1])
                    return gh[k] + (gh[k + 1] - gh[k]) * f
            return 0 if pp > gp[0] else gh[-1]
        grid["hAt"] = hAt
        sb = _lift_parcel(grid, sfc.p, sfc.t, sfc.td)
        thS = wS = 0.0
        n = 0
        p = sfc.p
        while p >= sfc.p - 100:
            t, td = _interp_logp(lv, "t", p), _interp_logp(lv, "td", p)
            if math.isfinite(t) and math.isfinite(td):
                thS += (t + 273.15) * math.pow(1000 / p, 0.2857)
                wS += mixr(p, td)
                n += 1
            p -= 1
        thS /= n
        wS /= n
        mlT = thS * math.pow(sfc.p / 1000, 0.2857) - 273.15
        eML = wS * sfc.p / (EPS + wS)
        lnE = math.log(eML / 6.112)
        mlTd = 243.5 * lnE / (17.67 - lnE)
        ml = _lift_parcel(grid, sfc.p, mlT, min(mlTd, mlT))
        best, bestTe = None, -1
        for l in lv:
            if l.p < sfc.p - 300 or not _isfinite(l.t) or not _isfinite(l.td):
                continue
            w = mixr(l.p, l.td)
            te = (l.t + 273.15) * math.pow(1000 / l.p, 0.2857) * math.exp(LV * w / (CP * (l.t + 273.15)))
            if te > bestTe:
                bestTe, best = te, l
        mu = _lift_parcel(grid, best.p, best.t, best.td) if best else sb
        P.update(sbcape=sb["cape"], sbcin=sb["cin"], sblcl=sb["lclH"], mlcape=ml["cape"], mlcin=ml["cin"],
                 mllcl=ml["lclH"], mllfc=ml["lfcH"], mucape=mu["cape"],
                 el=mu["elH"] if math.isfinite(mu["elH"]) else 11000)
        lclTerm = 1 if P["mllcl"] < 1000 else 0 if P["mllcl"] > 2000 else (2000 - P["mllcl"]) / 1000
        shrTerm = 0 if P["shr6"] < 12.5 else min(1.5, P["shr6"] / 20)
        cinTerm = 1 if P["mlcin"] > -50 else 0 if P["mlcin"] < -200 else (200 + P["mlcin"]) / 150
        P["stp"] = max(0, (P["mlcape"] / 1500) * lclTerm * (P["srh1"] / 150) * shrTerm * cinTerm)
    A.P = P
    return A


def base_state(snd: SoundingData, nz: int, dz: float, motion=(0.0, 0.0)):
    """sounding.js:143-197. Returns (B float32[(nz+1)*8], sfcP hPa, sfcH m). Per level k: theta0, qv0, rho0 (centre),
    rho0 (bottom face), pi0, p0 (Pa), u0, v0; level nz holds the lid density in slot 3."""
    lv = sorted([l for l in snd.levels if _isfinite(l.h) and _isfinite(l.t)], key=lambda l: l.h)
    sfcH, sfcP = lv[0].h, lv[0].p

    def byH(key, zAgl):
        h = zAgl + sfcH
        if h <= lv[0].h:
            return getattr(lv[0], key)
        for i in range(len(lv) - 1):
            if h <= lv[i + 1].h:
                a, b = lv[i], lv[i + 1]
                f = (h - a.h) / max(b.h - a.h, 1e-3)
                va, vb = getattr(a, key), getattr(b, key)
                if not (_isfinite(va) and _isfinite(vb)):
                    return va if _isfinite(va) else vb
                if key == "p":
                    return math.exp(math.log(va) + (math.log(vb) - math.log(va)) * f)
                return va + (vb - va) * f
        return float("nan")

    top = lv[-1]
    A = analyze(snd, parcels=False)
    B = np.zeros((nz + 1) * 8, dtype=np.float32)
    th, qv = [], []
    for k in range(nz):
        z = (k + 0.5) * dz
        T, Td, p = byH("t", z), byH("td", z), byH("p", z)
        if not (math.isfinite(T) and math.isfinite(p)):
            dzt = z + sfcH - top.h
            T = top.t
            p = top.p * math.exp(-G * dzt / (RD * (top.t + 273.15)))
            Td = min(top.td, -80)
        if not math.isfinite(Td):
            Td = T - 30
        Td = min(Td, T - 0.3)
        th.append((T + 273.15) * math.pow(1000 / p, RD / CP))
        qv.append(max(1e-7, mixr(p, Td)))
    piF = [0.0] * (nz + 1)
    piF[0] = math.pow(sfcP / 1000, RD / CP)
    for k in range(nz):
        piF[k + 1] = piF[k] - G * dz / (CP * th[k] * (1 + 0.61 * qv[k]))
    for k in range(nz):
        pi = 0.5 * (piF[k] + piF[k + 1])
        p = 100000 * math.pow(pi, CP / RD)
        T = th[k] * pi
        esx = 611.2 * math.exp(17.67 * (T - 273.15) / (T - 29.65))
        qvs = EPS * esx / (p - esx)
        qv[k] = min(qv[k], 0.97 * qvs)
        rho = p / (RD * T * (1 + 0.61 * qv[k]))
        w = A.wind_at((k + 0.5) * dz / 1000)
        B[k * 8:k * 8 + 8] = [th[k], qv[k], rho, 0, pi, p, w[0] - motion[0], w[1] - motion[1]]
    # face densities (read back from the float32 array, as the reference does)
    for k in range(nz + 1):
        if k == 0:
            r = float(B[2]) + (float(B[2]) - float(B[10])) * 0.5
        elif k == nz:
            r = float(B[(nz - 1) * 8 + 2]) * 0.94
        else:
            r = 0.5 * (float(B[(k - 1) * 8 + 2]) + float(B[k * 8 + 2]))
        B[k * 8 + 3] = r
    return B, sfcP, sfcH
