"""Hurricane mode on the B200 model: the host side of RegionalModel.setSurface / setVortex (model.js:1290-1365).

The kernels' hurricane branches (sea fluxes, drag, radiative relaxation, far-field hold, boundary-layer thermals,
K-profile boundary layer, warm-bubble storm starts, settling ice, maritime graupel, midpoint trajectories, the
trajectory-averaged pressure force and the 2-dx filter) run on the GPU once a model has a surface and a hurricane
(`RegionalModel.set_surface`). This module builds the initial vortex's table the way setVortex does: a Rankine-type
tangential wind made inertially stable, its pressure in gradient-wind balance and its warm core in hydrostatic
balance with that pressure. The tropical soundings, the sea-surface temperature and land maps and the storm tracker of
the reference's hurricane.js belong to its app and are not restated; `tropical_case` gives a synthetic stand-in (an
analytic moist sounding over a uniform sea with a strip of land) for tests and runs.
"""
from __future__ import annotations

import math

import numpy as np

VX_MAXR = 2048   # model.js:38, the most radii of the vortex table
DEG = math.pi / 180.0


def smooth(a, b, x):
    t = min(max((x - a) / (b - a), 0.0), 1.0)
    return t * t * (3 - 2 * t)


def js_round(x):
    """Math.round: halves go up."""
    return math.floor(x + 0.5)


def vortex_table(nz, dz, dx, lat, B, x, y, vmax, rmw, r0, ztop, moist_r=0.0, moist_rh=0.0, shape="deep"):
    """setVortex (model.js:1318-1365). B: the base state (nz+1)*8. Returns (table float32 (nz, nr, 4), info dict with
    nr, dr, the centre, the moist core, the central pressure deficit pc (hPa), the least core stability minStab (K/km)
    and the warm core's peak (K))."""
    f = 2 * 7.292e-5 * math.sin(lat * DEG)
    dr = max(500.0, dx / 2)
    nr = min(VX_MAXR, math.ceil(r0 * 2 / dr) + 3)
    sg = -1.0 if f < 0 else 1.0     # cyclonic in either hemisphere
    fa, al = abs(f), 0.6
    vs = np.zeros(nr)
    Mp = 0.0
    for i in range(nr):
        r = i * dr
        xx = r / rmw
        s = vmax * (1 + al) * xx / (al + xx ** (1 + al)) * (1 - smooth(0.5 * r0, r0, r))
        if r > 0:   # inertial stability: the absolute angular momentum never decreases outward
            s = max(s, (Mp - 0.5 * fa * r * r) / r, 0.0)
        vs[i] = s
        Mp = r * s + 0.5 * fa * r * r

    def Vs(r):
        return sg * vs[min(nr - 1, js_round(r / dr))]

    if shape == "mid":
        def Fz(z):
            return math.exp(-((z - 5000) / 2500) ** 2)
    else:
        def Fz(z):
            return 0.0 if z >= ztop else 1 - (z / ztop - math.sin(2 * math.pi * z / ztop) / (2 * math.pi))
    vt, ph = [], []
    for k in range(nz):
        F = Fz((k + 0.5) * dz)
        vk = np.array([Vs(i * dr) * F for i in range(nr)])
        pk = np.zeros(nr)

        def g(i):
            return 0.0 if i == 0 else vk[i] * vk[i] / (i * dr) + f * vk[i]
        for i in range(nr - 2, -1, -1):   # phi(r) = -int_r^inf (v^2/r' + f v) dr'
            pk[i] = pk[i + 1] - 0.5 * (g(i) + g(i + 1)) * dr
        vt.append(vk)
        ph.append(pk)
    tab = np.zeros((nz, nr, 4), np.float32)
    for k in range(nz):
        k0, k1 = max(k - 1, 0), min(k + 1, nz - 1)
        b = (ph[k1] - ph[k0]) / ((k1 - k0) * dz)
        tab[k, :, 0] = vt[k]
        tab[k, :, 1] = float(B[k * 8]) * b / 9.81
    min_stab, warm = 1e9, 0.0
    for k in range(1, nz):
        z = k * dz
        if z < 2000 or z > ztop:
            continue
        for i in range(min(nr, math.ceil(2 * rmw / dr))):
            a = float(B[(k - 1) * 8]) + float(tab[k - 1, i, 1])
            bb = float(B[k * 8]) + float(tab[k, i, 1])
            min_stab = min(min_stab, (bb - a) / dz * 1000)
        warm = max(warm, float(tab[k, 0, 1]))
    info = {"x": x, "y": y, "dr": dr, "nr": nr, "moistR": moist_r or 1.0, "moistRH": moist_rh if moist_r else 0.0,
            "pc": ph[0][0] * float(B[2]) / 100, "minStab": min_stab, "warm": warm}
    return tab, info


def tropical_case(nx=96, ny=96, nz=40, dx=2000.0, sst=302.0, land_cols=0, seed=3):
    """A synthetic hurricane setup: an analytic moist tropical sounding (the Weisman-Klemp family with no shear, warm
    and moist), a uniform sea of temperature sst with `land_cols` columns of land on the west edge, and a vortex at
    the domain centre. Returns (StormCase, surf (ny, nx, 4) float32, vortex kwargs)."""
    from . import workloads as W
    case = W.StormCase("hurricane", nx, ny, nz, dx, 6.0 * dx / 1000.0, 1, scheme=0, bubbles=[], seed=seed,
                       wk={"theta_sfc": 300.0, "qv_max": 0.018, "shear_u": 0.0})
    surf = np.zeros((ny, nx, 4), np.float32)
    surf[..., 1] = sst
    if land_cols:
        surf[:, :land_cols, 0] = 1.0
        surf[:, :land_cols, 1] = sst - 4.0
    Lx, Ly = nx * dx, ny * dx
    vort = {"x": Lx / 2, "y": Ly / 2, "vmax": 25.0, "rmw": 8 * dx, "r0": 0.35 * min(Lx, Ly), "ztop": 15000.0,
            "moist_r": 0.2 * min(Lx, Ly), "moist_rh": 0.9}
    return case, surf, vort


def default_hurricane():
    """ObHurricane with the library's defaults (ob_hurricane_default)."""
    import ctypes as C
    from . import _native as N
    h = N.ObHurricane()
    N.lib().ob_hurricane_default(C.byref(h))
    return h


def setup(case, surf, vort, lat=20.0, hur=None, noise=0.0):
    """A RegionalModel in hurricane mode, set up in the app's order (app.js:1611-1650): base state, parameters
    (latitude, Lin scheme), surface and hurricane, vortex, reset. Returns (model, B, hurricane, table, info)."""
    from . import model as M, sounding as snd_mod, workloads as W
    m = M.RegionalModel().allocate(spec={"dx": case.dx, "n": [case.nx, case.ny, case.nz]})
    m.params["noise"] = noise
    m.params["lat"] = lat
    m.params["scheme"] = "thompson" if case.scheme == 1 else "lin"
    text = W.weisman_klemp_sharppy(**case.wk)
    B, sfcP, _ = snd_mod.base_state(snd_mod.parse_sharppy(text), case.nz, case.dz)
    m.set_base_state(B)
    h = hur or default_hurricane()
    h.sfcP = float(sfcP) * 100.0
    h.centreX, h.centreY = float(vort["x"]), float(vort["y"])
    m.set_surface(surf, h)
    tab, info = vortex_table(case.nz, case.dz, case.dx, lat, B, **vort)
    m.set_vortex(tab, info)
    m.reset()
    return m, B, h, tab, info
