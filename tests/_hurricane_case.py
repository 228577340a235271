"""The hurricane-mode case of the tests (shared by the CPU and GPU tests): the synthetic tropical setup of
outbreaklab_b200.hurricane on a small domain with a strip of land, and the oracle set up the way
hurricane.setup sets up the GPU model."""

from outbreaklab_b200 import hurricane as H, sounding as snd_mod, workloads as W

from oracle import oracle as O

LAT = 20.0


def case():
    return H.tropical_case(nx=40, ny=36, nz=40, dx=2000.0, land_cols=6)


def base_state(c):
    text = W.weisman_klemp_sharppy(**c.wk)
    B, sfcP, _ = snd_mod.base_state(snd_mod.parse_sharppy(text), c.nz, c.dz)
    return B, sfcP


def oracle_setup(c, surf, vort, precision, lat=LAT):
    B, sfcP = base_state(c)
    m = O.OracleModel(c.nx, c.ny, c.nz, c.dx, precision)
    p = O.default_params()
    p.noise = 0.0
    p.lat = lat
    p.scheme = float(c.scheme)
    m.set_params(p)
    m.set_base_state(B)
    h = O.default_hurricane()
    h.sfcP = float(sfcP) * 100.0
    h.centreX, h.centreY = float(vort["x"]), float(vort["y"])
    m.set_surface(surf, h)
    tab, info = H.vortex_table(c.nz, c.dz, c.dx, lat, B, **vort)
    m.set_vortex(tab, info["nr"], info["x"], info["y"], info["dr"], info["moistR"], info["moistRH"])
    m.reset()
    return m, B, tab, info
