"""A small storm state, a projection and a radar site for the radar tests (shared by the CPU and GPU tests).

The state is a seeded hydrometeor blob (workloads.hydrometeor_blob) on a 48 x 40 x 40 domain at 1 km, plus a few
steps of the model so the winds carry structure; the site sits 20 km west and 15 km south of the domain's corner so
every cut's beams cross the storm."""
import numpy as np

from outbreaklab_b200 import radar as RD, workloads as W

LAT0, LON0, GROUND = 35.9, -97.2, 350.0


def case(scheme=0):
    return W.case_small(nx=48, ny=40, nz=40, dx=1000.0, dt=6.0, scheme=scheme)


def geo_for(c):
    return RD.Geo(LAT0, LON0, c.nx * c.dx, c.ny * c.dx, GROUND)


def site_for(c, geo, dx_m=-20000.0, dy_m=-15000.0):
    lat, lon = geo.from_model(dx_m, dy_m)
    return {"id": "KTST", "lat": lat, "lon": lon, "h": GROUND + 5.0}


class _ModelDims:
    """What RadarSim.cut_uniforms reads from a model, for a model that is not a RegionalModel (the oracle)."""

    def __init__(self, c, rho_sfc, scheme):
        self.nx, self.ny, self.nz, self.dx = c.nx, c.ny, c.nz, c.dx
        self.dz = 20000.0 / c.nz
        self.Lx, self.Ly = c.nx * c.dx, c.ny * c.dx
        self.rho_sfc = rho_sfc
        self.params = {"scheme": "thompson" if scheme == 1 else "lin"}


def cut_plan(c, geo, site, B, scheme=0, cut_indices=(0, 1, 8), az0=0.37, vol=2, sim_t=600.0, min_dbz=0.0, ntor=0):
    """The uniform blocks RadarSim.enc_cut would build for the given VCP 212 cuts, without a GPU."""
    sim = RD.RadarSim.__new__(RD.RadarSim)
    sim.m, sim.geo, sim.nTor = _ModelDims(c, float(B[2]), scheme), geo, ntor
    vcp = RD.VCPS[212]
    sx, sy = geo.to_model(site["lat"], site["lon"])
    ngr, ngd, cuts, nbytes = RD.radar_layout(c.nx * c.dx, c.ny * c.dx, sx, sy, vcp)
    R = {"site": site, "opts": {"minDbz": min_dbz}, "sx": sx, "sy": sy, "ngRef": ngr, "ngDop": ngd, "vol": vol,
         "az0": az0}
    return [(cuts[i], sim.cut_uniforms(R, cuts[i], sim_t)) for i in cut_indices], ngr, ngd, nbytes


TORNADO = [{"x": 24000.0, "y": 20000.0, "R": 150.0, "v": 60.0, "debrisTop": 1500.0, "debrisDbz": 55.0, "debris": 1.0}]


def tornado_array(lst=TORNADO):
    f = np.zeros(max(1, len(lst)) * 8, np.float32)
    for i, t in enumerate(lst):
        f[i * 8:(i + 1) * 8] = [t["x"], t["y"], t["R"], t["v"], t["debrisTop"], t["debrisDbz"], t["debris"], 0]
    return f
