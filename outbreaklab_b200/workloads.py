"""Synthetic workloads: the Weisman-Klemp analytic sounding, warm bubbles and seeded theta noise.

None of these exist in the reference, which starts storms by updraft nudging (model.js:683-694) from SHARPpy
soundings. The analytic sounding is written as SHARPpy text so that it goes through the reference's own base-state
path (``sounding.base_state``, sounding.js:143-197); bubbles and noise are added to theta after ``reset`` on the host
so that the oracle and the GPU start from identical bytes.

Configurations (sizes and spacings of the headline benchmark and the parity cases):
  C1  64 x 64 x 40, dx 2 km, dt 12 s, one bubble, Lin-type microphysics
  C2  640 x 640 x 40, dx 1 km, dt 6 s, 8 bubbles >= 35 km apart and >= 40 km from the edges, Lin-type
  C3  1024 x 1024 x 80 pressure solve, Gaussian random field RHS with 5 km correlation length
  C4  512 x 512 x 40, dx 500 m, dt 3 s, Thompson-style microphysics
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

from . import sounding as snd_mod

G, CP, RD = 9.80665, 1005.7, 287.04


# ---------------------------------------------------------------------------------------------------------------
# mulberry32 (app.js:1308), vectorised: the n-th draw depends only on seed + n * 0x6D2B79F5
# ---------------------------------------------------------------------------------------------------------------
def mulberry32_block(seed: int, n: int, start: int = 0) -> np.ndarray:
    """Draws start .. start+n-1 of mulberry(seed) as float64 in [0, 1)."""
    with np.errstate(over="ignore"):
        idx = np.arange(start + 1, start + n + 1, dtype=np.uint64)
        a = ((np.uint64(seed & 0xFFFFFFFF) + idx * np.uint64(0x6D2B79F5)) & np.uint64(0xFFFFFFFF)).astype(np.uint32)
        t = (a ^ (a >> np.uint32(15))) * (a | np.uint32(1))
        t = (t + (t ^ (t >> np.uint32(7))) * (t | np.uint32(61))) ^ t
        return (t ^ (t >> np.uint32(14))).astype(np.float64) / 4294967296.0


class Mulberry32:
    def __init__(self, seed: int):
        self.seed = seed & 0xFFFFFFFF
        self.n = 0

    def __call__(self) -> float:
        v = mulberry32_block(self.seed, 1, self.n)[0]
        self.n += 1
        return float(v)


# ---------------------------------------------------------------------------------------------------------------
# Weisman & Klemp (1982) analytic sounding
# ---------------------------------------------------------------------------------------------------------------
def weisman_klemp_sharppy(theta_sfc=300.0, z_tr=12000.0, theta_tr=343.0, T_tr=213.0, qv_max=0.014,
                          shear_u=25.0, shear_depth=6000.0, p_sfc=1000.0, dz=50.0, ztop=20000.0,
                          rh_scale=1.0) -> str:
    """theta(z) = theta_s + (theta_tr - theta_s)(z/z_tr)^(5/4) below the tropopause, isothermal (T_tr) above;
    RH = 1 - 3/4 (z/z_tr)^(5/4) (0.25 above), qv capped at qv_max; u rising linearly to shear_u over shear_depth,
    v = 0. Hydrostatic pressure from p_sfc with the virtual potential temperature. Rows every dz to ztop."""
    z = np.arange(0.0, ztop + 0.5 * dz, dz)
    th = np.where(z <= z_tr, theta_sfc + (theta_tr - theta_sfc) * (z / z_tr) ** 1.25,
                  theta_tr * np.exp(G / (CP * T_tr) * (z - z_tr)))
    rh = np.where(z <= z_tr, 1.0 - 0.75 * (z / z_tr) ** 1.25, 0.25) * rh_scale
    qv = np.zeros_like(z)
    for _ in range(6):
        thv = th * (1 + 0.61 * qv)
        pi = np.empty_like(z)
        pi[0] = (p_sfc / 1000.0) ** (RD / CP)
        for k in range(1, len(z)):
            pi[k] = pi[k - 1] - G * (z[k] - z[k - 1]) / (CP * 0.5 * (thv[k] + thv[k - 1]))
        p = 1000.0 * pi ** (CP / RD)
        T = th * pi
        tc = T - 273.15
        es = 6.112 * np.exp(17.67 * tc / (tc + 243.5))
        qvs = 0.622 * es / np.maximum(p - es, 1e-3)
        qv = np.minimum(rh * qvs, qv_max)
    e = qv * p / (0.622 + qv)
    L = np.log(np.maximum(e, 1e-10) / 6.112)
    td = 243.5 * L / (17.67 - L)
    u = shear_u * np.minimum(z / shear_depth, 1.0)
    ws = u / snd_mod.KT
    lines = ["%TITLE%", " WK82   analytic", "", "   LEVEL       HGHT       TEMP       DWPT       WDIR       WSPD",
             "-------------------------------------------------------------------", "%RAW%"]
    for k in range(len(z)):
        lines.append("%.4f, %.2f, %.4f, %.4f, %.2f, %.4f" % (p[k], z[k], tc[k], td[k], 270.0, ws[k]))
    lines.append("%END%")
    return "\n".join(lines)


# ---------------------------------------------------------------------------------------------------------------
# configurations
# ---------------------------------------------------------------------------------------------------------------
@dataclass
class StormCase:
    name: str
    nx: int
    ny: int
    nz: int
    dx: float
    dt: float
    steps: int
    scheme: int = 0                       # 0 Lin-type, 1 Thompson-style
    bubbles: list = field(default_factory=list)   # (xc, yc) model metres
    bubble_dth: float = 3.0
    bubble_rh: float = 10000.0
    bubble_rz: float = 1500.0
    bubble_zc: float = 1500.0
    noise: float = 0.1
    seed: int = 1
    wk: dict = field(default_factory=dict)

    @property
    def dz(self):
        return 20000.0 / self.nz

    @property
    def cells(self):
        return self.nx * self.ny * self.nz


def place_bubbles(n, Lx, Ly, seed, min_sep=35000.0, edge=40000.0, max_tries=100000):
    """Rejection sampling of n centres >= min_sep apart and >= edge from the domain edges (mulberry32(seed))."""
    rng = Mulberry32(seed)
    pts = []
    tries = 0
    while len(pts) < n and tries < max_tries:
        tries += 1
        x = edge + (Lx - 2 * edge) * rng()
        y = edge + (Ly - 2 * edge) * rng()
        if all(math.hypot(x - a, y - b) >= min_sep for a, b in pts):
            pts.append((x, y))
    if len(pts) < n:
        raise ValueError("could not place %d bubbles" % n)
    return pts


def case_c1(steps=120):
    nx = ny = 64
    dx = 2000.0
    return StormCase("C1", nx, ny, 40, dx, 12.0, steps, bubbles=[(nx * dx / 2, ny * dx / 2)])


def case_c2(steps=600):
    nx = ny = 640
    dx = 1000.0
    return StormCase("C2", nx, ny, 40, dx, 6.0, steps, bubbles=place_bubbles(8, nx * dx, ny * dx, seed=2))


def case_c4(steps=1200):
    nx = ny = 512
    dx = 500.0
    return StormCase("C4", nx, ny, 40, dx, 3.0, steps, scheme=1, bubbles=place_bubbles(8, nx * dx, ny * dx, seed=4))


def case_small(nx=32, ny=24, nz=16, dx=2000.0, scheme=0, dt=12.0, steps=1, seed=1):
    """A small parity case (ragged sizes: nx != ny, neither a multiple of 8)."""
    return StormCase("small", nx, ny, nz, dx, dt, steps, scheme=scheme,
                     bubbles=[(nx * dx / 2, ny * dx / 2)], bubble_rh=min(10000.0, nx * dx / 4), seed=seed)


def base_state_for(case: StormCase):
    text = weisman_klemp_sharppy(**case.wk)
    s = snd_mod.parse_sharppy(text)
    B, sfcP, sfcH = snd_mod.base_state(s, case.nz, case.dz)
    return B, text


def perturb_theta(case: StormCase, V: np.ndarray) -> np.ndarray:
    """Adds the bubbles and the seeded +/- noise to theta of the interior cells of a V texel array
    ((nz+1)(ny+1)(nx+1) x 4, float32). Noise order: x fastest, then y, then z, one draw per cell."""
    nx, ny, nz, dx, dz = case.nx, case.ny, case.nz, case.dx, case.dz
    V = V.reshape(nz + 1, ny + 1, nx + 1, 4).copy()
    th = V[:nz, :ny, :nx, 3].astype(np.float64)
    z = (np.arange(nz) + 0.5) * dz
    y = (np.arange(ny) + 0.5) * dx
    x = (np.arange(nx) + 0.5) * dx
    Z, Y, X = np.meshgrid(z, y, x, indexing="ij")
    for (xc, yc) in case.bubbles:
        r = np.sqrt(((X - xc) / case.bubble_rh) ** 2 + ((Y - yc) / case.bubble_rh) ** 2
                    + ((Z - case.bubble_zc) / case.bubble_rz) ** 2)
        th += np.where(r < 1.0, case.bubble_dth * np.cos(0.5 * np.pi * r) ** 2, 0.0)
    if case.noise > 0:
        th += case.noise * (2.0 * mulberry32_block(case.seed, nx * ny * nz).reshape(nz, ny, nx) - 1.0)
    V[:nz, :ny, :nx, 3] = th.astype(np.float32)
    return V.reshape(-1)


def gaussian_rhs(nx, ny, nz, dx, corr_len=5000.0, seed=3, dtype=np.float64):
    """Seeded white noise low-passed by a Gaussian of the given correlation length (spectral filter), horizontal
    mean removed per level: the pressure-solve right-hand side of the 1024 x 1024 x 80 case."""
    rng = np.random.default_rng(seed)
    w = rng.standard_normal((nz, ny, nx))
    kx = np.fft.rfftfreq(nx, d=dx) * 2 * np.pi
    ky = np.fft.fftfreq(ny, d=dx) * 2 * np.pi
    K2 = ky[:, None] ** 2 + kx[None, :] ** 2
    filt = np.exp(-0.5 * K2 * corr_len ** 2)
    f = np.fft.irfft2(np.fft.rfft2(w, axes=(1, 2)) * filt[None], s=(ny, nx), axes=(1, 2))
    f -= f.mean(axis=(1, 2), keepdims=True)
    f /= max(np.abs(f).max(), 1e-30)
    return f.astype(dtype)


def hydrometeor_blob(case: StormCase, B, seed=5, thompson=False):
    """Seeded cloud / rain / ice / snow / graupel blobs and a supersaturated core (Q1, Q2 texel arrays, float32), so
    that one step exercises every microphysics process of both schemes: warm rain, riming, freezing, melting,
    evaporation, sublimation, the saturation adjustment and (Thompson) the rain-number budget."""
    nx, ny, nz, dx, dz = case.nx, case.ny, case.nz, case.dx, case.dz
    rng = np.random.default_rng(seed)
    z = (np.arange(nz) + 0.5) * dz
    y = (np.arange(ny) + 0.5) * dx
    x = (np.arange(nx) + 0.5) * dx
    Z, Y, X = np.meshgrid(z, y, x, indexing="ij")
    xc, yc = nx * dx / 2, ny * dx / 2
    r = np.sqrt(((X - xc) / (nx * dx / 4)) ** 2 + ((Y - yc) / (ny * dx / 4)) ** 2)
    blob = np.clip(1 - r, 0, 1) * (0.6 + 0.4 * rng.random((nz, ny, nx)))
    Bz = B.reshape(-1, 8)[:nz]
    qv0 = Bz[:, 1][:, None, None]
    T = Bz[:, 0][:, None, None] * Bz[:, 4][:, None, None]
    cold = (T < 268.0).astype(np.float64)
    warm = (T > 276.0).astype(np.float64)
    q1 = np.zeros((nz, ny, nx, 4))
    q2 = np.zeros((nz, ny, nx, 4))
    q1[..., 0] = qv0 * (1 + 0.08 * blob)                          # supersaturated core
    q1[..., 1] = 1.5e-3 * blob * (Z < 9000)                        # cloud water
    q1[..., 2] = 8e-4 * blob * cold                                # cloud ice
    q1[..., 3] = 3e-3 * blob * (Z < 7000) + 2e-5 * (1 - blob)      # rain (light rain outside: evaporation)
    q2[..., 0] = 1.2e-3 * blob * (Z > 4000)                        # snow (melts below the freezing level)
    q2[..., 1] = 4e-3 * blob * (Z > 2000) + 1e-5 * warm * (1 - blob)  # graupel
    if thompson:
        q2[..., 2] = q1[..., 3] * 10 ** (5 + 2 * rng.random((nz, ny, nx)))  # rain number per kg
    return q1.astype(np.float32).reshape(-1), q2.astype(np.float32).reshape(-1)


# ---------------------------------------------------------------------------------------------------------------
# Air-mass boundaries and storm starts (app.js:52-56, 527-545, 1321-1345; model.js:1371-1389)
# ---------------------------------------------------------------------------------------------------------------
TRIPLE_POINT = (36.3, -99.9)   # where the example cold front, warm front and dryline meet (app.js:53-55)


def case_fronts(nx=96, ny=88, nz=40, dx=2000.0, scheme=0):
    """A parity case for the large-scale forcing: the reference's example fronts over a domain centred on their
    triple point (2 km, dt 12 s: the LSF pass reruns after 5 steps), one warm bubble in the warm sector."""
    Lx, Ly = nx * dx, ny * dx
    return StormCase("fronts", nx, ny, nz, dx, 12.0, 6, scheme=scheme, bubbles=[(0.7 * Lx, 0.3 * Ly)],
                     bubble_rh=min(10000.0, Lx / 8))


def fronts_setup(case: StormCase, n_towers=2, seed=7, t0=-300.0):
    """The boundaries and storm-start towers of ``case_fronts``: the reference's default cold front, warm front and
    dryline (boundaries.default_bounds) projected about their triple point at the domain centre, with the surface lows'
    joined motion and the sounding's 150 m wind (boundaries.boundary_models), and ``n_towers`` main towers drawn by
    the run's storm-start scheduler in the warm sector, already pushing at t = 0 (started at ``t0``, no satellites).
    Returns (bounds, events)."""
    from . import boundaries as BND
    from .radar import Geo
    from .runloop import CIScheduler
    text = weisman_klemp_sharppy(**case.wk)
    A = snd_mod.analyze(snd_mod.parse_sharppy(text))
    geo = Geo(TRIPLE_POINT[0], TRIPLE_POINT[1], case.nx * case.dx, case.ny * case.dx)
    bounds = BND.boundary_models(BND.default_bounds(), geo, A.wind_at(0.15))

    class _Dom:
        Lx, Ly = case.nx * case.dx, case.ny * case.dx
        time = 0.0

        def set_ci(self, ev):
            pass

    sch = CIScheduler(_Dom(), {"seed": seed}, motion=A.rm)
    events = []
    spots = [(0.72, 0.28), (0.62, 0.42), (0.80, 0.40)]   # the warm sector: south-east of the triple point
    for k in range(n_towers):
        x, y = spots[k % len(spots)]
        events.append(sch.tower_cluster(x * case.nx * case.dx, y * case.ny * case.dx, t0, "warm sector")[0])
    return bounds, events
