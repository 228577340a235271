"""Air-mass boundaries on the host (app.js:12-65, 479-563; model.js:1371-1380) and the storm starts along them
(app.js:1416-1432), on CPU: geometry, surface lows, the packed record, the oracle's large-scale forcing with the
reference's example fronts, and the scheduler's boundary draws."""
import math

import numpy as np
import pytest

from outbreaklab_b200 import boundaries as BND, runloop as RL, workloads as W
from outbreaklab_b200.radar import Geo


def _fronts():
    case = W.case_fronts()
    bounds, events = W.fronts_setup(case)
    return case, bounds, events


def test_default_fronts_meet_in_one_low_that_moves_as_one_point():
    geo = Geo(*W.TRIPLE_POINT, 192000.0, 176000.0)
    bnds = BND.default_bounds()
    lows = BND.find_lows(bnds, geo)
    assert len(lows) == 1 and len(lows[0]["members"]) == 3 and lows[0]["front"]
    assert abs(lows[0]["x"]) < 1.0 and abs(lows[0]["y"]) < 1.0      # the triple point is the projection's centre
    vel = BND.boundary_vels(bnds, geo)
    mean = [sum(BND.bnd_motion(b)[c] for b in bnds) / 3 for c in range(2)]
    assert vel[0][2] == vel[1][0] == vel[2][0] == pytest.approx(mean)
    assert vel[0][0] == BND.bnd_motion(bnds[0])                         # other vertices move with their boundary
    # a fixed low motion overrides the mean (app.js:517-518)
    vel2 = BND.boundary_vels(bnds, geo, {"auto": False, "speed": 10.0, "dir": 90.0})
    assert vel2[1][0] == pytest.approx([10.0, 0.0], abs=1e-12)


def test_sides_put_the_other_air_mass_behind_fronts_and_west_of_the_dryline():
    case, bounds, _ = _fronts()
    Lx, Ly = case.nx * case.dx, case.ny * case.dx
    warm_sector = (0.75 * Lx, 0.25 * Ly)
    for mb in bounds:
        d, over = BND.sdist(mb, *warm_sector, 0.0)
        assert d < 0, mb["b"]["type"]                                  # outside every air mass
    assert BND.other_weight(bounds, *warm_sector, 0.0) == 0.0
    assert BND.other_weight(bounds, 0.05 * Lx, 0.3 * Ly, 0.0) == 1.0   # west: behind the dryline
    assert BND.other_weight(bounds, 0.8 * Lx, 0.95 * Ly, 0.0) == 1.0   # north: the cold air of the warm front
    # flip turns a boundary's side around
    b = dict(BND.default_bounds()[2], flip=True)
    geo = Geo(*W.TRIPLE_POINT, Lx, Ly)
    assert BND.bnd_model(b, geo, (0.0, 0.0))["side"] == -bounds[2]["side"]


def test_packed_record_layout():
    _, bounds, _ = _fronts()
    f, n = BND.pack_boundaries(bounds)
    assert n == 3 and f.dtype == np.float32 and f.size == BND.MAX_BOUNDS * 148
    for i, mb in enumerate(bounds):
        r = f[i * 148:(i + 1) * 148]
        want = [len(mb["pts"]), *mb["motion"], mb["halfW"], mb["dT"], mb["Hmax"], mb["slope"], mb["Hmin"], mb["dq"],
                mb["qRatio"], mb["du"], mb["dv"], mb["wRatio"], 1.0, mb["dFree"], mb["side"], mb["vary"], mb["seed"],
                mb["varyL"], 0.0]
        assert np.array_equal(r[:20], np.array(want, np.float32))
        for k, p in enumerate(mb["pts"]):
            assert np.array_equal(r[20 + 4 * k:24 + 4 * k], np.array([p[0], p[1], *mb["vel"][k]], np.float32))
        assert not r[20 + 4 * len(mb["pts"]):].any()
    assert not f[3 * 148:].any()
    # at most 8 boundaries of at most 32 points
    many = [dict(bounds[0], pts=[[float(k), 0.0]] * 40, vel=None) for _ in range(10)]
    f, n = BND.pack_boundaries(many)
    assert n == 8 and f[0] == 32 and f[20 + 4 * 31 + 2] == np.float32(bounds[0]["motion"][0])


def test_oracle_forcing_with_the_example_fronts(oracle_lib):
    """The restated LSF pass with the fronts: FP32 and FP64 instantiations agree, and the anomalies have the fronts'
    signs (cold air behind the cold and warm fronts, hot dry air behind the dryline, nudging deep in the air masses)."""
    case, bounds, events = _fronts()
    f, _ = oracle_lib.setup_case(case, 4, bounds=bounds, ci=events)
    d, _ = oracle_lib.setup_case(case, 8, bounds=bounds, ci=events)
    nx, ny = case.nx, case.ny
    A = d.get(oracle_lib.FIELD_LSF_A, f64=True).reshape(ny, nx, 4)
    B = d.get(oracle_lib.FIELD_LSF_B, f64=True).reshape(ny, nx, 4)
    for fld in (oracle_lib.FIELD_LSF_A, oracle_lib.FIELD_LSF_B, oracle_lib.FIELD_PHT):
        a, r = f.get(fld).astype(np.float64), d.get(fld, f64=True)
        assert np.abs(a - r).max() <= 2e-4 * np.abs(r).max()
    assert A[-1, nx // 2, 0] < -3.0          # north: cold air
    assert A[4, nx // 4, 0] > 1.0             # south-west: behind the dryline
    assert A[ny // 4, 3 * nx // 4, 0] == 0.0  # warm sector
    assert B[:, :, 3].max() == 1.0 and B[ny // 4, 3 * nx // 4, 3] == 0.0
    for m in (f, d):
        m.step(case.dt, 1)
    C = d.get(oracle_lib.FIELD_CI_MAP, f64=True).reshape(-1, 4)
    assert ((C[:, 0] * C[:, 1]) > 0.5).sum() > 10


def _sched(bounds, case, **ci):
    class Dom:
        Lx, Ly = case.nx * case.dx, case.ny * case.dx
        nx, ny, dx = case.nx, case.ny, case.dx
        time = 0.0

        def set_ci(self, ev):
            pass

    return RL.CIScheduler(Dom(), dict({"seed": 7}, **ci), motion=(10.0, 2.0), bounds=bounds)


def test_starts_along_boundaries_land_on_their_warm_side():
    case, bounds, _ = _fronts()
    for mb in bounds:
        mb["b"] = dict(mb["b"], rate=4000.0)
    s = _sched(bounds, case, warmRate=0.0)
    t = 1800.0
    n = s.schedule(t, 60.0)
    mains = [e for e in s.events if e["zc"] == 2000.0 and e["rz"] == 2000.0]
    assert n > 5 and len(mains) == n
    labels = {BND.BND_TYPES[k]["label"].lower() for k in ("cold", "warm", "dry")}
    mar, warm = s.margin(), 0
    for e in mains:
        assert e["why"] in labels
        mb = next(m for m in bounds if BND.BND_TYPES[m["b"]["type"]]["label"].lower() == e["why"])
        d, _ = BND.sdist(mb, e["x"], e["y"], t)
        warm += d < 0
        assert abs(d) <= 22000.0 + 1.0          # at most 22 km off the polyline (nearer where segments meet)
        assert mar <= e["x"] <= s.m.Lx - mar and mar <= e["y"] <= s.m.Ly - mar
    assert warm >= 0.9 * len(mains)             # on the warm side, but for starts near a bend of the polyline


def test_warm_sector_draws_avoid_air_masses_and_rate_zero_boundaries_draw_nothing():
    case, bounds, _ = _fronts()
    for mb in bounds:
        mb["b"] = dict(mb["b"], rate=0.0)
    s = _sched(bounds, case, warmRate=2000.0)
    s.schedule(1800.0, 60.0)
    assert s.events and all(e["why"] == "warm sector" for e in s.events)
    for e in s.events:
        if e["zc"] == 2000.0 and e["rz"] == 2000.0:
            assert BND.other_weight(bounds, e["x"], e["y"], 1800.0) <= 0.25


def test_boundary_draws_follow_the_reference_order():
    """The draw order of scheduleCI's boundary loop (app.js:1419-1431): Poisson count, then per start the position
    along the polyline and the offset, then towerCluster's draws; replayed here with a plain mulberry32 stream."""
    case, bounds, _ = _fronts()
    mb = dict(bounds[0], b=dict(bounds[0]["b"], rate=3000.0))
    s = _sched([mb], case, warmRate=0.0, start=0.0)
    t = 600.0
    s.schedule(t, 60.0)
    rng = W.Mulberry32(7 * 7919 + 13)
    mar = s.margin()
    Lx, Ly = s.m.Lx, s.m.Ly
    area = (Lx - 2 * mar) * (Ly - 2 * mar) / 1e6
    # warm-sector Poisson draw with rate 0: one draw
    L0, k, p = math.exp(-0.0 * area / 1e5), 0, 1.0
    while True:
        k += 1
        p *= rng()
        if not (p > L0 and k < 50):
            break
    P = BND.pts_at(mb, t)
    segs = [(P[i], P[i + 1], math.hypot(P[i + 1][0] - P[i][0], P[i + 1][1] - P[i][1])) for i in range(len(P) - 1)]
    L = sum(sg[2] for sg in segs)
    lam, k, p, Lp = 3000.0 * (L / 1e6) * 60.0 / 3600, 0, 1.0, None
    Lp = math.exp(-lam)
    while True:
        k += 1
        p *= rng()
        if not (p > Lp and k < 50):
            break
    n = k - 1
    first = None
    for _ in range(n):
        sv, seg = rng() * L, segs[0]
        for sg in segs:
            if sv <= sg[2]:
                seg = sg
                break
            sv -= sg[2]
        a, e, ln = seg
        f = sv / max(ln, 1)
        ux, uy = (e[0] - a[0]) / ln, (e[1] - a[1]) / ln
        off = (6000 + rng() * 16000) * -mb["side"]
        x, y = a[0] + (e[0] - a[0]) * f - uy * off, a[1] + (e[1] - a[1]) * f + ux * off
        if mar <= x <= Lx - mar and mar <= y <= Ly - mar:
            first = (x, y)
            break
    assert first is not None
    assert (s.events[0]["x"], s.events[0]["y"]) == first
