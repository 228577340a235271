"""The sub-grid tornado scheme on CPU (app.js:1435-1572): the oracle's two candidate searches against each other,
and the host logic (mesocyclone tracking, spawning, following, roping out, the per-step tick) with the oracle's
candidate search standing in for the GPU one."""
import math

import numpy as np
import pytest

from outbreaklab_b200 import runloop as RL, tornado as TS, workloads as W

from oracle import tornado_oracle as TO


def blank_maps(nx, ny):
    m0 = np.zeros((ny, nx, 4), np.float32)
    m1 = np.zeros((ny, nx, 4), np.float32)
    m0[..., 0] = m0[..., 1] = -30.0
    return {"m0": m0, "m1": m1, "t": 0.0}


def plant(maps, x, y, dx, zeta=0.012, uh=300.0, w=30.0, core=55.0, cold=-3.0):
    """A mesocyclone at (x, y): a 1-km vortex under an updraft with helicity, a rain core and a cold pool."""
    m0, m1 = maps["m0"], maps["m1"]
    ny, nx = m0.shape[:2]
    X, Y = np.meshgrid((np.arange(nx) + 0.5) * dx, (np.arange(ny) + 0.5) * dx)
    r2 = ((X - x) ** 2 + (Y - y) ** 2) / (3 * dx) ** 2
    g = np.exp(-r2).astype(np.float32)
    m0[..., 3] = np.maximum(m0[..., 3], zeta * g)
    m1[..., 1] = np.maximum(m1[..., 1], uh * g)
    m1[..., 0] = np.maximum(m1[..., 0], w * g)
    m0[..., 1] = np.maximum(m0[..., 1], core * np.exp(-r2 / 4).astype(np.float32))
    m0[..., 2] = np.minimum(m0[..., 2], cold * np.exp(-r2 / 6).astype(np.float32))
    return maps


def oracle_candidates(maps, dx, zmin):
    return [{"i": c[0], "j": c[1], "x": c[2], "y": c[3], "z1": c[4], "uh": c[5], "w": c[6]}
            for c in TO.candidates(maps["m0"], maps["m1"], dx, zmin)]


class FakeModel:
    def __init__(self, nx=120, ny=100, dx=1500.0):
        self.nx, self.ny, self.dx = nx, ny, dx
        self.Lx, self.Ly = nx * dx, ny * dx
        self.time = 0.0


class FakeRadar:
    def __init__(self):
        self.nTor = 0
        self.calls = []

    def set_tornadoes(self, lst):
        self.calls.append(list(lst))
        self.nTor = len(lst)


# ---------------------------------------------------------------------------------------------------------------
# the oracle
# ---------------------------------------------------------------------------------------------------------------
@pytest.mark.parametrize("nx,ny", [(12, 12), (13, 13), (14, 19), (40, 33), (96, 80)])
def test_loop_and_vectorised_candidates_agree(nx, ny):
    rng = np.random.default_rng(nx * 100 + ny)
    m0 = np.zeros((ny, nx, 4), np.float32)
    m1 = np.zeros((ny, nx, 4), np.float32)
    m0[..., 3] = rng.gamma(1.0, 0.003, (ny, nx)).astype(np.float32)
    m0[..., 2] = rng.normal(-2.0, 2.5, (ny, nx)).astype(np.float32)
    m1[..., 0] = rng.gamma(2.0, 8.0, (ny, nx)).astype(np.float32)
    m1[..., 1] = rng.gamma(1.5, 80.0, (ny, nx)).astype(np.float32)
    if nx > 20:
        m0[10, 10:16, 3] = 0.05            # a plateau: equal neighbours do not stop a maximum
    for dx, zmin in ((1000.0, None), (1500.0, None), (1000.0, 0.0), (3000.0, -1.0)):
        a = TO.candidates_loop(m0, m1, dx, zmin)
        b = TO.candidates(m0, m1, dx, zmin)
        assert a == b
    if nx <= 12 or ny <= 12:
        assert TO.candidates(m0, m1, 1000.0, -1.0) == []


def test_candidate_rules():
    dx = 1500.0
    maps = plant(blank_maps(60, 60), 30 * dx, 30 * dx, dx)
    c = TO.candidates(maps["m0"], maps["m1"], dx)
    assert len(c) == 1 and c[0][:2] == (30, 30)
    # too weak a vortex, a cold-pool core, too little helicity or updraft: no candidate
    for kw in ({"zeta": 0.0029}, {"uh": 59.0}, {"w": 11.9}):
        m = plant(blank_maps(60, 60), 30 * dx, 30 * dx, dx, **kw)
        assert TO.candidates(m["m0"], m["m1"], dx) == []
    m = plant(blank_maps(60, 60), 30 * dx, 30 * dx, dx)
    m["m0"][..., 2] = -5.0
    assert TO.candidates(m["m0"], m["m1"], dx) == []


def test_threshold_in_float32():
    for x in (0.0045, 0.003, 0.003 * 1500 / 1234.5, 1e-3 / 3):
        f = TS.float_at_least(x)
        assert float(f) >= x and float(np.nextafter(f, np.float32(-np.inf))) < x
        z = np.float32(x)
        assert (float(z) < x) == (z < f)


# ---------------------------------------------------------------------------------------------------------------
# the scheme
# ---------------------------------------------------------------------------------------------------------------
def scheme(model=None, **kw):
    model = model or FakeModel()
    kw.setdefault("candidates", oracle_candidates)
    return TS.TornadoScheme(model, **kw)


def test_random_stream_is_seeded_as_the_run():
    s = scheme(ci_seed=7)
    ref = W.Mulberry32(7 * 104729 + 71)
    assert [s.rng() for _ in range(4)] == [ref() for _ in range(4)]


def test_off_for_hurricanes_and_fine_grids():
    assert scheme().active()
    assert not scheme(hurricane=True).active()
    assert not scheme(FakeModel(dx=300.0)).active()
    assert not scheme(on=False).active()
    r = FakeRadar()
    r.nTor = 2
    s = scheme(on=False, radar=r)
    s.tick(10.0, 6.0)
    assert r.calls == [[]]


def test_mesocyclone_is_tracked_and_dropped():
    m = FakeModel()
    s = scheme(m)
    dx, vx = m.dx, 15.0
    ids = []
    for k in range(6):
        t = 60.0 * (k + 1)
        maps = plant(blank_maps(m.nx, m.ny), 40 * dx + vx * t, 50 * dx, dx)
        s.update(maps, t)
        assert s.cands >= 1
        ids.append(sorted(M["id"] for M in s.meso))
    assert ids[0] == [1] and all(i == [1] for i in ids)
    M = s.meso[0]
    assert 5.0 < M["vx"] < 25.0 and abs(M["vy"]) < 5.0
    assert M["strongFor"] == pytest.approx(60.0 * 5)
    # no candidate for six minutes: the mesocyclone is forgotten
    s.update(blank_maps(m.nx, m.ny), 60.0 * 6 + 400.0)
    assert s.meso == []


def test_spawn_only_from_a_mature_mesocyclone_then_rope_out():
    m = FakeModel()
    r = FakeRadar()
    s = scheme(m, radar=r, stp=6.0, rate=1e6)     # a spawn draw always succeeds once the rules allow one
    dx = m.dx
    spawned_at = None
    for k in range(1, 30):
        t = 60.0 * k
        s.update(plant(blank_maps(m.nx, m.ny), 50 * dx, 50 * dx, dx), t)
        if s.list and spawned_at is None:
            spawned_at = t
    M = s.meso[0]
    assert spawned_at is not None
    # born at t = 60; it has to be 900 s old and strong for 480 s
    assert spawned_at >= 60.0 + 900.0
    T = s.list[0]
    assert 0 <= T["ef"] <= 5 and T["t1"] > T["t0"] == spawned_at and M["lastTor"] >= spawned_at
    assert len(s.list) == 1          # one at a time near a mesocyclone (20 km) and 600 s between spawns
    assert any(x.startswith("TORNADO #1 EF") for x in s.log)
    # the tick advances it and hands it to the radar
    act = s.tick(spawned_at + 30.0, 6.0)
    assert len(act) == 1 and r.calls[-1] == act
    a = act[0]
    assert a["v"] <= TS.EF_V[T["ef"]] and a["debrisTop"] == 500 + 800 * T["ef"] and a["debrisDbz"] == 40 + 4 * T["ef"]
    if T["ef"] == 0:
        assert a["debris"] == 0.0
    # the mesocyclone goes away: after 300 s lost the tornado has 120 s left, then lifts
    t = 60.0 * 30
    while not T["done"] and t < 60.0 * 60:
        t += 60.0
        s.update(blank_maps(m.nx, m.ny), t)
    assert T["done"] and any("lifted" in x for x in s.log)
    assert s.tick(t + 6.0, 6.0) == [] and r.calls[-1] == []


def test_forced_storm_blocks_spawning():
    m = FakeModel()
    dx = m.dx
    ev = [{"x": 50 * dx, "y": 50 * dx, "rh": 4000.0, "t0": 0.0, "t1": 1e9, "vx": 0.0, "vy": 0.0}]
    s = scheme(m, stp=6.0, rate=1e6, events=lambda: ev)
    for k in range(1, 40):
        s.update(plant(blank_maps(m.nx, m.ny), 50 * dx, 50 * dx, dx), 60.0 * k)
    assert s.list == [] and s.meso[0]["strongFor"] == 0.0


def test_no_spawn_without_core_or_outflow():
    m = FakeModel()
    dx = m.dx
    s = scheme(m, stp=6.0, rate=1e6)
    for k in range(1, 30):
        s.update(plant(blank_maps(m.nx, m.ny), 50 * dx, 50 * dx, dx, core=35.0), 60.0 * k)
    assert s.list == [] and s.mature == 0
    s = scheme(m, stp=6.0, rate=1e6)
    for k in range(1, 30):
        s.update(plant(blank_maps(m.nx, m.ny), 50 * dx, 50 * dx, dx, cold=-0.5), 60.0 * k)
    assert s.list == []


def test_tick_envelope_and_track():
    s = scheme()
    s.list.append({"id": 1, "ef": 3, "x": 0.0, "y": 0.0, "mx": 0.0, "my": 0.0, "vx": 20.0, "vy": 0.0, "t0": 0.0,
                   "t1": 1200.0, "R": 200.0, "lost": 0.0, "track": [], "done": False})
    vs = []
    for k in range(200):
        t = 6.0 * (k + 1)
        a = s.tick(t, 6.0)[0]
        vs.append(a["v"])
        age = t / 1200.0
        env = TS.smooth(0, 0.15, age) * (1 - TS.smooth(0.7, 1, age))
        assert a["v"] == pytest.approx(68 * env * (0.92 + 0.08 * math.sin(t / 47 + 1)))
        assert a["R"] == pytest.approx(200.0 * (0.6 + 0.4 * env))
    tr = s.list[0]["track"]
    assert len(tr) >= 2 and all(math.hypot(b[0] - a[0], b[1] - a[1]) > 1500 for a, b in zip(tr, tr[1:]))
    assert max(vs) <= 68.0


def test_run_loop_counts_tornadoes():
    class Model(FakeModel):
        steps = 0

        def enc_step(self, dt):
            self.time += dt
            self.steps += 1

        def sync(self):
            pass

        def set_ci(self, ev):
            pass

        def request_maps(self):
            mp = plant(blank_maps(self.nx, self.ny), 50 * self.dx, 50 * self.dx, self.dx)
            mp["t"] = self.time
            return mp

    m = Model()
    loop = RL.RunLoop(m, 6.0, 1800.0, tornadoes={"stp": 6.0, "rate": 1e6, "candidates": oracle_candidates},
                      replay_every=1e9)
    res = loop.run()
    assert res["time"] >= 1800.0
    active, total = res["tornadoes"]
    assert total == 1 and active == 1
