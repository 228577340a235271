"""The storm-initiation scheduler of the run loop (app.js:1306-1433) on CPU, with a stand-in model: its random
stream, Poisson draws, tower clusters, margins and the echo and time-window tests."""
import math

import numpy as np

from outbreaklab_b200 import runloop as RL, workloads as W


class FakeModel:
    def __init__(self, nx=200, ny=160, dx=1000.0):
        self.nx, self.ny, self.dx = nx, ny, dx
        self.Lx, self.Ly = nx * dx, ny * dx
        self.time = 0.0
        self.sets = []

    def set_ci(self, events):
        self.sets.append(len(events))


def test_random_stream_is_the_runs_mulberry32():
    m = FakeModel()
    s = RL.CIScheduler(m, {"seed": 7})
    ref = W.Mulberry32(7 * 7919 + 13)
    assert [s.rng() for _ in range(5)] == [ref() for _ in range(5)]


def test_poisson_mean_and_cap():
    s = RL.CIScheduler(FakeModel(), {"seed": 3})
    draws = [s.poisson(2.5) for _ in range(4000)]
    assert abs(np.mean(draws) - 2.5) < 0.1
    assert max(s.poisson(200.0) for _ in range(20)) <= 49   # at most 50 factors (app.js:1309)


def test_tower_cluster_shape():
    s = RL.CIScheduler(FakeModel(), {"seed": 11}, motion=(12.0, 5.0))
    for _ in range(50):
        ev = s.tower_cluster(100000.0, 80000.0, 900.0, "warm sector")
        main, sats = ev[0], ev[1:]
        assert 0 <= len(sats) <= 5
        assert 0.8 * 12000 <= main["rh"] <= 1.2 * 12000 and 9.0 <= main["wt"] <= 11.0
        assert 900 + 600 + 900 <= main["t1"] <= 900 + 1080 + 1200
        sp = math.hypot(main["vx"], main["vy"])
        assert 0.85 * 13.0 - 1e-9 <= sp <= 1.15 * 13.0 + 1e-9
        for e in sats:
            assert math.hypot(e["x"] - 100000.0, e["y"] - 80000.0) <= 0.7 * main["rh"] + 1e-6
            assert main["t0"] <= e["t0"] <= main["t0"] + 600 and (e["vx"], e["vy"]) == (main["vx"], main["vy"])


def test_schedule_window_margin_and_echo():
    m = FakeModel()
    s = RL.CIScheduler(m, {"seed": 5, "warmRate": 4000.0, "start": 0.25, "end": 4.5})
    assert s.schedule(100.0, 60.0) == 0          # before ci.start
    assert s.schedule(5 * 3600.0, 60.0) == 0     # after ci.end
    n = s.schedule(1800.0, 60.0)
    assert n > 0 and m.sets[-1] == len(s.events)
    mar = s.margin()
    assert mar == min(max(0.08 * min(m.Lx, m.Ly), 5000.0), 40000.0) + 12000.0 + 5000.0
    for e in s.events:
        if e is s.events[0] or e["zc"] == 2000.0:
            assert mar <= e["x"] <= m.Lx - mar and mar <= e["y"] <= m.Ly - mar
    # echoes above 35 dBZ everywhere: every try lands near a storm, nothing is added
    maps = {"m0": np.full((m.ny, m.nx, 4), 50.0, np.float32)}
    before = len(s.events)
    assert s.schedule(1900.0, 60.0, maps) == 0 and len(s.events) == before
