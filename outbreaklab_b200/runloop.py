"""The caller of the step: the reference's run loop and storm-initiation scheduler, on the B200 model.

RunLoop mirrors loop() (app.js:1678-1732): steps in batches sized to about 60 ms of GPU work each
(stepsPerBatch, 1..40), storm-initiation scheduling every 60 s of model time, the radars' due cuts after every step
(RadarSim.enc_due), the sub-grid tornadoes advanced after every step and updated from each batch's last map readback
(tornadoTick / tornadoUpdate, tornado.py), a map readback for each replay frame (every `replay_every` s of model time)
and for the scheduler's echo test, finished volumes written as Archive II files (RadarSim.collect_level2, the server's write,
server.py:249-284), optional pacing to a multiple of real time, and the simulation rate. The browser parts (status
bar, map painting, upload retries, the replay UI) have no counterpart here.

CIScheduler mirrors scheduleCI and towerCluster (app.js:1306-1433) for outbreak mode: Poisson-drawn starts in the open
warm sector, each a 0-4 km updraft push that moves with the storm motion (the sounding's Bunkers right mover) plus
0-5 satellite towers, all drawn from the run's mulberry32 stream (seeded as app.js:1646), and Poisson-drawn starts
along each boundary with a trigger rate, 6-22 km into its warm side, their satellite ellipse laid along the boundary
(app.js:1416-1432). The warm-sector draw skips points inside any boundary's air mass (other_weight > 0.25). The
boundaries are boundaries.boundary_models records (the run's RUN.mbs).
"""
from __future__ import annotations

import math
import os
import time

import numpy as np

from . import boundaries as BND
from . import workloads as W

CI_DEFAULTS = {"warmRate": 1.2, "start": 0.25, "end": 4.5, "seed": 7, "wt": 10.0, "rh": 12000.0, "auto": True}  # app.js:27


class CIScheduler:
    def __init__(self, model, ci=None, motion=(0.0, 0.0), log=None, bounds=None):
        self.m = model
        self.mbs = list(bounds or [])
        self.ci = dict(CI_DEFAULTS, **(ci or {}))
        self.rng = W.Mulberry32((int(self.ci["seed"]) | 0) * 7919 + 13)
        self.motion = motion
        self.events = []
        self.log = log if log is not None else []

    # app.js:1308-1309, 1318-1319
    def poisson(self, lam):
        L, k, p = math.exp(-lam), 0, 1.0
        while True:
            k += 1
            p *= self.rng()
            if not (p > L and k < 50):
                break
        return k - 1

    def uniform(self, a, b):
        return a + (b - a) * self.rng()

    def pick_weighted(self, w):
        r = self.rng() * sum(w)
        for i, x in enumerate(w):
            r -= x
            if r < 0:
                return i
        return len(w) - 1

    # app.js:1321-1345
    def tower_cluster(self, x, y, t0, why, axis=None, opts=None):
        opts = opts or {}
        ci, rm = self.ci, opts.get("motion", self.motion)
        rh = opts.get("rh", ci["rh"]) * self.uniform(0.8, 1.2)
        wt = opts.get("wt", ci["wt"]) * self.uniform(0.9, 1.1)
        ramp = self.uniform(600, 1080)
        dur = ramp + self.uniform(900, 1200)
        sp = math.hypot(rm[0], rm[1]) * self.uniform(0.85, 1.15)
        dm = math.atan2(rm[1], rm[0]) + self.uniform(-0.2, 0.2)
        vx, vy = sp * math.cos(dm), sp * math.sin(dm)
        out = [{"x": x, "y": y, "zc": 2000.0, "rh": rh, "rz": 2000.0, "wt": wt, "t0": t0, "t1": t0 + dur, "vx": vx, "vy": vy,
                "seed": self.rng() * 100, "ramp": ramp, "why": why}]
        n = self.pick_weighted([0.08, 0.17, 0.25, 0.25, 0.15, 0.10])
        ang = axis + self.uniform(-0.4, 0.4) if axis is not None else self.rng() * math.pi
        aspect = self.uniform(1.8, 4) if axis is not None else self.uniform(1, 3.5)
        ca, sa = math.cos(ang), math.sin(ang)
        for _ in range(n):
            r = math.sqrt(self.rng()) * 0.7 * rh
            th = self.rng() * 2 * math.pi
            a, b = r * math.cos(th), r * math.sin(th) / aspect
            start = t0 + self.uniform(0, 600)
            zc, rhs, rz, wts = self.uniform(1600, 2100), rh * self.uniform(0.25, 0.5), self.uniform(1500, 1900), wt * self.uniform(0.7, 1.1)
            t1 = start + self.uniform(360, 960)
            out.append({"x": x + a * ca - b * sa, "y": y + a * sa + b * ca, "zc": zc, "rh": rhs, "rz": rz, "wt": wts,
                        "t0": start, "t1": t1, "vx": vx, "vy": vy, "seed": self.rng() * 100, "ramp": self.uniform(90, 300),
                        "why": why})
        return out

    # app.js:1348-1351
    def margin(self):
        L = min(self.m.Lx, self.m.Ly)
        return min(max(0.08 * L, 5000.0), 40000.0) + self.ci["rh"] + 5000.0

    def add_event(self, x, y, t0, why, axis=None, opts=None):
        self.events.extend(self.tower_cluster(x, y, t0, why, axis, opts))
        self.m.set_ci(self.events)
        self.log.append("storm start (%s) at (%.1f, %.1f) km, t+%.0f min" % (why, x / 1000, y / 1000, t0 / 60))

    # app.js:1395-1401
    def echo_near(self, maps, x, y, rad):
        if maps is None:
            return False
        m0 = maps["m0"]
        nx, ny, dx = self.m.nx, self.m.ny, self.m.dx
        r = math.ceil(rad / dx)
        i0, j0 = math.floor(x / dx), math.floor(y / dx)
        sub = m0[max(0, j0 - r):min(ny - 1, j0 + r) + 1:2, max(0, i0 - r):min(nx - 1, i0 + r) + 1:2, 0]
        return bool((sub > 35).any())

    # app.js:1402-1433, outbreak mode: the open warm sector, then along each boundary
    def schedule(self, t, dt_win, maps=None):
        ci = self.ci
        if not ci["auto"] or t < ci["start"] * 3600 or t > ci["end"] * 3600:
            return 0
        Lx, Ly, mar = self.m.Lx, self.m.Ly, self.margin()
        area = (Lx - 2 * mar) * (Ly - 2 * mar) / 1e6
        n = self.poisson(ci["warmRate"] * area / 1e5 * dt_win / 3600)
        added = 0
        for _ in range(n):
            for _try in range(6):
                x = mar + self.rng() * (Lx - 2 * mar)
                y = mar + self.rng() * (Ly - 2 * mar)
                # not into another storm (its push would stir its outflow), nor into a boundary's air mass
                if BND.other_weight(self.mbs, x, y, t) > 0.25 or self.echo_near(maps, x, y, 35000.0):
                    continue
                self.add_event(x, y, t, "warm sector")
                added += 1
                break
        for mb in self.mbs:
            b = mb.get("b")
            if not b or not (b.get("rate", 0) > 0):
                continue
            P = BND.pts_at(mb, t)
            segs, L = [], 0.0
            for i in range(len(P) - 1):
                a, e = P[i], P[i + 1]
                ln = math.hypot(e[0] - a[0], e[1] - a[1])
                segs.append((a, e, ln))
                L += ln
            n = self.poisson(b["rate"] * (L / 1e6) * dt_win / 3600)
            for _ in range(n):
                s, seg = self.rng() * L, segs[0]
                for sg in segs:
                    if s <= sg[2]:
                        seg = sg
                        break
                    s -= sg[2]
                a, e, ln = seg
                f = s / max(ln, 1)
                ux, uy = (e[0] - a[0]) / ln, (e[1] - a[1]) / ln
                off = (6000 + self.rng() * 16000) * -mb["side"]          # into the warm side
                x = a[0] + (e[0] - a[0]) * f + (-uy) * off
                y = a[1] + (e[1] - a[1]) * f + ux * off
                if x < mar or y < mar or x > Lx - mar or y > Ly - mar:
                    continue
                if self.echo_near(maps, x, y, 25000.0):
                    continue
                self.add_event(x, y, t, BND.BND_TYPES[b["type"]]["label"].lower(), math.atan2(uy, ux))
                added += 1
        return added


class RunLoop:
    def __init__(self, model, dt, t_end, radar=None, ci=None, motion=(0.0, 0.0), replay_every=180.0, out_dir=None,
                 run="run", epoch0_ms=None, pace=0.0, batch_ms=60.0, tornadoes=None, bounds=None):
        self.m, self.dt, self.t_end = model, float(dt), float(t_end)
        self.radar = radar
        self.log = []
        self.ci = CIScheduler(model, ci, motion, self.log, bounds) if ci is not None else None
        # tornadoes: None, or the keyword arguments of TornadoScheme (stp, rate, on, hurricane, ...)
        self.tor = None
        if tornadoes is not None:
            from .tornado import TornadoScheme
            seed = (ci or {}).get("seed", CI_DEFAULTS["seed"])
            self.tor = TornadoScheme(model, radar, ci_seed=seed, events=(lambda: self.ci.events if self.ci else []),
                                     log=self.log, **tornadoes)
        self.replay_every, self.replay_next = float(replay_every), 0.0
        self.out_dir, self.run_name = out_dir, run
        self.epoch0 = int(time.time() * 1000) if epoch0_ms is None else int(epoch0_ms)
        self.pace, self.batch_ms = float(pace), float(batch_ms)
        self.steps_per_batch = 4
        self.ci_next = 0.0
        self.maps = None
        self.frames = []
        self.volumes = []
        self.batches = []
        self.sim_rate = 0.0

    def _volume(self, v):
        out = self.radar.collect_level2(v, self.run_name, self.epoch0)
        rec = {"icao": out["header"]["icao"], "name": out["name"], "size": len(out["bytes"]), "epoch_ms": out["header"]["epoch_ms"]}
        if self.out_dir:
            d = os.path.join(self.out_dir, self.run_name, out["header"]["icao"])
            os.makedirs(d, exist_ok=True)
            p = os.path.join(d, out["name"])
            with open(p + ".part", "wb") as f:   # written whole, then renamed (server.py:270-273)
                f.write(out["bytes"])
            os.replace(p + ".part", p)
            rec["path"] = p
        self.volumes.append(rec)

    def run(self):
        m = self.m
        wall0, sim0 = time.perf_counter(), m.time
        while m.time < self.t_end:
            nb, t0, ran = self.steps_per_batch, time.perf_counter(), 0
            for _ in range(nb):
                if m.time >= self.t_end:
                    break
                if self.ci is not None and m.time >= self.ci_next:
                    self.ci.schedule(m.time, 60.0, self.maps)
                    self.ci_next = m.time + 60.0
                m.enc_step(self.dt)
                ran += 1
                if self.tor is not None:
                    self.tor.tick(m.time, self.dt)
                due = self.radar.enc_due(m.time) if self.radar is not None else []
                if m.time >= self.replay_next:
                    self.frames.append(m.request_maps())
                    self.maps = self.frames[-1]
                    self.replay_next = math.floor(m.time / self.replay_every + 1) * self.replay_every
                for v in due:
                    self._volume(v)
            m.sync()
            el = (time.perf_counter() - t0) * 1000.0
            self.batches.append((ran, el))
            # aim for ~batch_ms of GPU work per batch (app.js:1711)
            self.steps_per_batch = int(min(max(round(max(ran, 1) * (self.batch_ms / max(el, 5.0))), 1), 40))
            if (self.ci is not None and self.ci.ci["auto"]) or self.tor is not None:
                self.maps = m.request_maps()   # the scheduler's echo test reads the latest composite reflectivity
            if self.tor is not None:
                self.tor.update(self.maps, self.maps["t"])   # candidates from the device copy of these maps
            if self.pace > 0:
                want = wall0 + (m.time - sim0) / self.pace
                wait = want - time.perf_counter()
                if wait > 0:
                    time.sleep(min(wait, 2.0))
        el = time.perf_counter() - wall0
        self.sim_rate = (m.time - sim0) / max(el, 1e-9)
        return {"time": m.time, "steps": m.steps, "sim_rate": self.sim_rate, "frames": len(self.frames),
                "volumes": self.volumes, "events": len(self.ci.events) if self.ci else 0, "log": self.log,
                "steps_per_batch": self.steps_per_batch,
                "tornadoes": self.tor.counts() if self.tor else (0, 0)}
