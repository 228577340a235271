"""Batched ensembles of storm runs (no counterpart in the reference, which runs one domain per browser tab).

Members differ in grid size, spacing and sounding: nx x ny drawn in [128, 384] x [128, 320] (multiples of 8), dx in
{1, 1.5, 2} km with the reference's step dt = 6 dx_km s (app.js:1666), 40 levels, a Weisman-Klemp sounding whose
surface theta and moisture are drawn until its mixed-layer CAPE (sounding.analyze, sounding.js:86-137) lies in
1500-4000 J/kg, and a 0-6 km shear drawn in 10-35 m/s; Thompson-style microphysics; one or two warm bubbles.

Two ways to step them. `run` gives each member its own CUDA stream and replays each member's captured step there, so
small members run side by side (24 graph launches per ensemble step, 21 kernels each). `run_grouped` makes the
members one ObEnsemble: every pass of the step is ONE launch over all members (the members' grids, uniforms and
field pointers sit in a table the kernels index by block; the solve's transforms take their tiles from every
member's problem list), 22 launches per ensemble step whatever the member count (16 with a one-pass solve), captured as one CUDA graph. Its
tile shapes (block widths of the stencil passes, the widest transform tile of the solve) are picked by the
project's autotuner (ob_ensemble_tune) and cached per member set (TileCache). Across GPUs the members are
independent units: plan_shards balances them over ranks by cell count, and the only collective is the final gather
of the metrics.
"""
from __future__ import annotations

import ctypes as C
import json
import math
import os
import time

import numpy as np

from . import sounding as snd_mod
from . import workloads as W


def draw_members(n: int = 24, seed: int = 5, nz: int = 40, scheme: int = 1, steps: int = 100):
    """n seeded StormCases of the C5 ensemble (mulberry32 draws, app.js:1308)."""
    rng = W.Mulberry32(seed)
    out = []
    for i in range(n):
        nx = 128 + 8 * int(rng() * 33)      # 128 .. 384
        ny = 128 + 8 * int(rng() * 25)      # 128 .. 320
        dx = (1000.0, 1500.0, 2000.0)[min(2, int(rng() * 3))]
        shear = 10.0 + 25.0 * rng()
        wk = None
        for _ in range(200):
            cand = {"theta_sfc": 297.0 + 7.0 * rng(), "qv_max": 0.010 + 0.008 * rng(), "shear_u": shear}
            a = snd_mod.analyze(snd_mod.parse_sharppy(W.weisman_klemp_sharppy(**cand)))
            if 1500.0 <= a.P["mlcape"] <= 4000.0:
                wk = cand
                wk_cape = a.P["mlcape"]
                break
        if wk is None:
            raise ValueError("member %d: no sounding with MLCAPE in 1500-4000 J/kg" % i)
        Lx, Ly = nx * dx, ny * dx
        nb = 1 + int(rng() * 2)
        bubbles = [(Lx * (0.3 + 0.4 * rng()), Ly * (0.3 + 0.4 * rng())) for _ in range(nb)]
        c = W.StormCase("C5-%02d" % i, nx, ny, nz, dx, 6.0 * dx / 1000.0, steps, scheme=scheme, bubbles=bubbles,
                        bubble_rh=min(10000.0, 0.15 * min(Lx, Ly)), seed=seed * 100 + i, wk=wk)
        c.mlcape = wk_cape
        out.append(c)
    return out


def plan_shards(cases, world: int):
    """Members per rank: largest first onto the least-loaded rank (cell count), ties to the lowest rank."""
    load = [0] * world
    plan = [[] for _ in range(world)]
    for i in sorted(range(len(cases)), key=lambda i: (-cases[i].cells, i)):
        r = min(range(world), key=lambda r: (load[r], r))
        plan[r].append(i)
        load[r] += cases[i].cells
    return [sorted(p) for p in plan]


def run(cases, steps: int = 50, warmup: int = 3):
    """Steps every member `steps` times concurrently (one stream each). Returns the metrics of this process: total
    cell-steps per second over the device span of the timed steps, and per-member step latency percentiles."""
    import torch
    from . import _native as N, model as M
    models = []
    for c in cases:
        m, _ = M.setup_case(c)
        models.append(m)
    streams = [torch.cuda.ExternalStream(int(N.lib().ob_model_stream(m.h) or 0)) for m in models]
    for m, c in zip(models, cases):
        N.check(N.lib().ob_model_step(m.h, c.dt, warmup))
    for m in models:
        m.sync()
    ev = [[(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
          for _ in models]
    t0 = time.perf_counter()
    for s in range(steps):
        for i, (m, c) in enumerate(zip(models, cases)):
            ev[i][s][0].record(streams[i])
            N.check(N.lib().ob_model_step(m.h, c.dt, 1))
            ev[i][s][1].record(streams[i])
    host_s = time.perf_counter() - t0
    for m in models:
        m.sync()
    lat = np.array([[ev[i][s][0].elapsed_time(ev[i][s][1]) for s in range(steps)] for i in range(len(models))])
    # device span: earliest start to latest end, all relative to one event (events on different streams share the
    # device clock)
    ref = ev[0][0][0]
    start = min(ref.elapsed_time(ev[i][0][0]) for i in range(len(models)))
    end = max(ref.elapsed_time(ev[i][steps - 1][1]) for i in range(len(models)))
    span_ms = end - start
    cells = sum(c.cells for c in cases)
    out = {"members": len(cases), "cells": cells, "steps": steps, "device_ms": span_ms, "host_launch_ms": host_s * 1e3,
           "cell_steps_per_s": cells * steps / (span_ms / 1000.0),
           "latency_ms_p50": float(np.percentile(lat, 50)), "latency_ms_p99": float(np.percentile(lat, 99)),
           "latency_ms_all": lat.tolist(), "nan_guard_count": int(sum(m.nan_count for m in models))}
    for m in models:
        m.destroy()
    return out


def gather(local: dict, dist=None):
    """Combines the ranks' metrics (all_gather of a fixed-size vector; the only collective of an ensemble run).
    Throughput is the total cell-steps over the slowest rank's device span; latency percentiles pool every rank's
    member-step samples."""
    lat = np.asarray(local["latency_ms_all"], np.float64).reshape(-1)
    if dist is None:
        parts = [(local["cells"] * local["steps"], local["device_ms"], lat)]
    else:
        torch, td = dist
        dev = "cuda" if td.get_backend() == "nccl" else "cpu"
        world = td.get_world_size()
        n = torch.tensor([lat.size], dtype=torch.int64, device=dev)
        ns = [torch.zeros_like(n) for _ in range(world)]
        td.all_gather(ns, n)
        mx = int(max(int(x.item()) for x in ns))
        buf = torch.zeros(mx + 3, dtype=torch.float64, device=dev)
        buf[0] = float(local["cells"] * local["steps"])
        buf[1] = float(local["device_ms"])
        buf[2] = float(lat.size)
        buf[3:3 + lat.size] = torch.from_numpy(lat).to(dev)
        bufs = [torch.zeros_like(buf) for _ in range(world)]
        td.all_gather(bufs, buf)
        parts = []
        for b in bufs:
            b = b.cpu().numpy()
            k = int(b[2])
            parts.append((b[0], b[1], b[3:3 + k]))
    cell_steps = sum(p[0] for p in parts)
    span = max(p[1] for p in parts)
    allat = np.concatenate([p[2] for p in parts]) if parts else np.zeros(1)
    return {"cell_steps_per_s": cell_steps / (span / 1000.0), "device_ms_max": span,
            "latency_ms_p50": float(np.percentile(allat, 50)), "latency_ms_p99": float(np.percentile(allat, 99)),
            "ranks": len(parts)}


class TileCache:
    """Autotuned tiles per member set, in a JSON file: {signature: {"tiles": [...], "ms": [...]}}. The signature
    names the device and every member's grid, spacing and dt, so a cached choice is reused only for the same work."""

    def __init__(self, path=None):
        self.path = path or os.path.join(os.path.expanduser("~"), ".cache", "outbreaklab_b200", "ensemble_tiles.json")

    @staticmethod
    def signature(cases, device=""):
        parts = ["%dx%dx%d@%g/%g" % (c.nx, c.ny, c.nz, c.dx, c.dt) for c in cases]
        return device + "|" + ";".join(parts)

    def load(self):
        try:
            with open(self.path) as f:
                return json.load(f)
        except (OSError, ValueError):
            return {}

    def get(self, sig):
        e = self.load().get(sig)
        if e and isinstance(e.get("tiles"), list):
            return [int(x) for x in e["tiles"]]
        return None

    def get_lanes(self, sig):
        e = self.load().get(sig)
        return int(e["lanes"]) if e and "lanes" in e else None

    def put(self, sig, tiles, ms, lanes=None):
        d = self.load()
        d[sig] = {"tiles": [int(x) for x in tiles], "ms": [float(x) for x in ms]}
        if lanes is not None:
            d[sig]["lanes"] = int(lanes)
        os.makedirs(os.path.dirname(self.path) or ".", exist_ok=True)
        tmp = self.path + ".part"
        with open(tmp, "w") as f:
            json.dump(d, f, indent=1, sort_keys=True)
        os.replace(tmp, self.path)


class Ensemble:
    """An ObEnsemble over RegionalModels (members keep their handles)."""

    def __init__(self, models, dts):
        from . import _native as N
        self.N = N
        self.models = list(models)
        arr = (C.c_void_p * len(self.models))(*[m.h for m in self.models])
        d = np.asarray(dts, np.float32)
        h = C.c_void_p()
        N.check(N.lib().ob_ensemble_create(arr, N.fptr(d), len(self.models), C.byref(h)))
        self.h = h
        self.dts = d

    def step(self, n=1):
        self.N.check(self.N.lib().ob_ensemble_step(self.h, int(n)))

    def sync(self):
        self.N.check(self.N.lib().ob_ensemble_sync(self.h))

    def timed_steps(self, n):
        ms = C.c_float()
        self.N.check(self.N.lib().ob_ensemble_timed_steps(self.h, int(n), C.byref(ms)))
        return ms.value

    def set_graphs(self, on):
        self.N.check(self.N.lib().ob_ensemble_set_graphs(self.h, int(bool(on))))

    def set_lanes(self, k):
        self.N.check(self.N.lib().ob_ensemble_set_lanes(self.h, int(k)))

    @property
    def lanes(self):
        return int(self.N.lib().ob_ensemble_lanes(self.h))

    def tiles(self):
        t = (C.c_int * self.N.ENS_NTILES)()
        self.N.check(self.N.lib().ob_ensemble_get_tiles(self.h, t))
        return list(t)

    def set_tiles(self, tiles):
        t = (C.c_int * self.N.ENS_NTILES)(*[int(x) for x in tiles])
        self.N.check(self.N.lib().ob_ensemble_set_tiles(self.h, t))

    def tune(self, reps=5):
        t = (C.c_int * self.N.ENS_NTILES)()
        ms = np.zeros(self.N.ENS_NTILES, np.float32)
        self.N.check(self.N.lib().ob_ensemble_tune(self.h, int(reps), t, self.N.fptr(ms)))
        return list(t), ms.tolist()

    def lsf_times(self):
        t = (C.c_double * len(self.models))()
        self.N.check(self.N.lib().ob_ensemble_lsf_times(self.h, t))
        return list(t)

    @property
    def stream(self):
        return self.N.lib().ob_ensemble_stream(self.h)

    def destroy(self):
        if self.h:
            self.N.lib().ob_ensemble_destroy(self.h)
            self.h = None


def train_surrogate(cases, rec_minutes=20.0, rate=0.3, pairs=20_000_000, train_steps=6000, batch=16384, lr=1e-3, seed=7,
                    margin=0.05):
    """The members' learned microphysics: pairs recorded from a plain Thompson run of a donor member (a fresh copy of
    the first 1-km member, or of the first member), normalised with a margin on the trusted input range, trained on
    the GPU. The network serves every member; its tendencies scale with each member's dt (the surrogate kernel's
    dt ratio), the saturation adjustment after them does not need to."""
    from . import model as M, surrogate as S
    donor = next((c for c in cases if c.dx == 1000.0), cases[0])
    net = S.MicroSurrogate(seed=seed)
    net.reserve(pairs)
    m, _ = M.setup_case(donor)
    t0 = time.time()
    S.record(m, net, max(1, int(rec_minutes * 60 / donor.dt)), donor.dt, rate)
    m.sync()
    m.destroy()
    info = {"donor": [donor.nx, donor.ny, donor.nz, donor.dx], "record_s": time.time() - t0, "pairs": net.count()}
    net.fit_norm(donor.dt, margin=margin)
    t0 = time.time()
    losses = [net.train(batch, max(1, int(train_steps * frac)), l) for l, frac in ((lr, 0.6), (lr * 0.3, 0.25), (lr * 0.1, 0.15))]
    info.update({"train_s": time.time() - t0, "train_loss": losses})
    return net, info


def run_grouped(cases, steps: int = 50, warmup: int = 3, tune: bool = True, cache: TileCache = None, reps: int = 5,
                lanes=None, surrogate=None):
    """Steps every member `steps` times as one ObEnsemble. Tiles and the lane count come from the cache for this
    member set, else from the autotuner (tiles) and from timing a few warm-up steps with one and with two lanes (the
    lane count changes no result, only which launches overlap); both are then cached. surrogate: None (the
    Thompson-style scheme as it is) or the keyword arguments of train_surrogate (the members then run the learned
    microphysics). Returns the metrics of this process: cell-steps per second over the device time of the timed
    steps, the ensemble step's latency percentiles (per-step CUDA events), the tiles and lanes used."""
    import torch
    from . import _native as N, model as M
    net, sinfo = (None, None)
    if surrogate is not None:
        net, sinfo = train_surrogate(cases, **surrogate)
    models = []
    for c in cases:
        m, _ = M.setup_case(c)
        if m.solver < 1:
            m.set_solver(2)
        if net is not None:
            m.set_surrogate(net)
        models.append(m)
    ens = Ensemble(models, [c.dt for c in cases])
    try:
        out = _run_grouped(ens, models, cases, steps, warmup, tune, cache, reps, lanes)
        if net is not None:
            q = [m.surrogate_stats() for m in models]
            out["surrogate"] = dict(sinfo, queued_last_step=int(sum(a for a, _ in q)), fallbacks_last_step=int(sum(b for _, b in q)))
        return out
    finally:
        ens.destroy()
        for m in models:
            m.destroy()
        if net is not None:
            net.close()


def _run_grouped(ens, models, cases, steps, warmup, tune, cache, reps, lanes):
    import torch
    tiles_src, tune_ms, lane_ms = "default", None, None
    if lanes is not None:
        ens.set_lanes(lanes)
    if tune:
        cache = cache or TileCache()
        sig = TileCache.signature(cases, torch.cuda.get_device_name(0) if torch.cuda.is_available() else "")
        t = cache.get(sig)
        if t is not None:
            ens.set_tiles(t)
            tiles_src = "cache"
            if lanes is None and cache.get_lanes(sig):
                ens.set_lanes(min(cache.get_lanes(sig), len(models)))
        else:
            ens.step(1)           # a state with motion in it for the timing
            ens.sync()
            t, tune_ms = ens.tune(reps)
            if lanes is None and len(models) > 1:
                lane_ms = {}
                for k in (1, 2):
                    ens.set_lanes(k)
                    ens.step(2)   # capture
                    lane_ms[k] = ens.timed_steps(4) / 4
                ens.set_lanes(min(lane_ms, key=lane_ms.get))
            cache.put(sig, t, tune_ms, ens.lanes)
            tiles_src = "autotuned"
    ens.step(warmup)
    ens.sync()
    stream = torch.cuda.ExternalStream(int(ens.stream or 0))
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
    t0 = time.perf_counter()
    for s in range(steps):
        ev[s][0].record(stream)
        ens.step(1)
        ev[s][1].record(stream)
    host_s = time.perf_counter() - t0
    ens.sync()
    lat = np.array([a.elapsed_time(b) for a, b in ev])
    span_ms = ev[0][0].elapsed_time(ev[-1][1])
    cells = sum(c.cells for c in cases)
    out = {"members": len(cases), "cells": cells, "steps": steps, "device_ms": span_ms, "host_launch_ms": host_s * 1e3,
           "cell_steps_per_s": cells * steps / (span_ms / 1000.0),
           "latency_ms_p50": float(np.percentile(lat, 50)), "latency_ms_p99": float(np.percentile(lat, 99)),
           "latency_ms_all": lat.tolist(), "nan_guard_count": int(sum(m.nan_count for m in models)),
           "tiles": ens.tiles(), "tiles_source": tiles_src, "tune_ms": tune_ms, "lanes": ens.lanes, "lane_step_ms": lane_ms,
           "launches_per_step": ens.lanes * (11 + {1: 5, 4: 17}.get(models[0].solver, 11) + (1 if getattr(models[0], "surrogate", False) else 0))}
    return out
