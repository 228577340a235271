"""Batched ensembles of storm runs (no counterpart in the reference, which runs one domain per browser tab).

Members differ in grid size, spacing and sounding: nx x ny drawn in [128, 384] x [128, 320] (multiples of 8), dx in
{1, 1.5, 2} km with the reference's step dt = 6 dx_km s (app.js:1666), 40 levels, a Weisman-Klemp sounding whose
surface theta and moisture are drawn until its mixed-layer CAPE (sounding.analyze, sounding.js:86-137) lies in
1500-4000 J/kg, and a 0-6 km shear drawn in 10-35 m/s; Thompson-style microphysics; one or two warm bubbles.

Each member is an independent model with its own CUDA stream; an ensemble step queues every member's step without
waiting, so small members run side by side and fill the GPU. The per-step uniforms (model time among them) are
kernel parameters, so the steps are launched, not replayed from captured graphs; with 21 launches per member step
the host stays ahead of the GPU (its launch time is reported next to the device time). Across GPUs the members are
independent units: plan_shards balances them over ranks by cell count, and the only collective is the final gather
of the metrics.
"""
from __future__ import annotations

import math
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
