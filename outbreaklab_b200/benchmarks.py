"""Secondary benchmarks (one JSON line each): the pressure solve in isolation and the step on other configurations.

  python -m outbreaklab_b200.benchmarks solve --nx 1024 --ny 1024 --nz 80 --precision 2 --reps 20
  python -m outbreaklab_b200.benchmarks step --case c4 --steps 50
  python -m outbreaklab_b200.benchmarks surrogate [--nx 512] [--minutes 60] [--pairs 100000000]
  python -m outbreaklab_b200.benchmarks ensemble [--members 24] [--steps 50] [--mode grouped|streams]
                                                                               (torchrun: members shard over ranks)

The solve benchmark's right-hand side is the 5 km-correlated Gaussian random field of the 1024 x 1024 x 80 case
(zero horizontal mean per level), with the Weisman-Klemp densities. Its residual at this size and at the 640 x 640 x 40
step's solve grid is held to the solve tests' bar in tests/test_gpu_full_size.py.
"""
from __future__ import annotations

import argparse
import json
import os
import time

import numpy as np

from . import model as M, workloads as W


def _density(nz, dz):
    B, _ = W.base_state_for(W.StormCase("solve", 8, 8, nz, 1000.0, 6.0, 1))
    Bz = B.reshape(nz + 1, 8)
    return Bz[:nz, 2].astype(np.float32).copy(), Bz[:, 3].astype(np.float32).copy()


def solve(args):
    nx, ny, nz, dx = args.nx, args.ny, args.nz, args.dx
    dz = 20000.0 / nz
    rc, rw = _density(nz, dz)
    rhs = W.gaussian_rhs(nx, ny, nz, dx, corr_len=5000.0, seed=3).astype(np.float32)
    P = M.PoissonDirect(nx, ny, nz, dx, dz, args.precision)
    P.set_density(rc, rw)
    if args.pair_tiles is not None:
        P.set_pair_tiles(bool(args.pair_tiles))
    if args.bn:
        P.set_tile_widths(args.bn, args.bn)
    P.solve(rhs)   # uploads the right-hand side that device_ms solves again
    ms = P.device_ms(args.reps)
    # MMAs per transform element: 1 (fp32 SIMT), 3 (bf16x3), 3 + 3 (refined), 3 + 1 (refined in plain bf16),
    # 3 + 3 + 3 (two refinement sweeps)
    flops = 4.0 * nx * ny * nz * (nx + ny) * {0: 1, 1: 3, 2: 6, 3: 4, 4: 9, 5: 4}[args.precision]
    out = {"bench": "pressure solve", "nx": nx, "ny": ny, "nz": nz, "precision": args.precision, "ms": ms,
           "pair_tiles": args.pair_tiles, "bn": args.bn,
           "dst_flops": flops, "tflops": flops / (ms * 1e-3) / 1e12}
    print(json.dumps(out), flush=True)


def step(args):
    case = {"c1": W.case_c1, "c2": W.case_c2, "c4": W.case_c4}[args.case]()
    m, _ = M.setup_case(case)
    if args.solver is not None:
        m.set_solver(args.solver)
    if args.pair_tiles is not None:
        m.set_pair_tiles(bool(args.pair_tiles))
    import ctypes as C
    from . import _native as N
    N.check(N.lib().ob_model_step(m.h, case.dt, args.warmup))
    t = C.c_float()
    N.check(N.lib().ob_model_timed_steps(m.h, case.dt, args.steps, C.byref(t)))
    print(json.dumps({"bench": "step", "case": case.name, "cells": case.cells, "steps": args.steps, "ms_per_step": t.value / args.steps,
                      "sim_s_per_wall_s": args.steps * case.dt / (t.value / 1000.0), "solver": m.solver}), flush=True)


def _storm_metrics(m):
    """Accumulated surface rain (kg), maximum composite reflectivity (dBZ), maximum updraft (m/s), and the cells
    holding any condensate / at least the surrogate's 1e-5 kg/kg of it."""
    from . import _native as N
    mp = m.request_maps()
    q1 = m.get_field(N.FIELD_Q1).reshape(-1, 4)
    q2 = m.get_field(N.FIELD_Q2).reshape(-1, 4)
    cond = q1[:, 1:4].astype(np.float64).sum(1) + q2[:, 0:2].astype(np.float64).sum(1)
    return {"rain_kg": m.budgets()["rain"], "max_dbz": float(mp["m0"][..., 0].max()), "max_w": float(mp["m1"][..., 0].max()),
            "cells_with_condensate": int((cond > 0).sum()), "cells_above_1e-5": int((cond >= 1e-5).sum())}


def surrogate_compare(nx=512, minutes=60.0, pairs=100_000_000, rate=0.3, batch=16384, train_steps=20000, lr=1e-3,
                      seed=1, margin=0.05):
    """Plain Thompson-style microphysics vs the MLP surrogate on the 512 x 512 x 40 (500 m, dt 3 s) case: training
    pairs recorded from a plain run of the same grid and step with other seeded bubbles, training on the GPU, then
    two runs of the evaluation case from the same initial state, timed on the device (CUDA events). Returns a dict."""
    import ctypes as C
    from . import _native as N, surrogate as S
    args = argparse.Namespace(nx=nx, minutes=minutes, pairs=pairs, rate=rate, batch=batch, train_steps=train_steps, lr=lr,
                              seed=seed, margin=margin)
    dx, dt = 500.0, 3.0
    steps = int(round(args.minutes * 60 / dt))
    L = nx * dx
    edge = min(40000.0, 0.15 * L)
    sep = min(35000.0, 0.2 * L)
    mk = lambda name, seed: W.StormCase(name, nx, nx, 40, dx, dt, steps, scheme=1,
                                        bubbles=W.place_bubbles(8, L, L, seed=seed, min_sep=sep, edge=edge))
    out = {"bench": "microphysics surrogate", "grid": [nx, nx, 40], "dx": dx, "dt": dt, "minutes": args.minutes}
    net = S.MicroSurrogate(seed=args.seed)
    net.reserve(args.pairs)
    # training data: a plain run with another bubble draw (one-step tendencies of an instantaneous saturation
    # adjustment do not scale with dt, so the pairs come from the same time step as the runs they serve)
    tm, _ = M.setup_case(mk("train", args.seed + 100))
    t0 = time.time()
    S.record(tm, net, steps, dt, args.rate)
    tm.sync()
    out["record_s"] = time.time() - t0
    tm.destroy()
    out["pairs"] = net.count()
    net.fit_norm(dt, margin=args.margin)
    out["range_margin"] = args.margin
    t0 = time.time()
    losses = []
    for lr, frac in ((args.lr, 0.6), (args.lr * 0.3, 0.25), (args.lr * 0.1, 0.15)):
        losses.append(net.train(args.batch, max(1, int(args.train_steps * frac)), lr))
    out["train_s"] = time.time() - t0
    out["train_loss"] = losses
    out["train_steps"] = args.train_steps
    out["batch"] = args.batch
    res = {}
    for mode in ("plain", "surrogate"):
        m, _ = M.setup_case(mk("eval", 4))
        if mode == "surrogate":
            m.set_surrogate(net)
        t = C.c_float()
        N.check(N.lib().ob_model_timed_steps(m.h, dt, steps, C.byref(t)))
        r = {"ms_per_step": t.value / steps, "sim_s_per_wall_s": steps * dt / (t.value / 1000.0),
             "cell_steps_per_s": m.nx * m.ny * m.nz * steps / (t.value / 1000.0)}
        r.update(_storm_metrics(m))
        if mode == "surrogate":
            r["queued_last_step"], r["fallbacks_last_step"] = m.surrogate_stats()
        res[mode] = r
        m.destroy()
    out.update(res)
    p, q = res["plain"], res["surrogate"]
    out["speedup"] = q["sim_s_per_wall_s"] / p["sim_s_per_wall_s"]
    out["rain_rel_diff"] = (q["rain_kg"] - p["rain_kg"]) / max(abs(p["rain_kg"]), 1e-30)
    out["max_dbz_diff"] = q["max_dbz"] - p["max_dbz"]
    out["max_w_rel_diff"] = (q["max_w"] - p["max_w"]) / max(abs(p["max_w"]), 1e-30)
    return out


def surrogate(args):
    print(json.dumps(surrogate_compare(args.nx, args.minutes, args.pairs, args.rate, args.batch, args.train_steps, args.lr,
                                       args.seed, args.margin)), flush=True)


def ensemble(args):
    """The C5 ensemble: members drawn by seed, sharded over ranks by cell count (torchrun sets WORLD_SIZE), each
    rank stepping its members concurrently; rank 0 prints the gathered metrics."""
    from . import ensemble as E
    rank, world = int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1"))
    dist = None
    if world > 1:
        import datetime
        import torch
        import torch.distributed as td
        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
        td.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
        dist = (torch, td)
    cases = E.draw_members(args.members, args.seed, steps=args.steps)
    mine = [cases[i] for i in E.plan_shards(cases, world)[rank]]
    if args.mode == "grouped":
        local = E.run_grouped(mine, args.steps, args.warmup, tune=not args.no_tune,
                              surrogate={} if args.surrogate else None)
    else:
        local = E.run(mine, args.steps, args.warmup)
    res = E.gather(local, dist)
    if rank == 0:
        res.update({"bench": "ensemble", "members": len(cases), "cells": sum(c.cells for c in cases), "steps": args.steps,
                    "n_gpus": world, "host_launch_ms_rank0": local["host_launch_ms"],
                    "device_ms_rank0": local["device_ms"], "nan_guard_count_rank0": local["nan_guard_count"],
                    "grids": [[c.nx, c.ny, c.nz, c.dx] for c in cases], "mode": args.mode})
        for k in ("tiles", "tiles_source", "tune_ms", "lanes", "lane_step_ms", "launches_per_step", "surrogate"):
            if k in local:
                res[k + "_rank0"] = local[k]
        print(json.dumps(res), flush=True)
    if dist:
        dist[1].destroy_process_group()


def main(argv=None):
    ap = argparse.ArgumentParser()
    sub = ap.add_subparsers(dest="cmd", required=True)
    a = sub.add_parser("solve")
    a.add_argument("--nx", type=int, default=1024)
    a.add_argument("--ny", type=int, default=1024)
    a.add_argument("--nz", type=int, default=80)
    a.add_argument("--dx", type=float, default=1000.0)
    a.add_argument("--precision", type=int, default=2)
    a.add_argument("--reps", type=int, default=10)
    a.add_argument("--pair-tiles", type=int, choices=[0, 1], default=None,
                   help="1: transforms on SM pairs (256-row tiles); 0: on single SMs; default: the library's choice")
    a.add_argument("--bn", type=int, default=0, help="outputs per transform tile (multiple of 16, 32..256); 0: automatic")
    b = sub.add_parser("step")
    b.add_argument("--case", default="c4")
    b.add_argument("--steps", type=int, default=50)
    b.add_argument("--warmup", type=int, default=5)
    b.add_argument("--solver", type=int, default=None)
    b.add_argument("--pair-tiles", type=int, choices=[0, 1], default=None)
    c = sub.add_parser("surrogate")
    c.add_argument("--nx", type=int, default=512)
    c.add_argument("--minutes", type=float, default=60.0)
    c.add_argument("--pairs", type=int, default=100_000_000)
    c.add_argument("--rate", type=float, default=0.3)
    c.add_argument("--batch", type=int, default=16384)
    c.add_argument("--train-steps", type=int, default=20000)
    c.add_argument("--lr", type=float, default=1e-3)
    c.add_argument("--seed", type=int, default=1)
    c.add_argument("--margin", type=float, default=0.05, help="trusted input range: training range widened by this share")
    e = sub.add_parser("ensemble")
    e.add_argument("--members", type=int, default=24)
    e.add_argument("--steps", type=int, default=50)
    e.add_argument("--warmup", type=int, default=3)
    e.add_argument("--seed", type=int, default=5)
    e.add_argument("--mode", choices=["grouped", "streams"], default="grouped",
                   help="grouped: one launch per pass over all members (ObEnsemble); streams: one stream per member")
    e.add_argument("--no-tune", action="store_true", help="grouped mode: default tiles, no autotuner")
    e.add_argument("--surrogate", action="store_true", help="grouped mode: the members run the MLP microphysics surrogate")
    args = ap.parse_args(argv)
    {"solve": solve, "step": step, "surrogate": surrogate, "ensemble": ensemble}[args.cmd](args)


if __name__ == "__main__":
    main()
