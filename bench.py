#!/usr/bin/env python
"""Benchmark of the B200 storm-model time step.

Workload (the headline configuration): 640 x 640 x 40 cells at 1 km x 500 m, dt 6 s, Lin-type microphysics, Weisman-
Klemp analytic sounding, 8 seeded +3 K warm bubbles; synthetic inputs (no dataset exists for this model). A bench
"step" is one model time step (the reference's encStep, model.js:1442-1476). The 2.8 GB state is larger than the
126 MB L2, so no flush is needed between steps.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

value  = simulated seconds per wall second over the K timed steps (device time, CUDA events, max over ranks);
e2e    = the same metric through the public Python API (RegionalModel.enc_step) over the same K steps of a second copy
         of the case, with the per-step forcing upload from pinned host memory and a device-to-host read of every
         step's FP64 budgets (requested after the step, read while the next one runs) inside the timed region (wall
         clock, max over ranks);
roofline = the dominant kernel of the step against the measured HBM copy peak (MEASURED_PEAKS.json), and
           solve_roofline the pressure solve's MMA work against the measured bf16 peak;
cpu_baseline = the CPU restatement of the reference step (oracle, fp32, OpenMP) on a bounded sample.
With --gpus N > 1 each rank runs an independent replica of the domain ("replicas only": a single domain does not
shard); value sums the simulated seconds of all ranks over the slowest rank's time.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "sim-sec/wall-sec + cell-steps/s, plain vs MLP microphysics (1 B200, stated err)"


def _rank_env():
    return int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("LOCAL_RANK", "0"))


def _pin_device(local_rank, world):
    if world > 1:
        vis = os.environ.get("CUDA_VISIBLE_DEVICES")
        devs = vis.split(",") if vis else [str(i) for i in range(64)]
        os.environ["CUDA_VISIBLE_DEVICES"] = devs[local_rank]


class ClockSampler:
    """nvidia-smi samples of SM clock and throttle reasons during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self):
        self.proc = None
        self.lines = []

    def start(self, period_ms=20):
        """Starts sampling every period_ms and returns once the first sample is in (at most 3 s), so that the
        sampler is live when the timed region begins."""
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "--query-gpu=" + self.Q, "--format=csv,noheader,nounits",
                                          "-lms", str(period_ms)], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL,
                                         text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
            t0 = time.time()
            while not self.lines and time.time() - t0 < 3.0:
                time.sleep(0.005)
            self.skip = len(self.lines)   # samples taken before the timed region are not counted
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        dev = os.environ.get("CUDA_VISIBLE_DEVICES", "0").split(",")[0]
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines[getattr(self, "skip", 0):] or self.lines[-1:]:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9 or (dev.isdigit() and f[0] != dev):
                continue
            try:
                sm.append(float(f[1]))
                smax.append(float(f[2]))
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def pass_bytes(nx, ny, nz, pad, dt):
    """Algorithmic bytes per pass of one step (each array counted once per pass, fp32, structure of arrays)."""
    Nv = (nx + 1) * (ny + 1) * (nz + 1)
    Nc = nx * ny * nz
    Np = (nx + 2 * pad) * (ny + 2 * pad) * nz
    N2 = nx * ny
    lsf_every = math.ceil(60.0 / dt)
    return {
        "LSF+CI": (4 * Nc + 32 * N2) / lsf_every + 16 * N2,
        "NUT": 16 * Nv + 16 * Nc,
        "ADVV": 32 * Nv + 48 * Nv,
        "ADVQ": (12 * Nv + 64 * Nc) + (12 * Nv + 96 * Nc),
        "PHYS": 32 * Nv + 76 * Nc,
        "DIV": 12 * Nv + 4 * Nc,
        "SOLVE": 40 * Np,
        "PROJ+RAIN": 32 * Nv + 4 * Np + 4 * 3 * N2 + 16 * N2,
    }


def solve_flops(nx, ny, nz, pad):
    nxp, nyp = nx + 2 * pad, ny + 2 * pad
    return 4.0 * nxp * nyp * nz * (nxp + nyp)


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return p["hbm_gbs"], p["bf16_tflops"], "measured (MEASURED_PEAKS.json)"
    except Exception:
        return 6650.0, 1590.0, "fallback (no MEASURED_PEAKS.json: the pool's earlier measurement)"


def ncu_traffic(pass_name, cells):
    """DRAM bytes of one pass from the committed ncu summary (profiles/ncu_traffic.json), scaled from the captured
    workload to this one by the cell count; None when the pass has no entry."""
    try:
        with open(os.path.join(ROOT, "profiles", "ncu_traffic.json")) as f:
            j = json.load(f)
        v = j.get(pass_name)
        return None if v is None else v["bytes"] * cells / v["cells"]
    except Exception:
        return None


def cpu_baseline(case, steps=1):
    from oracle import oracle as O
    O.build()
    m, _ = O.setup_case(case, 4)
    t0 = time.perf_counter()
    m.step(case.dt, steps)
    el = time.perf_counter() - t0
    cores = os.cpu_count() or 1
    try:
        cores = len(os.sched_getaffinity(0))
    except Exception:
        pass
    return {"value": steps * case.dt / el, "unit": "sim-s/wall-s", "cores": cores, "kind": "port",
            "sample": "%d model step(s) of the %dx%dx%d case from t=0 (fp32 C++ oracle, OpenMP, %.1f s)"
                      % (steps, case.nx, case.ny, case.nz, el), "cell_steps_per_s": steps * case.cells / el}


def full_run(case):
    """All steps of the configuration the metric is quoted on (600 steps = 60 simulated minutes of the 640 x 640 x 40
    case), from t = 0 on a fresh copy, device time (CUDA events around the steps on the model's stream). The first
    occurrence of each step graph (parity x LSF due) is captured inside the timed steps."""
    import ctypes as C
    from outbreaklab_b200 import _native as N, model as M
    m, _ = M.setup_case(case)
    try:
        ms = C.c_float()
        clocks = ClockSampler()
        clocks.start(50)
        N.check(N.lib().ob_model_timed_steps(m.h, case.dt, case.steps, C.byref(ms)))
        clk = clocks.stop()
        b = m.budgets()
        maps = m.request_maps()
        import numpy as np
        m0 = maps["m0"].reshape(case.ny, case.nx, 4)
        return {"steps": case.steps, "sim_minutes": case.steps * case.dt / 60.0, "ms": ms.value,
                "ms_per_step": ms.value / case.steps, "sim_s_per_wall_s": case.steps * case.dt / (ms.value / 1000.0),
                "cell_steps_per_s": case.steps * case.cells / (ms.value / 1000.0),
                "max_dbz": float(np.max(m0[..., 0])), "rain_kg": b["rain"], "nan_guard_count": m.nan_count,
                "clocks": clk}
    finally:
        m.destroy()


def c3_solve():
    """The pressure solve alone at 1024 x 1024 x 80 (dx 1 km, dz 250 m, Weisman-Klemp densities, 5 km-correlated
    Gaussian right-hand side): device ms per solve and the FP64 residual (on the device) for the refined precisions."""
    import numpy as np
    from outbreaklab_b200 import model as M, workloads as W
    nx = ny = 1024
    nz, dx = 80, 1000.0
    dz = 20000.0 / nz
    B, _ = W.base_state_for(W.StormCase("solve", 8, 8, nz, dx, 6.0, 1))
    Bz = B.reshape(nz + 1, 8)
    rc, rw = Bz[:nz, 2].astype(np.float32).copy(), Bz[:, 3].astype(np.float32).copy()
    rhs = W.gaussian_rhs(nx, ny, nz, dx, corr_len=5000.0, seed=3, dtype=np.float32)
    out = {"workload": "solve 1024x1024x80, dx 1 km, dz 250 m, Gaussian RHS (5 km correlation)",
           "dst_flops": 4.0 * nx * ny * nz * (nx + ny)}
    for prec, name in ((5, "bf16+1 bf16x3 refinement (the model's default)"), (2, "bf16x3+1 refinement"),
                       (4, "bf16x3+2 refinements"), (0, "fp32 SIMT")):
        P = M.PoissonDirect(nx, ny, nz, dx, dz, prec)
        try:
            P.set_density(rc, rw)
            P.solve(rhs)
            r_inf, r_l2 = P.residual()
            ms = P.device_ms(5)
        finally:
            P.destroy()
        out["precision_%d" % prec] = {"solver": name, "ms": ms, "residual_max_rel": r_inf, "residual_l2_rel": r_l2}
    return out


def c5_ensemble():
    """The batched ensemble: 24 members drawn by seed (128-384 x 128-320 x 40 at 1-2 km, Weisman-Klemp soundings with
    CAPE 1500-4000 J/kg), Thompson-style microphysics, every pass one grouped launch per lane, autotuned tiles;
    ensemble cell-steps/s and the ensemble step's p50 / p99 latency over 50 steps."""
    from outbreaklab_b200 import ensemble as E
    cases = E.draw_members(24, 5, steps=50)
    r = E.run_grouped(cases, 50, 3, tune=True)
    keep = ("cell_steps_per_s", "latency_ms_p50", "latency_ms_p99", "device_ms", "tiles", "tiles_source", "lanes",
            "launches_per_step")
    out = {k: r[k] for k in keep if k in r}
    out.update({"members": len(cases), "cells": sum(c.cells for c in cases), "steps": 50})
    return out


def run_reference(args, rank, world):
    """The reference's own CPU implementation is WGSL run by a browser WebGPU device, which cannot run here; its
    CPU restatement (oracle/, fp32, all host threads) stands in for it."""
    if rank != 0:
        return
    from outbreaklab_b200 import workloads as W
    case = W.case_c2()
    nsample = max(1, min(args.steps, 3))
    from oracle import oracle as O
    O.build()
    m, _ = O.setup_case(case, 4)
    m.step(case.dt, min(args.warmup, 1))
    t0 = time.perf_counter()
    m.step(case.dt, nsample)
    el = time.perf_counter() - t0
    val = nsample * case.dt / el
    cores = len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else os.cpu_count()
    line = {"impl": "reference", "metric": METRIC, "value": val, "unit": "sim-s/wall-s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000 * el / nsample,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "cell_steps_per_s": nsample * case.cells / el,
            "config": {"workload": "640x640x40 dx 1 km dz 500 m dt 6 s, Lin, 8 warm bubbles (Weisman-Klemp)",
                       "cells": case.cells, "parallelism": "replicas" if world > 1 else "single domain",
                       "l2": "state 2.8 GB > 126 MB L2 (no flush needed)"},
            "cpu_baseline": {"value": val, "unit": "sim-s/wall-s", "cores": cores, "kind": "port",
                             "sample": "%d of the timed model steps after %d warm-up step(s); the reference's WGSL "
                                       "needs a WebGPU device (unavailable on this box), so its fp32 C++ restatement "
                                       "runs" % (nsample, min(args.warmup, 1))},
            "e2e": {"value": val, "unit": "sim-s/wall-s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def run_ours(args, rank, world):
    import numpy as np
    from outbreaklab_b200 import _native as N, model as M, workloads as W

    dist = None
    if world > 1:
        import torch
        import torch.distributed as td
        import datetime
        torch.cuda.set_device(0)
        td.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
        dist = (torch, td)

    def barrier():
        if dist:
            dist[1].barrier()

    def allmax(x):
        if not dist:
            return x
        t = dist[0].tensor([float(x)], device="cuda")
        dist[1].all_reduce(t, op=dist[1].ReduceOp.MAX)
        return float(t.item())

    case = W.case_c2()
    if args.nx:
        case = W.StormCase("C2-%d" % args.nx, args.nx, args.nx, 40, 1000.0, 6.0, args.steps,
                           bubbles=W.place_bubbles(4, args.nx * 1000.0, args.nx * 1000.0, seed=2, min_sep=20000.0,
                                                   edge=min(40000.0, args.nx * 250.0)))
    m, _ = M.setup_case(case)
    import ctypes as C
    lib = N.lib()
    ms = C.c_float()
    # warm-up
    N.check(lib.ob_model_step(m.h, case.dt, args.warmup))
    m.sync()
    # per-pass profile (3 steps, averaged) for the roofline
    prof = np.zeros(16, np.float32)
    acc = np.zeros(16)
    nprof = 3
    for _ in range(nprof):
        n = lib.ob_model_profile_step(m.h, case.dt, prof.ctypes.data_as(C.POINTER(C.c_float)), 16)
        if n < 0:
            N.check(-n)
        acc[:n] += prof[:n]
    names = ["LSF+CI", "NUT", "ADVV", "ADVQ", "PHYS", "DIV", "SOLVE", "PROJ+RAIN"]
    pass_ms = {nm: acc[i] / nprof for i, nm in enumerate(names)}
    # timed region: K steps, device time
    clocks = ClockSampler()
    barrier()
    m.sync()
    clocks.start()
    N.check(lib.ob_model_timed_steps(m.h, case.dt, args.steps, C.byref(ms)))
    clk = clocks.stop()
    barrier()
    t_ms = allmax(ms.value)
    per_rank_sim = args.steps * case.dt
    value = world * per_rank_sim / (t_ms / 1000.0)
    cell_steps = world * args.steps * case.cells / (t_ms / 1000.0)
    # end to end through the public API, on a second copy of the case over the same steps as the timed region (the
    # storms grow, so later steps cost more): every step uploads the app's storm-start list (setCI, model.js:1383)
    # from pinned host memory, steps, and requests the step's FP64 water / mass / rain budgets, whose copy to the host
    # is read back while the next step runs (the reference app reads its maps back the same way, double-buffered:
    # model.js:1478-1494); the last step's budgets are read inside the timed region. The list holds one event
    # scheduled after the run (its window opens at 1e9 s), so the CI pass reads it every step while the workload stays
    # the bubbles-only case. The untimed warm-up has as many steps as precede the device-timed region, which also
    # captures every step graph of the list's uniforms before the timing starts.
    import torch
    pinned_t = torch.zeros(N.CI_FLOATS, dtype=torch.float32, pin_memory=True)
    pinned = pinned_t.numpy()
    pinned[:] = [0.5 * case.nx * case.dx, 0.5 * case.ny * case.dx, 1500.0, 10000.0, 1500.0, 5.0, 1e9, 1e9 + 1800.0,
                 0.0, 0.0, 0.0, 600.0]
    h2d_bytes = int(pinned.nbytes)
    d2h_bytes = 8 * 8   # each request copies back its block of 8 FP64 sums
    m2, _ = M.setup_case(case)

    def e2e_step(prev):
        N.check(lib.ob_model_set_ci(m2.h, N.fptr(pinned), 1))
        m2.enc_step(case.dt)
        ticket = m2.request_budgets()
        if prev is not None:
            m2.read_budgets(prev)
        return ticket

    prev = None
    for _ in range(args.warmup + nprof):
        prev = e2e_step(prev)
    m2.read_budgets(prev)
    barrier()
    m2.sync()
    ke = args.steps
    t0 = time.perf_counter()
    prev = None
    for _ in range(ke):
        prev = e2e_step(prev)
    last = m2.read_budgets(prev)
    e2e_s = allmax(time.perf_counter() - t0)
    if not all(math.isfinite(v) for v in last.values()):
        raise RuntimeError("end-to-end run: non-finite budgets %s" % last)
    e2e_val = world * ke * case.dt / e2e_s
    m2.destroy()
    # roofline of the dominant kernel: the pass with the longest time per kernel launch (PHYS, NUT and DIV are one
    # kernel each; ADVV, ADVQ, PROJ+RAIN and LSF+CI two; the refined solve eleven)
    hbm, bf16, src = peaks()
    pb = pass_bytes(case.nx, case.ny, case.nz, m.pad, case.dt)
    kernels = {"LSF+CI": 2, "NUT": 1, "ADVV": 2, "ADVQ": 2, "PHYS": 1, "DIV": 1, "SOLVE": 11 if m.solver >= 2 else 5,
               "PROJ+RAIN": 2}
    dom = max(pass_ms, key=lambda k: pass_ms[k] / kernels[k])
    achieved = pb[dom] / (pass_ms[dom] / 1000.0) / 1e9
    roof = {"pass": dom, "kernel": {"PHYS": "k_phys", "NUT": "k_nut", "DIV": "k_div"}.get(dom, dom), "bound": "hbm",
            "achieved": achieved, "peak": hbm, "unit": "GB/s", "frac": achieved / hbm,
            "peak_source": src, "traffic": ncu_traffic(dom, case.cells),
            "algorithmic_bytes": pb[dom], "ms": pass_ms[dom], "launches_per_step": kernels[dom],
            "note": "algorithmic bytes: every array the reference's pass reads and writes; the clear-air skips of ADVQ "
                    "and PHYS leave zero hydrometeor channels untouched, so their DRAM traffic is below them"}
    # the solve's transforms against the tensor-core peak: the MMA work of the bf16x3 split (3 products per
    # element) and of the refinement pass (3 more, or 1 in plain bf16)
    mult = {0: 1, 1: 3, 2: 6, 3: 4, 4: 9, 5: 4}[m.solver]
    fl = solve_flops(case.nx, case.ny, case.nz, m.pad) * mult
    solve_roof = {"bound": "tensor", "flops": fl, "dst_flops": fl / mult, "ms": pass_ms["SOLVE"],
                  "achieved": fl / (pass_ms["SOLVE"] / 1000.0) / 1e12, "peak": bf16, "unit": "TFLOP/s",
                  "frac": fl / (pass_ms["SOLVE"] / 1000.0) / 1e12 / bf16, "traffic": ncu_traffic("SOLVE", case.cells),
                  "note": "achieved over the whole pass (transforms, tridiagonals, residual) at the burst bf16 peak"}
    step_bytes = sum(pb.values())
    step_ms = t_ms / args.steps
    line = {"metric": METRIC, "value": value, "unit": "sim-s/wall-s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": step_ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic (Weisman-Klemp sounding, seeded bubbles)",
            "cell_steps_per_s": cell_steps,
            "config": {"workload": ("640x640x40 dx 1 km dz 500 m dt 6 s, Lin, 8 warm bubbles (Weisman-Klemp)" if not args.nx
                                    else "%dx%dx40 dx 1 km dz 500 m dt 6 s, Lin, 4 warm bubbles (Weisman-Klemp)" % (args.nx, args.nx)),
                       "cells": case.cells, "parallelism": "replicas" if world > 1 else "single domain",
                       "l2": "state %.1f GB > 126 MB L2 (no flush needed)" % (2.8 * case.cells / 16384000),
                       "solver": {0: "fp32 SIMT DST", 1: "bf16x3 tensor-core DST",
                                  2: "bf16x3 tensor-core DST + 1 refinement sweep",
                                  3: "bf16x3 tensor-core DST + 1 plain-bf16 refinement sweep",
                                  4: "bf16x3 tensor-core DST + 2 refinement sweeps",
                                  5: "plain-bf16 tensor-core DST + 1 bf16x3 refinement sweep"}[m.solver]},
            "pass_ms": {k: round(v, 4) for k, v in pass_ms.items()},
            "step_hbm": {"algorithmic_bytes": step_bytes, "gbs": step_bytes / (step_ms / 1000.0) / 1e9,
                         "frac_of_measured_peak": step_bytes / (step_ms / 1000.0) / 1e9 / hbm},
            "roofline": roof, "solve_roofline": solve_roof, "clocks": clk,
            "e2e": {"value": e2e_val, "unit": "sim-s/wall-s", "h2d_bytes_per_step": h2d_bytes,
                    "d2h_bytes_per_step": d2h_bytes, "steps": ke},
            "gpu_launches": None, "nan_guard_count": m.nan_count}
    # CI, NUT, ADVV x2, ADVQ x2, PHYS, DIV, the refined solve (8 transforms, 2 tridiagonals, 1 residual), PROJ, RAIN;
    # LSF every 60 s of model time
    launches_per_step = 21
    line["gpu_launches"] = int(args.steps * launches_per_step + math.ceil(args.steps * case.dt / 60.0))
    if rank == 0 and world == 1 and not args.no_extras:
        for key, fn in (("full_run", lambda: full_run(W.case_c2())), ("c3", c3_solve), ("c5", c5_ensemble)):
            try:
                line[key] = fn()
            except Exception as e:  # the headline line still prints
                line[key] = {"error": str(e)[:300]}
    if rank == 0 and world == 1 and not args.no_mlp:
        # the metric's second half: plain vs MLP microphysics on the 512 x 512 x 40 Thompson case, 60 minutes
        from outbreaklab_b200 import benchmarks as BM
        try:
            r = BM.surrogate_compare()
            line["mlp"] = {
                "workload": "512x512x40 dx 500 m dz 500 m dt 3 s, Thompson-style, 8 warm bubbles, 60 min; surrogate "
                            "12->3x128 GELU->10, BF16 weights / FP32 accumulation on tcgen05",
                "plain_sim_s_per_wall_s": r["plain"]["sim_s_per_wall_s"],
                "mlp_sim_s_per_wall_s": r["surrogate"]["sim_s_per_wall_s"],
                "plain_cell_steps_per_s": r["plain"]["cell_steps_per_s"],
                "mlp_cell_steps_per_s": r["surrogate"]["cell_steps_per_s"],
                "speedup": r["speedup"], "rain_rel_diff": r["rain_rel_diff"], "max_dbz_diff": r["max_dbz_diff"],
                "max_w_rel_diff": r["max_w_rel_diff"], "pairs": r["pairs"], "train_s": r["train_s"],
                "train_loss": r["train_loss"][-1], "queued_last_step": r["surrogate"]["queued_last_step"],
                "fallbacks_last_step": r["surrogate"]["fallbacks_last_step"]}
        except Exception as e:  # the headline line still prints
            line["mlp"] = {"error": str(e)[:300]}
    if rank == 0:
        if not args.no_cpu_baseline:
            line["cpu_baseline"] = cpu_baseline(case, 1)
        print(json.dumps(line), flush=True)
    if dist:
        dist[1].destroy_process_group()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=600)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-mlp", action="store_true", help="skip the plain vs MLP microphysics leg")
    ap.add_argument("--no-extras", action="store_true", help="skip the 60-minute run, the 1024x1024x80 solve and the "
                                                             "24-member ensemble")
    ap.add_argument("--nx", type=int, default=0, help="smaller square domain (profiling captures); 0 = 640")
    args = ap.parse_args()
    args.warmup = max(3, args.warmup)
    rank, world, local = _rank_env()
    _pin_device(local, world)
    if args.impl == "reference":
        run_reference(args, rank, world)
    else:
        run_ours(args, rank, world)


if __name__ == "__main__":
    main()
