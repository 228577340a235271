"""Secondary benchmarks (one JSON line each): the pressure solve in isolation and the step on other configurations.

  python -m outbreaklab_b200.benchmarks solve --nx 1024 --ny 1024 --nz 80 --precision 2 --reps 20
  python -m outbreaklab_b200.benchmarks step --case c4 --steps 50

The solve benchmark's right-hand side is the 5 km-correlated Gaussian random field of the 1024 x 1024 x 80 case
(zero horizontal mean per level), with the Weisman-Klemp densities; errors and residuals are computed in FP64 on the
host when --check is given (the FP64 solve of the CPU oracle takes minutes at full size).
"""
from __future__ import annotations

import argparse
import json
import os
import sys
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
    phi = P.solve(rhs)
    ms = P.device_ms(args.reps)
    flops = 4.0 * nx * ny * nz * (nx + ny) * (3 if args.precision >= 1 else 1) * (2 if args.precision == 2 else 1)
    out = {"bench": "pressure solve", "nx": nx, "ny": ny, "nz": nz, "precision": args.precision, "ms": ms,
           "dst_flops": flops, "tflops": flops / (ms * 1e-3) / 1e12}
    if args.check:
        sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
        from oracle import oracle as O
        r64, w64 = rc.astype(np.float64), rw.astype(np.float64)
        ref = O.poisson_solve(rhs.astype(np.float64), dx, dz, r64, w64, 8)
        res = O.poisson_apply(phi.astype(np.float64), dx, dz, r64, w64) - rhs
        out.update(err_inf=float(np.abs(phi - ref).max() / np.abs(ref).max()),
                   err_l2=float(np.sqrt(((phi - ref) ** 2).sum() / (ref ** 2).sum())),
                   resid_inf=float(np.abs(res).max() / np.abs(rhs).max()),
                   resid_l2=float(np.sqrt((res ** 2).sum() / (rhs.astype(np.float64) ** 2).sum())))
    print(json.dumps(out), flush=True)


def step(args):
    case = {"c1": W.case_c1, "c2": W.case_c2, "c4": W.case_c4}[args.case]()
    m, _ = M.setup_case(case)
    if args.solver is not None:
        m.set_solver(args.solver)
    import ctypes as C
    from . import _native as N
    N.check(N.lib().ob_model_step(m.h, case.dt, args.warmup))
    t = C.c_float()
    N.check(N.lib().ob_model_timed_steps(m.h, case.dt, args.steps, C.byref(t)))
    print(json.dumps({"bench": "step", "case": case.name, "cells": case.cells, "steps": args.steps, "ms_per_step": t.value / args.steps,
                      "sim_s_per_wall_s": args.steps * case.dt / (t.value / 1000.0), "solver": m.solver}), flush=True)


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
    a.add_argument("--check", action="store_true")
    b = sub.add_parser("step")
    b.add_argument("--case", default="c4")
    b.add_argument("--steps", type=int, default=50)
    b.add_argument("--warmup", type=int, default=5)
    b.add_argument("--solver", type=int, default=None)
    args = ap.parse_args(argv)
    {"solve": solve, "step": step}[args.cmd](args)


if __name__ == "__main__":
    main()
