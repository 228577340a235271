"""Host-side mirror of the reference's step and field-buffer API over the C ABI.

``RegionalModel`` keeps the method names and argument meaning of the reference class (model.js:1156-1496):
``allocate``, ``set_sounding``, ``set_boundaries``, ``set_ci``, ``set_surface``, ``set_vortex``, ``reset``,
``enc_step``, ``request_maps``, ``destroy``, ``params``, ``time``, ``steps``, ``parity``. ``PoissonDirect`` mirrors
solver.js:105-165. Errors surface as ``ObError`` (the reference throws a JS ``Error``, model.js:1194-1200).
All compute runs in the CUDA library; nothing here falls back to the CPU.
"""
from __future__ import annotations

import ctypes as C
import math

import numpy as np

from . import _native as N
from . import boundaries
from . import sounding as snd_mod

# grid presets (model.js:1143-1154)
GRID_PRESETS = {
    "quick": {"dx": 2000, "n": [320, 320, 56]},
    "standard": {"dx": 1500, "n": [448, 448, 60]},
    "large": {"dx": 1500, "n": [640, 640, 60]},
    "fine": {"dx": 1000, "n": [640, 640, 64]},
    "m500": {"dx": 500, "n": [512, 512, 80]},
    "m250": {"dx": 250, "n": [512, 512, 100]},
    "m100": {"dx": 100, "n": [512, 512, 160]},
}

# RegionalModel.params (model.js:1176-1180) -> ObParams field
_PARAM_MAP = {"cs": "cs", "nu0": "nu0", "drag": "drag", "z0": "z0", "spongeW": "spongeW", "spongeTau": "spongeTau",
              "dampZ": "dampZ", "dampTau": "dampTau", "auto": "autoc", "qc0": "qc0", "freeze": "freeze",
              "noise": "noise", "mc": "mc", "vcap": "vcap", "evap": "evap", "sortQ": "sortQ", "ciRate": "ciRate",
              "nudgeTau": "nudgeTau", "lat": "lat", "moistMix": "moistMix", "mcFloor": "mcFloor", "evapT": "evapT"}


def grid_pad(dx: float) -> int:
    return N.lib().ob_grid_pad(float(dx))


class RegionalModel:
    """The B200 storm model of one domain (model.js:1156)."""

    def __init__(self):
        p = N.default_params()
        self.params = {k: float(getattr(p, v)) for k, v in _PARAM_MAP.items()}
        self.params["scheme"] = "lin"
        self.h = None
        self.bounds = []
        self.ci_events = []
        self.rho_sfc = None
        self.base = None
        self.analysis = None

    # ---- allocation (model.js:1186-1238) ----
    def allocate(self, key=None, spec=None):
        self.destroy()
        pr = spec or GRID_PRESETS[key]
        nx, ny, nz = pr["n"]
        g = N.ObGrid(int(nx), int(ny), int(nz), float(pr["dx"]))
        h = C.c_void_p()
        N.check(N.lib().ob_model_create(C.byref(g), C.byref(h)))
        self.h = h
        self.key = key or pr.get("key")
        self.nx, self.ny, self.nz, self.dx = int(nx), int(ny), int(nz), float(pr["dx"])
        self.dz = 20000.0 / nz
        self.Lx, self.Ly = nx * self.dx, ny * self.dx
        self.pad = grid_pad(self.dx)
        self.params["spongeW"] = min(max(0.08 * min(self.Lx, self.Ly), 5000.0), 40000.0)
        return self

    def destroy(self):
        self._params_sent = None   # a later handle may reuse this one's address
        if self.h:
            N.lib().ob_model_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.destroy()
        except Exception:
            pass

    def _sync_params(self):
        """Sends `params` to the library when they differ from what this handle last received (only
        ob_model_set_params writes the library's copy, so an unchanged dict needs no call on every step)."""
        vals = tuple(float(self.params[k]) for k in _PARAM_MAP) + (self.params.get("scheme") == "thompson",)
        if getattr(self, "_params_sent", None) == (self.h.value, vals):
            return
        p = N.default_params()
        for k, v in _PARAM_MAP.items():
            setattr(p, v, float(self.params[k]))
        p.scheme = 1.0 if self.params.get("scheme") == "thompson" else 0.0
        N.check(N.lib().ob_model_set_params(self.h, C.byref(p)))
        self._params_sent = (self.h.value, vals)

    # ---- inputs ----
    def set_sounding(self, text: str):
        """model.js:1276-1288: SHARPpy text -> analysis + base state on the model grid."""
        s = snd_mod.parse_sharppy(text)
        self.analysis = snd_mod.analyze(s)
        B, sfcP, sfcH = snd_mod.base_state(s, self.nz, self.dz)
        self.set_base_state(B)
        self.base = {"B": B, "sfcP": sfcP, "sfcH": sfcH}
        return self.analysis

    def set_base_state(self, B):
        B = np.ascontiguousarray(B, np.float32).reshape(-1)
        if B.size != (self.nz + 1) * 8:
            raise N.ObError(N.OB_ERR_INVALID, "base state: %d values, expected (nz+1)*8 = %d" % (B.size, (self.nz + 1) * 8))
        N.check(N.lib().ob_model_set_base_state(self.h, N.fptr(B), self.nz))
        self.rho_sfc = float(B[2])

    def set_boundaries(self, bnds):
        """model.js:1371-1380: [{pts, motion, vel, halfW, dT, Hmax, slope, Hmin, dq, qRatio, du, dv, wRatio, nudge,
        dFree, side, vary, seed, varyL}] in model metres and m/s (boundaries.boundary_models builds them from the
        boundaries drawn on the map). Like the reference, takes effect at the next reset or LSF pass."""
        f, n = boundaries.pack_boundaries(bnds)
        self.bounds = list(bnds)[:n]
        N.check(N.lib().ob_model_set_boundaries(self.h, N.fptr(f), n))

    def set_ci(self, events):
        """model.js:1383-1389: towers [{x, y, zc, rh, rz, wt, t0, t1, vx, vy, seed, ramp}]; those that ended before
        the model's time are dropped."""
        f, act = pack_ci(events, self.time)
        self.ci_events = act
        N.check(N.lib().ob_model_set_ci(self.h, N.fptr(f), len(act)))

    # ---- stepping (model.js:1427-1476) ----
    def reset(self):
        self._sync_params()
        N.check(N.lib().ob_model_reset(self.h))

    # ---- hurricane mode (model.js:1290-1365) ----
    def set_surface(self, surf=None, hur=None):
        """setSurface: surf (ny, nx, 4) float32 (land fraction, SST K, 0, 0) or None; hur an ObHurricane or None."""
        a = None if surf is None else np.ascontiguousarray(surf, np.float32).reshape(-1)
        if a is not None and a.size != self.nx * self.ny * 4:
            raise N.ObError(N.OB_ERR_INVALID, "set_surface: %d floats, want nx * ny * 4 = %d" % (a.size, self.nx * self.ny * 4))
        if hur is not None and not isinstance(hur, N.ObHurricane):
            raise N.ObError(N.OB_ERR_INVALID, "set_surface: the hurricane is an ObHurricane (hurricane.default_hurricane())")
        N.check(N.lib().ob_model_set_surface(self.h, N.fptr(a) if a is not None else None,
                                             C.byref(hur) if hur is not None else None))
        self.hurricane = hur

    def set_hurricane(self, hur):
        N.check(N.lib().ob_model_set_hurricane(self.h, C.byref(hur)))
        self.hurricane = hur

    def set_vortex(self, tab=None, info=None):
        """setVortex's table (hurricane.vortex_table) or None to clear it; read by reset."""
        if tab is None:
            N.check(N.lib().ob_model_set_vortex(self.h, None, 0, 0.0, 0.0, 1.0, 1.0, 0.0))
            return
        t = np.ascontiguousarray(tab, np.float32)
        if t.ndim != 3 or t.shape[0] != self.nz or t.shape[2] != 4:
            raise N.ObError(N.OB_ERR_INVALID, "set_vortex: the table is (nz, nr, 4)")
        N.check(N.lib().ob_model_set_vortex(self.h, N.fptr(t.reshape(-1)), int(t.shape[1]), float(info["x"]), float(info["y"]),
                                            float(info["dr"]), float(info["moistR"]), float(info["moistRH"])))

    def enc_step(self, dt, nsteps=1):
        self._sync_params()
        N.check(N.lib().ob_model_step(self.h, float(dt), int(nsteps)))

    step = enc_step

    def sync(self):
        N.check(N.lib().ob_model_sync(self.h))

    @property
    def time(self):
        t, s, p = C.c_double(), C.c_int(), C.c_int()
        N.check(N.lib().ob_model_time(self.h, C.byref(t), C.byref(s), C.byref(p)))
        return t.value

    @property
    def steps(self):
        t, s, p = C.c_double(), C.c_int(), C.c_int()
        N.check(N.lib().ob_model_time(self.h, C.byref(t), C.byref(s), C.byref(p)))
        return s.value

    @property
    def parity(self):
        t, s, p = C.c_double(), C.c_int(), C.c_int()
        N.check(N.lib().ob_model_time(self.h, C.byref(t), C.byref(s), C.byref(p)))
        return p.value

    def set_pair_tiles(self, on: bool):
        """The solve's transforms on SM pairs (True) or single SMs (False); bit-identical results."""
        N.check(N.lib().ob_model_set_pair_tiles(self.h, int(bool(on))))

    def set_tile_widths(self, bn_x: int = 0, bn_y: int = 0):
        """Outputs per tile of the solve's x and y transforms (multiples of 16 in 32..256; 0: automatic)."""
        N.check(N.lib().ob_model_set_tile_widths(self.h, int(bn_x), int(bn_y)))

    def set_solver(self, precision: int):
        """Pressure-solve precision: 0 = fp32 transforms, 1 = bf16x3 tensor-core transforms."""
        N.check(N.lib().ob_model_set_solver(self.h, int(precision)))

    @property
    def solver(self):
        return int(N.lib().ob_model_solver(self.h))

    # ---- microphysics surrogate (no counterpart in the reference; see surrogate.py) ----
    def set_surrogate(self, net=None):
        """From the next step on, the microphysics of queued cells runs through a copy of net's current weights on
        the tensor cores (None: the plain scheme)."""
        N.check(N.lib().ob_model_set_surrogate(self.h, net.h if net is not None else None))
        self.surrogate = net is not None

    def surrogate_stats(self):
        """(cells the last step queued for the surrogate, how many of them fell back to the scheme)."""
        q, f = C.c_uint(), C.c_uint()
        N.check(N.lib().ob_model_surrogate_stats(self.h, C.byref(q), C.byref(f)))
        return q.value, f.value

    @property
    def nan_count(self):
        return int(N.lib().ob_model_nan_count(self.h))

    # ---- readback ----
    def request_maps(self):
        """model.js:1478-1494: {m0, m1, m2, m3: float32 (ny, nx, 4), t}."""
        out = np.empty(self.nx * self.ny * 16, np.float32)
        N.check(N.lib().ob_model_maps(self.h, N.fptr(out)))
        a = out.reshape(4, self.ny, self.nx, 4)
        return {"m0": a[0], "m1": a[1], "m2": a[2], "m3": a[3], "t": self.time}

    def field_shape(self, field):
        nx, ny, nz, p = self.nx, self.ny, self.nz, self.pad
        return {N.FIELD_V: ((nz + 1) * (ny + 1) * (nx + 1) * 4, np.float32),
                N.FIELD_Q1: (nx * ny * nz * 4, np.float32), N.FIELD_Q2: (nx * ny * nz * 4, np.float32),
                N.FIELD_AUX: (nx * ny * nz * 2, np.float32),
                N.FIELD_PHI: ((nx + 2 * p) * (ny + 2 * p) * nz, np.float32),
                N.FIELD_RAIN: (nx * ny, np.float64),
                N.FIELD_LSF_A: (nx * ny * 4, np.float32), N.FIELD_LSF_B: (nx * ny * 4, np.float32),
                N.FIELD_CI_MAP: (nx * ny * 4, np.float32), N.FIELD_PHT: (nx * ny * nz, np.float32)}[field]

    def get_field(self, field):
        n, dt = self.field_shape(field)
        out = np.empty(n, dt)
        N.check(N.lib().ob_model_get_field(self.h, field, out.ctypes.data, out.nbytes))
        return out

    def set_field(self, field, arr):
        n, dt = self.field_shape(field)
        a = np.ascontiguousarray(arr, dt).reshape(-1)
        if a.size != n:
            raise N.ObError(N.OB_ERR_INVALID, "field %d: %d values, expected %d" % (field, a.size, n))
        N.check(N.lib().ob_model_set_field(self.h, field, a.ctypes.data, a.nbytes))

    def budgets(self):
        w, m, r = C.c_double(), C.c_double(), C.c_double()
        N.check(N.lib().ob_model_budgets(self.h, C.byref(w), C.byref(m), C.byref(r)))
        return {"water": w.value, "mass": m.value, "rain": r.value}

    def request_budgets(self) -> int:
        """Queues the budgets after the work queued so far and returns a ticket for read_budgets (no wait)."""
        t = C.c_longlong()
        N.check(N.lib().ob_model_request_budgets(self.h, C.byref(t)))
        return t.value

    def read_budgets(self, ticket: int):
        """Waits for the budgets of a request (one of the last 4) and returns them."""
        w, m, r = C.c_double(), C.c_double(), C.c_double()
        N.check(N.lib().ob_model_read_budgets(self.h, C.c_longlong(ticket), C.byref(w), C.byref(m), C.byref(r)))
        return {"water": w.value, "mass": m.value, "rain": r.value}

    @property
    def Vcur(self):
        return self.get_field(N.FIELD_V)


class PoissonDirect:
    """solver.js:105-165: exact solve of rho_c lap_h(phi) + d/dz(rho_w dphi/dz) = rhs on an nx x ny x nz grid.
    precision 0: fp32 transforms; 1: bf16x3 tensor-core transforms; 2: plus one bf16x3 refinement sweep on the
    FP64-accumulated residual; 3: that sweep in plain bf16; 4: two bf16x3 refinement sweeps."""

    def __init__(self, nx, ny, nz, dx, dz, precision=0):
        self.nx, self.ny, self.nz, self.dx, self.dz = nx, ny, nz, dx, dz
        h = C.c_void_p()
        N.check(N.lib().ob_poisson_create(nx, ny, nz, float(dx), float(dz), int(precision), C.byref(h)))
        self.h = h

    def set_density(self, rhoC, rhoW):
        rc = np.ascontiguousarray(rhoC, np.float32)
        rw = np.ascontiguousarray(rhoW, np.float32)
        assert rc.size == self.nz and rw.size == self.nz + 1
        N.check(N.lib().ob_poisson_set_density(self.h, N.fptr(rc), N.fptr(rw)))

    def solve(self, rhs):
        r = np.ascontiguousarray(rhs, np.float32)
        out = np.empty_like(r)
        N.check(N.lib().ob_poisson_solve(self.h, N.fptr(r), N.fptr(out)))
        return out

    def device_ms(self, reps=10):
        """Device time of one solve (CUDA events) on the last right-hand side."""
        t = C.c_float()
        N.check(N.lib().ob_poisson_time(self.h, int(reps), C.byref(t)))
        return t.value

    def set_pair_tiles(self, on: bool):
        """Transforms on tiles of 256 rows computed by SM pairs (True) or 128-row tiles on single SMs (False);
        bit-identical results."""
        N.check(N.lib().ob_poisson_set_pair_tiles(self.h, int(bool(on))))

    def set_tile_widths(self, bn_x: int = 0, bn_y: int = 0):
        """Outputs per tile of the x and y transforms (multiples of 16 in 32..256; 0: automatic)."""
        N.check(N.lib().ob_poisson_set_tile_widths(self.h, int(bn_x), int(bn_y)))

    def residual(self):
        """FP64 residual of the last solve on the device: (max|r| / max|rhs|, ||r||_2 / ||rhs||_2)."""
        a, b = C.c_double(), C.c_double()
        N.check(N.lib().ob_poisson_residual(self.h, C.byref(a), C.byref(b)))
        return a.value, b.value

    def destroy(self):
        if getattr(self, "h", None):
            N.lib().ob_poisson_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.destroy()
        except Exception:
            pass


def pack_ci(events, time=0.0):
    """setCI's record (model.js:1383-1389): the towers still active after ``time`` (at most the last OB_MAX_CI),
    12 float32 each. Returns (array, active events)."""
    act = [e for e in events if e["t1"] > time][-N.MAX_CI:]
    f = np.zeros(max(1, len(act)) * N.CI_FLOATS, np.float32)
    for i, e in enumerate(act):
        f[i * 12:(i + 1) * 12] = [e["x"], e["y"], e["zc"], e["rh"], e["rz"], e["wt"], e["t0"], e["t1"],
                                  e.get("vx", 0) or 0, e.get("vy", 0) or 0, e.get("seed", i * 1.37),
                                  e.get("ramp", 150) or 150]
    return f, act


def setup_case(case, bounds=None, ci=None):
    """A RegionalModel for a workloads.StormCase: defaults, INIT noise 0, scheme, analytic sounding, optional
    boundaries (boundaries.boundary_models records) and storm-start towers, reset, then the bubbles and seeded theta
    noise. Returns (model, B)."""
    from . import workloads
    m = RegionalModel().allocate(spec={"dx": case.dx, "n": [case.nx, case.ny, case.nz]})
    m.params["noise"] = 0.0
    m.params["scheme"] = "thompson" if case.scheme == 1 else "lin"
    B, _ = workloads.base_state_for(case)
    m.set_base_state(B)
    if bounds:
        m.set_boundaries(bounds)
    if ci:
        m.set_ci(ci)
    m.reset()
    V = m.get_field(N.FIELD_V)
    m.set_field(N.FIELD_V, workloads.perturb_theta(case, V))
    return m, B
