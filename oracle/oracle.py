"""ctypes loader of the CPU oracle (TEST INFRASTRUCTURE ONLY).

Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg import this module. It drives the C++
restatement in ob_oracle.cpp (float = parity oracle and CPU baseline, double = FP64 error reference).
PARITY UNPINNED: the reference has no tests or golden vectors and its WGSL cannot run on this machine.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "liboboracle.so")

_lib = None


def build(force: bool = False) -> str:
    src = os.path.join(HERE, "ob_oracle.cpp")
    if force or not os.path.exists(LIB_PATH) or os.path.getmtime(LIB_PATH) < os.path.getmtime(src):
        subprocess.check_call(["make", "-s", "-C", HERE])
    return LIB_PATH


def lib():
    global _lib
    if _lib is None:
        try:
            _lib = C.CDLL(LIB_PATH)
        except OSError:
            build(force=True)
            _lib = C.CDLL(LIB_PATH)
        _declare(_lib)
    return _lib


class ObParams(C.Structure):
    _fields_ = [(n, C.c_float) for n in (
        "cs", "nu0", "drag", "z0", "spongeW", "spongeTau", "dampZ", "dampTau", "autoc", "qc0", "freeze", "noise",
        "mc", "vcap", "evap", "sortQ", "ciRate", "nudgeTau", "lat", "moistMix", "mcFloor", "scheme", "evapT",
        "dtScale")]


class ObHurricane(C.Structure):
    """include/ob.h ObHurricane (hurricane mode)."""
    _fields_ = [(n, C.c_float) for n in (
        "ck", "landMoist", "sfcP", "tauRad", "radCap", "blDepth", "u10f", "gust", "thermals", "thermalScale", "maritime",
        "filter4", "cdCap", "dissHeat", "centreX", "centreY", "thermalR", "envR", "cnOld", "traj2")]


def _declare(L):
    vp, i, d, f = C.c_void_p, C.c_int, C.c_double, C.c_float
    fp = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
    dp = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
    L.oro_create.restype = vp
    L.oro_create.argtypes = [i, i, i, d, i]
    L.oro_destroy.argtypes = [vp]
    L.oro_set_base_state.argtypes = [vp, fp]
    L.oro_set_params.argtypes = [vp, C.POINTER(ObParams)]
    L.oro_set_boundaries.argtypes = [vp, fp, i]
    L.oro_set_ci.argtypes = [vp, fp, i]
    L.oro_reset.argtypes = [vp]
    L.oro_set_surface.argtypes = [vp, vp, C.POINTER(ObHurricane)]
    L.oro_set_vortex.argtypes = [vp, vp, i, d, d, d, d, d]
    L.ob_hurricane_default.argtypes = [C.POINTER(ObHurricane)]
    L.oro_step.argtypes = [vp, d, i]
    L.oro_time.restype = d
    L.oro_time.argtypes = [vp]
    L.oro_parity.restype = i
    L.oro_parity.argtypes = [vp]
    L.oro_maps.argtypes = [vp, fp]
    L.oro_get_field.restype = i
    L.oro_get_field.argtypes = [vp, i, fp, C.c_size_t]
    L.oro_get_field_f64.restype = i
    L.oro_get_field_f64.argtypes = [vp, i, dp, C.c_size_t]
    L.oro_set_field.restype = i
    L.oro_set_field.argtypes = [vp, i, fp, C.c_size_t]
    L.oro_rain.argtypes = [vp, dp]
    L.oro_budgets.argtypes = [vp, C.POINTER(d), C.POINTER(d)]
    L.oro_poisson_solve_f32.argtypes = [i, i, i, d, d, fp, fp, fp, fp]
    L.oro_poisson_solve_f64.argtypes = [i, i, i, d, d, dp, dp, dp, dp]
    L.oro_poisson_apply_f64.argtypes = [i, i, i, d, d, dp, dp, dp, dp]
    L.oro_pcg.restype = C.c_uint32
    L.oro_pcg.argtypes = [C.c_uint32]
    L.oro_hash3i.restype = C.c_uint32
    L.oro_hash3i.argtypes = [i, i, i]
    L.oro_gnoise2.restype = f
    L.oro_gnoise2.argtypes = [f, f]
    L.oro_dst_matrix.argtypes = [i, dp]
    u8 = np.ctypeslib.ndpointer(np.uint8, flags="C_CONTIGUOUS")
    L.oro_radar_cut.argtypes = [vp, fp, fp, u8, fp, C.c_void_p]
    L.oro_radar_cut_f64.argtypes = [vp, fp, fp, u8, dp, C.c_void_p]
    L.oro_radar_code.restype = C.c_uint32
    L.oro_radar_code.argtypes = [f, f, f]
    L.oro_radar_phi.argtypes = [fp, fp, i, i, u8]
    L.ob_params_default.argtypes = [C.POINTER(ObParams)]
    L.ob_grid_pad.restype = i
    L.ob_grid_pad.argtypes = [f]


FIELD_V, FIELD_Q1, FIELD_Q2, FIELD_AUX, FIELD_PHI = 0, 1, 2, 3, 4
FIELD_LSF_A, FIELD_LSF_B, FIELD_CI_MAP, FIELD_PHT = 6, 7, 8, 9


def default_params() -> ObParams:
    p = ObParams()
    lib().ob_params_default(C.byref(p))
    return p


def default_hurricane() -> ObHurricane:
    h = ObHurricane()
    lib().ob_hurricane_default(C.byref(h))
    return h


class OracleModel:
    """The reference's RegionalModel step on the CPU (precision 4 = float, 8 = double)."""

    def __init__(self, nx, ny, nz, dx, precision=4):
        self.nx, self.ny, self.nz, self.dx = nx, ny, nz, float(dx)
        self.dz = 20000.0 / nz
        self.pad = lib().ob_grid_pad(float(dx))
        self.h = lib().oro_create(nx, ny, nz, float(dx), precision)
        self.precision = precision

    def __del__(self):
        if getattr(self, "h", None):
            lib().oro_destroy(self.h)
            self.h = None

    def field_count(self, field):
        nx, ny, nz, p = self.nx, self.ny, self.nz, self.pad
        return {FIELD_V: (nx + 1) * (ny + 1) * (nz + 1) * 4, FIELD_Q1: nx * ny * nz * 4, FIELD_Q2: nx * ny * nz * 4,
                FIELD_AUX: nx * ny * nz * 2, FIELD_PHI: (nx + 2 * p) * (ny + 2 * p) * nz,
                FIELD_LSF_A: nx * ny * 4, FIELD_LSF_B: nx * ny * 4, FIELD_CI_MAP: nx * ny * 4,
                FIELD_PHT: nx * ny * nz}[field]

    def set_base_state(self, B):
        lib().oro_set_base_state(self.h, np.ascontiguousarray(B, np.float32))

    def set_params(self, p: ObParams):
        lib().oro_set_params(self.h, C.byref(p))

    def set_boundaries(self, packed, n):
        lib().oro_set_boundaries(self.h, np.ascontiguousarray(packed, np.float32).reshape(-1), n)

    def set_ci(self, ev, n):
        lib().oro_set_ci(self.h, np.ascontiguousarray(ev, np.float32).reshape(-1), n)

    def reset(self):
        lib().oro_reset(self.h)

    def set_surface(self, surf, hur):
        """setSurface (model.js:1296-1303): surf (ny, nx, 4) float32 or None, hur an ObHurricane or None."""
        a = None if surf is None else np.ascontiguousarray(surf, np.float32).reshape(-1)
        lib().oro_set_surface(self.h, a.ctypes.data if a is not None else None, C.byref(hur) if hur is not None else None)

    def set_vortex(self, tab, nr, x, y, dr, moist_r, moist_rh):
        """setVortex's table (nz, nr, 4) float32, or nr = 0 to clear it."""
        a = None if tab is None else np.ascontiguousarray(tab, np.float32).reshape(-1)
        lib().oro_set_vortex(self.h, a.ctypes.data if a is not None else None, int(nr), float(x), float(y), float(dr),
                             float(moist_r), float(moist_rh))

    def step(self, dt, n=1):
        lib().oro_step(self.h, float(dt), int(n))

    @property
    def time(self):
        return lib().oro_time(self.h)

    def get(self, field, f64=False):
        n = self.field_count(field)
        if f64:
            out = np.empty(n, np.float64)
            rc = lib().oro_get_field_f64(self.h, field, out, n)
        else:
            out = np.empty(n, np.float32)
            rc = lib().oro_get_field(self.h, field, out, n)
        assert rc == 0
        return out

    def set(self, field, arr):
        arr = np.ascontiguousarray(arr, np.float32).reshape(-1)
        assert lib().oro_set_field(self.h, field, arr, arr.size) == 0

    def maps(self):
        out = np.empty(self.nx * self.ny * 16, np.float32)
        lib().oro_maps(self.h, out)
        return out

    def rain(self):
        out = np.empty(self.nx * self.ny, np.float64)
        lib().oro_rain(self.h, out)
        return out

    def budgets(self):
        w, m = C.c_double(), C.c_double()
        lib().oro_budgets(self.h, C.byref(w), C.byref(m))
        return w.value, m.value

    def radar_cut(self, U, tor, volume_bytes, ng_dop, moments=True):
        """One radar cut on the current state (radar.js:229-268): returns (volume bytes, KDP (nrad, ngDop),
        moments (nrad, ngRef, 6) or None) in this model's precision."""
        U = np.ascontiguousarray(U, np.float32).reshape(-1)
        assert U.size == 44
        nrad, ngr = int(U[11]), int(U[12])
        tor = np.ascontiguousarray(tor if tor is not None else np.zeros(8), np.float32).reshape(-1)
        out = np.zeros(volume_bytes, np.uint8)
        dt = np.float64 if self.precision == 8 else np.float32
        kdp = np.zeros(720 * ng_dop, dt)
        mom = np.zeros(nrad * ngr * 6, dt) if moments else None
        fn = lib().oro_radar_cut_f64 if self.precision == 8 else lib().oro_radar_cut
        fn(self.h, U, tor, out, kdp, mom.ctypes.data if moments else None)
        return out, kdp[:nrad * ng_dop].reshape(nrad, ng_dop), (mom.reshape(nrad, ngr, 6) if moments else None)


def radar_code(v, sc, ofs):
    """WGSL code() of radar.js:140 on fp32 values (vectorised over v)."""
    v = np.asarray(v, np.float32)
    return np.array([lib().oro_radar_code(float(x), float(sc), float(ofs)) for x in v.reshape(-1)], np.uint32).reshape(v.shape)


def radar_phi(U, kdp):
    """WGSL_R_PHI (radar.js:243-268) on a given fp32 KDP array (nrad, ng): the PHI codes."""
    kdp = np.ascontiguousarray(kdp, np.float32)
    nrad, ng = kdp.shape
    out = np.zeros(nrad * ng, np.uint8)
    lib().oro_radar_phi(np.ascontiguousarray(U, np.float32).reshape(-1), kdp.reshape(-1), nrad, ng, out)
    return out.reshape(nrad, ng)


def poisson_solve(rhs, dx, dz, rhoC, rhoW, precision=4):
    nz, ny, nx = rhs.shape
    if precision == 8:
        out = np.empty_like(rhs, dtype=np.float64)
        lib().oro_poisson_solve_f64(nx, ny, nz, dx, dz, np.ascontiguousarray(rhoC, np.float64),
                                    np.ascontiguousarray(rhoW, np.float64),
                                    np.ascontiguousarray(rhs, np.float64).reshape(-1), out.reshape(-1))
        return out
    out = np.empty(rhs.shape, np.float32)
    lib().oro_poisson_solve_f32(nx, ny, nz, dx, dz, np.ascontiguousarray(rhoC, np.float32),
                                np.ascontiguousarray(rhoW, np.float32),
                                np.ascontiguousarray(rhs, np.float32).reshape(-1), out.reshape(-1))
    return out


def poisson_apply(phi, dx, dz, rhoC, rhoW):
    nz, ny, nx = phi.shape
    out = np.empty(phi.shape, np.float64)
    lib().oro_poisson_apply_f64(nx, ny, nz, dx, dz, np.ascontiguousarray(rhoC, np.float64),
                                np.ascontiguousarray(rhoW, np.float64),
                                np.ascontiguousarray(phi, np.float64).reshape(-1), out.reshape(-1))
    return out


def setup_case(case, precision=4, bounds=None, ci=None):
    """Creates an oracle model for a workloads.StormCase: defaults, noise 0, scheme, base state, optional boundaries
    and storm-start towers (packed by the same host code as the model's), reset, perturbed theta. Returns
    (model, B)."""
    from outbreaklab_b200 import workloads, boundaries, model as M
    B, _ = workloads.base_state_for(case)
    m = OracleModel(case.nx, case.ny, case.nz, case.dx, precision)
    p = default_params()
    p.noise = 0.0
    p.scheme = float(case.scheme)
    m.set_params(p)
    m.set_base_state(B)
    if bounds:
        m.set_boundaries(*boundaries.pack_boundaries(bounds))
    if ci:
        f, act = M.pack_ci(ci, 0.0)
        m.set_ci(f, len(act))
    m.reset()
    V = m.get(FIELD_V)
    m.set(FIELD_V, workloads.perturb_theta(case, V))
    return m, B
