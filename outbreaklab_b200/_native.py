"""ctypes binding of the C ABI (include/ob.h) exported by _lib/libob_b200.so.

There is no fallback: if the library is missing or no CUDA device is present, the calls fail with an error.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_lib", "libob_b200.so")

OB_OK, OB_ERR_OOM, OB_ERR_INVALID, OB_ERR_DEVICE, OB_ERR_TIMEOUT, OB_ERR_NAN = 0, 1, 2, 3, 4, 5
FIELD_V, FIELD_Q1, FIELD_Q2, FIELD_AUX, FIELD_PHI, FIELD_RAIN = 0, 1, 2, 3, 4, 5
FIELD_LSF_A, FIELD_LSF_B, FIELD_CI_MAP, FIELD_PHT = 6, 7, 8, 9
BOUNDARY_FLOATS, MAX_BOUNDS, CI_FLOATS, MAX_CI = 148, 8, 12, 256
OB_STATIC_POISSON_MAX_SIDE, OB_STATIC_POISSON_MAX_NZ, OB_STATIC_POISSON_MAX_CELLS = 256, 512, 1 << 20
RADAR_MAX_RADIALS, RADAR_MAX_TORNADOES, RADAR_TORNADO_FLOATS = 720, 64, 8
ENS_NTILES, ENS_MAX_MEMBERS = 6, 48


class ObError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__("%s (code %d)" % (msg, code))
        self.code = code


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


class ObGrid(C.Structure):
    _fields_ = [("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int), ("dx", C.c_float)]


# every symbol include/ob.h declares: name -> (restype, argtypes)
_vp, _i, _f, _d, _sz = C.c_void_p, C.c_int, C.c_float, C.c_double, C.c_size_t
_fp = C.POINTER(C.c_float)
SYMBOLS = {
    "ob_last_error": (C.c_char_p, []),
    "ob_version": (C.c_char_p, []),
    "ob_params_default": (None, [C.POINTER(ObParams)]),
    "ob_grid_pad": (_i, [_f]),
    "ob_model_create": (_i, [C.POINTER(ObGrid), C.POINTER(_vp)]),
    "ob_model_destroy": (_i, [_vp]),
    "ob_model_set_base_state": (_i, [_vp, _fp, _i]),
    "ob_model_set_params": (_i, [_vp, C.POINTER(ObParams)]),
    "ob_model_set_boundaries": (_i, [_vp, _fp, _i]),
    "ob_model_set_ci": (_i, [_vp, _fp, _i]),
    "ob_model_reset": (_i, [_vp]),
    "ob_model_step": (_i, [_vp, _f, _i]),
    "ob_model_sync": (_i, [_vp]),
    "ob_model_maps": (_i, [_vp, _fp]),
    "ob_model_get_field": (_i, [_vp, _i, _vp, _sz]),
    "ob_model_set_field": (_i, [_vp, _i, _vp, _sz]),
    "ob_model_time": (_i, [_vp, C.POINTER(_d), C.POINTER(_i), C.POINTER(_i)]),
    "ob_model_budgets": (_i, [_vp, C.POINTER(_d), C.POINTER(_d), C.POINTER(_d)]),
    "ob_model_nan_count": (C.c_uint, [_vp]),
    "ob_model_stream": (_vp, [_vp]),
    "ob_model_set_solver": (_i, [_vp, _i]),
    "ob_model_solver": (_i, [_vp]),
    "ob_model_timed_steps": (_i, [_vp, _f, _i, _fp]),
    "ob_model_profile_step": (_i, [_vp, _f, _fp, _i]),
    "ob_poisson_create": (_i, [_i, _i, _i, _f, _f, _i, C.POINTER(_vp)]),
    "ob_poisson_destroy": (_i, [_vp]),
    "ob_poisson_set_density": (_i, [_vp, _fp, _fp]),
    "ob_poisson_solve": (_i, [_vp, _fp, _fp]),
    "ob_poisson_solve_device": (_i, [_vp, _vp, _vp, _vp]),
    "ob_poisson_time": (_i, [_vp, _i, _fp]),
    "ob_poisson_residual": (_i, [_vp, C.POINTER(C.c_double), C.POINTER(C.c_double)]),
    "ob_poisson_set_pair_tiles": (_i, [_vp, _i]),
    "ob_model_set_pair_tiles": (_i, [_vp, _i]),
    "ob_poisson_set_tile_widths": (_i, [_vp, _i, _i]),
    "ob_model_request_budgets": (_i, [_vp, C.POINTER(C.c_longlong)]),
    "ob_model_read_budgets": (_i, [_vp, C.c_longlong, C.POINTER(C.c_double), C.POINTER(C.c_double), C.POINTER(C.c_double)]),
    "ob_model_set_tile_widths": (_i, [_vp, _i, _i]),
    "ob_dst_tc_selftest": (_i, [_i, _i, _i, _i, _fp, _fp, _fp]),
    "ob_poisson_solve_static": (_i, [_i, _i, _i, _f, _f, _vp, _vp, _vp, _vp, _vp]),
    "ob_radar_create": (_i, [_vp, _sz, _i, C.POINTER(_vp)]),
    "ob_radar_destroy": (_i, [_vp]),
    "ob_radar_set_tornadoes": (_i, [_vp, _fp, _i]),
    "ob_radar_cut": (_i, [_vp, _vp]),
    "ob_radar_read": (_i, [_vp, _vp, _sz]),
    "ob_radar_cut_moments": (_i, [_vp, _vp, _fp, _sz]),
    "ob_radar_kdp": (_i, [_vp, _fp, _sz]),
    "ob_radar_level2": (_i, [_vp, _vp, _i, _vp, _sz, _vp, _sz]),
    "ob_radar_write": (_i, [_vp, _vp, _sz]),
    "ob_mlp_create": (_i, [C.c_uint, C.POINTER(_vp)]),
    "ob_mlp_destroy": (_i, [_vp]),
    "ob_mlp_set_params": (_i, [_vp, _fp, _i]),
    "ob_mlp_get_params": (_i, [_vp, _fp, _i]),
    "ob_mlp_set_norm": (_i, [_vp, _fp, _i]),
    "ob_mlp_get_norm": (_i, [_vp, _fp, _i]),
    "ob_mlp_reserve_pairs": (_i, [_vp, C.c_longlong]),
    "ob_mlp_pair_count": (_i, [_vp, C.POINTER(C.c_longlong)]),
    "ob_mlp_read_pairs": (_i, [_vp, C.c_longlong, C.c_longlong, _fp]),
    "ob_mlp_write_pairs": (_i, [_vp, _fp, C.c_longlong]),
    "ob_mlp_grad": (_i, [_vp, _fp, _i, C.POINTER(_d), _fp]),
    "ob_mlp_eval": (_i, [_vp, _fp, _i, _fp]),
    "ob_mlp_train": (_i, [_vp, _i, _i, _f, C.c_uint, C.POINTER(_d)]),
    "ob_mlp_set_training": (_i, [_vp, _i]),
    "ob_mlp_sort_pairs": (_i, [_vp]),
    "ob_model_record_micro": (_i, [_vp, _vp, _f]),
    "ob_model_set_graphs": (_i, [_vp, _i]),
    "ob_model_tornado_candidates": (_i, [_vp, _f, _fp, _i, C.POINTER(_i)]),
    "ob_hurricane_default": (None, [C.POINTER(ObHurricane)]),
    "ob_model_set_surface": (_i, [_vp, _fp, C.POINTER(ObHurricane)]),
    "ob_model_set_hurricane": (_i, [_vp, C.POINTER(ObHurricane)]),
    "ob_model_set_vortex": (_i, [_vp, _fp, _i, _f, _f, _f, _f, _f]),
    "ob_ensemble_create": (_i, [C.POINTER(_vp), _fp, _i, C.POINTER(_vp)]),
    "ob_ensemble_set_lanes": (_i, [_vp, _i]),
    "ob_ensemble_lanes": (_i, [_vp]),
    "ob_ensemble_step": (_i, [_vp, _i]),
    "ob_ensemble_timed_steps": (_i, [_vp, _i, _fp]),
    "ob_ensemble_sync": (_i, [_vp]),
    "ob_ensemble_set_graphs": (_i, [_vp, _i]),
    "ob_ensemble_set_tiles": (_i, [_vp, C.POINTER(_i)]),
    "ob_ensemble_get_tiles": (_i, [_vp, C.POINTER(_i)]),
    "ob_ensemble_time_pass": (_i, [_vp, _i, _i, _fp]),
    "ob_ensemble_tune": (_i, [_vp, _i, C.POINTER(_i), _fp]),
    "ob_ensemble_lsf_times": (_i, [_vp, C.POINTER(_d)]),
    "ob_ensemble_stream": (_vp, [_vp]),
    "ob_ensemble_destroy": (None, [_vp]),
    "ob_model_set_surrogate": (_i, [_vp, _vp]),
    "ob_model_surrogate_stats": (_i, [_vp, C.POINTER(C.c_uint), C.POINTER(C.c_uint)]),
}
MLP_NIN, MLP_NOUT, MLP_NPARAM, MLP_PAIR, MLP_NNORM = 12, 10, 35978, 24, 59

_lib = None


def lib():
    """Loads the library (raises OSError if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise OSError("outbreaklab_b200: %s is missing; run `python -m outbreaklab_b200.build`" % LIB_PATH)
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in SYMBOLS.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def check(rc: int):
    if rc != OB_OK:
        raise ObError(rc, lib().ob_last_error().decode(errors="replace"))
    return rc


def fptr(a: np.ndarray):
    assert a.dtype == np.float32 and a.flags.c_contiguous
    return a.ctypes.data_as(_fp)


def default_params() -> ObParams:
    p = ObParams()
    lib().ob_params_default(C.byref(p))
    return p
