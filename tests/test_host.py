"""Host-side tests that need no GPU: the C-ABI library loads and exports every symbol include/ob.h declares, the
parameter defaults agree with the reference's, the host mirror packs inputs in the reference's layouts."""
import ctypes as C
import os
import re
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared_symbols():
    names = set()
    for f in os.listdir(os.path.join(ROOT, "include")):
        if f.endswith(".h"):
            src = open(os.path.join(ROOT, "include", f)).read()
            src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
            names |= set(re.findall(r"\b(ob_[a-z0-9_]+)\s*\(", src))
    return names


def test_library_exports_every_declared_symbol(native):
    lib = native.LIB_PATH
    out = subprocess.run(["nm", "-D", "--defined-only", lib], capture_output=True, text=True, check=True).stdout
    exported = set(re.findall(r"\s[TW]\s+(ob_[a-z0-9_]+)$", out, flags=re.M))
    declared = _declared_symbols()
    assert declared, "no declarations found"
    missing = declared - exported
    assert not missing, "declared but not exported: %s" % sorted(missing)
    # the ctypes table covers the same set
    assert declared <= set(native.SYMBOLS), sorted(declared - set(native.SYMBOLS))
    L = native.lib()  # loads without a GPU
    assert L.ob_version().startswith(b"outbreaklab-b200")


def test_params_defaults_match_reference(native, oracle_lib):
    p = native.default_params()
    # model.js:1176-1180 with the app.js:1613 outbreak overrides (qc0 2e-3, dampZ 15 km, dampTau 150 s,
    # mcFloor 0.25, evap 0.22)
    ref = dict(cs=0.18, nu0=1.0, drag=1.0, z0=0.1, spongeTau=100, dampZ=15000, dampTau=150, autoc=1e-3, qc0=2e-3,
               freeze=1.0, noise=0.25, mc=1.0, vcap=110, evap=0.22, sortQ=5e-4, ciRate=0.5, nudgeTau=5400, lat=35,
               moistMix=0, mcFloor=0.25, scheme=0, evapT=0.3)
    for k, v in ref.items():
        assert getattr(p, k) == pytest.approx(v, rel=1e-6), k
    q = oracle_lib.default_params()
    for name, _ in native.ObParams._fields_:
        assert getattr(p, name) == getattr(q, name), name


def test_grid_pad_matches_reference(native):
    # gridPad (model.js:1122): Math.round(10 km / dx / 8) * 8 clamped to 8..64 (Math.round rounds halves up)
    import math
    for dx in [100, 250, 500, 1000, 1500, 2000, 4000]:
        want = int(min(max(math.floor(10000 / dx / 8 + 0.5) * 8, 8), 64))
        assert native.lib().ob_grid_pad(float(dx)) == want


def test_model_create_without_gpu_reports_device_error(native):
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("a GPU is present")
    except ImportError:
        pass
    g = native.ObGrid(16, 16, 8, 2000.0)
    h = C.c_void_p()
    rc = native.lib().ob_model_create(C.byref(g), C.byref(h))
    assert rc == native.OB_ERR_DEVICE
    assert b"CUDA" in native.lib().ob_last_error() or b"device" in native.lib().ob_last_error()


def test_invalid_grid_is_rejected(native):
    g = native.ObGrid(2, 16, 8, 2000.0)
    h = C.c_void_p()
    assert native.lib().ob_model_create(C.byref(g), C.byref(h)) == native.OB_ERR_INVALID
    assert b"bad grid" in native.lib().ob_last_error()


def test_perturb_theta_touches_interior_only():
    from outbreaklab_b200 import workloads as W
    case = W.case_small(nx=12, ny=10, nz=8)
    V = np.zeros((case.nz + 1) * (case.ny + 1) * (case.nx + 1) * 4, np.float32)
    P = W.perturb_theta(case, V).reshape(case.nz + 1, case.ny + 1, case.nx + 1, 4)
    assert np.all(P[..., :3] == 0)
    assert np.all(P[case.nz, :, :, 3] == 0) and np.all(P[:, case.ny, :, 3] == 0) and np.all(P[:, :, case.nx, 3] == 0)
    assert np.abs(P[:case.nz, :case.ny, :case.nx, 3]).max() > 1.0


def test_traffic_table_covers_the_bench_passes():
    """bench.py's roofline traffic comes from profiles/ncu_traffic.json: every pass with algorithmic bytes but LSF+CI
    (a few 2-D columns) has a positive entry with its captured cell count, and the solve's entry is the sum of its
    kernels' captures (transforms 622 MB, tridiagonals 73 + 89 MB, residual 181 MB per precision-5 solve)."""
    import json
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    with open(os.path.join(root, "profiles", "ncu_traffic.json")) as f:
        table = json.load(f)
    for name in ("NUT", "ADVV", "ADVQ", "PHYS", "DIV", "SOLVE", "PROJ+RAIN"):
        assert table[name]["bytes"] > 0 and table[name]["cells"] > 0, name
    assert abs(table["SOLVE"]["bytes"] - (622 + 73 + 89 + 181) * 1e6) < 1e6
