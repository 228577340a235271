"""Parity helpers shared by the tests.

Relative error of a field = max |a - ref| / max |ref| over the field (infinity norms), with ref the FP64 oracle.
The GPU passes when its error is within the FP32 restatement's own rounding envelope:
    err(GPU) <= max(TOL_ABS_REL, ENVELOPE * err(FP32 oracle))
TOL_ABS_REL = 1e-5 is the one-step relative tolerance; ENVELOPE = 2 allows the GPU's different (FMA-contracted,
differently ordered) fp32 summation to be up to twice as far from FP64 as the oracle's own fp32 arithmetic.
"""
import numpy as np

TOL_ABS_REL = 1e-5
ENVELOPE = 2.0

CHANNELS = {0: ("u", "v", "w", "theta"), 1: ("qv", "qc", "qi", "qr"), 2: ("qs", "qg", "Nr", "spare"), 3: ("nuh", "nuv"),
            4: ("phi",)}


def rel_errors(a, f32, f64, nch):
    a = np.asarray(a, np.float64).reshape(-1, nch)
    f32 = np.asarray(f32, np.float64).reshape(-1, nch)
    f64 = np.asarray(f64, np.float64).reshape(-1, nch)
    out = []
    for c in range(nch):
        scale = np.abs(f64[:, c]).max()
        if scale == 0:
            out.append((0.0 if np.abs(a[:, c]).max() == 0 else np.inf, 0.0 if np.abs(f32[:, c]).max() == 0 else np.inf))
            continue
        out.append((np.abs(a[:, c] - f64[:, c]).max() / scale, np.abs(f32[:, c] - f64[:, c]).max() / scale))
    return out


def check_field(name, a, f32, f64, nch, tol=TOL_ABS_REL, envelope=ENVELOPE):
    errs = rel_errors(a, f32, f64, nch)
    bad = []
    for c, (eg, ec) in enumerate(errs):
        if not np.isfinite(eg) or eg > max(tol, envelope * ec):
            bad.append("%s[%s]: GPU %.3e vs FP32 oracle %.3e" % (name, CHANNELS.get(name, [str(i) for i in range(nch)])[c]
                                                                  if isinstance(name, int) else c, eg, ec))
    return errs, bad
