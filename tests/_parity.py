"""Parity helpers shared by the tests.

Relative error of a field = max |a - ref| / max |ref| over the field (infinity norms), with ref the FP64 oracle.
The GPU passes when its error is within the FP32 restatement's own rounding envelope:
    err(GPU) <= max(TOL_ABS_REL, ENVELOPE * err(FP32 oracle))
TOL_ABS_REL = 1e-5 is the one-step relative tolerance; ENVELOPE = 2 allows the GPU's different (FMA-contracted,
differently ordered) fp32 summation to be up to twice as far from FP64 as the oracle's own fp32 arithmetic.
Each check records (test, field, channel, GPU error, FP32 oracle error, the bar applied) in RECORDS.
"""
import numpy as np

TOL_ABS_REL = 1e-5
ENVELOPE = 2.0

CHANNELS = {0: ("u", "v", "w", "theta"), 1: ("qv", "qc", "qi", "qr"), 2: ("qs", "qg", "Nr", "spare"), 3: ("nuh", "nuv"),
            4: ("phi",), 6: ("lsfA.dT", "lsfA.depth", "lsfA.dq", "lsfA.qdepth"),
            7: ("lsfB.du", "lsfB.dv", "lsfB.wdepth", "lsfB.nudge"), 8: ("ci.push", "ci.w", "ci.zc", "ci.rz"),
            9: ("phT",)}
FIELD_NAMES = {0: "V", 1: "Q1", 2: "Q2", 3: "AUX", 4: "PHI", 6: "LSF_A", 7: "LSF_B", 8: "CI_MAP", 9: "PHT"}

# Every check_field call is recorded here with the test that made it (tests/conftest.py sets CURRENT and, when the
# environment names a file in OB_PARITY_REPORT, writes the records there as JSON lines at the end of the session).
RECORDS = []
CURRENT = [""]


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
        ch = CHANNELS.get(name, [str(i) for i in range(nch)])[c] if isinstance(name, int) else str(c)
        bar = max(tol, envelope * ec)
        RECORDS.append({"test": CURRENT[0], "field": FIELD_NAMES.get(name, str(name)), "channel": ch,
                        "gpu": float(eg), "fp32": float(ec), "tol": tol, "envelope": envelope, "bar": float(bar)})
        if not np.isfinite(eg) or eg > bar:
            bad.append("%s[%s]: GPU %.3e vs FP32 oracle %.3e" % (name, ch, eg, ec))
    return errs, bad
