"""GPU parity of the storm-model step (C ABI) against the CPU oracle (FP32 restatement) and its FP64 instantiation.

Tolerance (tests/_parity.py): per field, max|GPU - FP64| / max|FP64| <= max(1e-5, 2 x the FP32 oracle's own error)."""
import numpy as np
import pytest

from outbreaklab_b200 import _native as N, model as M, workloads as W

from _parity import check_field

pytestmark = pytest.mark.gpu

FIELDS = ((N.FIELD_V, 4), (N.FIELD_Q1, 4), (N.FIELD_Q2, 4), (N.FIELD_AUX, 2), (N.FIELD_PHI, 1))


def _setup(oracle_lib, case, blob=False):
    g, B = M.setup_case(case)
    f, _ = oracle_lib.setup_case(case, 4)
    d, _ = oracle_lib.setup_case(case, 8)
    if blob:
        q1, q2 = W.hydrometeor_blob(case, B, thompson=case.scheme == 1)
        for m in (f, d):
            m.set(oracle_lib.FIELD_Q1, q1)
            m.set(oracle_lib.FIELD_Q2, q2)
        g.set_field(N.FIELD_Q1, q1)
        g.set_field(N.FIELD_Q2, q2)
    return g, f, d


def _compare(g, f, d, fields=FIELDS, tol=1e-5, envelope=2.0):
    bad, report = [], {}
    for fld, ch in fields:
        errs, b = check_field(fld, g.get_field(fld), f.get(fld), d.get(fld, f64=True), ch, tol, envelope)
        report[fld] = errs
        bad += b
    return bad, report


CASES = {
    "small-lin": lambda: W.case_small(),
    "small-lin-blob": lambda: W.case_small(nx=40, ny=36, nz=40, dx=1000.0, dt=6.0),
    "small-thompson-blob": lambda: W.case_small(nx=40, ny=36, nz=40, dx=1000.0, dt=6.0, scheme=1),
    "c1": lambda: W.case_c1(),
}


@pytest.mark.parametrize("solver", [2, 3, 5, 0])
@pytest.mark.parametrize("name", list(CASES))
def test_one_step_parity(oracle_lib, native, name, solver):
    """Solvers 2 (bf16x3 solve refined in bf16x3), 3 (refined in plain bf16), 5 (a plain-bf16 solve refined in
    bf16x3) and 0 (fp32 transforms) all within the envelope."""
    case = CASES[name]()
    g, f, d = _setup(oracle_lib, case, blob="blob" in name)
    g.set_solver(solver)
    for m in (g, f, d):
        m.step(case.dt, 1)
    g.sync()
    bad, rep = _compare(g, f, d)
    assert not bad, "\n".join(bad)
    assert g.nan_count == 0


def test_one_step_unrefined_bf16x3_stated_error(oracle_lib, native):
    """Solver 1 (bf16x3 without refinement): its stated one-step error bound, 5e-4 of each field's maximum."""
    case = CASES["small-lin-blob"]()
    g, f, d = _setup(oracle_lib, case, blob=True)
    g.set_solver(1)
    for m in (g, f, d):
        m.step(case.dt, 1)
    bad, _ = _compare(g, f, d, tol=5e-4, envelope=0.0)
    assert not bad, "\n".join(bad)


@pytest.mark.parametrize("name", ["small-lin-blob", "small-thompson-blob"])
def test_five_step_parity(oracle_lib, native, name):
    case = CASES[name]()
    g, f, d = _setup(oracle_lib, case, blob=True)
    for m in (g, f, d):
        m.step(case.dt, 5)
    bad, _ = _compare(g, f, d, tol=1e-4, envelope=3.0)
    assert not bad, "\n".join(bad)


def test_maps_parity(oracle_lib, native):
    case = CASES["small-lin-blob"]()
    g, f, d = _setup(oracle_lib, case, blob=True)
    for m in (g, f, d):
        m.step(case.dt, 2)
    mg = g.request_maps()
    a = np.stack([mg["m0"], mg["m1"], mg["m2"], mg["m3"]]).reshape(-1, 4)
    bad = check_field("maps", a, f.maps(), d.maps(), 4, tol=1e-4, envelope=4.0)[1]
    assert not bad, bad


def test_budgets_and_rain(oracle_lib, native):
    case = CASES["small-lin-blob"]()
    g, f, d = _setup(oracle_lib, case, blob=True)
    for m in (g, f, d):
        m.step(case.dt, 3)
    bg = g.budgets()
    wd, md = d.budgets()
    assert abs(bg["mass"] - md) / md < 1e-12
    assert abs(bg["water"] - wd) / wd < 1e-6
    rd = d.rain().sum() * case.dx * case.dx
    assert rd > 0
    assert abs(bg["rain"] - rd) / rd < 1e-4
    rain_g = g.get_field(N.FIELD_RAIN)
    assert np.allclose(rain_g, d.rain(), rtol=1e-4, atol=1e-12 * d.rain().max())


def test_field_roundtrip(native):
    case = W.case_small(nx=20, ny=17, nz=12)
    g = M.RegionalModel().allocate(spec={"dx": case.dx, "n": [case.nx, case.ny, case.nz]})
    rng = np.random.default_rng(1)
    for fld in (N.FIELD_V, N.FIELD_Q1, N.FIELD_Q2, N.FIELD_AUX, N.FIELD_PHI, N.FIELD_RAIN):
        n, dt = g.field_shape(fld)
        a = rng.standard_normal(n).astype(dt)
        g.set_field(fld, a)
        assert np.array_equal(g.get_field(fld), a)
    with pytest.raises(N.ObError):
        g.set_field(N.FIELD_V, np.zeros(5, np.float32))


def test_c1_30_minutes(oracle_lib, native):
    """Check (b): after 30 simulated minutes of the 64 x 64 x 40 case, max w, max reflectivity and accumulated rain
    agree with the FP32 oracle within 2 %."""
    case = W.case_c1()
    g, B = M.setup_case(case)
    f, _ = oracle_lib.setup_case(case, 4)
    for m in (g, f):
        m.step(case.dt, 150)
    Vg = g.get_field(N.FIELD_V).reshape(case.nz + 1, case.ny + 1, case.nx + 1, 4)
    Vf = f.get(oracle_lib.FIELD_V).reshape(case.nz + 1, case.ny + 1, case.nx + 1, 4)
    mg = g.request_maps()["m0"][..., 0].max()
    mf = f.maps().reshape(4, case.ny, case.nx, 4)[0, ..., 0].max()
    rg, rf = g.budgets()["rain"], f.rain().sum() * case.dx ** 2
    assert Vf[..., 2].max() > 20 and mf > 50 and rf > 0
    assert abs(Vg[..., 2].max() - Vf[..., 2].max()) / Vf[..., 2].max() < 0.02
    assert abs(mg - mf) / mf < 0.02
    assert abs(rg - rf) / rf < 0.02
    assert g.nan_count == 0


def test_step_errors(native):
    g = M.RegionalModel().allocate(spec={"dx": 2000.0, "n": [16, 16, 8]})
    with pytest.raises(N.ObError) as e:
        g.enc_step(-1.0)
    assert e.value.code == N.OB_ERR_INVALID
    with pytest.raises(N.ObError):
        g.set_base_state(np.zeros(5, np.float32))
    with pytest.raises(N.ObError):
        g.set_surface(np.zeros(4, np.float32), {"ck": 1})


def test_graph_replay_equals_direct_launches(native):
    """25 steps (LSF due at steps 1, 11, 21; both parities): replayed CUDA graphs give the bytes of direct launches."""
    case = CASES["small-thompson-blob"]()
    g1, B = M.setup_case(case)
    g2, _ = M.setup_case(case)
    q1, q2 = W.hydrometeor_blob(case, B, thompson=True)
    for g in (g1, g2):
        g.set_field(N.FIELD_Q1, q1)
        g.set_field(N.FIELD_Q2, q2)
    N.check(N.lib().ob_model_set_graphs(g2.h, 0))
    for _ in range(25):
        g1.step(case.dt, 1)
        g2.step(case.dt, 1)
    g1.sync()
    g2.sync()
    assert g1.time == g2.time and g1.steps == 25
    for f in (N.FIELD_V, N.FIELD_Q1, N.FIELD_Q2, N.FIELD_PHI):
        assert np.array_equal(g1.get_field(f), g2.get_field(f)), f
    # the FP64 budget sums use atomics (their order varies run to run): equal to rounding
    b1, b2 = g1.budgets(), g2.budgets()
    for k in b1:
        assert np.isclose(b1[k], b2[k], rtol=1e-12, atol=0), k
