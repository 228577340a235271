"""The clear-air skips of the scalar advection and of the physics pass (blocks whose reach holds no hydrometeor and no
nonzero spare channel neither read nor rewrite those channels) against the oracle, which restates the reference's
step without any skip: a storm case runs dry, then set_field writes hydrometeors and a nonzero spare fourth Q2
channel into air that held none (the brick flags are rebuilt from the new state), and five more steps carry them
through bricks that turn from dry to wet; every field, the spare channel included, stays within the five-step parity
envelope of the step tests."""
import numpy as np
import pytest

from outbreaklab_b200 import _native as N, model as M, workloads as W

from _parity import check_field

pytestmark = pytest.mark.gpu

FIELDS = ((N.FIELD_V, 4), (N.FIELD_Q1, 4), (N.FIELD_Q2, 4), (N.FIELD_AUX, 2), (N.FIELD_PHI, 1))


def _blob(nz, ny, nx, cz, cy, cx, r, amp):
    z, y, x = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    b = amp * np.exp(-(((x - cx) / r) ** 2 + ((y - cy) / r) ** 2 + ((z - cz) / (r / 2)) ** 2))
    return np.where(b > 1e-3 * amp, b, 0.0).astype(np.float32)


@pytest.mark.parametrize("scheme", [0, 1])
def test_dry_then_wet_mid_run(oracle_lib, native, scheme):
    case = W.case_small(nx=48, ny=40, nz=40, dx=1000.0, dt=6.0, scheme=scheme)
    g, _ = M.setup_case(case)
    f, _ = oracle_lib.setup_case(case, 4)
    d, _ = oracle_lib.setup_case(case, 8)
    for m in (g, f, d):
        m.step(case.dt, 3)
    g.sync()
    nz, ny, nx = case.nz, case.ny, case.nx
    q1 = f.get(oracle_lib.FIELD_Q1).reshape(nz, ny, nx, 4).copy()
    q2 = f.get(oracle_lib.FIELD_Q2).reshape(nz, ny, nx, 4).copy()
    assert not q1[..., 1:].any() and not q2[..., :2].any(), "the case condensed before the injection"
    q1[..., 1] += _blob(nz, ny, nx, 8, 10, 12, 4.0, 1.5e-3)    # cloud water
    q1[..., 3] += _blob(nz, ny, nx, 6, 12, 14, 3.0, 8e-4)     # rain, falling into the dry air below it
    q2[..., 0] += _blob(nz, ny, nx, 14, 28, 34, 3.0, 5e-4)    # snow
    q2[..., 3] += _blob(nz, ny, nx, 5, 26, 30, 4.0, 1e-3)     # the spare channel, which no scheme sets
    if scheme == 1:
        q2[..., 2] = np.where(q1[..., 3] > 0, q1[..., 3] * 3.183e8, 0.0).astype(np.float32)   # rain number
    for m in (f, d):
        m.set(oracle_lib.FIELD_Q1, q1)
        m.set(oracle_lib.FIELD_Q2, q2)
    g.set_field(N.FIELD_Q1, q1)
    g.set_field(N.FIELD_Q2, q2)
    for m in (g, f, d):
        m.step(case.dt, 5)
    g.sync()
    bad = []
    for fld, ch in FIELDS:
        _, b = check_field(fld, g.get_field(fld), f.get(fld), d.get(fld, f64=True), ch, 1e-4, 3.0)
        bad += b
    assert not bad, "\n".join(bad)
    spare = g.get_field(N.FIELD_Q2).reshape(-1, 4)[:, 3]
    assert spare.max() > 0 and g.nan_count == 0
    g.destroy()
