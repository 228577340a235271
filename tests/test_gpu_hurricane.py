"""Hurricane mode on the GPU against the oracle (FP32 restatement and FP64), through the C ABI: the initial vortex,
one step (sea fluxes, drag, boundary layer, radiative relaxation, far-field hold, thermals, settling ice, maritime
graupel, midpoint trajectories), five steps (the trajectory-averaged pressure force from step 2, the 2-dx filter at
step 4), the maps, graphs against direct launches, and back to outbreak mode."""
import numpy as np
import pytest

from outbreaklab_b200 import _native as N, hurricane as H

import _hurricane_case as HC
from _parity import check_field

pytestmark = pytest.mark.gpu

FIELDS = ((N.FIELD_V, 4), (N.FIELD_Q1, 4), (N.FIELD_Q2, 4), (N.FIELD_AUX, 2), (N.FIELD_PHI, 1))


def _setup():
    c, surf, vort = HC.case()
    g, B, h, tab, info = H.setup(c, surf, vort, lat=HC.LAT)
    f, _, _, _ = HC.oracle_setup(c, surf, vort, 4)
    d, _, _, _ = HC.oracle_setup(c, surf, vort, 8)
    return c, g, f, d


def _compare(g, f, d, fields=FIELDS, tol=1e-5, envelope=2.0):
    bad = []
    for fld, ch in fields:
        bad += check_field(fld, g.get_field(fld), f.get(fld), d.get(fld, f64=True), ch, tol, envelope)[1]
    return bad


def test_initial_vortex_parity(native):
    c, g, f, d = _setup()
    bad = _compare(g, f, d, fields=((N.FIELD_V, 4), (N.FIELD_Q1, 4)))
    assert not bad, "\n".join(bad)
    V = g.get_field(N.FIELD_V).reshape(c.nz + 1, c.ny + 1, c.nx + 1, 4)
    assert 15.0 < np.abs(V[0, :, :, :2]).max() < 30.0
    g.destroy()


def test_one_step_parity(native):
    c, g, f, d = _setup()
    for m in (g, f, d):
        m.step(c.dt, 1)
    g.sync()
    bad = _compare(g, f, d)
    assert not bad, "\n".join(bad)
    assert g.nan_count == 0
    g.destroy()


def test_five_step_parity_with_pressure_carry_and_filter(native):
    c, g, f, d = _setup()
    for m in (g, f, d):
        m.step(c.dt, 5)
    g.sync()
    bad = _compare(g, f, d, tol=1e-4, envelope=3.0)
    assert not bad, "\n".join(bad)
    mg = g.request_maps()
    a = np.stack([mg["m0"], mg["m1"], mg["m2"], mg["m3"]]).reshape(-1, 4)
    bad = check_field("maps", a, f.maps(), d.maps(), 4, tol=1e-4, envelope=4.0)[1]
    assert not bad, bad
    g.destroy()


def test_graphs_equal_direct_launches(native):
    c, g1, _, _ = _setup()
    c, g2, _, _ = _setup()
    N.check(N.lib().ob_model_set_graphs(g2.h, 0))
    for _ in range(10):       # filter steps 4 and 8, both parities
        g1.step(c.dt, 1)
        g2.step(c.dt, 1)
    g1.sync()
    g2.sync()
    for fld in (N.FIELD_V, N.FIELD_Q1, N.FIELD_Q2, N.FIELD_PHI):
        assert np.array_equal(g1.get_field(fld), g2.get_field(fld)), fld
    g1.destroy()
    g2.destroy()


def test_back_to_outbreak_mode(native):
    c, g, _, _ = _setup()
    g.step(c.dt, 2)
    g.set_surface(None, None)
    g.set_vortex(None)
    g.step(c.dt, 3)
    g.sync()
    assert g.nan_count == 0
    with pytest.raises(N.ObError):
        g.set_hurricane(H.default_hurricane())   # not in hurricane mode any more
    g.destroy()
