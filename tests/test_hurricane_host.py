"""Hurricane mode on CPU: setVortex's table (model.js:1318-1365) and the oracle's hurricane branches (FP32 against
FP64 over the steps that bring in the trajectory-averaged pressure force and the 2-dx filter)."""
import math

import numpy as np
import pytest

from outbreaklab_b200 import hurricane as H, sounding as snd_mod, workloads as W

from oracle import oracle as O


from _hurricane_case import base_state, oracle_setup


def test_vortex_table_balance():
    case, surf, vort = H.tropical_case(nx=64, ny=64)
    B, _ = base_state(case)
    lat = 20.0
    tab, info = H.vortex_table(case.nz, case.dz, case.dx, lat, B, **vort)
    nr, dr = info["nr"], info["dr"]
    assert tab.shape == (case.nz, nr, 4) and dr == max(500.0, case.dx / 2)
    v0 = tab[0, :, 0].astype(np.float64)
    r = np.arange(nr) * dr
    # the wind peaks near the radius of maximum wind at about vmax (the taper starts at r0 / 2)
    i_max = int(np.argmax(v0))
    assert abs(r[i_max] - vort["rmw"]) <= 2 * dr and 0.9 * vort["vmax"] <= v0.max() <= 1.0001 * vort["vmax"]
    # inertially stable: the absolute angular momentum r v + f r^2 / 2 never decreases outward
    f = 2 * 7.292e-5 * math.sin(lat * math.pi / 180)
    M = r * v0 + 0.5 * f * r * r
    assert np.all(np.diff(M) >= -1e-6 * M.max())
    # the wind weakens with height to nothing at the top of the vortex; a warm core above the lowest kilometres
    z = (np.arange(case.nz) + 0.5) * case.dz
    assert tab[z >= vort["ztop"], :, 0].max() == 0.0
    assert info["warm"] > 0.5 and info["pc"] < 0
    assert np.all(tab[..., 2:] == 0)


def test_vortex_southern_hemisphere_turns_the_other_way():
    case, surf, vort = H.tropical_case(nx=48, ny=48)
    B, _ = base_state(case)
    tn, _ = H.vortex_table(case.nz, case.dz, case.dx, 20.0, B, **vort)
    ts, _ = H.vortex_table(case.nz, case.dz, case.dx, -20.0, B, **vort)
    assert tn[0, :, 0].max() > 0 and ts[0, :, 0].min() < 0
    assert np.allclose(tn[0, :, 0], -ts[0, :, 0], atol=1e-5)


@pytest.fixture(scope="module")
def hurricane_runs():
    import _hurricane_case as HC
    case, surf, vort = HC.case()
    f, B, tab, info = oracle_setup(case, surf, vort, 4)
    d, _, _, _ = oracle_setup(case, surf, vort, 8)
    out = {"case": case, "f": f, "d": d, "info": info}
    yield out


def test_oracle_hurricane_fp32_tracks_fp64(hurricane_runs):
    r = hurricane_runs
    case, f, d = r["case"], r["f"], r["d"]
    # step 0: no pressure carried yet; step 1: the carried pressure starts; step 3: the first 2-dx filter
    for s in range(5):
        f.step(case.dt, 1)
        d.step(case.dt, 1)
    for fld, nch in ((O.FIELD_V, 4), (O.FIELD_Q1, 4), (O.FIELD_Q2, 4), (O.FIELD_PHI, 1)):
        a = f.get(fld).astype(np.float64).reshape(-1, nch)
        b = d.get(fld, f64=True).reshape(-1, nch)
        assert np.isfinite(a).all() and np.isfinite(b).all()
        for c in range(nch):
            scale = np.abs(b[:, c]).max()
            if scale > 0:
                assert np.abs(a[:, c] - b[:, c]).max() <= 1e-3 * scale, (fld, c)
    V = d.get(O.FIELD_V, f64=True).reshape(case.nz + 1, case.ny + 1, case.nx + 1, 4)
    # the vortex spins: tangential winds of the order of vmax near the surface, cyclonic (positive vorticity)
    assert 15.0 < np.abs(V[0, :, :, 0]).max() < 40.0
    u, v = V[0, :-1, :-1, 0], V[0, :-1, :-1, 1]
    zeta = (v[:, 1:] - v[:, :-1])[:-1] - (u[1:, :] - u[:-1, :])[:, :-1]
    assert zeta.sum() > 0


def test_outbreak_mode_unchanged_by_clearing_the_surface():
    case = W.case_small()
    a, _ = O.setup_case(case, 4)
    b, _ = O.setup_case(case, 4)
    b.set_surface(None, None)
    b.set_vortex(None, 0, 0, 0, 1, 1, 0)
    for m in (a, b):
        m.step(case.dt, 3)
    for fld in (O.FIELD_V, O.FIELD_Q1, O.FIELD_Q2, O.FIELD_PHI):
        assert np.array_equal(a.get(fld), b.get(fld))
