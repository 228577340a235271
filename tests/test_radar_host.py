"""CPU tests of the radar path: the oracle's gate restatement pinned by known answers, the host layout and
scheduling of RadarSim (radar.js:288-367), and the Level II code table shared with the reference's l2writer.py."""
import json
import math
import os

import numpy as np
import pytest

from outbreaklab_b200 import radar as RD

import _radar_case as RC

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def test_level2_table_matches_reference_writer():
    """radar.js:21 quantises with the scale/offset l2writer.py:19-27 decodes with (fixture made from l2writer.py)."""
    g = json.load(open(os.path.join(GOLDEN, "l2writer_moments.json")))
    assert g["GATE_FIRST_M"] == RD.GATE0 and g["GATE_SIZE_M"] == RD.GATEDR
    for name, (sc, ofs) in RD.L2_SCALE.items():
        assert g["MOMENTS"][name]["scale"] == pytest.approx(sc, rel=0, abs=0)
        assert g["MOMENTS"][name]["offset"] == ofs
    assert g["MOMENT_ORDER"] == ["REF", "VEL", "SW", "ZDR", "PHI", "RHO"]


def test_code_rounds_half_to_even_and_clamps(oracle_lib):
    """WGSL round() is half-to-even; codes clamp to [2, 255] (radar.js:140)."""
    v = np.array([10.0, 10.25, 10.75, 11.25, -40.0, 200.0, 0.0], np.float32)
    assert list(oracle_lib.radar_code(v, 2, 66)) == [86, 86, 88, 88, 2, 255, 66]
    # decoding with l2writer's table recovers the value to half a step
    sc, ofs = RD.L2_SCALE["ZDR"]
    z = np.linspace(-7.9, 7.9, 101, dtype=np.float32)
    dec = (oracle_lib.radar_code(z, sc, ofs).astype(np.float64) - ofs) / sc
    assert np.abs(dec - z).max() <= 0.5 / sc + 1e-6


def test_phi_accumulates_in_gate_order(oracle_lib):
    """PhiDP = offset + sum 2 KDP dr (km), mod 360, empty gates (KDP < 0) coded 0 and skipped (radar.js:251-264)."""
    U = np.zeros(44, np.float32)
    U[15] = 250.0   # gate spacing
    U[19] = 25.0    # system PhiDP
    kdp = np.full((2, 8), 0.5, np.float32)
    kdp[1, 3] = -1.0
    codes = oracle_lib.radar_phi(U, kdp)
    acc, exp0 = np.float32(25.0), []
    for _ in range(8):
        acc = np.float32(acc + np.float32(np.float32(np.float32(2.0) * np.float32(0.5)) * np.float32(250.0)) * np.float32(0.001))
        exp0.append(int(min(max(round(float(np.float32(np.float32(acc * np.float32(253)) / np.float32(360)) + 2)), 2), 255)))
    assert list(codes[0]) == exp0
    assert codes[1, 3] == 0 and codes[1, 4] == exp0[3]


def test_layout_and_timing_vcp212():
    """addRadar's volume layout: 14 cuts, 3 split pairs at 720 radials, moments back to back; cut times sum to
    the VCP's duration (radar.js:293-318)."""
    ngr, ngd, cuts, nbytes = RD.radar_layout(640e3, 640e3, -50e3, 320e3, RD.VCPS[212])
    assert len(cuts) == 17 and ngr % 4 == 0 and ngd == min(ngr, RD.MAX_DOP_GATES)
    far = math.hypot(640e3 + 50e3, 320e3)
    assert ngr == min(RD.MAX_REF_GATES, max(64, math.ceil(math.ceil((min(460e3, far + 10e3) - 2125) / 250) / 4) * 4))
    off = 0
    for c in cuts:
        for mo in c["mom"]:
            assert mo["off"] == off
            off += c["nrad"] * mo["ngates"]
    assert off == nbytes
    assert cuts[-1]["t0"] + cuts[-1]["dur"] == pytest.approx(270.0)
    assert [c["kind"] for c in cuts[:6]] == ["surv", "dop"] * 3


def test_geo_round_trip():
    g = RD.Geo(35.9, -97.2, 200e3, 150e3, 350.0)
    for x, y in [(0, 0), (-20e3, -15e3), (180e3, 140e3)]:
        lat, lon = g.from_model(x, y)
        x2, y2 = g.to_model(lat, lon)
        assert abs(x2 - x) < 1e-3 and abs(y2 - y) < 1e-3


def test_oracle_cut_sees_the_storm(oracle_lib):
    """On the hydrometeor blob the oracle's cut has echoes inside the domain and none beyond it, velocities within
    the Nyquist interval, and the FP32 and FP64 restatements agree on the codes of almost every gate."""
    from outbreaklab_b200 import workloads as W
    c = RC.case()
    geo = RC.geo_for(c)
    site = RC.site_for(c, geo)
    f, B = oracle_lib.setup_case(c, 4)
    d, _ = oracle_lib.setup_case(c, 8)
    q1, q2 = W.hydrometeor_blob(c, B)
    for m in (f, d):
        m.set(oracle_lib.FIELD_Q1, q1)
        m.set(oracle_lib.FIELD_Q2, q2)
    plan, ngr, ngd, nbytes = RC.cut_plan(c, geo, site, B, cut_indices=(8,))
    cut, U = plan[0]
    ua = U.as_array()
    of, kf, mf = f.radar_cut(ua, None, nbytes, ngd)
    od, kd, md = d.radar_cut(ua, None, nbytes, ngd)
    ref = next(o for o in cut["mom"] if o["name"] == "REF")
    rf = of[ref["off"]:ref["off"] + cut["nrad"] * ngr]
    rd = od[ref["off"]:ref["off"] + cut["nrad"] * ngr]
    assert (rf > 0).sum() > 1000, "no echo"
    assert (rf == rd).mean() > 0.995
    vel = mf[:, :ngd, 1]
    ok = np.isfinite(vel)
    assert ok.any() and np.abs(vel[ok]).max() <= U.nyq[0] + 1e-3
