"""The run loop on the GPU model: 12 minutes of a small Thompson storm with automatic storm starts, a virtual radar
whose finished volumes are written as Archive II files, replay frames every minute and adaptive batches."""
import bz2
import os
import struct

import pytest

from outbreaklab_b200 import _native as N, model as M, radar as RD, runloop as RL

import _radar_case as RC

pytestmark = pytest.mark.gpu


def test_run_loop_with_radar_and_storm_starts(native, tmp_path):
    c = RC.case(scheme=1)
    g, B = M.setup_case(c)
    geo = RC.geo_for(c)
    sim = RD.RadarSim(g, geo, seed=3)
    sim.add_radar(RC.site_for(c, geo))
    loop = RL.RunLoop(g, c.dt, 720.0, radar=sim, ci={"warmRate": 3000.0, "start": 0.0, "rh": 4000.0}, replay_every=60.0,
                      out_dir=str(tmp_path), run="t", epoch0_ms=1714586400000)
    res = loop.run()
    assert res["time"] >= 720.0 and res["steps"] == 120
    assert res["frames"] == 13                      # t = 6 s, then every minute to 12 min
    assert 1 <= res["steps_per_batch"] <= 40
    assert res["events"] > 0 and any("storm start" in s for s in res["log"])
    assert len(res["volumes"]) >= 1
    v = res["volumes"][0]
    data = open(v["path"], "rb").read()
    assert data[:12] == b"AR2V0006.001" and len(data) == v["size"] and os.path.basename(v["path"]).startswith("KTST")
    n = struct.unpack(">i", data[24:28])[0]
    meta = bz2.decompress(data[28:28 + n])
    assert len(meta) == 134 * 2432
    assert g.nan_count == 0
    sim.destroy()


def test_run_loop_with_fronts_starts_storms_along_them(native):
    """The reference's example fronts over their triple point: the run loop's scheduler starts storms along the
    boundaries (on their warm side) as well as in the warm sector, and the model runs the nudged forcing with them."""
    from outbreaklab_b200 import boundaries as BND, workloads as W
    case = W.case_fronts(nx=96, ny=88, nz=40)
    bounds, _ = W.fronts_setup(case)
    for mb in bounds:
        mb["b"] = dict(mb["b"], rate=400.0)        # a start on each boundary about every minute
    g, _ = M.setup_case(case, bounds=bounds)
    loop = RL.RunLoop(g, case.dt, 300.0, ci={"warmRate": 300.0, "start": 0.0, "rh": 6000.0}, replay_every=60.0,
                      bounds=bounds)
    res = loop.run()
    labels = [s for s in res["log"] if "storm start" in s]
    kinds = {BND.BND_TYPES[k]["label"].lower() for k in ("cold", "warm", "dry")}
    assert any(any(k in s for k in kinds) for s in labels), labels
    assert res["events"] > 0 and g.nan_count == 0
    A = g.get_field(N.FIELD_LSF_A).reshape(case.ny, case.nx, 4)
    assert A[..., 0].min() < -3.0 and A[..., 0].max() > 1.0


class _Recorder:
    """The GPU model as the run loop sees it, recording every storm-start list the scheduler sends (setCI) with the
    number of steps taken before it, packed as the model packs it."""

    def __init__(self, model):
        self._m = model
        self.calls = []

    def __getattr__(self, name):
        return getattr(self._m, name)

    def set_ci(self, events):
        f, act = M.pack_ci(events, self._m.time)
        self.calls.append((self._m.steps, f.copy(), len(act)))
        self._m.set_ci(events)


@pytest.mark.parametrize("scheme", [0, 1])
def test_run_loop_storm_starts_match_the_oracle(oracle_lib, native, scheme):
    """The run loop's scheduler (warm sector and along the reference's example fronts) drives the GPU model for 132 s
    (11 steps through the LSF pass at t = 60 s, scheduler windows at t = 0, 60 and 120 s); every storm-start list it
    sent, at the step it was sent, is replayed on the FP32 oracle and its FP64 instantiation, and the state is held
    to the five-step bar: max(1e-4, 3 x the FP32 oracle's error) per field and channel against FP64."""
    from outbreaklab_b200 import workloads as W
    from _parity import check_field
    case = W.case_fronts(scheme=scheme)
    bounds, _ = W.fronts_setup(case)
    for mb in bounds:
        mb["b"] = dict(mb["b"], rate=400.0)
    g, _ = M.setup_case(case, bounds=bounds)
    rec = _Recorder(g)
    loop = RL.RunLoop(rec, case.dt, 132.0, ci={"warmRate": 3000.0, "start": 0.0, "rh": 6000.0}, replay_every=60.0,
                      bounds=bounds)
    res = loop.run()
    g.sync()
    assert res["steps"] == 11 and res["events"] > 0 and rec.calls, res
    f, _ = oracle_lib.setup_case(case, 4, bounds=bounds)
    d, _ = oracle_lib.setup_case(case, 8, bounds=bounds)
    calls = list(rec.calls)
    for step in range(res["steps"]):
        while calls and calls[0][0] == step:
            _, packed, n = calls.pop(0)
            for o in (f, d):
                o.set_ci(packed, n)
        for o in (f, d):
            o.step(case.dt, 1)
    assert not calls
    assert abs(d.time - g.time) < 1e-9
    C = d.get(N.FIELD_CI_MAP, f64=True).reshape(-1, 4)
    assert ((C[:, 0] * C[:, 1]) > 0.5).sum() > 10, "no storm-start push on the oracle side"
    bad = []
    for fld, ch in ((N.FIELD_V, 4), (N.FIELD_Q1, 4), (N.FIELD_Q2, 4), (N.FIELD_PHI, 1)):
        errs, b = check_field(fld, g.get_field(fld), f.get(fld), d.get(fld, f64=True), ch, 1e-4, 3.0)
        print(fld, ["%.2e/%.2e" % e for e in errs])
        bad += b
    bad += check_field(N.FIELD_CI_MAP, g.get_field(N.FIELD_CI_MAP), f.get(N.FIELD_CI_MAP),
                       d.get(N.FIELD_CI_MAP, f64=True), 4, 1e-5, 2.0)[1]
    assert not bad, "\n".join(bad)
    assert g.nan_count == 0
