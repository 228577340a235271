"""The run loop on the GPU model: 12 minutes of a small Thompson storm with automatic storm starts, a virtual radar
whose finished volumes are written as Archive II files, replay frames every minute and adaptive batches."""
import bz2
import os
import struct

import pytest

from outbreaklab_b200 import model as M, radar as RD, runloop as RL

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
