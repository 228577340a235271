"""The tornado-candidate search on the GPU (ob_model_tornado_candidates) against the oracle's restatement of
tornadoCandidates (app.js:1453-1466), on the maps of a growing Thompson supercell, at the scheme's threshold and at
lower ones that let many more lattice points through to the maximum and helicity / updraft tests; then the scheme and
the run loop on the GPU candidates."""

import numpy as np
import pytest

from outbreaklab_b200 import model as M, runloop as RL, tornado as TS, workloads as W

from oracle import tornado_oracle as TO

pytestmark = pytest.mark.gpu


def _key(c):
    return (c["i"], c["j"], c["z1"], c["uh"], c["w"])


def _oracle(maps, dx, zmin):
    return [(c[0], c[1], c[4], c[5], c[6]) for c in TO.candidates(maps["m0"], maps["m1"], dx, zmin)]


@pytest.fixture(scope="module")
def storm(native):
    c = W.StormCase("tor", 96, 88, 40, 1000.0, 6.0, 1, scheme=1, bubbles=[(40000.0, 36000.0)], bubble_rh=8000.0,
                    bubble_dth=3.0, seed=3)
    g, _ = M.setup_case(c)
    yield g
    g.destroy()


def test_candidates_match_oracle_as_the_storm_grows(storm):
    g = storm
    seen = 0
    for k in range(6):
        g.enc_step(6.0, 50)                     # 5 minutes of model time per readback
        maps = g.request_maps()
        for zmin in (TO.zeta_min(g.dx), 0.001, 0.0, -1.0):
            got = [_key(c) for c in TS.gpu_candidates(g, zmin)]
            assert got == _oracle(maps, g.dx, zmin), (k, zmin)
            seen += len(got)
        # a tiny output buffer: the call reports the full count and the host retries with room for all
        full = TS.gpu_candidates(g, -1.0)
        assert [_key(c) for c in TS.gpu_candidates(g, -1.0, cap=1)] == [_key(c) for c in full]
    assert seen > 0, "the storm never made a rotating updraft"
    assert g.nan_count == 0


def test_scheme_and_run_loop_on_gpu_candidates(native):
    c = W.StormCase("tor2", 96, 88, 40, 1000.0, 6.0, 1, scheme=1, bubbles=[(40000.0, 36000.0)], bubble_rh=8000.0,
                    seed=4)
    g, _ = M.setup_case(c)
    loop = RL.RunLoop(g, c.dt, 1200.0, replay_every=1e9, tornadoes={"stp": 2.0})
    res = loop.run()
    assert res["time"] >= 1200.0 and g.nan_count == 0
    s = loop.tor
    assert s.last_t > 0 and s.cands >= 0
    active, total = res["tornadoes"]
    assert 0 <= active <= total
    g.destroy()
