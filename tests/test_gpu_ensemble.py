"""GPU tests of the batched ensemble (C5): members stepped concurrently on their own streams give exactly the fields
each member gives stepped alone, and the ensemble runner reports finite throughput and latency."""
import numpy as np
import pytest

from outbreaklab_b200 import _native as N, ensemble as E, model as M, workloads as W

pytestmark = pytest.mark.gpu


def _small_members():
    cs = E.draw_members(3, 7, steps=3)
    for c, (nx, ny) in zip(cs, ((48, 40), (64, 56), (40, 72))):
        c.nx, c.ny = nx, ny
        c.bubbles = [(nx * c.dx / 2, ny * c.dx / 2)]
        c.bubble_rh = min(10000.0, 0.2 * min(nx, ny) * c.dx)
    return cs


def test_concurrent_members_match_members_alone(native):
    cs = _small_members()
    together = [M.setup_case(c)[0] for c in cs]
    for _ in range(3):
        for m, c in zip(together, cs):
            N.check(N.lib().ob_model_step(m.h, c.dt, 1))   # queued, no waiting between members
    for m in together:
        m.sync()
    for m, c in zip(together, cs):
        alone, _ = M.setup_case(c)
        alone.step(c.dt, 3)
        alone.sync()
        for f in (N.FIELD_V, N.FIELD_Q1, N.FIELD_Q2):
            assert np.array_equal(m.get_field(f), alone.get_field(f)), (c.name, f)
        alone.destroy()
    for m in together:
        m.destroy()


def test_ensemble_runner_metrics(native):
    cs = _small_members()
    r = E.run(cs, steps=4, warmup=1)
    g = E.gather(r)
    assert r["members"] == 3 and r["nan_guard_count"] == 0
    assert np.isfinite(g["cell_steps_per_s"]) and g["cell_steps_per_s"] > 0
    assert 0 < g["latency_ms_p50"] <= g["latency_ms_p99"]
