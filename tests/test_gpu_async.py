"""Host hand-offs that do not wait for the model's stream: the storm-start list's upload (setCI, model.js:1383) and
requested budgets (the requestMaps pattern, model.js:1478-1494)."""
import numpy as np
import pytest

from outbreaklab_b200 import _native as N, model as M, workloads as W

pytestmark = pytest.mark.gpu


def _events(case, wt):
    return [{"x": 0.5 * case.nx * case.dx, "y": 0.5 * case.ny * case.dx, "zc": 1500.0, "rh": 6000.0, "rz": 1500.0,
             "wt": wt, "t0": 0.0, "t1": 1e6, "vx": 0.0, "vy": 0.0, "seed": 1.0, "ramp": 60.0}]


def test_requested_budgets_equal_the_blocking_call(native):
    case = W.case_small(nx=40, ny=32, nz=16, dx=2000.0, dt=12.0)
    a, _ = M.setup_case(case)
    try:
        tickets, blocking = [], []
        for _ in range(3):
            a.enc_step(case.dt)
            tickets.append(a.request_budgets())
            blocking.append(a.budgets())
        assert tickets == sorted(tickets) and len(set(tickets)) == 3
        for t, b in zip(tickets, blocking):
            assert a.read_budgets(t) == b          # the same reductions after the same steps, bit for bit
        for _ in range(4):                          # four newer requests reuse every slot
            a.request_budgets()
        with pytest.raises(N.ObError):
            a.read_budgets(tickets[0])
        with pytest.raises(N.ObError):
            a.read_budgets(10 ** 6)                 # never requested
    finally:
        a.destroy()


def test_storm_start_list_is_copied_at_the_call(native):
    """The caller may change its array right after ob_model_set_ci: the upload queued on the stream sends the list
    as it was at the call, so the steps equal those with the list never changed (and differ from those without the
    tower's push)."""
    case = W.case_small(nx=40, ny=32, nz=16, dx=2000.0, dt=12.0)
    ms = [M.setup_case(case)[0] for _ in range(3)]
    ref, a, z = ms
    try:
        f, act = M.pack_ci(_events(case, 8.0))
        f0, _ = M.pack_ci(_events(case, 0.0))
        N.check(N.lib().ob_model_set_ci(ref.h, N.fptr(f), len(act)))
        N.check(N.lib().ob_model_set_ci(z.h, N.fptr(f0), len(act)))
        buf = f.copy()
        N.check(N.lib().ob_model_set_ci(a.h, N.fptr(buf), len(act)))
        buf[5] = 0.0                                # the tower's strength, zeroed right after the call
        for m in ms:
            m.enc_step(case.dt, 3)
        for fld in (N.FIELD_V, N.FIELD_Q1):
            assert np.array_equal(a.get_field(fld).view(np.uint32), ref.get_field(fld).view(np.uint32)), fld
        assert not np.array_equal(z.get_field(N.FIELD_V), ref.get_field(N.FIELD_V))
    finally:
        for m in ms:
            m.destroy()
