"""The allocation-free pressure solve (ob_poisson_solve_static) against the handle-based one (ob_poisson_solve).

Some callers cannot allocate GPU memory: a plugin bound to another runtime that owns the GPU's memory and hands out
only its own fixed budget, or a host that forbids device allocation after start-up. ob_poisson_solve_static serves
them from a fixed device array; this test calls it through the C ABI twice in a row (the array keeps the previous
call's contents) and checks each result against the allocating entry point within the tests' one-step tolerance
(1e-5 relative). It sits in its own file, collected last, and works both alone in a fresh process and after the other
tests.
"""
import ctypes as C

import numpy as np
import pytest

from outbreaklab_b200 import _native as N, model as M, workloads as W

pytestmark = pytest.mark.gpu

TOL = 1e-5


def _density(nz, dz):
    rc = 1.15 * np.exp(-(np.arange(nz) + 0.5) * dz / 9000.0)
    rw = np.concatenate([[rc[0] * 1.02], 0.5 * (rc[1:] + rc[:-1]), [rc[-1] * 0.94]])
    return rc.astype(np.float32), rw.astype(np.float32)


def _static_solve(torch, nx, ny, nz, dx, dz, rc, rw, rhs):
    dev = torch.device("cuda")
    t_rc = torch.from_numpy(rc).to(dev)
    t_rw = torch.from_numpy(rw).to(dev)
    t_rhs = torch.from_numpy(np.ascontiguousarray(rhs)).to(dev)
    t_phi = torch.full_like(t_rhs, float("nan"))
    stream = torch.cuda.current_stream()
    torch.cuda.synchronize()
    rc_ = N.lib().ob_poisson_solve_static(nx, ny, nz, float(dx), float(dz), C.c_void_p(t_rc.data_ptr()),
                                          C.c_void_p(t_rw.data_ptr()), C.c_void_p(t_rhs.data_ptr()),
                                          C.c_void_p(t_phi.data_ptr()), C.c_void_p(stream.cuda_stream))
    N.check(rc_)
    stream.synchronize()
    return t_phi.cpu().numpy()


def test_static_solve_matches_allocating_solve_twice(native):
    torch = pytest.importorskip("torch")
    assert torch.cuda.is_available()
    # two different problems back to back: the second call must not see the first one's leftovers
    for (nx, ny, nz, seed) in [(70, 52, 40, 1), (96, 64, 24, 2)]:
        dx, dz = 1000.0, 20000.0 / nz
        rc, rw = _density(nz, dz)
        rhs = W.gaussian_rhs(nx, ny, nz, dx, corr_len=5000.0, seed=seed).astype(np.float32)
        P = M.PoissonDirect(nx, ny, nz, dx, dz, 0)
        P.set_density(rc, rw)
        want = P.solve(rhs)
        P.destroy()
        got = _static_solve(torch, nx, ny, nz, dx, dz, rc, rw, rhs)
        assert np.isfinite(got).all()
        err = np.abs(got - want).max() / np.abs(want).max()
        assert err <= TOL, (nx, ny, nz, err)


def test_static_solve_rejects_oversize(native):
    rc = C.c_void_p(1)
    n = N.OB_STATIC_POISSON_MAX_SIDE + 1
    assert N.lib().ob_poisson_solve_static(n, 8, 8, 1000.0, 500.0, rc, rc, rc, rc, None) == N.OB_ERR_INVALID
    assert b"exceeds the static limits" in N.lib().ob_last_error()
    assert N.lib().ob_poisson_solve_static(256, 256, 40, 1000.0, 500.0, rc, rc, rc, rc, None) == N.OB_ERR_INVALID
