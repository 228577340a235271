"""GPU pressure solve (solver.js) against the FP64 oracle: parity, FP64 residual, the near-singular lowest mode."""
import numpy as np
import pytest

from outbreaklab_b200 import model as M, workloads as W

pytestmark = pytest.mark.gpu


def _density(nz, dz):
    rc = 1.15 * np.exp(-(np.arange(nz) + 0.5) * dz / 9000.0)
    rw = np.concatenate([[rc[0] * 1.02], 0.5 * (rc[1:] + rc[:-1]), [rc[-1] * 0.94]])
    return rc.astype(np.float32), rw.astype(np.float32)


@pytest.mark.parametrize("shape", [(70, 52, 16), (96, 96, 40), (64, 80, 80)])
@pytest.mark.parametrize("precision", [0])
def test_poisson_parity_and_residual(oracle_lib, native, shape, precision):
    nx, ny, nz = shape
    dx, dz = 1000.0, 20000.0 / nz
    rc, rw = _density(nz, dz)
    rhs = W.gaussian_rhs(nx, ny, nz, dx, corr_len=5000.0, seed=nx).astype(np.float32)
    P = M.PoissonDirect(nx, ny, nz, dx, dz, precision)
    P.set_density(rc, rw)
    phi = P.solve(rhs)
    ref = oracle_lib.poisson_solve(rhs.astype(np.float64), dx, dz, rc.astype(np.float64), rw.astype(np.float64), 8)
    f32 = oracle_lib.poisson_solve(rhs, dx, dz, rc, rw, 4)
    scale = np.abs(ref).max()
    e_gpu = np.abs(phi - ref).max() / scale
    e_f32 = np.abs(f32 - ref).max() / scale
    assert e_gpu <= max(1e-5, 2 * e_f32), (e_gpu, e_f32)
    # FP64 residual of the GPU solution, relative to the right-hand side
    res = oracle_lib.poisson_apply(phi.astype(np.float64), dx, dz, rc.astype(np.float64), rw.astype(np.float64)) - rhs
    res_f32 = oracle_lib.poisson_apply(f32.astype(np.float64), dx, dz, rc.astype(np.float64), rw.astype(np.float64)) - rhs
    r_gpu = np.abs(res).max() / np.abs(rhs).max()
    r_f32 = np.abs(res_f32).max() / np.abs(rhs).max()
    assert r_gpu <= max(1e-5, 2 * r_f32), (r_gpu, r_f32)


def test_lowest_mode_solve(oracle_lib, native):
    """A right-hand side that is the (0, 0) sine mode in x, y with structure in z: the near-singular tridiagonal."""
    nx, ny, nz, dx, dz = 48, 40, 40, 1000.0, 500.0
    rc, rw = _density(nz, dz)
    i = np.arange(nx) + 0.5
    j = np.arange(ny) + 0.5
    mode = np.outer(np.sin(np.pi * j / ny), np.sin(np.pi * i / nx))
    rhs = (np.cos(np.pi * (np.arange(nz) + 0.5) / nz)[:, None, None] * mode[None]).astype(np.float32)
    P = M.PoissonDirect(nx, ny, nz, dx, dz, 0)
    P.set_density(rc, rw)
    phi = P.solve(rhs)
    ref = oracle_lib.poisson_solve(rhs.astype(np.float64), dx, dz, rc.astype(np.float64), rw.astype(np.float64), 8)
    assert np.abs(phi - ref).max() / np.abs(ref).max() < 1e-5
