"""The bf16x3 tcgen05 transform kernel in isolation, and the precision-1 pressure solve."""
import numpy as np
import pytest

from outbreaklab_b200 import _native as N, model as M, workloads as W

pytestmark = pytest.mark.gpu


def _tc(A, B):
    Mr, K = A.shape
    P, Nn, K2 = B.shape
    assert K == K2
    C = np.empty((P, Mr, Nn), np.float32)
    A = np.ascontiguousarray(A, np.float32)
    B = np.ascontiguousarray(B, np.float32)
    N.check(N.lib().ob_dst_tc_selftest(Mr, Nn, K, P, N.fptr(A), N.fptr(B.reshape(-1)), N.fptr(C.reshape(-1))))
    return C


@pytest.mark.parametrize("shape", [(128, 128, 64, 1), (128, 128, 128, 2), (200, 136, 72, 3), (656, 96, 656, 2)])
def test_tc_transform_matches_fp64(native, shape):
    Mr, Nn, K, P = shape
    rng = np.random.default_rng(Mr + K)
    A = rng.standard_normal((Mr, K)).astype(np.float32)
    B = rng.standard_normal((P, Nn, K)).astype(np.float32)
    C = _tc(A, B)
    ref = np.einsum("mk,pnk->pmn", A.astype(np.float64), B.astype(np.float64))
    # bf16x3 keeps ~16 significant bits per product; the error of a K-term sum is ~2^-16 sqrt(K) of the sum's scale
    err = np.abs(C - ref).max() / np.abs(ref).max()
    assert err < 2e-4, err


def test_tc_transform_identity_exact(native):
    """With the identity as A (exact in bf16), C = hi(B) + lo(B) reproduces B to bf16x2 precision."""
    K = 64
    A = np.eye(128, K, dtype=np.float32)
    rng = np.random.default_rng(3)
    B = rng.standard_normal((1, 128, K)).astype(np.float32)
    C = _tc(A, B)[0]
    ref = B[0].T[:128]
    assert np.abs(C[:K] - B[0].T).max() <= 1e-5 * np.abs(B).max()


def _density(nz, dz):
    rc = 1.15 * np.exp(-(np.arange(nz) + 0.5) * dz / 9000.0)
    rw = np.concatenate([[rc[0] * 1.02], 0.5 * (rc[1:] + rc[:-1]), [rc[-1] * 0.94]])
    return rc.astype(np.float32), rw.astype(np.float32)


@pytest.mark.parametrize("precision", [1, 2, 3, 5])
@pytest.mark.parametrize("shape", [(96, 80, 40), (150, 130, 16), (256, 200, 80)])
def test_poisson_bf16x3_vs_fp64(oracle_lib, native, shape, precision):
    nx, ny, nz = shape
    dx, dz = 1000.0, 20000.0 / nz
    rc, rw = _density(nz, dz)
    rhs = W.gaussian_rhs(nx, ny, nz, dx, corr_len=5000.0, seed=nx).astype(np.float32)
    P = M.PoissonDirect(nx, ny, nz, dx, dz, precision)
    P.set_density(rc, rw)
    phi = P.solve(rhs)
    r64, w64 = rc.astype(np.float64), rw.astype(np.float64)
    ref = oracle_lib.poisson_solve(rhs.astype(np.float64), dx, dz, r64, w64, 8)
    f32 = oracle_lib.poisson_solve(rhs, dx, dz, rc, rw, 4)
    err = np.abs(phi - ref).max() / np.abs(ref).max()
    err32 = np.abs(f32 - ref).max() / np.abs(ref).max()
    res = np.abs(oracle_lib.poisson_apply(phi.astype(np.float64), dx, dz, r64, w64) - rhs).max() / np.abs(rhs).max()
    if precision == 1:
        assert err < 5e-4, err                     # stated error of the unrefined bf16x3 solve
    elif precision == 3:
        # the plain-bf16 correction: ~5e-4 (the first pass) x a few 1e-3 (bf16 of the correction)
        assert err <= max(1e-5, 2 * err32), (err, err32)
        assert res < 3e-3, res
    else:
        assert err <= max(1e-5, 2 * err32), (err, err32)   # refined: at least as accurate as the fp32 restatement
        assert res < 3e-4, res                     # one sweep cuts the ~1e-2 residual of a single pass ~100x


@pytest.mark.parametrize("nx,ny,nz,precision,bn", [(656, 656, 40, 2, 144), (656, 656, 40, 3, 112), (336, 320, 40, 1, 64),
                                                   (1024, 1024, 80, 2, 176), (48, 40, 16, 2, 32), (656, 656, 40, 5, 96),
                                                   (1024, 1024, 80, 5, 0)])
def test_pair_tiles_are_bit_identical(native, nx, ny, nz, precision, bn):
    """The transforms on SM pairs (tiles of 256 rows, tcgen05.mma.cta_group::2, each SM loading half of the matrix
    tile) and with other tile widths give the same bits as the automatic single-SM tiles: the same bf16 products
    accumulated over the same k-steps. Shapes cover automatic widths 224, 176 / 160, 256 and 48, narrowed last tiles
    (656 outputs in tiles of 144, 112 or 96), ring depths 3 to 8, the plain-bf16 passes (the correction of precision
    3, the first pass of precision 5) and a grid smaller than one pair tile."""
    import numpy as np
    from outbreaklab_b200 import model as M, workloads as W
    dz = 20000.0 / nz
    B, _ = W.base_state_for(W.StormCase("solve", 8, 8, nz, 1000.0, 6.0, 1))
    Bz = B.reshape(nz + 1, 8)
    rc, rw = Bz[:nz, 2].astype(np.float32).copy(), Bz[:, 3].astype(np.float32).copy()
    rhs = W.gaussian_rhs(nx, ny, nz, 1000.0, corr_len=5000.0, seed=5, dtype=np.float32)
    out = {}
    for pairs, width in ((False, 0), (True, 0), (True, bn), (False, bn)) if bn else ((False, 0), (True, 0)):
        P = M.PoissonDirect(nx, ny, nz, 1000.0, dz, precision)
        try:
            P.set_density(rc, rw)
            P.set_pair_tiles(pairs)
            P.set_tile_widths(width, width)
            out[pairs, width] = P.solve(rhs)
        finally:
            P.destroy()
    ref = out[False, 0]
    assert np.isfinite(ref).all()
    for key, phi in out.items():
        assert np.array_equal(phi.view(np.uint32), ref.view(np.uint32)), key


def test_pair_tiles_in_the_model_step(native):
    import numpy as np
    from outbreaklab_b200 import _native as N, model as M, workloads as W
    case = W.case_small(nx=120, ny=100, nz=40, dx=1000.0, dt=6.0)
    a, _ = M.setup_case(case)
    b, _ = M.setup_case(case)
    try:
        a.set_pair_tiles(False)   # single-SM tiles; b keeps the default, SM pairs
        for m in (a, b):
            m.enc_step(case.dt, 3)
            m.sync()
        for f in (N.FIELD_V, N.FIELD_Q1, N.FIELD_PHI):
            assert np.array_equal(a.get_field(f).view(np.uint32), b.get_field(f).view(np.uint32)), f
    finally:
        a.destroy()
        b.destroy()
