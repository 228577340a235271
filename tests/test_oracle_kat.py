"""Known-answer tests that pin the CPU oracle (the reference ships no tests or golden vectors, so the restatement is
pinned by mathematics: solver.js's DST and tridiagonal, noise.js's integer hash, app.js's mulberry32, sounding.js's
hydrostatic base state)."""
import math

import numpy as np
import pytest

from outbreaklab_b200 import sounding as S, workloads as W


# ---- pure-Python references written from the published algorithms ----
def pcg_py(v):
    """PCG-RXS-M-XS 32-bit hash (noise.js:4) in plain integer arithmetic."""
    M = 0xFFFFFFFF
    s = (v * 747796405 + 2891336453) & M
    w = (((s >> ((s >> 28) + 4)) ^ s) * 277803737) & M
    return ((w >> 22) ^ w) & M


def hash3i_py(x, y, z):
    M = 0xFFFFFFFF
    return pcg_py((x & M) ^ pcg_py((y & M) ^ pcg_py(((z & M) + 0x7F4A7C15) & M)))


def imul(a, b):
    """JavaScript Math.imul: low 32 bits of the product, as a signed int32."""
    r = ((a & 0xFFFFFFFF) * (b & 0xFFFFFFFF)) & 0xFFFFFFFF
    return r - (1 << 32) if r & 0x80000000 else r


def to_i32(x):
    x &= 0xFFFFFFFF
    return x - (1 << 32) if x & 0x80000000 else x


def mulberry_js(seed, n):
    """app.js:1308 with JavaScript int32 / uint32 semantics emulated step by step."""
    a = to_i32(seed)
    out = []
    for _ in range(n):
        a = to_i32(a + 0x6D2B79F5)
        t = imul(a ^ ((a & 0xFFFFFFFF) >> 15), 1 | a)
        t = to_i32((t + imul(t ^ ((t & 0xFFFFFFFF) >> 7), 61 | t)) ^ t)
        out.append(((t ^ ((t & 0xFFFFFFFF) >> 14)) & 0xFFFFFFFF) / 4294967296)
    return np.array(out)


def test_pcg_and_hash(oracle_lib):
    L = oracle_lib.lib()
    for v in [0, 1, 2, 12345, 0xFFFFFFFF, 0x9E3779B9, 747796405]:
        assert L.oro_pcg(v) == pcg_py(v)
    for (x, y, z) in [(0, 0, 0), (17, 3, 5), (-1, 2, -3), (640, 640, 40), (123456, -98765, 7)]:
        assert L.oro_hash3i(x, y, z) == hash3i_py(x, y, z)


def test_mulberry32_vectorised_matches_js_semantics():
    for seed in [1, 2, 7 * 7919 + 13, 0x7FFFFFFF, -5]:
        ref = mulberry_js(seed, 200)
        got = W.mulberry32_block(seed & 0xFFFFFFFF, 200)
        assert np.array_equal(ref, got)
        r = W.Mulberry32(seed & 0xFFFFFFFF)
        assert [r() for _ in range(5)] == list(ref[:5])


@pytest.mark.parametrize("N", [8, 37, 80])
def test_dst_orthonormal_and_eigen(oracle_lib, N):
    q = np.empty(N * N)
    oracle_lib.lib().oro_dst_matrix(N, q)
    Q = q.reshape(N, N)  # Q[i, l] = v_l(i)
    assert np.abs(Q.T @ Q - np.eye(N)).max() < 1e-12
    # 1-D Laplacian with phi = 0 on the faces outside cells 0 and N-1 (antisymmetric ghosts), solver.js:113-114
    h = 1000.0
    L1 = (np.diag(-2 * np.ones(N)) + np.diag(np.ones(N - 1), 1) + np.diag(np.ones(N - 1), -1))
    L1[0, 0] = L1[-1, -1] = -3
    L1 /= h * h
    lam = -4 / (h * h) * np.sin(np.pi * (np.arange(N) + 1) / (2 * N)) ** 2
    assert np.abs(L1 @ Q - Q * lam[None, :]).max() < 1e-12 * np.abs(lam).max() * 10


def _dense_operator(O, nx, ny, nz, dx, dz, rc, rw):
    n = nx * ny * nz
    A = np.empty((n, n))
    e = np.zeros((nz, ny, nx))
    for j in range(n):
        e.reshape(-1)[:] = 0
        e.reshape(-1)[j] = 1
        A[:, j] = O.poisson_apply(e, dx, dz, rc, rw).reshape(-1)
    return A


def test_poisson_oracle_vs_dense_solve(oracle_lib):
    O = oracle_lib
    nx, ny, nz, dx, dz = 7, 5, 6, 1500.0, 400.0
    rng = np.random.default_rng(0)
    rc = 1.2 * np.exp(-np.arange(nz) * dz / 9000.0)
    rw = np.concatenate([[rc[0] * 1.02], 0.5 * (rc[1:] + rc[:-1]), [rc[-1] * 0.94]])
    rhs = rng.standard_normal((nz, ny, nx))
    A = _dense_operator(O, nx, ny, nz, dx, dz, rc, rw)
    ref = np.linalg.solve(A, rhs.reshape(-1)).reshape(nz, ny, nx)
    got64 = O.poisson_solve(rhs, dx, dz, rc, rw, precision=8)
    assert np.abs(got64 - ref).max() / np.abs(ref).max() < 1e-10
    got32 = O.poisson_solve(rhs.astype(np.float32), dx, dz, rc.astype(np.float32), rw.astype(np.float32), 4)
    assert np.abs(got32 - ref).max() / np.abs(ref).max() < 1e-4
    # the residual of the FP64 solve through the operator
    res = O.poisson_apply(got64, dx, dz, rc, rw) - rhs
    assert np.abs(res).max() / np.abs(rhs).max() < 1e-10


def test_base_state_hydrostatic():
    nz = 40
    dz = 20000.0 / nz
    text = W.weisman_klemp_sharppy()
    snd = S.parse_sharppy(text)
    B, sfcP, sfcH = S.base_state(snd, nz, dz)
    B = B.reshape(nz + 1, 8).astype(np.float64)
    th, qv, rho, rhow, pi, p = B[:nz, 0], B[:nz, 1], B[:nz, 2], B[:, 3], B[:nz, 4], B[:nz, 5]
    # Exner integrated upward on faces: pi(centre) = mean of the faces, faces from the hydrostatic recurrence
    piF = np.empty(nz + 1)
    piF[0] = (sfcP / 1000.0) ** (S.RD / S.CP)
    # th and qv are stored after the 97 % cap; the recurrence used the uncapped qv, which only differs where capped
    for k in range(nz):
        piF[k + 1] = piF[k] - S.G * dz / (S.CP * th[k] * (1 + 0.61 * qv[k]))
    assert np.abs(0.5 * (piF[:-1] + piF[1:]) - pi).max() < 2e-4
    assert np.allclose(p, 1e5 * pi ** (S.CP / S.RD), rtol=1e-6)
    T = th * pi
    assert np.allclose(rho, p / (S.RD * T * (1 + 0.61 * qv)), rtol=1e-6)
    es = 611.2 * np.exp(17.67 * (T - 273.15) / (T - 29.65))
    assert np.all(qv <= 0.97 * 0.622 * es / (p - es) * (1 + 1e-6))
    assert np.isclose(rhow[0], rho[0] + 0.5 * (rho[0] - rho[1]), rtol=1e-6)
    assert np.isclose(rhow[nz], rho[nz - 1] * 0.94, rtol=1e-6)
    assert np.allclose(rhow[1:nz], 0.5 * (rho[:-1] + rho[1:]), rtol=1e-6)
    # Weisman-Klemp: theta_sfc ~ 300 K, qv capped at 14 g/kg, westerly shear 25 m/s over 6 km
    assert abs(th[0] - 300.3) < 0.5 and qv.max() <= 0.014 + 1e-9
    assert abs(B[12, 6] - 25.0) < 0.2 and abs(B[2, 6] - 25.0 * 1250 / 6000) < 0.2


def test_sharppy_parser_rejects_short_input():
    with pytest.raises(ValueError):
        S.parse_sharppy("%RAW%\n1000, 0, 20, 15, 180, 10\n%END%")
    snd = S.parse_sharppy(W.weisman_klemp_sharppy())
    assert snd.levels[0].p > snd.levels[-1].p and len(snd.levels) == 401


def test_bubble_placement_constraints():
    pts = W.place_bubbles(8, 640e3, 640e3, seed=2)
    assert len(pts) == 8
    for i, (x, y) in enumerate(pts):
        assert 40e3 <= x <= 600e3 and 40e3 <= y <= 600e3
        for (a, b) in pts[:i]:
            assert math.hypot(x - a, y - b) >= 35e3


def test_oracle_c1_short_run_is_physical(oracle_lib):
    """A few steps of the 64 x 64 x 40 case: the bubble rises, mass is constant, no NaN."""
    case = W.case_c1()
    m, B = oracle_lib.setup_case(case, 4)
    w0, m0 = m.budgets()
    m.step(case.dt, 10)
    V = m.get(oracle_lib.FIELD_V).reshape(case.nz + 1, case.ny + 1, case.nx + 1, 4)
    assert np.isfinite(V).all()
    assert V[..., 2].max() > 0.5
    w1, m1 = m.budgets()
    assert m1 == m0
    assert abs(w1 - w0) / w0 < 1e-3
