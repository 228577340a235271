"""The float64 restatement of the surrogate network (oracle/mlp_oracle.py) pinned by mathematics: its analytic
gradient against central finite differences, and the bf16 rounding helper against exact bfloat16 values."""
import numpy as np

from oracle import mlp_oracle as O


def _case(seed=0, n=24):
    rng = np.random.default_rng(seed)
    params = rng.standard_normal(O.NPARAM) * 0.2
    pairs = np.zeros((n, O.PAIR))
    pairs[:, 0] = rng.uniform(230, 300, n)
    pairs[:, 1] = rng.uniform(3e4, 1e5, n)
    pairs[:, 2] = rng.uniform(0.4, 1.2, n)
    pairs[:, 3:9] = rng.uniform(0, 5e-3, (n, 6))
    pairs[:, 9] = rng.uniform(0, 1e5, n)
    pairs[:, 11] = rng.normal(0, 5, n)
    pairs[:, 12:20] = rng.normal(0, 1e-4, (n, 8))
    norm = np.concatenate([rng.normal(0, 1, 12), rng.uniform(0.1, 1.0, 12), np.r_[rng.uniform(1e-5, 1e-3, 8), 0, 0],
                           np.full(12, -1e30), np.full(12, 1e30), [3.0]])
    return params, pairs, norm


def test_gradient_matches_finite_differences():
    params, pairs, norm = _case()
    loss, g = O.loss_and_grad(params, pairs, norm)
    rng = np.random.default_rng(1)
    idx = np.concatenate([rng.choice(O.NPARAM, 40, replace=False), [0, O.NPARAM - 1, O.NPARAM - 11]])
    h = 1e-6
    for i in idx:
        p1, p2 = params.copy(), params.copy()
        p1[i] += h
        p2[i] -= h
        fd = (O.loss_and_grad(p1, pairs, norm)[0] - O.loss_and_grad(p2, pairs, norm)[0]) / (2 * h)
        # central differences carry O(h^2) truncation and O(eps loss / h) rounding: 1e-4 relative
        assert abs(fd - g[i]) <= 1e-4 * max(1.0, abs(fd)), (i, fd, g[i])


def test_loss_is_forward_mse():
    params, pairs, norm = _case(2)
    X, T = O.normalise(pairs, norm)
    Y, _ = O.forward(params, X)
    loss, _ = O.loss_and_grad(params, pairs, norm)
    assert np.isclose(loss, ((Y[:, :8] - T[:, :8]) ** 2).mean(), rtol=1e-12)


def test_bf16_rounding():
    x = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 2 ** -9, 1.0 + 3 * 2 ** -9, -3.14159, 0.0, 1.0 + 3 * 2 ** -8], np.float64)
    r = O.bf16(x)
    assert r[0] == 1.0
    assert r[1] == 1.0                    # bf16 ulp at 1 is 2^-7: 1 + 2^-8 is a tie, to even (down)
    assert r[2] == 1.0                    # below half an ulp
    assert r[3] == 1.0 + 2 ** -7          # above half an ulp
    assert r[6] == 1.0 + 2 ** -6          # a tie between odd 1 + 2^-7 and even 1 + 2^-6
    assert abs(r[4] + 3.140625) < 1e-12
    assert r[5] == 0.0
