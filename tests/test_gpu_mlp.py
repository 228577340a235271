"""GPU tests of the microphysics surrogate (C ABI): the training kernels' loss and gradient against the float64 oracle
(oracle/mlp_oracle.py), pair recording in the physics pass, the tensor-core inference inside the step against the
oracle's bf16-emulating forward, the scheme fallback, and what a trained network gains over no network."""
import numpy as np
import pytest

from oracle import mlp_oracle as MO
from outbreaklab_b200 import _native as N, model as M, surrogate as S, workloads as W

pytestmark = pytest.mark.gpu


def _synthetic(seed, n):
    rng = np.random.default_rng(seed)
    pairs = np.zeros((n, S.PAIR), np.float32)
    pairs[:, 0] = rng.uniform(230, 300, n)
    pairs[:, 1] = rng.uniform(3e4, 1e5, n)
    pairs[:, 2] = rng.uniform(0.4, 1.2, n)
    pairs[:, 3:9] = rng.uniform(0, 5e-3, (n, 6)) * (rng.random((n, 6)) > 0.3)
    pairs[:, 9] = rng.uniform(0, 1e5, n)
    pairs[:, 11] = rng.normal(0, 5, n)
    pairs[:, 12:20] = rng.normal(0, 1e-4, (n, 8))
    return pairs


def _norm_for(pairs, dt=3.0):
    f = MO.features(pairs[:, :12].astype(np.float64))
    sd = f.std(0)
    sc = np.where(sd > 0, 1 / np.where(sd > 0, sd, 1), 0)
    os_ = np.r_[np.sqrt((pairs[:, 12:20].astype(np.float64) ** 2).mean(0)), 0, 0]
    return np.concatenate([f.mean(0), sc, os_, np.full(12, -3e38), np.full(12, 3e38), [dt]]).astype(np.float32)


def test_training_gradient_matches_float64_oracle(native):
    """Loss and every parameter's gradient of one batch (300 pairs: not a multiple of any tile) vs float64."""
    net = S.MicroSurrogate(seed=3)
    pairs = _synthetic(1, 300)
    norm = _norm_for(pairs)
    net.set_norm(norm)
    params = (np.random.default_rng(2).standard_normal(S.NPARAM) * 0.1).astype(np.float32)
    net.set_params(params)
    loss, g = net.grad(pairs)
    lr, gr = MO.loss_and_grad(params.astype(np.float64), pairs.astype(np.float64), norm.astype(np.float64))
    assert abs(loss - lr) <= 1e-5 * abs(lr)
    # fp32 accumulation over the batch: each parameter block within 1e-4 of its float64 norm
    o = 0
    for name, shp in MO.SHAPES:
        n = int(np.prod(shp))
        a, b = g[o:o + n].astype(np.float64), gr[o:o + n]
        assert np.linalg.norm(a - b) <= 1e-4 * np.linalg.norm(b) + 1e-12, name
        o += n
    # the forward path alone (ob_mlp_eval) in physical units
    y = net.eval(pairs)
    X, _ = MO.normalise(pairs.astype(np.float64), norm.astype(np.float64))
    yr, _ = MO.forward(params.astype(np.float64), X)
    yr = yr * norm[24:34].astype(np.float64)
    assert np.abs(y - yr).max() <= 1e-4 * np.abs(yr).max()


def test_tensor_core_gradient_matches_bf16_oracle(native):
    """The bf16 tensor-core training kernels (the default for batches that are multiples of 128): loss and every
    parameter's gradient of one batch of 256 pairs against the float64 restatement that rounds to bf16 at the same
    points (oracle/mlp_oracle.py loss_and_grad_bf16), and against the exact float64 gradient at bf16's precision."""
    net = S.MicroSurrogate(seed=3)
    pairs = _synthetic(11, 256)
    norm = _norm_for(pairs)
    net.set_norm(norm)
    params = (np.random.default_rng(4).standard_normal(S.NPARAM) * 0.1).astype(np.float32)
    net.set_params(params)
    loss, g = net.grad(pairs)
    lb, gb = MO.loss_and_grad_bf16(params.astype(np.float64), pairs.astype(np.float64), norm.astype(np.float64))
    lr, gr = MO.loss_and_grad(params.astype(np.float64), pairs.astype(np.float64), norm.astype(np.float64))
    assert abs(loss - lb) <= 1e-4 * abs(lb), (loss, lb)
    assert abs(loss - lr) <= 2e-2 * abs(lr), (loss, lr)
    o = 0
    for name, shp in MO.SHAPES:
        n = int(np.prod(shp))
        a, b, r = g[o:o + n].astype(np.float64), gb[o:o + n], gr[o:o + n]
        # fp32 accumulation against exact sums, and the odd bf16 operand rounded the other way
        assert np.linalg.norm(a - b) <= 3e-3 * np.linalg.norm(b) + 1e-12, (name, np.linalg.norm(a - b) / np.linalg.norm(b))
        assert np.linalg.norm(a - r) <= 5e-2 * np.linalg.norm(r) + 1e-12, (name, np.linalg.norm(a - r) / np.linalg.norm(r))
        o += n
    # the same batch through the fp32 SIMT kernels (mode 0) matches the exact float64 gradient, as before
    net.set_training(0)
    loss0, g0 = net.grad(pairs)
    assert abs(loss0 - lr) <= 1e-5 * abs(lr)
    assert np.linalg.norm(g0.astype(np.float64) - gr) <= 1e-4 * np.linalg.norm(gr)


def test_adam_steps_reduce_the_loss(native):
    net = S.MicroSurrogate(seed=4)
    pairs = _synthetic(5, 20000)
    # learnable targets: every tendency a smooth function of the inputs
    x = pairs[:, :12].astype(np.float64)
    pairs[:, 12] = 1e-3 * np.tanh((x[:, 0] - 265) / 20)
    pairs[:, 13] = -2e-5 * x[:, 3] / 5e-3 + 1e-5 * np.sin(x[:, 11] / 3)
    for c in range(14, 20):
        pairs[:, c] = 1e-5 * np.tanh(x[:, c - 10] / 2.5e-3 - 1) * (x[:, 1] / 1e5)
    net.reserve(len(pairs))
    net.write_pairs(pairs)
    net.set_norm(_norm_for(pairs))
    first = net.train(1024, 5, 1e-3)
    net.train(1024, 800, 1e-3)
    last = net.train(1024, 20, 1e-4)
    assert last < 0.2 * first, (first, last)


def test_training_is_deterministic(native):
    """A seed fixes the trained network: two trainings from the same initial parameters on the same pairs give
    bit-identical parameters and losses (every batch reduction adds its partial sums in a fixed order)."""
    pairs = _synthetic(7, 6000)
    nets = []
    for _ in range(2):
        net = S.MicroSurrogate(seed=9)
        net.reserve(len(pairs))
        net.write_pairs(pairs)
        net.set_norm(_norm_for(pairs))
        loss = net.train(2048, 40, 1e-3, seed=11)
        nets.append((loss, net.params()))
    assert nets[0][0] == nets[1][0]
    assert np.array_equal(nets[0][1], nets[1][1])


def _thompson_blob_model():
    case = W.case_small(nx=40, ny=36, nz=40, dx=1000.0, dt=6.0, scheme=1)
    g, B = M.setup_case(case)
    q1, q2 = W.hydrometeor_blob(case, B, thompson=True)
    g.set_field(N.FIELD_Q1, q1)
    g.set_field(N.FIELD_Q2, q2)
    return case, g, B


def _record_one_step(rate=1.0):
    case, a, B = _thompson_blob_model()
    net = S.MicroSurrogate(seed=9)
    net.reserve(case.cells)
    S.record(a, net, 1, case.dt, rate)
    return case, a, B, net, net.read_pairs()


def test_recorded_pairs_have_a_canonical_order(native):
    """Two recordings of the same three steps give byte-identical pair buffers: after recording, ob_mlp_sort_pairs
    orders the pairs by (model time of their step, texel offset), whatever order the physics pass appended them in."""
    bufs = []
    for _ in range(2):
        case, a, B = _thompson_blob_model()
        net = S.MicroSurrogate(seed=9)
        net.reserve(3 * case.cells)
        S.record(a, net, 3, case.dt, 0.5)
        bufs.append(net.read_pairs())
        net.close()
    P, Q = bufs
    assert len(P) > 1000 and P.shape == Q.shape
    assert np.array_equal(P.view(np.uint32), Q.view(np.uint32))
    t, off = P[:, 23].astype(np.float64), P[:, 22].view(np.uint32).astype(np.int64)
    assert set(np.unique(t)) == {0.0, case.dt, 2 * case.dt}   # the model time of each recorded step
    key = t * 2 ** 32 + off
    assert (np.diff(key) > 0).all()                            # strictly increasing: (time, offset) is unique


def test_a_recording_past_capacity_drops_its_last_step(native):
    """A buffer that fills up in the middle of a step keeps a race-dependent subset of that step's pairs; the sort
    drops the step, so the count and the buffer are the same from run to run and end on a whole step."""
    case, a, B = _thompson_blob_model()
    full = S.MicroSurrogate(seed=9)
    full.reserve(3 * case.cells)
    S.record(a, full, 3, case.dt, 0.5)
    ref = full.read_pairs()
    full.close()
    per_step = [int((ref[:, 23] == k * case.dt).sum()) for k in range(3)]
    assert min(per_step) > 100
    cap = per_step[0] + per_step[1] // 2          # fills up half-way through the second step
    bufs = []
    for _ in range(2):
        case, a, B = _thompson_blob_model()
        net = S.MicroSurrogate(seed=9)
        net.reserve(cap)
        S.record(a, net, 3, case.dt, 0.5)
        assert net.count() == per_step[0]
        bufs.append(net.read_pairs())
        net.close()
    assert np.array_equal(bufs[0].view(np.uint32), bufs[1].view(np.uint32))
    assert np.array_equal(bufs[0].view(np.uint32), ref[:per_step[0]].view(np.uint32))


def test_recorded_pairs_are_scheme_tendencies(native):
    case, a, B, net, P = _record_one_step()
    assert len(P) > 1000
    assert np.isfinite(P).all()
    off = P[:, 22].view(np.uint32)
    px = ((case.nx + 1) + 31) // 32 * 32
    i, j, k = off % px, (off // px) % (case.ny + 1), off // (px * (case.ny + 1))
    assert (i < case.nx).all() and (j < case.ny).all() and (k < case.nz).all()
    assert len(np.unique(off)) == len(off)
    # the process rates conserve total water: the six water tendencies cancel to fp32 rounding
    dq = P[:, 13:19].astype(np.float64)
    q = P[:, 3:9].astype(np.float64)
    assert np.abs(dq.sum(1)).max() <= 1e-6 * q.sum(1).max()
    # pressure and density are the base state's at the cell's level
    Bz = B.reshape(-1, 8)
    assert np.allclose(P[:, 1], Bz[k, 5]) and np.allclose(P[:, 2], Bz[k, 2])


def _cell_state(model, case, B, off):
    """T and qv of the cells at the given texel offsets after a step."""
    px = ((case.nx + 1) + 31) // 32 * 32
    i, j, k = off % px, (off // px) % (case.ny + 1), off // (px * (case.ny + 1))
    V = model.get_field(N.FIELD_V).reshape(case.nz + 1, case.ny + 1, case.nx + 1, 4)
    Q1 = model.get_field(N.FIELD_Q1).reshape(case.nz, case.ny, case.nx, 4)
    pi0 = B.reshape(-1, 8)[k, 4].astype(np.float64)
    return V[k, j, i, 3].astype(np.float64) * pi0, Q1[k, j, i, 0].astype(np.float64)


def test_tensor_core_inference_in_the_step(native):
    """One surrogate step: the queued cells are exactly the recorded ones (those holding condensate), none falls
    back, and each cell's T and qv equal the oracle's bf16-emulating forward pass with the projection and the
    saturation adjustment applied."""
    case, a, B, rec, P = _record_one_step()
    net = S.MicroSurrogate(seed=11)
    net.reserve(len(P))
    net.write_pairs(P)
    norm = net.fit_norm(case.dt)
    _, b, _ = _thompson_blob_model()
    b.set_surrogate(net)
    b.step(case.dt, 1)
    queued, fallbacks = b.surrogate_stats()
    assert queued == len(P) and fallbacks == 0
    off = P[:, 22].view(np.uint32)
    T, qv = _cell_state(b, case, B, off)
    X, _ = MO.normalise(P.astype(np.float64), norm.astype(np.float64))
    Y, _ = MO.forward(net.params().astype(np.float64), X, emulate_bf16=True)
    ref = MO.apply(P, Y, norm.astype(np.float64), case.dt)
    sc = norm[24:34].astype(np.float64)
    # compare the changes the network made: after the saturation adjustment, with its latent heat
    dT, dq = np.abs(T - ref[:, 0]), np.abs(qv - ref[:, 1])
    # bf16 activations, the hardware tanh and the summation order: a few percent of an output's spread at most;
    # a wrong operand layout would be off by the spread itself
    # (cells at the edge of saturation can condense on one side and not the other, so the bound on the largest
    # difference is looser than on the 99th percentile)
    for d, s_ in ((dT, sc[0]), (dq, sc[1])):
        assert np.percentile(d, 99) <= 0.02 * s_, (np.percentile(d, 99), s_)
        assert d.max() <= 0.3 * s_, (d.max(), s_)


def test_out_of_range_cells_fall_back_to_the_scheme(native):
    """With an empty trusted range every queued cell runs the scheme: the step equals a plain step."""
    case, a, B, rec, P = _record_one_step()
    net = S.MicroSurrogate(seed=12)
    net.reserve(len(P))
    net.write_pairs(P)
    norm = net.fit_norm(case.dt)
    norm[34:46], norm[46:58] = 3e38, -3e38
    net.set_norm(norm)
    _, b, _ = _thompson_blob_model()
    _, c, _ = _thompson_blob_model()
    b.set_surrogate(net)
    b.step(case.dt, 1)
    c.step(case.dt, 1)
    queued, fallbacks = b.surrogate_stats()
    assert queued > 1000 and fallbacks == queued
    for f, ch in ((N.FIELD_V, 4), (N.FIELD_Q1, 4), (N.FIELD_Q2, 4)):
        x = b.get_field(f).reshape(-1, ch).astype(np.float64)
        y = c.get_field(f).reshape(-1, ch).astype(np.float64)
        for cc in range(ch):
            scale = max(np.abs(y[:, cc]).max(), 1e-30)
            assert np.abs(x[:, cc] - y[:, cc]).max() <= 1e-5 * scale, (f, cc)


def test_trained_network_beats_no_network(native):
    """Trained on 20 recorded steps, the network's loss on 5 later steps is well below that of no tendency at all
    (the method without it)."""
    case, a, B = _thompson_blob_model()
    net = S.MicroSurrogate(seed=21)
    tl = S.fit(a, net, record_steps=20, dt=case.dt, rate=1.0, capacity=40 * case.cells, batch=4096,
               train_steps=1500, lr=2e-3)
    hold = S.MicroSurrogate(seed=22)
    hold.reserve(6 * case.cells)
    S.record(a, hold, 5, case.dt, 1.0)
    H = hold.read_pairs()
    hl, _ = net.grad(H[:65536])
    zl = S.zero_tendency_loss(net, H[:65536])
    print("train loss %.4f held-out %.4f no-network %.4f" % (tl, hl, zl))
    assert hl < 0.5 * zl, (hl, zl)
