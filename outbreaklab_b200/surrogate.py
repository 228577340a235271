"""Host side of the microphysics surrogate: a per-cell MLP that emulates the Thompson-style microphysics block of the
physics pass (model.js:775-905). No counterpart in the reference (OutbreakLab has no learned component).

The network, its training and its inference all run on the GPU through the C ABI (include/ob.h, ob_mlp_*):

    net = MicroSurrogate(seed=1)
    net.reserve(n_pairs)
    record(model, net, steps, dt, rate)      # (state, tendency) pairs from plain Thompson steps of the model itself
    net.fit_norm(dt)                          # input/output scaling and the trusted input range, from the pairs
    net.train(batch, steps, lr)               # fp32 forward/backward kernels + Adam on the GPU
    model.set_surrogate(net)                  # from the next step on, tcgen05 inference in the step

The inputs of a pair are (T, p, rho, qv, qc, qr, qi, qs, qg, Nr, Ni, w) before the block, its targets the block's
change of (T, qv, qc, qi, qr, qs, qg, Nr) over one step; Ni (the reference's spare fourth Q2 channel) and the
changes of Ni and w are carried as documented zeros.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _native as N

NIN, NOUT, NLOSS, PAIR, NPARAM, NNORM = N.MLP_NIN, N.MLP_NOUT, 8, N.MLP_PAIR, N.MLP_NPARAM, N.MLP_NNORM
INPUTS = ("T", "p", "rho", "qv", "qc", "qr", "qi", "qs", "qg", "Nr", "Ni", "w")
OUTPUTS = ("T", "qv", "qc", "qi", "qr", "qs", "qg", "Nr", "Ni", "w")


def features(x: np.ndarray) -> np.ndarray:
    """The input transform of the network: log(q + 1e-9) for the mixing ratios, log(Nr + 1) for Nr."""
    f = np.array(x, np.float64)
    f[:, 3:9] = np.log(np.maximum(f[:, 3:9], 0.0) + 1e-9)
    f[:, 9] = np.log(np.maximum(f[:, 9], 0.0) + 1.0)
    return f


class MicroSurrogate:
    """One network (ObMlp): fp32 master weights, Adam state, normalisation and a device buffer of recorded pairs."""

    def __init__(self, seed: int = 1):
        h = C.c_void_p()
        N.check(N.lib().ob_mlp_create(C.c_uint(seed), C.byref(h)))
        self.h = h

    def sort_pairs(self):
        """Orders the recorded pairs by (model time of their step, texel offset) (ob_mlp_sort_pairs)."""
        N.check(N.lib().ob_mlp_sort_pairs(self.h))

    def set_training(self, mode: int):
        """1 (default): BF16 tensor-core training kernels for batches that are multiples of 128; 0: FP32 SIMT."""
        N.check(N.lib().ob_mlp_set_training(self.h, int(mode)))

    def close(self):
        if self.h:
            N.lib().ob_mlp_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # parameters and normalisation
    def params(self) -> np.ndarray:
        p = np.empty(NPARAM, np.float32)
        N.check(N.lib().ob_mlp_get_params(self.h, N.fptr(p), NPARAM))
        return p

    def set_params(self, p):
        p = np.ascontiguousarray(p, np.float32)
        N.check(N.lib().ob_mlp_set_params(self.h, N.fptr(p), NPARAM))

    def norm(self) -> np.ndarray:
        v = np.empty(NNORM, np.float32)
        N.check(N.lib().ob_mlp_get_norm(self.h, N.fptr(v), NNORM))
        return v

    def set_norm(self, v):
        v = np.ascontiguousarray(v, np.float32)
        N.check(N.lib().ob_mlp_set_norm(self.h, N.fptr(v), NNORM))

    # recorded pairs
    def reserve(self, capacity: int):
        N.check(N.lib().ob_mlp_reserve_pairs(self.h, C.c_longlong(int(capacity))))

    def count(self) -> int:
        c = C.c_longlong()
        N.check(N.lib().ob_mlp_pair_count(self.h, C.byref(c)))
        return int(c.value)

    def read_pairs(self, first: int = 0, count: int | None = None) -> np.ndarray:
        n = self.count() - first if count is None else count
        out = np.empty((max(n, 0), PAIR), np.float32)
        if n > 0:
            N.check(N.lib().ob_mlp_read_pairs(self.h, C.c_longlong(first), C.c_longlong(n), N.fptr(out.reshape(-1))))
        return out

    def write_pairs(self, pairs):
        pairs = np.ascontiguousarray(pairs, np.float32)
        N.check(N.lib().ob_mlp_write_pairs(self.h, N.fptr(pairs.reshape(-1)), C.c_longlong(len(pairs))))

    def fit_norm(self, dt: float, sample: int = 1_000_000, margin: float = 0.0):
        """Standardisation of the transformed inputs and the spread of each tendency, from up to `sample` pairs read
        back to the host; the trusted input range is the pairs' raw range (widened by `margin` of its width)."""
        n = self.count()
        step = max(1, n // sample)
        P = self.read_pairs(0, n)[::step].astype(np.float64)
        f = features(P[:, :NIN])
        mean, std = f.mean(0), f.std(0)
        scale = np.where(std > 1e-12, 1.0 / np.where(std > 1e-12, std, 1.0), 0.0)
        y = P[:, NIN:NIN + NOUT]
        out_scale = np.sqrt((y ** 2).mean(0))
        out_scale[NLOSS:] = 0.0
        out_scale = np.where(out_scale > 0, out_scale, 0.0)
        lo, hi = P[:, :NIN].min(0), P[:, :NIN].max(0)
        w = hi - lo
        v = np.concatenate([mean, scale, out_scale, lo - margin * w, hi + margin * w, [dt]]).astype(np.float32)
        self.set_norm(v)
        return v

    # training and evaluation
    def grad(self, pairs):
        pairs = np.ascontiguousarray(pairs, np.float32)
        g = np.empty(NPARAM, np.float32)
        loss = C.c_double()
        N.check(N.lib().ob_mlp_grad(self.h, N.fptr(pairs.reshape(-1)), len(pairs), C.byref(loss), N.fptr(g)))
        return loss.value, g

    def eval(self, pairs) -> np.ndarray:
        pairs = np.ascontiguousarray(pairs, np.float32)
        out = np.empty((len(pairs), NOUT), np.float32)
        N.check(N.lib().ob_mlp_eval(self.h, N.fptr(pairs.reshape(-1)), len(pairs), N.fptr(out.reshape(-1))))
        return out

    def train(self, batch: int, steps: int, lr: float, seed: int = 7) -> float:
        loss = C.c_double()
        N.check(N.lib().ob_mlp_train(self.h, int(batch), int(steps), C.c_float(lr), C.c_uint(seed), C.byref(loss)))
        return loss.value


def record(model, net: MicroSurrogate, steps: int, dt: float, rate: float):
    """Steps the model `steps` times with the plain scheme while recording pairs into net's buffer, then puts the
    buffer in its canonical order (model time, texel offset), so that what the network is trained on does not depend
    on the order in which the physics pass appended the pairs."""
    N.check(N.lib().ob_model_record_micro(model.h, net.h, C.c_float(rate)))
    try:
        model.step(dt, steps)
    finally:
        N.check(N.lib().ob_model_record_micro(model.h, None, C.c_float(0.0)))
    net.sort_pairs()


def fit(model, net: MicroSurrogate, *, record_steps: int, dt: float, rate: float, capacity: int, batch: int = 16384,
        train_steps: int = 4000, lr: float = 1e-3) -> float:
    """Record pairs from `record_steps` plain steps of the model, normalise, and train with a stepped learning rate
    (60 % of the steps at lr, 25 % at lr/3, 15 % at lr/10); returns the mean loss of the last stage."""
    net.reserve(capacity)
    record(model, net, record_steps, dt, rate)
    net.fit_norm(dt)
    tl = 0.0
    for lr_i, frac in ((lr, 0.6), (lr * 0.3, 0.25), (lr * 0.1, 0.15)):
        tl = net.train(batch, max(1, int(train_steps * frac)), lr_i)
    return tl


def zero_tendency_loss(net: MicroSurrogate, pairs) -> float:
    """The training loss of the method without the network (no microphysics tendency) on the given pairs."""
    sc = net.norm()[24:24 + NLOSS].astype(np.float64)
    t = np.asarray(pairs, np.float64)[:, NIN:NIN + NLOSS] / np.where(sc > 0, sc, 1.0)
    return float((np.where(sc > 0, t, 0.0) ** 2).mean())
