"""Float64 restatement of the microphysics surrogate network (TEST INFRASTRUCTURE ONLY).

Only tests/ import this module: it is the checker of the GPU training kernels (forward, loss, gradient of every
parameter) and of the tensor-core inference kernel (with bf16 rounding of weights and activations emulated). It
restates the network the library documents for ob_mlp_* (include/ob.h): 12 inputs -> 3 x 128 GELU (tanh form) ->
10 outputs, inputs log-transformed and standardised, loss = mean squared error of the first 8 outputs in normalised
units. The surrogate has no counterpart in the reference; the scheme it emulates is the Thompson-style block of
model.js:775-905, whose restatement is ob_oracle.cpp.
"""
from __future__ import annotations

import numpy as np

NIN, NH, NOUT, NLOSS, PAIR = 12, 128, 10, 8, 24
SHAPES = (("W1", (NH, NIN)), ("b1", (NH,)), ("W2", (NH, NH)), ("b2", (NH,)), ("W3", (NH, NH)), ("b3", (NH,)),
          ("W4", (NOUT, NH)), ("b4", (NOUT,)))
NPARAM = sum(int(np.prod(s)) for _, s in SHAPES)
GC, GA = 0.7978845608028654, 0.044715


def unpack(flat):
    out, o = {}, 0
    for name, shp in SHAPES:
        n = int(np.prod(shp))
        out[name] = np.asarray(flat[o:o + n], np.float64).reshape(shp)
        o += n
    return out


def pack(d):
    return np.concatenate([np.asarray(d[name], np.float64).reshape(-1) for name, _ in SHAPES])


def split_norm(norm):
    norm = np.asarray(norm, np.float64)
    return dict(in_mean=norm[0:12], in_scale=norm[12:24], out_scale=norm[24:34], in_lo=norm[34:46], in_hi=norm[46:58],
                dt=norm[58])


def features(x):
    """Raw inputs (n, 12) -> transformed inputs: log(q + 1e-9) for the mixing ratios, log(Nr + 1) for Nr."""
    f = np.array(x, np.float64)
    f[:, 3:9] = np.log(np.maximum(f[:, 3:9], 0.0) + 1e-9)
    f[:, 9] = np.log(np.maximum(f[:, 9], 0.0) + 1.0)
    return f


def gelu(z):
    return 0.5 * z * (1.0 + np.tanh(GC * (z + GA * z ** 3)))


def gelu_grad(z):
    t = np.tanh(GC * (z + GA * z ** 3))
    return 0.5 * (1.0 + t) + 0.5 * z * (1.0 - t * t) * GC * (1.0 + 3.0 * GA * z * z)


def bf16(a):
    """Round to the nearest bfloat16 (ties to even), returned as float64."""
    a32 = np.asarray(a, np.float32)
    u = a32.view(np.uint32).astype(np.uint64)
    u = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def forward(params, X, emulate_bf16=False):
    """Normalised inputs X (n, 12) -> outputs (n, 10) and the pre-activations of the hidden layers."""
    p = unpack(params)
    r = bf16 if emulate_bf16 else (lambda a: a)
    h = r(X)
    zs = []
    for l in (1, 2, 3):
        z = h @ r(p["W%d" % l]).T + p["b%d" % l]
        zs.append(z)
        h = r(gelu(z))
    return h @ r(p["W4"]).T + p["b4"], zs


def normalise(pairs, norm):
    n = split_norm(norm)
    X = (features(pairs[:, :NIN]) - n["in_mean"]) * n["in_scale"]
    sc = n["out_scale"]
    T = np.where(sc > 0, pairs[:, NIN:NIN + NOUT] / np.where(sc > 0, sc, 1.0), 0.0)
    return X, T


def loss_and_grad(params, pairs, norm):
    """The training kernels' loss and gradient in float64."""
    p = unpack(params)
    X, T = normalise(np.asarray(pairs, np.float64), norm)
    B = X.shape[0]
    hs = [X]
    zs = []
    h = X
    for l in (1, 2, 3):
        z = h @ p["W%d" % l].T + p["b%d" % l]
        zs.append(z)
        h = gelu(z)
        hs.append(h)
    Y = h @ p["W4"].T + p["b4"]
    D = np.zeros_like(Y)
    D[:, :NLOSS] = Y[:, :NLOSS] - T[:, :NLOSS]
    loss = float((D ** 2).sum() / (B * NLOSS))
    dY = 2.0 * D / (B * NLOSS)
    g = {"W4": dY.T @ hs[3], "b4": dY.sum(0)}
    dh = dY @ p["W4"]
    for l in (3, 2, 1):
        dz = dh * gelu_grad(zs[l - 1])
        g["W%d" % l] = dz.T @ hs[l - 1]
        g["b%d" % l] = dz.sum(0)
        dh = dz @ p["W%d" % l]
    return loss, pack(g)


def loss_and_grad_bf16(params, pairs, norm):
    """The tensor-core training kernels' loss and gradient (ob_mlp_train_tc.cu), in float64 with bf16 rounding at the
    same points: the normalised inputs, the weights, every hidden activation, dY and every dZ are bf16 operands; the
    products accumulate exactly (the kernels accumulate in fp32); GELU' is taken of the unrounded pre-activation. The
    bias gradients sum the bf16 operands (the kernels get them from a row of ones appended to the GEMM)."""
    p = unpack(params)
    pairs = np.asarray(pairs, np.float64)
    n = split_norm(norm)
    f32 = np.float32
    raw = pairs[:, :NIN].astype(f32)
    fe = raw.copy()
    fe[:, 3:9] = np.log(np.maximum(fe[:, 3:9], f32(0)) + f32(1e-9))
    fe[:, 9] = np.log(np.maximum(fe[:, 9], f32(0)) + f32(1))
    X = bf16((fe - n["in_mean"].astype(f32)) * n["in_scale"].astype(f32))
    sc = n["out_scale"]
    T = np.where(sc > 0, (pairs[:, NIN:NIN + NOUT].astype(f32) / np.where(sc > 0, sc, 1.0).astype(f32)).astype(np.float64), 0.0)
    B = X.shape[0]
    W = {l: bf16(p["W%d" % l]) for l in (1, 2, 3, 4)}
    hs, gs, h = [X], [], X
    for l in (1, 2, 3):
        z = h @ W[l].T + p["b%d" % l].astype(f32).astype(np.float64)
        gs.append(gelu_grad(z))
        h = bf16(gelu(z))
        hs.append(h)
    Y = h @ W[4].T + p["b4"]
    D = np.zeros_like(Y)
    D[:, :NLOSS] = Y[:, :NLOSS] - T[:, :NLOSS]
    loss = float((D ** 2).sum() / (B * NLOSS))
    dY = bf16(np.float32(2.0 / (B * NLOSS)) * D.astype(np.float32))
    g = {"W4": dY.T @ hs[3], "b4": dY.sum(0)}
    dh = dY @ W[4]
    for l in (3, 2, 1):
        dz = bf16(dh * gs[l - 1])
        g["W%d" % l] = dz.T @ hs[l - 1]
        g["b%d" % l] = dz.sum(0)
        dh = dz @ W[l]
    return loss, pack(g)


CPD, RV, LV, LF, LS, T0 = 1005.7, 461.5, 2.501e6, 3.337e5, 2.834e6, 273.15
NEW_SPECIES_FLOOR = 1e-8


def sat_adjust(T, qv, qc, qi, p):
    """The scheme's 3-iteration mixed-phase saturation adjustment (model.js:893-905), vectorised in float64."""
    T, qv, qc, qi = (np.array(a, np.float64) for a in (T, qv, qc, qi))
    fice = lambda t: np.clip((T0 - t) / 40.0, 0.0, 1.0)
    esl = lambda t: 611.2 * np.exp(17.67 * (t - T0) / (t - 29.65))
    esi = lambda t: 611.2 * np.exp(21.8745584 * (t - 273.16) / (t - 7.66))
    qi0 = qi.copy()
    qcl = qc + qi
    dsum = np.zeros_like(T)
    for _ in range(3):
        f = fice(T)
        e = esl(T) * (1 - f) + esi(T) * f
        qs = 0.622 * e / np.maximum(p - e, 100.0)
        Lh = LV * (1 - f) + LS * f
        d = (qv - qs) / (1.0 + Lh * Lh * qs / (CPD * RV * T * T))
        d = np.maximum(d, -qcl)
        qv, qcl, T, dsum = qv - d, qcl + d, T + Lh / CPD * d, dsum + d
    f = fice(T)
    qi = f * qcl
    qc = qcl - qi
    T = T + LF / CPD * (qi - qi0 - f * dsum)
    return T, qv, qc, qi


def apply(pairs, outputs, norm, dt):
    """The surrogate kernel's use of the outputs on each recorded cell: scaled process tendencies, the noise floor of
    empty species, positivity, total water, the rain-number bounds, then the saturation adjustment. Returns the new
    (T, qv, qc, qi, qr, qs, qg, Nr) before the sponge factor and the final clips."""
    n = split_norm(norm)
    x = np.asarray(pairs, np.float64)
    scale = dt / n["dt"] if n["dt"] > 0 else 1.0
    d = outputs[:, :NLOSS] * n["out_scale"][:NLOSS] * scale
    q = np.stack([x[:, 3], x[:, 4], x[:, 6], x[:, 5], x[:, 7], x[:, 8]], 1)  # qv, qc, qi, qr, qs, qg
    dq = np.where((q == 0) & (d[:, 1:7] < NEW_SPECIES_FLOOR), 0.0, d[:, 1:7])
    dq = np.maximum(dq, -q)
    gain = np.where(dq > 0, dq, 0).sum(1)
    loss = -np.where(dq < 0, dq, 0).sum(1)
    fg = np.where(gain > loss, loss / np.where(gain > 0, gain, 1), 1.0)
    fl = np.where(loss > gain, gain / np.where(loss > 0, loss, 1), 1.0)
    qn = q + dq * np.where(dq > 0, fg[:, None], fl[:, None])
    T = x[:, 0] + d[:, 0]
    nr = x[:, 9] + d[:, 7]
    qr = qn[:, 3]
    nr = np.where(qr > 1e-9, np.clip(nr, qr * 3.183e5, qr * 3.183e11), 0.0)
    T, qv, qc, qi = sat_adjust(T, qn[:, 0], qn[:, 1], qn[:, 2], x[:, 1])
    return np.column_stack([T, qv, qc, qi, qn[:, 3], qn[:, 4], qn[:, 5], nr])
